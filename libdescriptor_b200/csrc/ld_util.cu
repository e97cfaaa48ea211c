// ld_util.cu -- small device utilities: CSR row offsets, the FP64 rate probe.
#include <cub/cub.cuh>
#include <mutex>

#include "ld_bulk.cuh"
#include "ld_internal.h"

namespace ldb {
namespace {

__global__ void widen_counts(int n, const int *counts, long long *off) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r == 0) off[0] = 0;
    if (r < n) off[r + 1] = (long long)counts[r];
}

// Dependent FMA chains, 8 independent chains per thread (enough ILP to keep
// the FP64 pipe busy); the result is stored so the work cannot be removed.
__global__ void fp64_probe(int iters, double seed, double *out) {
    double a0 = seed + threadIdx.x * 1e-9, a1 = a0 + 1e-3, a2 = a0 + 2e-3, a3 = a0 + 3e-3;
    double a4 = a0 + 4e-3, a5 = a0 + 5e-3, a6 = a0 + 6e-3, a7 = a0 + 7e-3;
    const double m = 0.999999999, c = 1e-12;
    for (int k = 0; k < iters; ++k) {
#pragma unroll
        for (int u = 0; u < 16; ++u) {
            a0 = fma(a0, m, c); a1 = fma(a1, m, c); a2 = fma(a2, m, c); a3 = fma(a3, m, c);
            a4 = fma(a4, m, c); a5 = fma(a5, m, c); a6 = fma(a6, m, c); a7 = fma(a7, m, c);
        }
    }
    const double s = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
    if (s == 12345.678) out[0] = s;  // practically never; keeps the chains live
    if (threadIdx.x == 0 && blockIdx.x == 0) out[1] = s;
}

// Throughput probe of one FP64 library call (8 independent chains per
// thread); op: 0 exp, 1 sincos, 2 sqrt, 3 divide, 4 tan, 5 pow, 6 cos.
__global__ void op_probe(int op, int iters, double *out) {
    double v[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) v[c] = 0.3 + 0.01 * c + threadIdx.x * 1e-7;
    for (int k = 0; k < iters; ++k) {
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            const double x = v[c];
            double y;
            switch (op) {
            case 0: y = exp(-x); break;
            case 1: { double s, cc; sincos(x, &s, &cc); y = s + cc - 0.7; } break;
            case 2: y = sqrt(x + 0.5); break;
            case 3: y = 0.35 / (x + 0.6); break;
            case 4: y = tan(x) * 0.5; break;
            case 5: y = pow(x + 0.5, 1.7); break;
            default: y = cos(x); break;
            }
            v[c] = 0.25 + 0.5 * y;   // keeps x in (0.25, 0.75)
        }
    }
    double s = 0;
#pragma unroll
    for (int c = 0; c < 8; ++c) s += v[c];
    if (s == 12345.678) out[0] = s;
}

}  // namespace

int pool_alloc(void **p, size_t bytes, cudaStream_t s) {
    constexpr int kMaxDevices = 64;
    static std::mutex mu;
    static cudaMemPool_t pools[kMaxDevices] = {};
    int dev = 0;
    LDB_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return fail(LD_ERR_INVALID_ARG, "device ordinal outside the pool table");
    cudaMemPool_t pool = nullptr;
    {
        std::lock_guard<std::mutex> lk(mu);
        if (!pools[dev]) {
            cudaMemPoolProps props = {};
            props.allocType = cudaMemAllocationTypePinned;
            props.handleTypes = cudaMemHandleTypeNone;
            props.location.type = cudaMemLocationTypeDevice;
            props.location.id = dev;
            cudaMemPool_t created = nullptr;
            LDB_CUDA(cudaMemPoolCreate(&created, &props));
            unsigned long long keep = ~0ull;
            cudaError_t e = cudaMemPoolSetAttribute(created, cudaMemPoolAttrReleaseThreshold, &keep);
            if (e != cudaSuccess) {
                cudaMemPoolDestroy(created);
                return cuda_fail(e, "scratch pool");
            }
            pools[dev] = created;
        }
        pool = pools[dev];
    }
    if (int rc = count_alloc()) return rc;
    LDB_CUDA(cudaMallocFromPoolAsync(p, bytes ? bytes : 1, pool, s));
    const int f = scratch_fill();
    if (f >= 0) LDB_CUDA(cudaMemsetAsync(*p, f, bytes ? bytes : 1, s));
    return LD_OK;
}

size_t offsets_tmp_bytes(int n_rows) {
    size_t a = 0, b = 0;
    cub::DeviceScan::InclusiveSum(nullptr, a, (long long *)nullptr, (long long *)nullptr, n_rows);
    cub::DeviceReduce::Max(nullptr, b, (const int *)nullptr, (int *)nullptr, n_rows);
    return (a > b ? a : b) + 256;
}

int offsets_launch(int n_rows, const int *counts, long long *off, int *maxn, void *tmp,
                   size_t tmp_bytes, cudaStream_t s) {
    if (n_rows <= 0) {
        LDB_CUDA(cudaMemsetAsync(off, 0, sizeof(long long), s));
        if (maxn) LDB_CUDA(cudaMemsetAsync(maxn, 0, sizeof(int), s));
        return LD_OK;
    }
    const int bs = 256;
    widen_counts<<<(n_rows + bs - 1) / bs, bs, 0, s>>>(n_rows, counts, off);
    count_launch();
    LDB_CUDA(cudaGetLastError());
    size_t tb = tmp_bytes;
    LDB_CUDA(cub::DeviceScan::InclusiveSum(tmp, tb, off + 1, off + 1, n_rows, s));
    count_launch();
    if (maxn) {
        tb = tmp_bytes;
        LDB_CUDA(cub::DeviceReduce::Max(tmp, tb, counts, maxn, n_rows, s));
        count_launch();
    }
    return LD_OK;
}

// Self-test of the bounded bulk-copy wait: thread 0 arms the barrier for 16
// bytes that no copy delivers, every thread waits at most limit_ns, and the
// CTA reports kDevTimeout when the wait ran out (it always should).
__global__ void bulk_wait_probe(unsigned long long limit_ns, int *status) {
    __shared__ __align__(8) unsigned long long bar;
    if (threadIdx.x == 0) {
        bulk_barrier_init(&bar);
        bulk_expect(&bar, 16);
    }
    __syncthreads();
    const bool ok = bulk_copy_wait(&bar, limit_ns);
    if (__syncthreads_or(!ok) && threadIdx.x == 0) atomicCAS(status, 0, (int)kDevTimeout);
}

}  // namespace ldb

extern "C" int ld_debug_bulk_wait_timeout(long long limit_ns) {
    using namespace ldb;
    if (limit_ns <= 0 || limit_ns > 1000000000LL)
        return fail(LD_ERR_INVALID_ARG, "ld_debug_bulk_wait_timeout: limit_ns outside 1 .. 1e9");
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return fail(LD_ERR_NO_DEVICE, "no CUDA device visible");
    int *status = nullptr;
    LDB_CUDA(cudaMalloc(&status, sizeof(int)));
    int host = -1;
    cudaError_t e = cudaMemset(status, 0, sizeof(int));
    if (e == cudaSuccess) {
        bulk_wait_probe<<<1, 64>>>((unsigned long long)limit_ns, status);
        count_launch();
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(&host, status, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(status);
    if (e != cudaSuccess) return cuda_fail(e, "bulk_wait_probe");
    if (host == kDevTimeout)
        return fail(LD_ERR_TIMEOUT, "ld_debug_bulk_wait_timeout: the bounded wait ran out (as it should)");
    return LD_OK;
}

extern "C" int ld_measure_fp64_peak(int iters, double *tflops) {
    using namespace ldb;
    if (!tflops || iters <= 0) return fail(LD_ERR_INVALID_ARG, "ld_measure_fp64_peak: bad arguments");
    int dev = 0, nsm = 0;
    LDB_CUDA(cudaGetDevice(&dev));
    LDB_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    double *out = nullptr;
    LDB_CUDA(cudaMalloc(&out, 2 * sizeof(double)));
    const int threads = 256, blocks = nsm * 8;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    fp64_probe<<<blocks, threads>>>(iters / 4 + 1, 1.0, out);  // warm-up
    count_launch();
    cudaEventRecord(e0);
    fp64_probe<<<blocks, threads>>>(iters, 1.0, out);
    count_launch();
    cudaEventRecord(e1);
    cudaError_t err = cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (err != cudaSuccess) return cuda_fail(err, "fp64_probe");
    const double fmas = (double)blocks * threads * (double)iters * 16.0 * 8.0;
    *tflops = 2.0 * fmas / (ms * 1e-3) / 1e12;
    return LD_OK;
}

extern "C" int ld_measure_fp64_op_cost(int op, int iters, double fp64_tflops, double *flop_equiv) {
    using namespace ldb;
    if (!flop_equiv || iters <= 0 || op < 0 || op > 6 || !(fp64_tflops > 0))
        return fail(LD_ERR_INVALID_ARG, "ld_measure_fp64_op_cost: bad arguments");
    int dev = 0, nsm = 0;
    LDB_CUDA(cudaGetDevice(&dev));
    LDB_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    double *out = nullptr;
    LDB_CUDA(cudaMalloc(&out, sizeof(double)));
    const int threads = 256, blocks = nsm * 8;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    op_probe<<<blocks, threads>>>(op, iters / 4 + 1, out);
    count_launch();
    cudaEventRecord(e0);
    op_probe<<<blocks, threads>>>(op, iters, out);
    count_launch();
    cudaEventRecord(e1);
    cudaError_t err = cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (err != cudaSuccess) return cuda_fail(err, "op_probe");
    const double calls = (double)blocks * threads * (double)iters * 8.0;
    const double per_s = calls / (ms * 1e-3);
    // flops the FP64 pipe could have done in the time of one call (the
    // loop's own FMA per call is part of the call's cost)
    *flop_equiv = fp64_tflops * 1e12 / per_s;
    return LD_OK;
}
