// ld_sf_common.cuh -- helpers shared by the symmetry-function kernels:
// cutoff functions, warp reductions, the per-warp neighbour staging slice and
// the launch shape (warps per CTA, persistent grid, optional row queue).
#pragma once

#include <string>

#include "ld_csr.cuh"
#include "ld_internal.h"

namespace ldb {
namespace sfc {

constexpr double kPi = 3.1415926535897932;

__device__ __forceinline__ void raise_status(int *status, int code) {
    if (status) atomicCAS(status, 0, code);
}

__device__ __forceinline__ double cutc(double r, double rc) {
    return (r < rc) ? 0.5 * (cos(kPi * r / rc) + 1.0) : 0.0;
}
__device__ __forceinline__ double dcutc(double r, double rc) {
    return (r < rc) ? -0.5 * sin(kPi * r / rc) * (kPi / rc) : 0.0;
}
// the cosine cutoff and its derivative from r / rc = r * irc (irc = 1 / rc):
// one sincospi, no division, no reduction by pi
__device__ __forceinline__ double cutc_i(double r, double rc, double irc) {
    return (r < rc) ? 0.5 * (cospi(r * irc) + 1.0) : 0.0;
}
__device__ __forceinline__ void cutc_both(double r, double rc, double irc, double &fc, double &dfc) {
    if (r < rc) {
        double sn, cs;
        sincospi(r * irc, &sn, &cs);
        fc = 0.5 * (cs + 1.0);
        dfc = -0.5 * sn * (kPi * irc);
    } else {
        fc = 0.0;
        dfc = 0.0;
    }
}
__device__ __forceinline__ double ipow(double x, int n) {
    double r = 1.0;
    for (int k = 0; k < n; ++k) r *= x;
    return r;
}
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

struct WarpSlice {
    double *cx, *cy, *cz, *r, *ir, *rc, *fc, *dfc, *gx, *gy, *gz;
    int *spec, *idx, *inc, *nbl;
};

__device__ __forceinline__ WarpSlice slice(double *base, int cap, bool vjp) {
    WarpSlice s;
    double *p = base;
    s.cx = p; p += cap;
    s.cy = p; p += cap;
    s.cz = p; p += cap;
    s.r = p; p += cap;
    s.ir = p; p += cap;
    s.rc = p; p += cap;
    s.fc = p; p += cap;
    if (vjp) {
        s.dfc = p; p += cap;
        s.gx = p; p += cap;
        s.gy = p; p += cap;
        s.gz = p; p += cap;
    } else {
        s.dfc = s.gx = s.gy = s.gz = nullptr;
    }
    int *q = reinterpret_cast<int *>(p);
    s.spec = q; q += cap;
    s.idx = q; q += cap;
    s.inc = q; q += cap;
    s.nbl = q;
    return s;
}

// Per-warp staging size (doubles; the int arrays are packed after them).
inline int per_warp_doubles(int cap, bool vjp) { return cap * (vjp ? 11 : 7) + (4 * cap + 1) / 2 + 2; }

// Launch a warp-per-centre kernel kern(p, a, per_warp, queue) with the
// tuned shape: warps per CTA (a.sf_warps), CTA cap per SM, optional dynamic
// row queue (counter in the caller's work space or stream-ordered).
template <class K, class P>
int launch_rows_kernel(K kern, const P &p, const RowArgs &a, cudaStream_t s, bool vjp, const char *what,
                       int extra_doubles = 0) {
    const int cap = a.max_neigh > 0 ? a.max_neigh : 1;
    const int per_warp = per_warp_doubles(cap, vjp) + extra_doubles;
    const size_t per_warp_bytes = (size_t)per_warp * sizeof(double);
    int nw = (a.sf_warps == 1 || a.sf_warps == 2 || a.sf_warps == 4) ? a.sf_warps : 4;
    while (nw > 1 && per_warp_bytes * nw > 200 * 1024) --nw;
    if (per_warp_bytes * nw > 220 * 1024)
        return fail(LD_ERR_CAPACITY, "symmetry functions: max_neigh=" + std::to_string(a.max_neigh) +
                                         " exceeds the on-chip neighbour staging capacity");
    const size_t smem = per_warp_bytes * nw;
    LDB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int dev = 0, nsm = 148, per_sm = 1;
    LDB_CUDA(cudaGetDevice(&dev));
    LDB_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    LDB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, nw * 32, smem));
    if (per_sm < 1) per_sm = 1;
    if (a.ctas_per_sm > 0 && a.ctas_per_sm < per_sm) per_sm = a.ctas_per_sm;
    long long want = (a.n_rows + nw - 1) / nw;
    long long grid = (long long)nsm * per_sm;
    if (want < grid) grid = want;
    if (grid < 1) grid = 1;
    int *queue = nullptr;
    bool own = false;
    if (a.dynamic_queue) {
        if (a.work) {
            if (a.work_bytes < sizeof(int)) return fail(LD_ERR_INVALID_ARG, "work space too small");
            queue = static_cast<int *>(a.work);
        } else {
            const int rc = pool_alloc((void **)&queue, sizeof(int), s);
            if (rc) return rc;
            own = true;
        }
        LDB_CUDA(cudaMemsetAsync(queue, 0, sizeof(int), s));
    }
    kern<<<(unsigned)grid, nw * 32, smem, s>>>(p, a, per_warp, queue);
    count_launch();
    cudaError_t e = cudaGetLastError();
    if (own) {
        cudaError_t e2 = cudaFreeAsync(queue, s);
        if (e == cudaSuccess) e = e2;
    }
    if (e != cudaSuccess) return cuda_fail(e, what);
    return LD_OK;
}

}  // namespace sfc
}  // namespace ldb
