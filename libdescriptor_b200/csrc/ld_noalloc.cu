// ld_noalloc.cu -- descriptor + VJP entry point that allocates nothing.
//
// Some callers cannot call cudaMalloc at force-evaluation time: an MD engine
// or model driver that owns all device memory through its own pool, a
// real-time serving loop with a no-allocation policy, or code running where
// an allocation would synchronise the device or is simply forbidden.  For
// them the neighbour-row offsets, the prefix-sum work space and the device
// status word of one fused descriptor + VJP pass live in a fixed array in
// this library's own device memory instead of buffers from cudaMalloc.
//
// The array is a file-scope __device__ object of kScratchBytes: every GPU
// that loads the library holds it until the process exits.  It is shared by
// all calls and keeps the last call's contents; the status word is cleared
// at the start of every call.  Calls whose work overlaps on the GPU (two
// streams, two host threads) race on it: issue them on one stream or
// serialise them.  Like ld_gradient_dev, the call does not know the number
// of coordinate rows, so the caller keeps every centre and neighbour index
// inside the coordinates (no device-side index check runs).
#include <mutex>

#include "ld_internal.h"

namespace ldb {
int launch_rows(ld_descriptor *d, const RowArgs &a, cudaStream_t s);
}

namespace {

constexpr int kMaxRows = 1 << 18;                       // centre rows per call
constexpr size_t kStatusBytes = 256;                    // [0, 256): status word
constexpr size_t kOffsetBytes = ((size_t)(kMaxRows + 1) * 8 + 255) & ~(size_t)255;
constexpr size_t kScratchBytes = 4u << 20;              // 4 MiB in total
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

std::mutex g_mu;
void *g_base[kMaxDevices] = {nullptr};

// Device address of g_scratch for the current device (looked up once per
// device: host code only holds a stand-in symbol, never a device address).
// The current device must be the handle's: its parameter tables live there.
int scratch_base(const ld_descriptor *d, void **out) {
    int dev = 0;
    LDB_CUDA(cudaGetDevice(&dev));
    if (dev != ldb::handle_device(d))
        return ldb::fail(LD_ERR_INVALID_ARG, "ld_gradient_counts_dev_noalloc: the current device (" +
                                                 std::to_string(dev) + ") is not the descriptor's device (" +
                                                 std::to_string(ldb::handle_device(d)) + ")");
    if (dev < 0 || dev >= kMaxDevices) return ldb::fail(LD_ERR_INVALID_ARG, "device ordinal too large");
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_base[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess) return ldb::cuda_fail(e, "cudaGetSymbolAddress(g_scratch)");
        g_base[dev] = p;
    }
    *out = g_base[dev];
    return LD_OK;
}

}  // namespace

extern "C" int ld_gradient_counts_dev_noalloc(ld_descriptor *d, int n_rows, const int *row_centre,
                                              const int *species, const int *neighbor_list,
                                              const int *number_of_neighs, int max_neigh,
                                              const double *coords, const double *dE_ddesc,
                                              double *d_coords, double *desc_out, const int *image,
                                              ld_stream stream) {
    using namespace ldb;
    if (!d) return fail(LD_ERR_INVALID_ARG, "descriptor handle is NULL");
    if (n_rows < 0 || max_neigh < 0) return fail(LD_ERR_INVALID_ARG, "negative size");
    if (n_rows > kMaxRows)
        return fail(LD_ERR_CAPACITY, "ld_gradient_counts_dev_noalloc: n_rows=" + std::to_string(n_rows) +
                                         " exceeds the fixed scratch limit of " + std::to_string(kMaxRows) +
                                         " rows per call");
    if (n_rows == 0) return LD_OK;
    if (!species || !coords || !number_of_neighs || !dE_ddesc || !d_coords || (!neighbor_list && max_neigh > 0))
        return fail(LD_ERR_INVALID_ARG, "NULL device array");
    const size_t tmp_need = offsets_tmp_bytes(n_rows);
    const size_t tmp_have = kScratchBytes - kStatusBytes - kOffsetBytes;
    if (tmp_need > tmp_have)
        return fail(LD_ERR_CAPACITY, "ld_gradient_counts_dev_noalloc: prefix-sum work space does not fit");
    void *base = nullptr;
    int rc = scratch_base(d, &base);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    char *b = static_cast<char *>(base);
    int *status = reinterpret_cast<int *>(b);
    long long *off = reinterpret_cast<long long *>(b + kStatusBytes);
    void *tmp = b + kStatusBytes + kOffsetBytes;
    LDB_CUDA(cudaMemsetAsync(status, 0, sizeof(int), s));
    rc = offsets_launch(n_rows, number_of_neighs, off, nullptr, tmp, tmp_have, s);
    if (rc) return rc;
    RowArgs a;
    a.n_rows = n_rows;
    a.row_centre = row_centre;
    a.species = species;
    a.nbl = neighbor_list;
    a.off = off;
    a.max_neigh = max_neigh > 0 ? max_neigh : 1;
    a.coords = coords;
    a.desc = desc_out;
    a.dE = dE_ddesc;
    a.dcoords = d_coords;
    a.image = image;
    a.status = status;
    a.fused_only = true;   // single-kernel gradient: no stream-ordered work space
    rc = launch_rows(d, a, s);
    if (rc) return rc;
    int st = 0;
    LDB_CUDA(cudaMemcpyAsync(&st, status, sizeof(int), cudaMemcpyDeviceToHost, s));
    LDB_CUDA(cudaStreamSynchronize(s));
    if (st == kDevCapacity) return fail(LD_ERR_CAPACITY, "a centre has more neighbours than max_neigh");
    if (st != 0) return fail(LD_ERR_INVALID_ARG, "the kernels raised device status " + std::to_string(st));
    return LD_OK;
}
