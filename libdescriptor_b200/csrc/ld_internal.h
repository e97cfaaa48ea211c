// ld_internal.h -- shared declarations of the libdescriptor_b200 native core.
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <cstdint>
#include <string>
#include <vector>

#include "libdescriptor_b200.h"

namespace ldb {

// ---------------------------------------------------------------- errors
void set_error(const std::string &msg);
int fail(int code, const std::string &msg);
int cuda_fail(cudaError_t e, const char *what);

#define LDB_CUDA(expr)                                          \
    do {                                                        \
        cudaError_t _e = (expr);                                \
        if (_e != cudaSuccess) return ::ldb::cuda_fail(_e, #expr); \
    } while (0)

// Device-side error word: kernels raise a status with atomicCAS (first one
// wins) and the host reads it through ld_sync_status.
enum DeviceStatus : int {
    kDevOk = 0,
    kDevCapacity = 1,   // a row exceeded max_neigh
    kDevBadIndex = 2,   // neighbour / centre index outside coords
    kDevTimeout = 3,    // a bounded wait on an asynchronous copy ran out
};

// NVTX range over a scope (header-only NVTX 3: inert unless a profiler such
// as Nsight Systems or ncu's range filter is attached).
struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange &) = delete;
    NvtxRange &operator=(const NvtxRange &) = delete;
};

// Launch accounting (all kernels of the library).
void count_launch(int n = 1);
// Allocation accounting: every device allocation of the library (grow-only
// buffers, the stream-ordered scratch pool) calls this first; it returns
// LD_ERR_OOM when ld_fail_next_allocation armed a failure for this one.
int count_alloc();
// The byte new allocations are filled with (ld_debug_fill_scratch), or -1.
int scratch_fill();
// The device a descriptor handle was created on.
int handle_device(const ld_descriptor *d);

// ------------------------------------------------------------- device buf
struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    int ensure(size_t n);   // grow-only
    void release();
    template <class T> T *as() const { return static_cast<T *>(p); }
    ~DevBuf() { release(); }
};

// ------------------------------------------------------ symmetry functions
// Device view of the parameter tables (outputs re-ordered for the kernel:
// two-body outputs, then three-body outputs sorted by (type, eta) so that
// consecutive outputs can share one exp()).
// Factored form of a symmetry-function parameter set whose three-body
// outputs of each type (g4, g5) lie on a grid of at most kSFGA angular terms
// (lambda, zeta) x kSFGR radial terms (eta), with at most kSFG2 two-body
// outputs.  Passed by value to the kernels (constant bank), so parameter
// reads cost no memory instructions.
constexpr int kSFGA = 4;
constexpr int kSFGR = 4;
constexpr int kSFG2 = 16;
struct SFGrid {
    int n2 = 0;
    int t2[kSFG2] = {}, o2[kSFG2] = {};
    double a2[kSFG2] = {}, b2[kSFG2] = {};
    int na[2] = {0, 0}, nr[2] = {0, 0};            // [0]: g4, [1]: g5
    double lam[2][kSFGA] = {}, zeta[2][kSFGA] = {}, P[2][kSFGA] = {};
    int zi[2][kSFGA] = {};                          // integer zeta or -1
    double eta[2][kSFGR] = {};                      // ascending
    int ec[2][kSFGR] = {};                          // r > 0: k >= 2 -> E_0^k, else exp
    int out[2][kSFGA][kSFGR] = {};                  // output index, -1: empty cell
};

struct SFDev {
    int ns = 0, width = 0;
    int n2 = 0, n3 = 0;
    const double *rcut = nullptr;   // ns*ns
    const double *ircut = nullptr;  // ns*ns, 1 / rcut
    const int *o2 = nullptr;        // output index
    const int *t2 = nullptr;        // 1..3
    const double *a2 = nullptr;     // eta (g2) / kappa (g3)
    const double *b2 = nullptr;     // Rs (g2)
    const int *o3 = nullptr;        // output index
    const int *t3 = nullptr;        // 4 / 5
    const double *P3 = nullptr;     // 2^(1-zeta)
    const double *z3 = nullptr;     // zeta
    const double *l3 = nullptr;     // lambda
    const double *e3 = nullptr;     // eta
    const int *zi3 = nullptr;       // integer zeta (>=0) or -1
    // exp reuse per three-body output: -1 same factor as the previous output,
    // 0 evaluate exp(-eta S) (the first output of a type group sets the
    // group base), k >= 2 the group base raised to the k-th power (eta is
    // k times the group's smallest eta)
    const int *ec3 = nullptr;
    bool has_grid = false;
    SFGrid grid;
    // hyperparameter gradients: per output its type code (1..5), the offset
    // of its first parameter in the caller's flat parameter vector, and its
    // parameters (g2: eta, Rs; g3: kappa; g4/g5: zeta, lambda, eta) at
    // pv[3 * output]
    int nparams = 0;
    const int *pt = nullptr;
    const int *pofs = nullptr;
    const double *pv = nullptr;
};

// ------------------------------------------------------------- bispectrum
struct BSDev {
    int J = 0, style = 3, switch_flag = 1, bzero_flag = 0, ns = 0;
    int ncoeff = 0, nU = 0, nL = 0, ntrip = 0, nZall = 0, ncg = 0;
    double rfac0 = 0, rmin0 = 0, wself = 1.0;
    const double *rcut_flat = nullptr;  // per neighbour species (reference quirk)
    const double *ang_flat = nullptr;   // per neighbour species: rfac0 pi / (rc - rmin0)
    const double *isw_flat = nullptr;   // per neighbour species: 1 / (rc - rmin0)
    const double *wj = nullptr;         // per species weight
    const double *bzero = nullptr;      // J+1
    const double *rootpq = nullptr;     // (J+1)^2, [p*(J+1)+q] = sqrt(p/q)
    const int *ublock = nullptr;        // J+2: full-matrix layer offsets
    const int *lblock = nullptr;        // J+2: left-half layer offsets
    const int4 *trip = nullptr;         // (j1, j2, j, zoff)
    const int *cgoff = nullptr;         // per triple
    const double *cg = nullptr;
    // CG blocks packed by anti-diagonal m1 + m2 (the entries with a valid
    // output index only) for the tiled Z: entry (m1, output m) of triple t is
    // cgp[dbase[tri_off(t) + m] + m1]
    int ncgp = 0;
    const double *cgp = nullptr;
    const int *dbase = nullptr;
    const int *otrip = nullptr;         // per output: triple index
    const int *moff = nullptr;          // per triple CSR into (mo, mcoef)
    const int *mo = nullptr;
    const double *mcoef = nullptr;
    const int *jtoff = nullptr;         // J+2: triples with third index j
    const int *jtlist = nullptr;
    const int *lel = nullptr;           // nL: packed (j, ma, mb) of left element
    const int *toff_f = nullptr;        // NT+1 per-thread task offsets (forward)
    const int4 *task_f = nullptr;
    const int *toff_v = nullptr;        // NT+1 (gradient: all needed triples)
    const int4 *task_v = nullptr;
    // schedules of the twojmax-specialised per-centre kernel (nt2 threads):
    // Z tiles packed as x = j1 | j2 << 8 | j << 16 | a0 << 24,
    // y = b0 | rows << 8 | cols << 16, z = Z offset of the triple,
    // w = the triple's first entry in dbase
    int nt2 = 0;
    const int *toff2_f = nullptr;
    const int4 *task2_f = nullptr;
    const int *toff2_v = nullptr;
    const int4 *task2_v = nullptr;
    // rows-in-lanes Z kernel (kZWarps warps, one row per lane): items
    // (j | ma << 8), one output row of layer j each, scheduled per warp
    // (zoff: kZWarps+1); the triples of layer j are ztl[ztoff[j] ..
    // ztoff[j+1]) packed as x = j1 | j2 << 8 | c << 16 (c = (j1+j2-j)/2),
    // y = offset of its column weights in zg, z = cgoff of the triple,
    // w = triple index | (descriptor slot + 1) << 16 (slot -1: no output);
    // oslot maps an output to its slot
    int nbslot = 0;
    const int *oslot = nullptr;
    // per triple: its column weights by window step, G[mb][q] = cg(c + q -
    // mb, mb) (zero outside the triple's range), q padded to even, at zg +
    // the triple's ztl y field
    const double *zg = nullptr;
    int nzg = 0;
    const int *zoff_f = nullptr, *zitem_f = nullptr, *ztoff_f = nullptr;
    const int4 *ztl_f = nullptr;
    const int *zoff_v = nullptr, *zitem_v = nullptr, *ztoff_v = nullptr;
    const int4 *ztl_v = nullptr;
};

constexpr int kBSThreads = 128;   // threads per bispectrum CTA (one centre)
constexpr int kSFThreads = 128;   // threads per symmetry-function CTA (4 centres)
constexpr int kMaxTwoJ = 10;

// ----------------------------------------------------------- launch args
struct RowArgs {
    int n_rows = 0;
    const int *row_centre = nullptr;   // nullable: centre == row
    const int *row_list = nullptr;     // nullable: neighbour row == row
    const int *species = nullptr;
    const int *nbl = nullptr;
    const long long *off = nullptr;
    int max_neigh = 0;
    const double *coords = nullptr;
    int n_total = 0;                   // 0 = unknown (no index check)
    double *desc = nullptr;            // nullable for gradient
    const double *dE = nullptr;        // nullptr = forward only
    double *dcoords = nullptr;
    double *d_rfac0 = nullptr;         // bispectrum: dL/d rfac0 added here when set (pair kernel)
    long long dc_stride = 0;           // doubles between rows' gradients (0 = shared)
    const int *image = nullptr;
    int *status = nullptr;             // device error word
    bool fused_only = false;           // gradient in one kernel, no work space (no allocation)
    // ragged batches: start of each row's neighbours in nbl (nullable: off[row]);
    // off[] then only numbers the rows' neighbours consecutively
    const long long *nbl_begin = nullptr;
    // launch shape (0 = automatic); set through ld_set_tuning
    int sf_warps = 0;                  // warps (centre rows) per symmetry-function CTA: 1, 2, 4
    int ctas_per_sm = 0;               // per-centre bispectrum CTAs per SM
    int pair_grid_mult = 0;            // pair-parallel gradient grid = SMs x occupancy x this
    int dynamic_queue = 0;
    bool force_generic = false;        // symmetry functions: table-driven kernel even when a grid exists
    // host API overlap (nullable): the launches wait for in_ready before the
    // first kernel that reads dE, and record desc_done once the descriptors
    // are final (the bispectrum's pair-gradient kernel then still runs)
    cudaEvent_t in_ready = nullptr;
    cudaEvent_t desc_done = nullptr;
    // caller-provided device work space (nullable: stream-ordered allocation)
    void *work = nullptr;
    size_t work_bytes = 0;             // 1: rows claimed from an atomic counter instead of grid stride
};

// Z tiles of the twojmax-specialised per-centre kernel: one thread computes
// kZTileA x kZTileB output elements (rows ma x columns mb) of one triple
#ifndef LD_ZTILE_A
#define LD_ZTILE_A 2
#endif
#ifndef LD_ZTILE_B
#define LD_ZTILE_B 2
#endif
constexpr int kZTileA = LD_ZTILE_A;
constexpr int kZTileB = LD_ZTILE_B;

// warps of the rows-in-lanes Z kernel's CTA (32 rows per CTA)
#ifndef LD_ZWARPS
#define LD_ZWARPS 16
#endif
constexpr int kZWarps = LD_ZWARPS;
// shared memory of the rows-in-lanes Z kernel: the 32 rows' full U
// ([element][lane], 512 bytes per element) between zero guards of J+1
// elements before and J/2+1 after (reads just outside a row land there or
// in other elements of the lane, always finite, and meet a zero weight),
// then the descriptor sums [lane][slot]
inline size_t bs_smemZ_bytes(const BSDev &p, bool with_g = false) {
    return (size_t)(p.J + 1 + p.nU + p.J / 2 + 1) * 32 * 16 + (size_t)32 * (p.nbslot > 0 ? p.nbslot : 1) * 8 +
           (with_g ? (size_t)p.nzg * 8 + (size_t)p.ntrip * 32 * 8 : 0);
}
// The twojmax-specialised path runs U (per centre), Z/B/Y (rows in lanes)
// and the pair gradient as three kernels (the split form) where its Z kernel
// fits one SM's shared memory; otherwise (2J = 10) the per-centre kernel
// computes U, Z, B and Y together.  The column weights and the rows' betaj
// join the U block in shared memory when they fit too.
inline bool bs_split(const BSDev &p) { return bs_smemZ_bytes(p) <= 227 * 1024; }
inline bool bs_split_gshared(const BSDev &p) { return bs_smemZ_bytes(p, true) <= 227 * 1024; }

// warps of the twojmax-specialised per-centre bispectrum CTA (4..8): enough
// neighbour slots for about 32 neighbours in one round
#ifndef LD_BS2_WARPS
#define LD_BS2_WARPS 0
#endif
constexpr int bs2_warps(int J) {
    return LD_BS2_WARPS > 0 ? LD_BS2_WARPS
           : (32 + 32 / (J / 2 + 1) - 1) / (32 / (J / 2 + 1)) < 4 ? 4
           : (32 + 32 / (J / 2 + 1) - 1) / (32 / (J / 2 + 1)) > 8 ? 8
                                                                  : (32 + 32 / (J / 2 + 1) - 1) / (32 / (J / 2 + 1));
}

int sf_launch(const SFDev &p, const RowArgs &a, cudaStream_t s);
int sf_param_launch(const SFDev &p, const RowArgs &a, double *d_params, cudaStream_t s);
int sfg_launch(const SFDev &p, const RowArgs &a, cudaStream_t s);
int bs_launch(const BSDev &p, const RowArgs &a, cudaStream_t s);
size_t sf_work_bytes(const SFDev &p, int n_rows, bool vjp);
size_t bs_work_bytes(const BSDev &p, int n_rows, bool vjp);
size_t bs_smem_bytes(const BSDev &p, int max_neigh, bool vjp);

int offsets_launch(int n_rows, const int *counts, long long *off, int *maxn,
                   void *tmp, size_t tmp_bytes, cudaStream_t s);
size_t offsets_tmp_bytes(int n_rows);
// Stream-ordered scratch (free it with cudaFreeAsync) from a memory pool the
// library owns on each device.  The pool keeps what is freed (no release
// threshold), so calls that need scratch again reuse it instead of going back
// to the driver; it holds up to the largest scratch any call has needed.
int pool_alloc(void **p, size_t bytes, cudaStream_t s);

}  // namespace ldb
