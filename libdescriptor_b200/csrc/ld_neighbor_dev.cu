// ld_neighbor_dev.cu -- the neighbour builder on the device.
//
// Same ghosts (order, coordinates, species, image) and the same neighbour
// lists (order included) as the host builder in ld_neighbor.cpp, i.e. as the
// reference's nbl_create_paddings / nbl_build
// (python_bindings/neighbor/neighbor_list.cpp:78-243, 283-418): every product
// and sum is rounded separately (__dmul_rn / __dadd_rn, no fused multiply-add)
// in the host's evaluation order, so the cutoff and binning decisions agree
// bit for bit.
//
// Paddings: one flag per (image shell, atom), an exclusive scan gives each
// ghost its position in the reference's order (shells outer, atoms inner).
// Neighbour list: atoms binned into cells of side >= cutoff over the
// bounding box, sorted by cell with a stable radix sort (so a cell lists its
// atoms in index order), then one thread per query atom walks the 27 cells
// in the reference's order, twice: counts, then (after a scan) the list.
#include <cub/cub.cuh>

#include <string>
#include <vector>

#include "ld_internal.h"
#include "ld_neighbor_math.h"

namespace ldb {
namespace {

constexpr double kTol = 1.0e-10;

__device__ __forceinline__ double dot3(const double *m, double x, double y, double z) {
    return __dadd_rn(__dadd_rn(__dmul_rn(m[0], x), __dmul_rn(m[1], y)), __dmul_rn(m[2], z));
}

struct Mat9 {
    double v[9];
};

// fractional coordinates and their per-direction extrema (one block)
__global__ void frac_bounds(int n, const double *__restrict__ x, Mat9 fcell, double *__restrict__ frac,
                            double *__restrict__ bounds) {
    __shared__ double s_lo[3][32], s_hi[3][32];
    double lo[3] = {1e10, 1e10, 1e10}, hi[3] = {-1e10, -1e10, -1e10};
    for (int a = threadIdx.x; a < n; a += blockDim.x) {
        const double px = x[3 * a], py = x[3 * a + 1], pz = x[3 * a + 2];
        for (int d = 0; d < 3; ++d) {
            const double f = dot3(fcell.v + 3 * d, px, py, pz);
            frac[3 * a + d] = f;
            lo[d] = f < lo[d] ? f : lo[d];
            hi[d] = f > hi[d] ? f : hi[d];
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int d = 0; d < 3; ++d) {
        for (int o = 16; o > 0; o >>= 1) {
            const double l = __shfl_xor_sync(0xffffffffu, lo[d], o), h = __shfl_xor_sync(0xffffffffu, hi[d], o);
            lo[d] = l < lo[d] ? l : lo[d];
            hi[d] = h > hi[d] ? h : hi[d];
        }
        if (lane == 0) {
            s_lo[d][warp] = lo[d];
            s_hi[d][warp] = hi[d];
        }
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        const int d = threadIdx.x;
        double l = 1e10, h = -1e10;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            l = s_lo[d][w] < l ? s_lo[d][w] : l;
            h = s_hi[d][w] > h ? s_hi[d][w] : h;
        }
        bounds[d] = __dadd_rn(l, -kTol);
        bounds[3 + d] = __dadd_rn(h, kTol);
    }
}

struct PadShells {
    int size[3];
    double slack[3];
};

__device__ __forceinline__ bool keep_ghost(const int3 sh, const double *f, const double *bounds, const PadShells &g) {
    const double *lo = bounds, *hi = bounds + 3;
    const int c[3] = {sh.x, sh.y, sh.z};
    for (int d = 0; d < 3; ++d) {
        if (c[d] == -g.size[d] && __dadd_rn(f[d], -lo[d]) < g.slack[d]) return false;
        if (c[d] == g.size[d] && __dadd_rn(hi[d], -f[d]) < g.slack[d]) return false;
    }
    return true;
}

__global__ void pad_flags(int n, int n_shell, const int3 *__restrict__ shells, const double *__restrict__ frac,
                          const double *__restrict__ bounds, PadShells g, int *__restrict__ flags) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)n * n_shell) return;
    const int s = (int)(t / n), a = (int)(t - (long long)s * n);
    flags[t] = keep_ghost(shells[s], frac + 3 * a, bounds, g) ? 1 : 0;
}

__global__ void pad_write(int n, int n_shell, const int3 *__restrict__ shells, const double *__restrict__ frac,
                          const int *__restrict__ flags, const int *__restrict__ pos, Mat9 tcell,
                          const int *__restrict__ species, double *__restrict__ pc, int *__restrict__ ps,
                          int *__restrict__ pi) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)n * n_shell || !flags[t]) return;
    const int s = (int)(t / n), a = (int)(t - (long long)s * n);
    const int3 sh = shells[s];
    const double f0 = __dadd_rn((double)sh.x, frac[3 * a]), f1 = __dadd_rn((double)sh.y, frac[3 * a + 1]),
                 f2 = __dadd_rn((double)sh.z, frac[3 * a + 2]);
    const int o = pos[t];
    if (pc) {
        pc[3 * o] = dot3(tcell.v, f0, f1, f2);
        pc[3 * o + 1] = dot3(tcell.v + 3, f0, f1, f2);
        pc[3 * o + 2] = dot3(tcell.v + 6, f0, f1, f2);
    }
    if (ps) ps[o] = species[a];
    if (pi) pi[o] = a;
}

// bounding box as the reference's nbl_build starts it: lo = x0,
// hi = x0 + 1, then min / max over all atoms (one block)
__global__ void box_bounds(int n, const double *__restrict__ x, double *__restrict__ bounds) {
    __shared__ double s_lo[3][32], s_hi[3][32];
    double lo[3] = {x[0], x[1], x[2]};
    double hi[3] = {__dadd_rn(x[0], 1.0), __dadd_rn(x[1], 1.0), __dadd_rn(x[2], 1.0)};
    for (int a = threadIdx.x; a < n; a += blockDim.x)
        for (int d = 0; d < 3; ++d) {
            const double v = x[3 * a + d];
            lo[d] = v < lo[d] ? v : lo[d];
            hi[d] = v > hi[d] ? v : hi[d];
        }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int d = 0; d < 3; ++d) {
        for (int o = 16; o > 0; o >>= 1) {
            const double l = __shfl_xor_sync(0xffffffffu, lo[d], o), h = __shfl_xor_sync(0xffffffffu, hi[d], o);
            lo[d] = l < lo[d] ? l : lo[d];
            hi[d] = h > hi[d] ? h : hi[d];
        }
        if (lane == 0) {
            s_lo[d][warp] = lo[d];
            s_hi[d][warp] = hi[d];
        }
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        const int d = threadIdx.x;
        double l = s_lo[d][0], h = s_hi[d][0];
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
            l = s_lo[d][w] < l ? s_lo[d][w] : l;
            h = s_hi[d][w] > h ? s_hi[d][w] : h;
        }
        bounds[d] = l;
        bounds[3 + d] = h;
    }
}

struct Grid {
    int size[3];
    double lo[3], hi[3];
};

__device__ __forceinline__ void bin_of(double px, double py, double pz, const Grid &g, int *ix) {
    const double p[3] = {px, py, pz};
    for (int d = 0; d < 3; ++d) {
        const double t = __dmul_rn(__ddiv_rn(__dadd_rn(p[d], -g.lo[d]), __dadd_rn(g.hi[d], -g.lo[d])),
                                   (double)g.size[d]);
        int v = (int)t;
        ix[d] = v > g.size[d] - 1 ? g.size[d] - 1 : v;
    }
}

__global__ void cell_keys(int n, const double *__restrict__ x, Grid g, int *__restrict__ key, int *__restrict__ val,
                          int *__restrict__ cnt) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= n) return;
    int ix[3];
    bin_of(x[3 * a], x[3 * a + 1], x[3 * a + 2], g, ix);
    const int c = ix[0] + ix[1] * g.size[0] + ix[2] * g.size[0] * g.size[1];
    key[a] = c;
    val[a] = a;
    atomicAdd(cnt + c, 1);
}

// FILL = false: count the neighbours of every query atom; true: write them
template <bool FILL>
__global__ void walk_cells(int n_query, const int *__restrict__ need, const double *__restrict__ x, Grid g,
                           double cutsq, const int *__restrict__ cell_start, const int *__restrict__ cell_atoms,
                           int *__restrict__ counts, const long long *__restrict__ off, int *__restrict__ nbl,
                           int *__restrict__ status) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= n_query) return;
    if (!need[a]) {
        if (!FILL) counts[a] = 0;
        return;
    }
    const double px = x[3 * a], py = x[3 * a + 1], pz = x[3 * a + 2];
    int ix[3];
    bin_of(px, py, pz, g, ix);
    int cnt = 0;
    long long w = FILL ? off[a] : 0;
    for (int ii = max(0, ix[0] - 1); ii <= min(ix[0] + 1, g.size[0] - 1); ++ii)
        for (int jj = max(0, ix[1] - 1); jj <= min(ix[1] + 1, g.size[1] - 1); ++jj)
            for (int kk = max(0, ix[2] - 1); kk <= min(ix[2] + 1, g.size[2] - 1); ++kk) {
                const int c = ii + jj * g.size[0] + kk * g.size[0] * g.size[1];
                for (int q = cell_start[c]; q < cell_start[c + 1]; ++q) {
                    const int b = cell_atoms[q];
                    if (b == a) continue;
                    const double dx = __dadd_rn(x[3 * b], -px), dy = __dadd_rn(x[3 * b + 1], -py),
                                 dz = __dadd_rn(x[3 * b + 2], -pz);
                    const double rsq = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
                    if (rsq < kTol) {
                        if (status) atomicCAS(status, 0, 1);
                        continue;
                    }
                    if (rsq < cutsq) {
                        if (FILL) nbl[w++] = b;
                        ++cnt;
                    }
                }
            }
    if (!FILL) counts[a] = cnt;
}

// stream-ordered scratch, freed when the call returns
struct Scratch {
    cudaStream_t s;
    std::vector<void *> ptrs;
    explicit Scratch(cudaStream_t st) : s(st) {}
    template <class T>
    int get(T **p, size_t count) {
        void *q = nullptr;
        const int rc = pool_alloc(&q, (count ? count : 1) * sizeof(T), s);
        if (rc) return rc;
        ptrs.push_back(q);
        *p = static_cast<T *>(q);
        return LD_OK;
    }
    ~Scratch() {
        for (void *q : ptrs) cudaFreeAsync(q, s);
    }
};

template <class T>
int read_back(T *host, const T *dev, size_t count, cudaStream_t s) {
    LDB_CUDA(cudaMemcpyAsync(host, dev, count * sizeof(T), cudaMemcpyDeviceToHost, s));
    LDB_CUDA(cudaStreamSynchronize(s));
    return LD_OK;
}

}  // namespace
}  // namespace ldb

extern "C" int ld_create_paddings_dev(double cutoff, const double *cell, const int *pbc, const double *coords,
                                      const int *species, int n_atoms, int max_pad, double *pad_coords,
                                      int *pad_species, int *pad_image, int *n_pad, ld_stream stream) {
    using namespace ldb;
    if (!cell || !pbc || !n_pad || n_atoms < 0 || max_pad < 0 || (n_atoms > 0 && (!coords || !species)))
        return fail(LD_ERR_INVALID_ARG, "ld_create_paddings_dev: bad arguments");
    ldnb::PadGeom geo;
    if (!ldnb::pad_geometry(cutoff, cell, geo))
        return fail(LD_ERR_INVALID_ARG, "In inverting the cell matrix, the determinant is 0!");
    *n_pad = 0;
    if (n_atoms == 0) return LD_OK;
    std::vector<int3> shells;
    for (int i = -geo.size[0]; i <= geo.size[0]; ++i)
        for (int j = -geo.size[1]; j <= geo.size[1]; ++j)
            for (int k = -geo.size[2]; k <= geo.size[2]; ++k) {
                if (i == 0 && j == 0 && k == 0) continue;
                if ((pbc[0] == 0 && i != 0) || (pbc[1] == 0 && j != 0) || (pbc[2] == 0 && k != 0)) continue;
                shells.push_back(make_int3(i, j, k));
            }
    const int ns = (int)shells.size();
    if (ns == 0) return LD_OK;
    const long long total = (long long)ns * n_atoms;
    if (total >= (1LL << 31)) return fail(LD_ERR_CAPACITY, "ld_create_paddings_dev: too many image candidates");
    cudaStream_t s = (cudaStream_t)stream;
    Scratch sc(s);
    int3 *d_sh = nullptr;
    double *frac = nullptr, *bounds = nullptr;
    int *flags = nullptr, *pos = nullptr;
    void *tmp = nullptr;
    size_t tb = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tb, (int *)nullptr, (int *)nullptr, (int)total);
    int rc;
    if ((rc = sc.get(&d_sh, ns)) || (rc = sc.get(&frac, 3 * (size_t)n_atoms)) || (rc = sc.get(&bounds, 6)) ||
        (rc = sc.get(&flags, total)) || (rc = sc.get(&pos, total)) || (rc = sc.get((char **)&tmp, tb)))
        return rc;
    LDB_CUDA(cudaMemcpyAsync(d_sh, shells.data(), sizeof(int3) * ns, cudaMemcpyHostToDevice, s));
    Mat9 fc, tc;
    for (int k = 0; k < 9; ++k) {
        fc.v[k] = geo.fcell[k];
        tc.v[k] = geo.tcell[k];
    }
    frac_bounds<<<1, 1024, 0, s>>>(n_atoms, coords, fc, frac, bounds);
    count_launch();
    PadShells g;
    for (int d = 0; d < 3; ++d) {
        g.size[d] = geo.size[d];
        g.slack[d] = geo.slack[d];
    }
    const int bs = 256;
    const unsigned nb = (unsigned)((total + bs - 1) / bs);
    pad_flags<<<nb, bs, 0, s>>>(n_atoms, ns, d_sh, frac, bounds, g, flags);
    count_launch();
    LDB_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tb, flags, pos, (int)total, s));
    count_launch();
    int last[2] = {0, 0};
    if ((rc = read_back(&last[0], pos + total - 1, 1, s)) || (rc = read_back(&last[1], flags + total - 1, 1, s)))
        return rc;
    const int m = last[0] + last[1];
    *n_pad = m;
    if (!pad_coords && !pad_species && !pad_image) return LD_OK;   // count only
    if (m > max_pad)
        return fail(LD_ERR_CAPACITY, "ld_create_paddings_dev: " + std::to_string(m) + " ghosts > max_pad " +
                                         std::to_string(max_pad));
    pad_write<<<nb, bs, 0, s>>>(n_atoms, ns, d_sh, frac, flags, pos, tc, species, pad_coords, pad_species, pad_image);
    count_launch();
    LDB_CUDA(cudaGetLastError());
    LDB_CUDA(cudaStreamSynchronize(s));
    return LD_OK;
}

extern "C" int ld_build_neighbor_list_dev(const double *coords, int n_total, double cutoff, const int *need_neigh,
                                          int n_query, int *number_of_neighs, long long *neigh_offsets,
                                          long long max_nnz, int *neighbor_list, long long *nnz, int *max_neigh,
                                          ld_stream stream) {
    using namespace ldb;
    if (n_total < 0 || n_query < 0 || n_query > n_total || !nnz || max_nnz < 0 || !(cutoff > 0) ||
        (n_total > 0 && (!coords || !need_neigh)) || (n_query > 0 && (!number_of_neighs || !neigh_offsets)))
        return fail(LD_ERR_INVALID_ARG, "ld_build_neighbor_list_dev: bad arguments");
    cudaStream_t s = (cudaStream_t)stream;
    *nnz = 0;
    if (max_neigh) *max_neigh = 0;
    if (n_query == 0) {
        if (neigh_offsets) LDB_CUDA(cudaMemsetAsync(neigh_offsets, 0, sizeof(long long), s));
        return LD_OK;
    }
    Scratch sc(s);
    double *bounds = nullptr;
    int rc;
    if ((rc = sc.get(&bounds, 6))) return rc;
    box_bounds<<<1, 1024, 0, s>>>(n_total, coords, bounds);
    count_launch();
    double hb[6];
    if ((rc = read_back(hb, bounds, 6, s))) return rc;
    Grid g;
    long long cells = 1;
    for (int d = 0; d < 3; ++d) {
        g.lo[d] = hb[d];
        g.hi[d] = hb[3 + d];
        int sz = (int)((g.hi[d] - g.lo[d]) / cutoff);
        g.size[d] = sz <= 0 ? 1 : sz;
        cells *= g.size[d];
    }
    if (cells > (1LL << 28)) return fail(LD_ERR_INVALID_ARG, "Cell size too large! (particles fly away)");
    int *key = nullptr, *val = nullptr, *key2 = nullptr, *atoms = nullptr, *cnt = nullptr, *start = nullptr,
        *status = nullptr;
    void *tmp = nullptr;
    size_t tb_sort = 0, tb_scan = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tb_sort, (int *)nullptr, (int *)nullptr, (int *)nullptr, (int *)nullptr,
                                    n_total);
    cub::DeviceScan::ExclusiveSum(nullptr, tb_scan, (int *)nullptr, (int *)nullptr, (int)cells + 1);
    const size_t tb = tb_sort > tb_scan ? tb_sort : tb_scan;
    if ((rc = sc.get(&key, n_total)) || (rc = sc.get(&val, n_total)) || (rc = sc.get(&key2, n_total)) ||
        (rc = sc.get(&atoms, n_total)) || (rc = sc.get(&cnt, cells + 1)) || (rc = sc.get(&start, cells + 1)) ||
        (rc = sc.get(&status, 1)) || (rc = sc.get((char **)&tmp, tb)))
        return rc;
    LDB_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int) * (cells + 1), s));
    LDB_CUDA(cudaMemsetAsync(status, 0, sizeof(int), s));
    const int bs = 256;
    cell_keys<<<(n_total + bs - 1) / bs, bs, 0, s>>>(n_total, coords, g, key, val, cnt);
    count_launch();
    size_t t1 = tb;
    int end_bit = 1;
    while ((1LL << end_bit) < cells) ++end_bit;
    LDB_CUDA(cub::DeviceRadixSort::SortPairs(tmp, t1, key, key2, val, atoms, n_total, 0, end_bit, s));
    count_launch();
    size_t t2 = tb;
    LDB_CUDA(cub::DeviceScan::ExclusiveSum(tmp, t2, cnt, start, (int)cells + 1, s));
    count_launch();
    const double cutsq = cutoff * cutoff;
    walk_cells<false><<<(n_query + bs - 1) / bs, bs, 0, s>>>(n_query, need_neigh, coords, g, cutsq, start, atoms,
                                                            number_of_neighs, nullptr, nullptr, status);
    count_launch();
    int *d_max = nullptr;
    const size_t otb = offsets_tmp_bytes(n_query);
    void *otmp = nullptr;
    if ((rc = sc.get(&d_max, 1)) || (rc = sc.get((char **)&otmp, otb))) return rc;
    if ((rc = offsets_launch(n_query, number_of_neighs, neigh_offsets, d_max, otmp, otb, s))) return rc;
    long long total = 0;
    int st = 0, mx = 0;
    if ((rc = read_back(&total, neigh_offsets + n_query, 1, s)) || (rc = read_back(&st, status, 1, s)) ||
        (rc = read_back(&mx, d_max, 1, s)))
        return rc;
    if (st) return fail(LD_ERR_INVALID_ARG, "Collision of atoms (two atoms closer than 1e-5)");
    *nnz = total;
    if (max_neigh) *max_neigh = mx;
    if (!neighbor_list) return LD_OK;   // counts and offsets only
    if (total > max_nnz)
        return fail(LD_ERR_CAPACITY, "ld_build_neighbor_list_dev: " + std::to_string(total) +
                                         " neighbours > max_nnz " + std::to_string(max_nnz));
    walk_cells<true><<<(n_query + bs - 1) / bs, bs, 0, s>>>(n_query, need_neigh, coords, g, cutsq, start, atoms,
                                                           number_of_neighs, neigh_offsets, neighbor_list, nullptr);
    count_launch();
    LDB_CUDA(cudaGetLastError());
    LDB_CUDA(cudaStreamSynchronize(s));
    return LD_OK;
}
