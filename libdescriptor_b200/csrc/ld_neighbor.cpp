// ld_neighbor.cpp -- host neighbour lists: periodic ghost padding and a
// cell-list full neighbour list, as used to prepare descriptor inputs.
//
// Behaviour (and therefore the exact ghost ordering and neighbour order)
// follows the reference's KLIFF-derived builder,
// python_bindings/neighbor/neighbor_list.cpp: nbl_create_paddings (:283-418)
// and nbl_build (:78-243) with helper.hpp's vector/matrix helpers.  The same
// arithmetic order is kept so ghost coordinates and lists come out
// identical, which makes the descriptor inputs bit-identical too.
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "ld_internal.h"
#include "ld_neighbor_math.h"

namespace {

using namespace ldnb;
constexpr double kTol = 1.0e-10;

int paddings(double cutoff, const double *cell, const int *pbc, const double *x, const int *species, int n,
             std::vector<double> &pc, std::vector<int> &ps, std::vector<int> &pi) {
    PadGeom g;
    if (!pad_geometry(cutoff, cell, g))
        return ldb::fail(LD_ERR_INVALID_ARG, "In inverting the cell matrix, the determinant is 0!");
    const double *tcell = g.tcell, *fcell = g.fcell;
    std::vector<double> frac((size_t)3 * n);
    double lo[3] = {1e10, 1e10, 1e10}, hi[3] = {-1e10, -1e10, -1e10};
    for (int a = 0; a < n; ++a) {
        const double *p = x + 3 * a;
        const double f0 = vdot(fcell, p), f1 = vdot(fcell + 3, p), f2 = vdot(fcell + 6, p);
        frac[3 * a] = f0;
        frac[3 * a + 1] = f1;
        frac[3 * a + 2] = f2;
        const double f[3] = {f0, f1, f2};
        for (int d = 0; d < 3; ++d) {
            if (f[d] < lo[d]) lo[d] = f[d];
            if (f[d] > hi[d]) hi[d] = f[d];
        }
    }
    for (int d = 0; d < 3; ++d) {
        lo[d] -= kTol;
        hi[d] += kTol;
    }
    const int *size = g.size;
    const double *slack = g.slack;
    for (int i = -size[0]; i <= size[0]; ++i)
        for (int j = -size[1]; j <= size[1]; ++j)
            for (int k = -size[2]; k <= size[2]; ++k) {
                if (i == 0 && j == 0 && k == 0) continue;
                if ((pbc[0] == 0 && i != 0) || (pbc[1] == 0 && j != 0) || (pbc[2] == 0 && k != 0)) continue;
                for (int a = 0; a < n; ++a) {
                    const double fx = frac[3 * a], fy = frac[3 * a + 1], fz = frac[3 * a + 2];
                    // outermost image shells only keep atoms within reach
                    if (i == -size[0] && fx - lo[0] < slack[0]) continue;
                    if (i == size[0] && hi[0] - fx < slack[0]) continue;
                    if (j == -size[1] && fy - lo[1] < slack[1]) continue;
                    if (j == size[1] && hi[1] - fy < slack[1]) continue;
                    if (k == -size[2] && fz - lo[2] < slack[2]) continue;
                    if (k == size[2] && hi[2] - fz < slack[2]) continue;
                    const double f[3] = {i + fx, j + fy, k + fz};
                    pc.push_back(vdot(tcell, f));
                    pc.push_back(vdot(tcell + 3, f));
                    pc.push_back(vdot(tcell + 6, f));
                    ps.push_back(species[a]);
                    pi.push_back(a);
                }
            }
    return LD_OK;
}

inline void bin_of(const double *p, const int *size, const double *hi, const double *lo, int *idx) {
    for (int d = 0; d < 3; ++d) {
        idx[d] = (int)(((p[d] - lo[d]) / (hi[d] - lo[d])) * size[d]);
        if (idx[d] > size[d] - 1) idx[d] = size[d] - 1;
    }
}

int build(const double *x, int n, double cutoff, const int *need, int n_query, std::vector<int> &counts,
          std::vector<int> &flat) {
    if (n <= 0) {
        counts.assign(n_query > 0 ? n_query : 0, 0);
        return LD_OK;
    }
    double lo[3] = {x[0], x[1], x[2]};
    double hi[3] = {x[0] + 1.0, x[1] + 1.0, x[2] + 1.0};
    for (int a = 0; a < n; ++a)
        for (int d = 0; d < 3; ++d) {
            if (hi[d] < x[3 * a + d]) hi[d] = x[3 * a + d];
            if (lo[d] > x[3 * a + d]) lo[d] = x[3 * a + d];
        }
    int size[3];
    for (int d = 0; d < 3; ++d) {
        size[d] = (int)((hi[d] - lo[d]) / cutoff);
        if (size[d] <= 0) size[d] = 1;
    }
    const long long total = (long long)size[0] * size[1] * size[2];
    if (total > 1000000000LL)
        return ldb::fail(LD_ERR_INVALID_ARG, "Cell size too large! (particles fly away)");
    std::vector<std::vector<int>> cells((size_t)total);
    for (int a = 0; a < n; ++a) {
        int ix[3];
        bin_of(x + 3 * a, size, hi, lo, ix);
        cells[(size_t)ix[0] + (size_t)ix[1] * size[0] + (size_t)ix[2] * size[0] * size[1]].push_back(a);
    }
    const double cutsq = cutoff * cutoff;
    counts.assign(n_query, 0);
    flat.clear();
    for (int a = 0; a < n && a < n_query; ++a) {
        if (!need[a]) continue;
        const double px = x[3 * a], py = x[3 * a + 1], pz = x[3 * a + 2];
        int ix[3];
        bin_of(x + 3 * a, size, hi, lo, ix);
        int cnt = 0;
        for (int ii = std::max(0, ix[0] - 1); ii <= std::min(ix[0] + 1, size[0] - 1); ++ii)
            for (int jj = std::max(0, ix[1] - 1); jj <= std::min(ix[1] + 1, size[1] - 1); ++jj)
                for (int kk = std::max(0, ix[2] - 1); kk <= std::min(ix[2] + 1, size[2] - 1); ++kk) {
                    const auto &c = cells[(size_t)ii + (size_t)jj * size[0] + (size_t)kk * size[0] * size[1]];
                    for (int b : c) {
                        if (b == a) continue;
                        const double dx = x[3 * b] - px, dy = x[3 * b + 1] - py, dz = x[3 * b + 2] - pz;
                        const double rsq = dx * dx + dy * dy + dz * dz;
                        if (rsq < kTol)
                            return ldb::fail(LD_ERR_INVALID_ARG, "Collision of atoms " + std::to_string(a + 1) +
                                                                     " and " + std::to_string(b + 1));
                        if (rsq < cutsq) {
                            flat.push_back(b);
                            ++cnt;
                        }
                    }
                }
        counts[a] = cnt;
    }
    return LD_OK;
}

}  // namespace

extern "C" int ld_create_paddings(double cutoff, const double *cell, const int *pbc, const double *coords,
                                  const int *species, int n_atoms, int *n_pad, double *pad_coords,
                                  int *pad_species, int *pad_image) {
    if (!cell || !pbc || !n_pad || n_atoms < 0 || (n_atoms > 0 && (!coords || !species)))
        return ldb::fail(LD_ERR_INVALID_ARG, "ld_create_paddings: bad arguments");
    std::vector<double> pc;
    std::vector<int> ps, pi;
    int rc = paddings(cutoff, cell, pbc, coords, species, n_atoms, pc, ps, pi);
    if (rc) return rc;
    const int m = (int)pi.size();
    if (pad_coords || pad_species || pad_image) {
        if (*n_pad < m) return ldb::fail(LD_ERR_INVALID_ARG, "ld_create_paddings: output buffers too small");
        if (pad_coords && m) std::memcpy(pad_coords, pc.data(), sizeof(double) * pc.size());
        if (pad_species && m) std::memcpy(pad_species, ps.data(), sizeof(int) * m);
        if (pad_image && m) std::memcpy(pad_image, pi.data(), sizeof(int) * m);
    }
    *n_pad = m;
    return LD_OK;
}

extern "C" int ld_build_neighbor_list(const double *coords, int n_total, double cutoff, const int *need_neigh,
                                      int n_query, int *number_of_neighs, int *neighbor_list, long long *nnz) {
    if (n_total < 0 || n_query < 0 || n_query > n_total || !nnz || (n_total > 0 && (!coords || !need_neigh)) ||
        (n_query > 0 && !number_of_neighs) || !(cutoff > 0))
        return ldb::fail(LD_ERR_INVALID_ARG, "ld_build_neighbor_list: bad arguments");
    std::vector<int> counts, flat;
    int rc = build(coords, n_total, cutoff, need_neigh, n_query, counts, flat);
    if (rc) return rc;
    if (n_query) std::memcpy(number_of_neighs, counts.data(), sizeof(int) * n_query);
    if (neighbor_list) {
        if (*nnz < (long long)flat.size()) return ldb::fail(LD_ERR_INVALID_ARG, "ld_build_neighbor_list: neighbor_list too small");
        if (!flat.empty()) std::memcpy(neighbor_list, flat.data(), sizeof(int) * flat.size());
    }
    *nnz = (long long)flat.size();
    return LD_OK;
}
