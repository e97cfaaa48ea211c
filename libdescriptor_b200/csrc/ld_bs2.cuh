// ld_bs2.cuh -- bispectrum kernels specialised on twojmax ("column lanes").
//
// The Cayley-Klein / VMK recursion u(j,ma,mb) = -rq(ma,j-mb) conj(b) u(j-1,ma-1,mb)
// + rq(j-ma,j-mb) conj(a) u(j-1,ma,mb) (src/Bispectrum.cpp:490-554) only
// couples entries of ONE column mb across layers.  Here a lane owns one
// column of one neighbour and keeps it in registers for all layers: the
// update runs in place from the bottom row up, with compile-time indices
// (twojmax is a template parameter), so the recursion costs no shared-memory
// traffic.  A column mb enters the left half at layer j = 2 mb; its previous
// layer is then the inversion-symmetry image of column mb-1, fetched once
// from the neighbouring lane with a shuffle.  The middle column of an even
// layer gets the reference's copy step: centre conjugated, rows below it
// mirrored.  NC = J/2+1 lanes serve one neighbour ("slot"); a warp holds
// 32/NC slots.
//
// bsA_kernel<J, VJP, UOUT>  one CTA per centre: stage neighbours, U (column
//                     lanes, slots reduced through a per-warp buffer), Z (LPT
//                     task lists), B; for the gradient also Y = sum betaj Z ->
//                     HBM.  UOUT (the split form's first kernel at 2J = 9):
//                     U only, written as full U blocks [row / 32][element][row % 32].
// bsZ_kernel<J, VJP, GSH>  split form: one CTA per 32 rows, a row per lane;
//                     warp-uniform Z by rotating register windows over the
//                     rows' U in shared memory, B, and Y = sum betaj Z -> HBM.
// bsU_kernel<J>       split form's U for 2J <= 8: one warp per centre, slots of
//                     column lanes over the neighbours, each column's sums over
//                     all layers in registers, one slot reduction per centre.
// bsR_kernel<J>       pair-parallel gradient, reverse mode: one slot per
//                     (centre, neighbour) pair runs the column recursion
//                     forward (layer inputs kept in shared memory) and then
//                     carries dPhi/du backward to dPhi/da, dPhi/db; chained to
//                     the position with the Cayley-Klein derivatives, FP64
//                     atomics onto the neighbour and the centre.
#pragma once

#include "ld_internal.h"

namespace ldb {
namespace bs2 {

constexpr double kPi = 3.1415926535897932;

__host__ __device__ constexpr int ncols(int J) { return J / 2 + 1; }
__host__ __device__ constexpr int slots_per_warp(int J) { return 32 / ncols(J); }
// left-half layer offset: sum_{j'<j} (j'+1)(j'/2+1)
__host__ __device__ constexpr int lblock(int j) { return j <= 0 ? 0 : lblock(j - 1) + j * ((j - 1) / 2 + 1); }
// warps of the per-centre CTA: enough slots for ~32 neighbours, 4..8 warps
__host__ __device__ constexpr int warpsA(int J) { return bs2_warps(J); }

__device__ __forceinline__ void raise_status(int *status, int code) {
    if (status) atomicCAS(status, 0, code);
}

__device__ __forceinline__ double sfac_of(const BSDev &p, double r, double rc) {
    if (p.switch_flag == 0) return 1.0;
    if (p.switch_flag == 1) {
        if (r <= p.rmin0) return 1.0;
        if (r > rc) return 0.0;
        return 0.5 * (cospi((r - p.rmin0) / (rc - p.rmin0)) + 1.0);
    }
    return 0.0;
}
// the switching function and its derivative together (one sincospi of
// (r - rmin0) * isw, isw = 1 / (rc - rmin0) from the per-species table)
__device__ __forceinline__ void sfac_both(const BSDev &p, double r, double rc, double isw, double &sf,
                                          double &dsf) {
    sf = p.switch_flag == 0 ? 1.0 : 0.0;
    dsf = 0.0;
    if (p.switch_flag == 1) {
        if (r <= p.rmin0) {
            sf = 1.0;
        } else if (!(r > rc)) {
            const double inv = isw;
            double sn, cs;
            sincospi((r - p.rmin0) * inv, &sn, &cs);
            sf = 0.5 * (cs + 1.0);
            dsf = -0.5 * sn * (kPi * inv);
        }
    }
}
__device__ __forceinline__ double dsfac_of(const BSDev &p, double r, double rc) {
    if (p.switch_flag == 1) {
        if (r <= p.rmin0 || r > rc) return 0.0;
        const double f = kPi / (rc - p.rmin0);
        return -0.5 * sin((r - p.rmin0) * f) * f;
    }
    return 0.0;
}

// Cayley-Klein parameters of one neighbour (x, y, z relative to the centre)
// and, with TAN, their derivatives w.r.t. x, y, z.
struct CK {
    double ar, ai, br, bi;
    double dar[3], dai[3], dbr[3], dbi[3];
};

// with c0 = rfac0 pi / (rc - rmin0) given (the per-species table ang_flat)
template <bool TAN>
__device__ __forceinline__ void cayley_klein_c0(double rmin0, double x, double y, double z, double r, double c0,
                                                CK &c) {
    // theta0 = (r - rmin0) c0, z0 = r / tan(theta0) = r cos / sin: one
    // sincos and one reciprocal serve the parameters and their tangents
    const double theta0 = (r - rmin0) * c0;
    double sth, cth;
    sincos(theta0, &sth, &cth);
    const double isth = 1.0 / sth;
    const double z0 = r * cth * isth;
    const double r0inv = rsqrt(r * r + z0 * z0);
    c.ar = r0inv * z0;
    c.ai = -r0inv * z;
    c.br = r0inv * y;
    c.bi = -r0inv * x;
    if (TAN) {
        const double dz0 = cth * isth - r * c0 * isth * isth;
        const double dr0inv = -r0inv * r0inv * r0inv * (r + z0 * dz0);
        const double rinv = 1.0 / r;
        const double u3[3] = {x * rinv, y * rinv, z * rinv};
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            c.dar[d] = (dz0 * r0inv + z0 * dr0inv) * u3[d];
            c.dai[d] = -(z * dr0inv * u3[d] + (d == 2 ? r0inv : 0.0));
            c.dbr[d] = y * dr0inv * u3[d] + (d == 1 ? r0inv : 0.0);
            c.dbi[d] = -(x * dr0inv * u3[d] + (d == 0 ? r0inv : 0.0));
        }
    }
}

template <bool TAN>
__device__ __forceinline__ void cayley_klein(const BSDev &p, double x, double y, double z, double r, double rc,
                                             CK &c) {
    cayley_klein_c0<TAN>(p.rmin0, x, y, z, r, p.rfac0 * kPi / (rc - p.rmin0), c);
}

// One layer j of the column recursion for this lane's column mb (in place).
// ur/ui[D] hold the column's rows; with TAN also dr/di[3][D].  rq points at
// the rootpq table shifted by -mb so rq[p*D + (j)] = sqrt(p / (j - mb)).
template <int J, int j, bool TAN>
__device__ __forceinline__ void column_layer(int mb, const double *rq, const CK &c, double (&ur)[J + 1],
                                             double (&ui)[J + 1], double (&dr)[TAN ? 3 : 1][J + 1],
                                             double (&di)[TAN ? 3 : 1][J + 1]) {
    constexpr int D = J + 1;
    constexpr int hj = j / 2;
    constexpr bool even = (j % 2) == 0;
    if (even) {
        // birth of column hj: previous layer = mirror of column hj-1 (lane - 1)
#pragma unroll
        for (int m = 0; m < j; ++m) {
            const double s = ((m - hj) & 1) ? -1.0 : 1.0;
            const double tr = __shfl_up_sync(0xffffffffu, ur[j - 1 - m], 1);
            const double ti = __shfl_up_sync(0xffffffffu, ui[j - 1 - m], 1);
            double tdr[3] = {0, 0, 0}, tdi[3] = {0, 0, 0};
            if (TAN) {
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    tdr[d] = __shfl_up_sync(0xffffffffu, dr[TAN ? d : 0][j - 1 - m], 1);
                    tdi[d] = __shfl_up_sync(0xffffffffu, di[TAN ? d : 0][j - 1 - m], 1);
                }
            }
            if (mb == hj) {
                ur[m] = s * tr;
                ui[m] = -s * ti;
                if (TAN) {
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        dr[TAN ? d : 0][m] = s * tdr[d];
                        di[TAN ? d : 0][m] = -s * tdi[d];
                    }
                }
            }
        }
    }
    if (2 * mb <= j) {
#pragma unroll
        for (int ma = j; ma >= 0; --ma) {
            double nr = 0.0, ni = 0.0;
            double ndr[3] = {0, 0, 0}, ndi[3] = {0, 0, 0};
            if (ma >= 1) {
                const double q = -rq[ma * D + j];
                const double pr = ur[ma - 1], pi = ui[ma - 1];
                nr = q * (c.br * pr + c.bi * pi);
                ni = q * (c.br * pi - c.bi * pr);
                if (TAN) {
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        const double wr = dr[TAN ? d : 0][ma - 1], wi = di[TAN ? d : 0][ma - 1];
                        ndr[d] = q * (c.dbr[d] * pr + c.dbi[d] * pi + c.br * wr + c.bi * wi);
                        ndi[d] = q * (c.dbr[d] * pi - c.dbi[d] * pr + c.br * wi - c.bi * wr);
                    }
                }
            }
            if (ma < j) {
                const double q = rq[(j - ma) * D + j];
                const double pr = ur[ma], pi = ui[ma];
                nr += q * (c.ar * pr + c.ai * pi);
                ni += q * (c.ar * pi - c.ai * pr);
                if (TAN) {
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        const double wr = dr[TAN ? d : 0][ma], wi = di[TAN ? d : 0][ma];
                        ndr[d] += q * (c.dar[d] * pr + c.dai[d] * pi + c.ar * wr + c.ai * wi);
                        ndi[d] += q * (c.dar[d] * pi - c.dai[d] * pr + c.ar * wi - c.ai * wr);
                    }
                }
            }
            ur[ma] = nr;
            ui[ma] = ni;
            if (TAN) {
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    dr[TAN ? d : 0][ma] = ndr[d];
                    di[TAN ? d : 0][ma] = ndi[d];
                }
            }
        }
        if (even && mb == hj) {
            // the reference's inversion-symmetry copy on the middle column:
            // centre conjugated, rows below the centre mirrored from above
            ui[hj] = -ui[hj];
            if (TAN) {
#pragma unroll
                for (int d = 0; d < 3; ++d) di[TAN ? d : 0][hj] = -di[TAN ? d : 0][hj];
            }
#pragma unroll
            for (int ma = hj + 1; ma <= j; ++ma) {
                const double s = ((ma - hj) & 1) ? -1.0 : 1.0;
                ur[ma] = s * ur[j - ma];
                ui[ma] = -s * ui[j - ma];
                if (TAN) {
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        dr[TAN ? d : 0][ma] = s * dr[TAN ? d : 0][j - ma];
                        di[TAN ? d : 0][ma] = -s * di[TAN ? d : 0][j - ma];
                    }
                }
            }
        }
    }
}

// compile-time loop over layers 1..J
template <int J, int j, bool TAN, class F>
struct Layers {
    __device__ __forceinline__ static void run(int mb, const double *rq, const CK &c, double (&ur)[J + 1],
                                               double (&ui)[J + 1], double (&dr)[TAN ? 3 : 1][J + 1],
                                               double (&di)[TAN ? 3 : 1][J + 1], F &f) {
        column_layer<J, j, TAN>(mb, rq, c, ur, ui, dr, di);
        f.template after<j>(mb, ur, ui, dr, di);
        Layers<J, j + 1, TAN, F>::run(mb, rq, c, ur, ui, dr, di, f);
    }
};
template <int J, bool TAN, class F>
struct Layers<J, J + 1, TAN, F> {
    __device__ __forceinline__ static void run(int, const double *, const CK &, double (&)[J + 1],
                                               double (&)[J + 1], double (&)[TAN ? 3 : 1][J + 1],
                                               double (&)[TAN ? 3 : 1][J + 1], F &) {}
};

}  // namespace bs2

template <int J>
int bs2_launch_t(const BSDev &p, const RowArgs &a, cudaStream_t s);

}  // namespace ldb
