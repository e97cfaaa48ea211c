// ld_sfg.cu -- symmetry functions with a factored three-body parameter set.
//
// Same semantics as sf_kernel (SymmetryFunctions::compute,
// src/SymmetryFunctions.cpp:141-259: g4 = 2^(1-zeta) sum (1 + lambda cos)^zeta
// exp(-eta (r_ij^2 + r_ik^2 + r_jk^2)) fc fc fc, g5 without the r_jk terms).
// When the three-body outputs of each type lie on a grid of angular terms
// (lambda, zeta) x radial terms (eta) -- the usual Behler sets, e.g. 2 zeta x
// 2 lambda x 4 eta -- a triplet needs only one power per angular term and one
// exponential (or integer power of it) per radial term:
//   acc(a, r) += cp_a * E_r * F,   output = 2^(1-zeta_a) * acc(a, r),
// and the gradient's per-type sums A = sum g P cp E, B = sum g P cp eta E,
// C = sum g P lambda dcp E factor the same way through
//   s_a = sum_r gP(a, r) E_r,  t_a = sum_r gP(a, r) eta_r E_r.
// Every parameter is a compile-time-indexed member of the by-value SFGrid,
// so it is read from the constant bank; the upstream gradient of the row is
// read once per centre into registers.
#include "ld_sf_common.cuh"

namespace ldb {
namespace {
using namespace sfc;

constexpr int NA = kSFGA, NR = kSFGR;
#ifndef LD_SFG_MINB
#define LD_SFG_MINB 4
#endif
// the row's gP(a, r) = dL/dG * 2^(1-zeta) live at the end of the warp's
// shared slice (warp-uniform reads) instead of in registers
constexpr int kGPExtra = 2 * NA * NR;
// radial terms of a triplet: E0 = exp(-eta_0 S) once, its squarings
// E0^(2^k) once, and each integer multiple eta_r = k eta_0 (k < 2^kSFGPowBits)
// as a balanced product of the squarings its bits select: a dependent chain
// of 7 squarings + 3 products, shared by all radial terms (binary powering
// per term ran 3% slower on the 24-d set, one exp per term 1.5% slower)
constexpr int kSFGPowBits = 8;

// Paths the usual parameter sets never take (non-integer zeta, an eta that
// is not an integer multiple of its group's smallest, cosine radial terms)
// are kept out of line: with hundreds of rows per warp the warps of an SM
// drift into different phases of the kernel, and the hot code must then fit
// the instruction cache.
__device__ __noinline__ double exp_cold(double x) { return exp(x); }
__device__ __noinline__ double pow_cold(double b, double z) { return pow(b, z); }
__device__ __noinline__ void sincos_cold(double x, double *s, double *c) { sincos(x, s, c); }

// PH: 0 both sums, 2 the two-body sums only, 3 the three-body sums only
// (large batches run 2 then 3, see launch_g)
template <bool VJP, bool HAS4, bool HAS5, int PH = 0>
__global__ void __launch_bounds__(kSFThreads, VJP ? LD_SFG_MINB : 4)
sfg_kernel(const __grid_constant__ SFDev p, RowArgs a, int per_warp, int *queue) {
    extern __shared__ double smem[];
    const SFGrid &g = p.grid;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int nw = blockDim.x >> 5;
    const int cap = a.max_neigh;
    WarpSlice S = slice(smem + (size_t)warp * per_warp, cap, VJP);
    const int width = p.width;

    int row = blockIdx.x * nw + warp;
    if (queue) {
        int r0 = 0;
        if (lane == 0) r0 = atomicAdd(queue, 1);
        row = __shfl_sync(0xffffffffu, r0, 0);
    }
    RowMeta nxt{};
    if (row < a.n_rows) {
        nxt = row_meta(a, row);
        csr_prefetch(a, nxt, cap, S.nbl);
    }
    for (; row < a.n_rows;) {
        const RowMeta m = nxt;
        const int i = m.i, n = m.n;
        const int cur_row = row;
        if (queue) {
            int r1 = 0;
            if (lane == 0) r1 = atomicAdd(queue, 1);
            row = __shfl_sync(0xffffffffu, r1, 0);
        } else {
            row += gridDim.x * nw;
        }
        // the next row's list metadata, loaded now and used once this row's
        // segment has left the slice
        if (row < a.n_rows) nxt = row_meta(a, row);
        double *const dco = VJP ? a.dcoords + (size_t)cur_row * a.dc_stride : nullptr;
        csr_wait();
        if (n > cap || n < 0 || (a.n_total > 0 && (i < 0 || i >= a.n_total))) {
            raise_status(a.status, n > cap ? kDevCapacity : kDevBadIndex);
            if (a.desc)
                for (int q = lane; q < width; q += 32)
                    a.desc[(size_t)cur_row * width + q] = __longlong_as_double(0x7ff8000000000000LL);
            if (row < a.n_rows) csr_prefetch(a, nxt, cap, S.nbl);
            continue;
        }
        const double cix = a.coords[3 * i], ciy = a.coords[3 * i + 1], ciz = a.coords[3 * i + 2];
        const int is = a.species[i];
        // ---- stage the neighbours of this row (list from the slice)
        for (int jj = lane; jj < n; jj += 32) {
            int j = S.nbl[jj];
            int ok = 1;
            if (a.n_total > 0 && (j < 0 || j >= a.n_total)) {
                raise_status(a.status, kDevBadIndex);
                j = i;
                ok = 0;
            }
            const int js = a.species[j];
            const double x = a.coords[3 * j], y = a.coords[3 * j + 1], z = a.coords[3 * j + 2];
            const double rx = x - cix, ry = y - ciy, rz = z - ciz;
            const double r = sqrt(rx * rx + ry * ry + rz * rz);
            const double rc = p.rcut[is * p.ns + js], irc = p.ircut[is * p.ns + js];
            S.cx[jj] = x;
            S.cy[jj] = y;
            S.cz[jj] = z;
            S.r[jj] = r;
            S.ir[jj] = 1.0 / r;
            S.rc[jj] = rc;
            S.spec[jj] = js;
            S.idx[jj] = ok ? j : -1;
            S.inc[jj] = ok && !(r > rc);
            if (VJP) {
                double fc, dfc;
                cutc_both(r, rc, irc, fc, dfc);
                S.fc[jj] = fc;
                S.dfc[jj] = dfc;
                S.gx[jj] = 0.0;
                S.gy[jj] = 0.0;
                S.gz[jj] = 0.0;
            } else {
                S.fc[jj] = cutc_i(r, rc, irc);
            }
        }
        __syncwarp();
        if (row < a.n_rows) csr_prefetch(a, nxt, cap, S.nbl);
        const double *dE = VJP ? a.dE + (size_t)cur_row * width : nullptr;
        double gix = 0.0, giy = 0.0, giz = 0.0;
        // ---- two-body terms
        if (PH != 3 && g.n2 > 0) {
            double acc2[kSFG2];
#pragma unroll
            for (int q = 0; q < kSFG2; ++q) acc2[q] = 0.0;
            double g2[kSFG2];
            if (VJP) {
#pragma unroll
                for (int q = 0; q < kSFG2; ++q) g2[q] = q < g.n2 ? __ldg(dE + g.o2[q]) : 0.0;
            }
            for (int jj = lane; jj < n; jj += 32) {
                if (!S.inc[jj]) continue;
                const double r = S.r[jj], fc = S.fc[jj];
                const double dfc = VJP ? S.dfc[jj] : 0.0;
                double dsum = 0.0;
#pragma unroll
                for (int q = 0; q < kSFG2; ++q) {
                    if (q < g.n2) {
                        const int t = g.t2[q];
                        const double pa = g.a2[q], pb = g.b2[q];
                        double v, dv = 0.0;
                        if (t == 1) {
                            v = fc;
                            if (VJP) dv = dfc;
                        } else if (t == 2) {
                            const double e = exp(-pa * (r - pb) * (r - pb));
                            v = e * fc;
                            if (VJP) dv = e * (-2.0 * pa * (r - pb) * fc + dfc);
                        } else {
                            double sn, cs;
                            sincos_cold(pa * r, &sn, &cs);
                            v = cs * fc;
                            if (VJP) dv = -pa * sn * fc + cs * dfc;
                        }
                        acc2[q] += v;
                        if (VJP) dsum += g2[q] * dv;
                    }
                }
                if (VJP) {
                    const double inv = S.ir[jj];
                    const double gx = dsum * (S.cx[jj] - cix) * inv;
                    const double gy = dsum * (S.cy[jj] - ciy) * inv;
                    const double gz = dsum * (S.cz[jj] - ciz) * inv;
                    S.gx[jj] += gx;
                    S.gy[jj] += gy;
                    S.gz[jj] += gz;
                    gix -= gx;
                    giy -= gy;
                    giz -= gz;
                }
            }
#pragma unroll
            for (int q = 0; q < kSFG2; ++q) {
                if (q < g.n2) {
                    const double v = warp_sum(acc2[q]);
                    if (lane == 0 && a.desc) a.desc[(size_t)cur_row * width + g.o2[q]] = v;
                }
            }
        }
        // ---- three-body terms
        if (PH != 2 && (HAS4 || HAS5)) {
            constexpr int NT = 2;
            double acc[NT][NA][NR];
            double(*gP)[NA][NR] = reinterpret_cast<double(*)[NA][NR]>(smem + (size_t)warp * per_warp + per_warp - kGPExtra);
#pragma unroll
            for (int ty = 0; ty < NT; ++ty)
#pragma unroll
                for (int x = 0; x < NA; ++x)
#pragma unroll
                    for (int y = 0; y < NR; ++y) {
                        const bool on = (ty == 0 ? HAS4 : HAS5);
                        acc[ty][x][y] = 0.0;
                        double v = 0.0;
                        if (VJP && on && g.out[ty][x][y] >= 0) v = __ldg(dE + g.out[ty][x][y]) * g.P[ty][x];
                        // the slice has room for gP only in the gradient kernel
                        if (VJP && lane == 0) gP[ty][x][y] = v;
                    }
            if (VJP) __syncwarp();
            // Lane l owns neighbours jj = l, l + 32, ...; at step dd it takes the
            // triplet (jj, kk = (jj + dd) mod n), dd = 1 .. n/2 (the last step,
            // for even n, only for jj < n/2): every unordered pair once, and
            // within a step the lanes' kk are distinct, so the kk gradients are
            // plain read-modify-writes (steps ordered by __syncwarp) and the jj
            // gradient stays in registers.
            const int dmax = (n - 1) / 2, dlast = n / 2;
            for (int m0 = 0; m0 < n; m0 += 32) {
              const int jj = m0 + lane;
              const bool own = jj < n;
              const int jjs = own ? jj : 0;
              const bool incj = own && S.inc[jjs];
              const int js = S.spec[jjs];
              const double cxj = S.cx[jjs], cyj = S.cy[jjs], czj = S.cz[jjs];
              const double av = S.r[jjs], ia = S.ir[jjs], fa = S.fc[jjs];
              const double dfa = VJP ? S.dfc[jjs] : 0.0;
              double gjx = 0.0, gjy = 0.0, gjz = 0.0;
              for (int dd = 1; dd <= dlast; ++dd) {
                int kk = jj + dd;
                if (kk >= n) kk -= n;
                if (incj && (dd <= dmax || jj < dlast) && S.inc[kk]) {
                    const int ks = S.spec[kk];
                    const double rcjk = p.rcut[js * p.ns + ks], ircjk = p.ircut[js * p.ns + ks];
                    const double jkx = S.cx[kk] - cxj, jky = S.cy[kk] - cyj, jkz = S.cz[kk] - czj;
                    const double d = sqrt(jkx * jkx + jky * jky + jkz * jkz);
                    const double b = S.r[kk];
                    const double ib = S.ir[kk];
                    const double asq = av * av, bsq = b * b, dsq = d * d;
                    const double cth = (asq + bsq - dsq) * (0.5 * ia * ib);
                    const double fb = S.fc[kk];
                    double fd = 0.0, dfd = 0.0;
                    if (HAS4) {
                        if (VJP)
                            cutc_both(d, rcjk, ircjk, fd, dfd);
                        else
                            fd = cutc_i(d, rcjk, ircjk);
                    }
                    const bool g4ok = !(d > rcjk);
                    double Aq[NT] = {0.0, 0.0}, Bq[NT] = {0.0, 0.0}, Cq[NT] = {0.0, 0.0};
                    double Fq[NT];
                    Fq[0] = fa * fb * fd;
                    Fq[1] = fa * fb;
#pragma unroll
                    for (int ty = 0; ty < NT; ++ty) {
                        if (!(ty == 0 ? HAS4 : HAS5)) continue;
                        if (ty == 0 && !g4ok) continue;
                        const double Ssum = ty == 0 ? asq + bsq + dsq : asq + bsq;
                        // radial terms: one exp for the smallest eta; its
                        // squarings E0^(2^k) once, then each integer multiple
                        // as a balanced product of the squarings its bits
                        // select (dependent chain: 7 squarings + 3 products)
                        double E[NR];
                        {
                            double P[kSFGPowBits];
                            P[0] = exp(-g.eta[ty][0] * Ssum);
#pragma unroll
                            for (int k = 1; k < kSFGPowBits; ++k) P[k] = P[k - 1] * P[k - 1];
                            E[0] = g.nr[ty] > 0 ? P[0] : 0.0;
#pragma unroll
                            for (int y = 1; y < NR; ++y) {
                                E[y] = 0.0;
                                if (y < g.nr[ty]) {
                                    const int ec = g.ec[ty][y];
                                    if (ec >= 2 && ec < (1 << kSFGPowBits)) {
                                        double m[kSFGPowBits];
#pragma unroll
                                        for (int k = 0; k < kSFGPowBits; ++k) m[k] = (ec >> k) & 1 ? P[k] : 1.0;
#pragma unroll
                                        for (int w = 1; w < kSFGPowBits; w *= 2)
#pragma unroll
                                            for (int k = 0; k + w < kSFGPowBits; k += 2 * w) m[k] *= m[k + w];
                                        E[y] = m[0];
                                    } else {
                                        E[y] = exp_cold(-g.eta[ty][y] * Ssum);
                                    }
                                }
                            }
                        }
                        // angular terms
                        double cp[NA], dcp[NA];
#pragma unroll
                        for (int x = 0; x < NA; ++x) {
                            cp[x] = 0.0;
                            dcp[x] = 0.0;
                            if (x < g.na[ty]) {
                                const double base = 1.0 + g.lam[ty][x] * cth;
                                if (base > 0) {
                                    const int zi = g.zi[ty][x];
                                    if (zi == 1) {
                                        cp[x] = base;
                                        dcp[x] = 1.0;
                                    } else if (zi == 2) {
                                        cp[x] = base * base;
                                        dcp[x] = 2.0 * base;
                                    } else if (zi == 4) {
                                        const double b2 = base * base;
                                        cp[x] = b2 * b2;
                                        dcp[x] = 4.0 * b2 * base;
                                    } else if (zi >= 0) {
                                        cp[x] = ipow(base, zi);
                                        dcp[x] = zi > 0 ? g.zeta[ty][x] * ipow(base, zi - 1) : 0.0;
                                    } else {
                                        cp[x] = pow_cold(base, g.zeta[ty][x]);
                                        dcp[x] = g.zeta[ty][x] * pow_cold(base, g.zeta[ty][x] - 1.0);
                                    }
                                }
                            }
                        }
                        const double F = Fq[ty];
#pragma unroll
                        for (int y = 0; y < NR; ++y) {
                            const double W = E[y] * F;
#pragma unroll
                            for (int x = 0; x < NA; ++x) acc[ty][x][y] = fma(cp[x], W, acc[ty][x][y]);
                        }
                        if (VJP) {
                            double Ee[NR];
#pragma unroll
                            for (int y = 0; y < NR; ++y) Ee[y] = g.eta[ty][y] * E[y];
#pragma unroll
                            for (int x = 0; x < NA; ++x) {
                                double sa = 0.0, ta = 0.0;
#pragma unroll
                                for (int y = 0; y < NR; ++y) {
                                    sa = fma(gP[ty][x][y], E[y], sa);
                                    ta = fma(gP[ty][x][y], Ee[y], ta);
                                }
                                Aq[ty] = fma(cp[x], sa, Aq[ty]);
                                Bq[ty] = fma(cp[x], ta, Bq[ty]);
                                Cq[ty] = fma(g.lam[ty][x] * dcp[x], sa, Cq[ty]);
                            }
                        }
                    }
                    if (VJP) {
                        const double F4 = Fq[0], F5 = Fq[1];
                        const double A4 = Aq[0], B4 = Bq[0], C4 = Cq[0], A5 = Aq[1], B5 = Bq[1], C5 = Cq[1];
                        const double dfb = S.dfc[kk];
                        const double dca = (asq - bsq + dsq) * (0.5 * ia * ia * ib);
                        const double dcb = (bsq - asq + dsq) * (0.5 * ia * ib * ib);
                        const double dcd = -d * ia * ib;
                        const double Ga = F4 * C4 * dca - 2.0 * av * F4 * B4 + dfa * fb * fd * A4 +
                                          F5 * C5 * dca - 2.0 * av * F5 * B5 + dfa * fb * A5;
                        const double Gb = F4 * C4 * dcb - 2.0 * b * F4 * B4 + fa * dfb * fd * A4 +
                                          F5 * C5 * dcb - 2.0 * b * F5 * B5 + fa * dfb * A5;
                        const double Gd = F4 * C4 * dcd - 2.0 * d * F4 * B4 + fa * fb * dfd * A4 + F5 * C5 * dcd;
                        const double id = d > 0 ? rsqrt(dsq) : 0.0;
                        const double ijx = (cxj - cix) * ia, ijy = (cyj - ciy) * ia, ijz = (czj - ciz) * ia;
                        const double ukx = (S.cx[kk] - cix) * ib, uky = (S.cy[kk] - ciy) * ib,
                                     ukz = (S.cz[kk] - ciz) * ib;
                        const double udx = jkx * id, udy = jky * id, udz = jkz * id;
                        gjx += Ga * ijx - Gd * udx;
                        gjy += Ga * ijy - Gd * udy;
                        gjz += Ga * ijz - Gd * udz;
                        S.gx[kk] += Gb * ukx + Gd * udx;
                        S.gy[kk] += Gb * uky + Gd * udy;
                        S.gz[kk] += Gb * ukz + Gd * udz;
                        gix -= Ga * ijx + Gb * ukx;
                        giy -= Ga * ijy + Gb * uky;
                        giz -= Ga * ijz + Gb * ukz;
                    }
                }
                __syncwarp();
              }
              if (VJP && own) {
                  S.gx[jj] += gjx;
                  S.gy[jj] += gjy;
                  S.gz[jj] += gjz;
              }
              __syncwarp();
            }
#pragma unroll
            for (int ty = 0; ty < NT; ++ty)
#pragma unroll
                for (int x = 0; x < NA; ++x)
#pragma unroll
                    for (int y = 0; y < NR; ++y) {
                        if ((ty == 0 ? HAS4 : HAS5) && g.out[ty][x][y] >= 0) {
                            const double v = warp_sum(acc[ty][x][y]) * g.P[ty][x];
                            if (lane == 0 && a.desc) a.desc[(size_t)cur_row * width + g.out[ty][x][y]] = v;
                        }
                    }
        }
        if (VJP) {
            __syncwarp();
            for (int jj = lane; jj < n; jj += 32) {
                const int j = S.idx[jj];
                if (j < 0) continue;
                const int tj = a.image ? a.image[j] : j;
                atomicAdd(dco + 3 * (size_t)tj, S.gx[jj]);
                atomicAdd(dco + 3 * (size_t)tj + 1, S.gy[jj]);
                atomicAdd(dco + 3 * (size_t)tj + 2, S.gz[jj]);
            }
            gix = warp_sum(gix);
            giy = warp_sum(giy);
            giz = warp_sum(giz);
            if (lane == 0) {
                const int ti = a.image ? a.image[i] : i;
                atomicAdd(dco + 3 * (size_t)ti, gix);
                atomicAdd(dco + 3 * (size_t)ti + 1, giy);
                atomicAdd(dco + 3 * (size_t)ti + 2, giz);
            }
        }
        __syncwarp();
    }
}

// Batches of at least this many rows run the two-body and the three-body
// sums as two launches: with hundreds of rows per warp the warps of an SM
// drift into different phases of the kernel, and a launch that holds one
// phase keeps its hot code in the instruction cache (the rows' neighbours
// are staged twice; 0 disables the split)
#ifndef LD_SFG_SPLIT_ROWS
#define LD_SFG_SPLIT_ROWS 8192
#endif
template <bool VJP, bool H4, bool H5>
int launch_g(const SFDev &p, const RowArgs &a, cudaStream_t s) {
    if (LD_SFG_SPLIT_ROWS > 0 && a.n_rows >= LD_SFG_SPLIT_ROWS && p.grid.n2 > 0 && (H4 || H5)) {
        int rc = launch_rows_kernel(sfg_kernel<VJP, H4, H5, 2>, p, a, s, VJP, "sfg_kernel", VJP ? kGPExtra : 0);
        if (rc) return rc;
        return launch_rows_kernel(sfg_kernel<VJP, H4, H5, 3>, p, a, s, VJP, "sfg_kernel", VJP ? kGPExtra : 0);
    }
    return launch_rows_kernel(sfg_kernel<VJP, H4, H5>, p, a, s, VJP, "sfg_kernel", VJP ? kGPExtra : 0);
}

template <bool VJP>
int launch_vjp(const SFDev &p, const RowArgs &a, cudaStream_t s) {
    const bool h4 = p.grid.na[0] > 0, h5 = p.grid.na[1] > 0;
    if (h4 && h5) return launch_g<VJP, true, true>(p, a, s);
    if (h4) return launch_g<VJP, true, false>(p, a, s);
    if (h5) return launch_g<VJP, false, true>(p, a, s);
    return launch_g<VJP, false, false>(p, a, s);
}

}  // namespace

int sfg_launch(const SFDev &p, const RowArgs &a, cudaStream_t s) {
    if (a.n_rows <= 0) return LD_OK;
    return a.dE ? launch_vjp<true>(p, a, s) : launch_vjp<false>(p, a, s);
}

}  // namespace ldb
