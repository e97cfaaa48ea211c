// ld_sf.cu -- Behler symmetry functions on sm_100a: forward and fused
// forward + VJP.
//
// Semantics follow SymmetryFunctions::compute (src/SymmetryFunctions.cpp:
// 141-259) and sym_g1..g5 / cut_cos (:67-139): pair terms for every
// neighbour with r_ij <= rc_ij, triplet terms for kk > jj with r_ik <= rc_ik,
// g4 additionally zero when r_jk > rc_jk, base <= 0 -> 0.
//
// Mapping: one warp owns one centre row.  The row's neighbours (absolute
// coordinates, distance, cutoff function, species, index) are staged once in
// the warp's slice of shared memory; lanes then stride over pairs and over
// the flattened upper triangle of (jj, kk) triplets.  Per-output sums live in
// registers (one accumulator per output and lane) and are reduced with warp
// shuffles.  Three-body outputs are pre-sorted by (type, eta) on the host so
// consecutive outputs reuse one exp().  The gradient kernel recomputes every
// term, folds the upstream dL/dG into three scalar sums per triplet and
// type, assembles d/dr_j, d/dr_k, d/dr_i from them, accumulates neighbour
// gradients in shared memory and scatters them with FP64 atomics (optionally
// straight onto the ghost's master row).
#include "ld_sf_common.cuh"

namespace ldb {
namespace {
using namespace sfc;

// PH: 0 both sums, 2 the two-body sums only, 3 the three-body sums only
// (large batches run 2 then 3, see launch_t)
template <bool VJP, int M2, int M3, int PH = 0>
__global__ void __launch_bounds__(kSFThreads, VJP ? 3 : 4)
sf_kernel(SFDev p, RowArgs a, int per_warp_doubles, int *queue) {
    extern __shared__ double smem[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int nw = blockDim.x >> 5;
    const int cap = a.max_neigh;
    WarpSlice S = slice(smem + (size_t)warp * per_warp_doubles, cap, VJP);
    const int width = p.width;

    int row = blockIdx.x * nw + warp;
    if (queue) {
        int r0 = 0;
        if (lane == 0) r0 = atomicAdd(queue, 1);
        row = __shfl_sync(0xffffffffu, r0, 0);
    }
    // the next row's list is copied into the slice (cp.async) while the
    // current row computes
    RowMeta nxt{};
    if (row < a.n_rows) {
        nxt = row_meta(a, row);
        csr_prefetch(a, nxt, cap, S.nbl);
    }
    for (; row < a.n_rows;) {
        const RowMeta m = nxt;
        const int i = m.i, n = m.n;
        const int cur_row = row;  // row being processed; `row` is the next one
        // next row: from the shared counter (dynamic) or by grid stride
        if (queue) {
            int r1 = 0;
            if (lane == 0) r1 = atomicAdd(queue, 1);
            row = __shfl_sync(0xffffffffu, r1, 0);
        } else {
            row += gridDim.x * nw;
        }
        if (row < a.n_rows) nxt = row_meta(a, row);
        double *const dco = VJP ? a.dcoords + (size_t)cur_row * a.dc_stride : nullptr;
        csr_wait();
        if (n > cap || n < 0 || (a.n_total > 0 && (i < 0 || i >= a.n_total))) {
            raise_status(a.status, n > cap ? kDevCapacity : kDevBadIndex);
            if (a.desc)
                for (int q = lane; q < width; q += 32) a.desc[(size_t)cur_row * width + q] = __longlong_as_double(0x7ff8000000000000LL);
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
                j = i;   // read in-bounds data; the entry is dropped below
                ok = 0;
            }
            const int js = a.species[j];
            const double x = a.coords[3 * j], y = a.coords[3 * j + 1], z = a.coords[3 * j + 2];
            const double rx = x - cix, ry = y - ciy, rz = z - ciz;
            const double rsq = rx * rx + ry * ry + rz * rz;
            const double r = sqrt(rsq);
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
        // ---- two-body terms (g1, g2, g3)
        if (PH != 3 && p.n2 > 0) {
            double acc2[M2];
#pragma unroll
            for (int q = 0; q < M2; ++q) acc2[q] = 0.0;
            for (int jj = lane; jj < n; jj += 32) {
                if (!S.inc[jj]) continue;
                const double r = S.r[jj], rc = S.rc[jj], fc = S.fc[jj];
                double dsum = 0.0;
#pragma unroll
                for (int q = 0; q < M2; ++q) {
                    if (q < p.n2) {
                        const int t = __ldg(p.t2 + q);
                        const double pa = __ldg(p.a2 + q), pb = __ldg(p.b2 + q);
                        double v, dv = 0.0;
                        if (t == 1) {
                            v = fc;
                            if (VJP) dv = S.dfc[jj];
                        } else if (t == 2) {
                            const double e = exp(-pa * (r - pb) * (r - pb));
                            v = e * fc;
                            if (VJP) dv = e * (-2.0 * pa * (r - pb) * fc + S.dfc[jj]);
                        } else {
                            double sn, cs;
                            sincos(pa * r, &sn, &cs);
                            v = cs * fc;
                            if (VJP) dv = -pa * sn * fc + cs * S.dfc[jj];
                        }
                        acc2[q] += v;
                        if (VJP) dsum += __ldg(dE + __ldg(p.o2 + q)) * dv;
                    }
                }
                if (VJP) {
                    const double inv = S.ir[jj];
                    const double gx = dsum * (S.cx[jj] - cix) * inv;
                    const double gy = dsum * (S.cy[jj] - ciy) * inv;
                    const double gz = dsum * (S.cz[jj] - ciz) * inv;
                    S.gx[jj] += gx;   // jj is owned by this lane in this phase
                    S.gy[jj] += gy;
                    S.gz[jj] += gz;
                    gix -= gx;
                    giy -= gy;
                    giz -= gz;
                }
            }
#pragma unroll
            for (int q = 0; q < M2; ++q) {
                if (q < p.n2) {
                    const double v = warp_sum(acc2[q]);
                    if (lane == 0 && a.desc) a.desc[(size_t)cur_row * width + __ldg(p.o2 + q)] = v;
                }
            }
        }
        // ---- three-body terms (g4, g5)
        if (PH != 2 && p.n3 > 0) {
            double acc3[M3];
#pragma unroll
            for (int q = 0; q < M3; ++q) acc3[q] = 0.0;
            // lane l owns neighbours jj = l, l + 32, ...; at step dd it takes the
            // triplet (jj, kk = (jj + dd) mod n), dd = 1 .. n/2 (the last step,
            // for even n, only for jj < n/2): every unordered pair once, the
            // lanes' kk distinct within a step (plain read-modify-writes of the
            // kk gradients, steps ordered by __syncwarp), jj's in registers
            __syncwarp();
            const int dmax = (n - 1) / 2, dlast = n / 2;
            for (int m0 = 0; m0 < n; m0 += 32) {
              const int jj = m0 + lane;
              double gjx = 0.0, gjy = 0.0, gjz = 0.0;
              for (int dd = 1; dd <= dlast; ++dd) {
                int kk = jj + dd;
                if (kk >= n) kk -= n;
                if (jj < n && (dd <= dmax || jj < dlast) && S.inc[jj] && S.inc[kk]) {
                    // r_ik and its cutoff functions are the staged pair values of kk
                    // (same coordinates, same species-pair cutoff as the reference's
                    // per-triplet recomputation)
                    const int ks = S.spec[kk], js = S.spec[jj];
                    const double rcjk = p.rcut[js * p.ns + ks], ircjk = p.ircut[js * p.ns + ks];
                    const double jkx = S.cx[kk] - S.cx[jj], jky = S.cy[kk] - S.cy[jj], jkz = S.cz[kk] - S.cz[jj];
                    const double rjksq = jkx * jkx + jky * jky + jkz * jkz;
                    const double d = sqrt(rjksq);
                    const double av = S.r[jj], b = S.r[kk];
                    const double ia = S.ir[jj], ib = S.ir[kk];
                    const double asq = av * av, bsq = b * b, dsq = d * d;
                    const double cth = (asq + bsq - dsq) * (0.5 * ia * ib);
                    const double fa = S.fc[jj], fb = S.fc[kk];
                    double fd = 0.0, dfd = 0.0;
                    if (VJP)
                        cutc_both(d, rcjk, ircjk, fd, dfd);
                    else
                        fd = cutc_i(d, rcjk, ircjk);
                    const bool g4ok = !(d > rcjk);
                    const double S4 = asq + bsq + dsq, S5 = asq + bsq;
                    const double F4 = fa * fb * fd, F5 = fa * fb;
                    double A4 = 0, B4 = 0, C4 = 0, A5 = 0, B5 = 0, C5 = 0;
                    double E = 0.0, E0 = 0.0;
                    int tprev = 0;
#pragma unroll
                    for (int q = 0; q < M3; ++q) {
                        if (q < p.n3) {
                            const int t = __ldg(p.t3 + q);
                            const double eta = __ldg(p.e3 + q);
                            const int ec = __ldg(p.ec3 + q);
                            // exp(-eta S): once per distinct eta; integer multiples of the
                            // group's smallest eta by powering (e^{kx} = (e^x)^k)
                            if (t != tprev) {
                                E0 = exp(-eta * (t == 4 ? S4 : S5));
                                E = E0;
                                tprev = t;
                            } else if (ec == 0) {
                                E = exp(-eta * (t == 4 ? S4 : S5));
                            } else if (ec > 0) {
                                double r = 1.0, x = E0;
                                for (int k = ec; k > 0; k >>= 1) {
                                    if (k & 1) r *= x;
                                    x *= x;
                                }
                                E = r;
                            }
                            if (t == 5 || g4ok) {
                                const double lam = __ldg(p.l3 + q);
                                const double base = 1.0 + lam * cth;
                                const int zi = __ldg(p.zi3 + q);
                                double cp = 0.0, dcp = 0.0;
                                if (base > 0) {
                                    if (zi == 1) {
                                        cp = base;
                                        dcp = 1.0;
                                    } else if (zi == 2) {
                                        cp = base * base;
                                        dcp = 2.0 * base;
                                    } else if (zi == 4) {
                                        const double b2 = base * base;
                                        cp = b2 * b2;
                                        dcp = 4.0 * b2 * base;
                                    } else {
                                        const double zeta = __ldg(p.z3 + q);
                                        if (zi >= 0) {
                                            cp = ipow(base, zi);
                                            dcp = zi > 0 ? zeta * ipow(base, zi - 1) : 0.0;
                                        } else {
                                            cp = pow(base, zeta);
                                            dcp = zeta * pow(base, zeta - 1.0);
                                        }
                                    }
                                }
                                const double P = __ldg(p.P3 + q);
                                acc3[q] += P * cp * E * (t == 4 ? F4 : F5);
                                if (VJP && base > 0) {
                                    const double g = __ldg(dE + __ldg(p.o3 + q));
                                    const double bq = g * P * E;
                                    if (t == 4) {
                                        A4 += bq * cp;
                                        B4 += bq * cp * eta;
                                        C4 += bq * dcp * lam;
                                    } else {
                                        A5 += bq * cp;
                                        B5 += bq * cp * eta;
                                        C5 += bq * dcp * lam;
                                    }
                                }
                            }
                        }
                    }
                    if (VJP) {
                        const double dfa = S.dfc[jj], dfb = S.dfc[kk];
                        const double dca = (asq - bsq + dsq) * (0.5 * ia * ia * ib);
                        const double dcb = (bsq - asq + dsq) * (0.5 * ia * ib * ib);
                        const double dcd = -d * ia * ib;
                        const double Ga = F4 * C4 * dca - 2.0 * av * F4 * B4 + dfa * fb * fd * A4 +
                                          F5 * C5 * dca - 2.0 * av * F5 * B5 + dfa * fb * A5;
                        const double Gb = F4 * C4 * dcb - 2.0 * b * F4 * B4 + fa * dfb * fd * A4 +
                                          F5 * C5 * dcb - 2.0 * b * F5 * B5 + fa * dfb * A5;
                        const double Gd = F4 * C4 * dcd - 2.0 * d * F4 * B4 + fa * fb * dfd * A4 +
                                          F5 * C5 * dcd;
                        const double id = d > 0 ? rsqrt(dsq) : 0.0;
                        const double ijx = (S.cx[jj] - cix) * ia, ijy = (S.cy[jj] - ciy) * ia,
                                     ijz = (S.cz[jj] - ciz) * ia;
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
              if (VJP && jj < n) {
                  S.gx[jj] += gjx;
                  S.gy[jj] += gjy;
                  S.gz[jj] += gjz;
              }
              __syncwarp();
            }
#pragma unroll
            for (int q = 0; q < M3; ++q) {
                if (q < p.n3) {
                    const double v = warp_sum(acc3[q]);
                    if (lane == 0 && a.desc) a.desc[(size_t)cur_row * width + __ldg(p.o3 + q)] = v;
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
// sums as two launches, so that each launch's hot code stays in the
// instruction cache while the warps drift apart over hundreds of rows (the
// rows' neighbours are staged twice; 0 disables the split)
#ifndef LD_SF_SPLIT_ROWS
#define LD_SF_SPLIT_ROWS 8192
#endif
template <bool VJP, int M2, int M3>
int launch_t(const SFDev &p, const RowArgs &a, cudaStream_t s) {
    if (LD_SF_SPLIT_ROWS > 0 && a.n_rows >= LD_SF_SPLIT_ROWS && p.n2 > 0 && p.n3 > 0) {
        int rc = launch_rows_kernel(sf_kernel<VJP, M2, M3, 2>, p, a, s, VJP, "sf_kernel");
        if (rc) return rc;
        return launch_rows_kernel(sf_kernel<VJP, M2, M3, 3>, p, a, s, VJP, "sf_kernel");
    }
    return launch_rows_kernel(sf_kernel<VJP, M2, M3>, p, a, s, VJP, "sf_kernel");
}

}  // namespace

size_t sf_work_bytes(const SFDev &, int, bool) { return 256; }

int sf_launch(const SFDev &p, const RowArgs &a, cudaStream_t s) {
    if (a.n_rows <= 0) return LD_OK;
    if (p.has_grid && !a.force_generic) return sfg_launch(p, a, s);
    const int m = p.n2 > p.n3 ? p.n2 : p.n3;
    const bool vjp = a.dE != nullptr;
    if (m <= 16) return vjp ? launch_t<true, 16, 16>(p, a, s) : launch_t<false, 16, 16>(p, a, s);
    if (m <= 32) return vjp ? launch_t<true, 32, 32>(p, a, s) : launch_t<false, 32, 32>(p, a, s);
    if (m <= 64) return vjp ? launch_t<true, 64, 64>(p, a, s) : launch_t<false, 64, 64>(p, a, s);
    return fail(LD_ERR_CAPACITY, "symmetry functions: more than 64 outputs of one body order");
}

}  // namespace ldb
