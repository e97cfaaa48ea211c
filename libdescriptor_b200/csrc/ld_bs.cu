// ld_bs.cu -- SNAP-style bispectrum on sm_100a: forward and fused
// forward + VJP, one CTA (4 warps) per centre atom.
//
// Forward semantics follow Bispectrum::compute (src/Bispectrum.cpp:229-297):
// neighbours with 1e-10 < r < rc are kept in list order; Utot = wself*I +
// sum_k sfac_k w_k U_k with U from the Cayley-Klein / VMK 4.8.2 recursion
// (:490-554, including the inversion-symmetry copy, whose side effect on the
// centre element -- its imaginary part is negated -- is reproduced);
// Z(j1,j2,j,ma,mb<=j/2) = sum CG CG U_j1 U_j2 (:345-389); B from the
// half-matrix sum with doubling (:391-427); outputs in diagonal-style order
// (:429-468).
//
// Phases per centre (one CTA):
//  P0  stage the in-cutoff neighbours into shared memory, order preserving
//      (ballot + warp prefix).
//  P1  U recursion, warp per neighbour, lanes over the left-half elements of
//      a layer; each warp accumulates its own partial Utot, then the CTA sums
//      the partials and fills the right half by the inversion symmetry.
//  P2  Z elements from a host-built longest-processing-time schedule (the
//      per-thread task lists balance the CG double sums).
//  P3  B outputs; for the gradient also the adjoint "Y" arrays
//      Y_j = sum_t betaj_t Z_t with betaj_t a fixed sparse combination of
//      dL/dB (bispectrum symmetry identity, see the host table builder).
//  P4  (gradient) warp per neighbour: U and dU/dr recursion on the left half
//      contracted with Y on the fly -- no per-neighbour Jacobian is stored;
//      dL/dr_k = 2 w_k (dsfac u_hat S + sfac V) then FP64 atomics.
#include "ld_internal.h"

namespace ldb {
namespace {

constexpr double kPi = 3.1415926535897932;
constexpr int NT = kBSThreads;
constexpr int NW = NT / 32;

__device__ __forceinline__ void raise_status(int *status, int code) {
    if (status) atomicCAS(status, 0, code);
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

struct Carve {
    double *utr, *uti;      // nU
    double *yr, *yi;        // nL
    double *beta;           // ncoeff
    double *betaj;          // ntrip
    double *sx, *sy, *sz, *sr, *sw, *src;  // cap
    int *sidx;              // cap
    double *scratch;
    int *misc;              // 16 ints
    double *gred;           // NW*3
};

__host__ __device__ inline size_t rup2(size_t x) { return (x + 1) & ~(size_t)1; }

__host__ __device__ inline size_t lmax_of(int J) { return (size_t)(J + 1) * (J / 2 + 1); }

__host__ __device__ inline size_t scratch_doubles(int J, int nL, int nZ, bool vjp) {
    const size_t L = lmax_of(J);
    size_t p1 = (size_t)NW * (4 * L + 2 * (size_t)nL);
    size_t p2 = 2 * (size_t)nZ;
    size_t p4 = vjp ? (size_t)NW * 16 * L : 0;
    size_t m = p1 > p2 ? p1 : p2;
    return m > p4 ? m : p4;
}

__device__ inline Carve carve(double *sm, const BSDev &p, int cap, bool vjp) {
    Carve c;
    double *q = sm;
    c.utr = q; q += p.nU;
    c.uti = q; q += p.nU;
    if (vjp) {
        c.yr = q; q += p.nL;
        c.yi = q; q += p.nL;
        c.beta = q; q += p.ncoeff;
        c.betaj = q; q += p.ntrip;
    } else {
        c.yr = c.yi = c.beta = c.betaj = nullptr;
    }
    c.sx = q; q += cap;
    c.sy = q; q += cap;
    c.sz = q; q += cap;
    c.sr = q; q += cap;
    c.sw = q; q += cap;
    c.src = q; q += cap;
    c.gred = q; q += NW * 3;
    c.scratch = q; q += scratch_doubles(p.J, p.nL, p.nZall, vjp);
    int *iq = reinterpret_cast<int *>(q);
    c.sidx = iq; iq += cap;
    c.misc = iq;
    return c;
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
__device__ __forceinline__ double dsfac_of(const BSDev &p, double r, double rc) {
    if (p.switch_flag == 1) {
        if (r <= p.rmin0 || r > rc) return 0.0;
        const double inv = 1.0 / (rc - p.rmin0);
        return -0.5 * sinpi((r - p.rmin0) * inv) * (kPi * inv);
    }
    return 0.0;
}

// previous-layer element (layer jp, row m, column mb) from a left-half layer
// buffer, through the inversion symmetry when mb is right of the half.
__device__ __forceinline__ void prev_elem(const double *lr, const double *li, int jp, int m,
                                          int mb, double &vr, double &vi) {
    const int hp = jp / 2, nc = hp + 1;
    if (mb <= hp) {
        vr = lr[m * nc + mb];
        vi = li[m * nc + mb];
    } else {
        const int mm = jp - m, bb = jp - mb;
        const double s = ((m - mb) & 1) ? -1.0 : 1.0;
        vr = s * lr[mm * nc + bb];
        vi = -s * li[mm * nc + bb];
    }
}

template <bool VJP>
__global__ void __launch_bounds__(NT) bs_kernel(BSDev p, RowArgs a, int cap) {
    extern __shared__ double smem[];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    Carve C = carve(smem, p, cap, VJP);
    const int J = p.J, D = J + 1;
    const size_t L = lmax_of(J);
    const int width = p.ncoeff;

    for (int row = blockIdx.x; row < a.n_rows; row += gridDim.x) {
        const int i = a.row_centre ? a.row_centre[row] : row;
        const int lrow = a.row_list ? a.row_list[row] : row;
        const long long off = a.nbl_begin ? a.nbl_begin[lrow] : a.off[lrow];
        const int n = (int)(a.off[lrow + 1] - a.off[lrow]);
        double *const dco = VJP ? a.dcoords + (size_t)row * a.dc_stride : nullptr;
        if (n > cap || n < 0 || (a.n_total > 0 && (i < 0 || i >= a.n_total))) {
            if (tid == 0) raise_status(a.status, n > cap ? kDevCapacity : kDevBadIndex);
            if (a.desc)
                for (int q = tid; q < width; q += NT)
                    a.desc[(size_t)row * width + q] = __longlong_as_double(0x7ff8000000000000LL);
            continue;
        }
        const double cix = a.coords[3 * i], ciy = a.coords[3 * i + 1], ciz = a.coords[3 * i + 2];

        // ------------------------------------------------------------ P0
        int nin = 0;
        for (int c0 = 0; c0 < n; c0 += NT) {
            const int jj = c0 + tid;
            bool flag = false;
            double rx = 0, ry = 0, rz = 0, r = 0, rc = 0, wgt = 0;
            int j = 0;
            if (jj < n) {
                j = a.nbl[off + jj];
                if (a.n_total > 0 && (j < 0 || j >= a.n_total)) {
                    raise_status(a.status, kDevBadIndex);
                } else {
                    const int js = a.species[j];
                    rx = a.coords[3 * j] - cix;
                    ry = a.coords[3 * j + 1] - ciy;
                    rz = a.coords[3 * j + 2] - ciz;
                    const double rsq = rx * rx + ry * ry + rz * rz;
                    r = sqrt(rsq);
                    rc = p.rcut_flat[js];
                    wgt = p.wj[js];
                    flag = (r < rc) && (r > 1e-10);
                }
            }
            const unsigned bal = __ballot_sync(0xffffffffu, flag);
            if (lane == 0) C.misc[warp] = __popc(bal);
            __syncthreads();
            int wbase = 0, tot = 0;
#pragma unroll
            for (int w = 0; w < NW; ++w) {
                const int cw = C.misc[w];
                if (w < warp) wbase += cw;
                tot += cw;
            }
            if (flag) {
                const int pos = nin + wbase + __popc(bal & ((1u << lane) - 1u));
                C.sx[pos] = rx;
                C.sy[pos] = ry;
                C.sz[pos] = rz;
                C.sr[pos] = r;
                C.src[pos] = rc;
                C.sw[pos] = wgt;
                C.sidx[pos] = j;
            }
            nin += tot;
            __syncthreads();
        }

        // ------------------------------------------------------------ P1
        {
            double *lay_r = C.scratch + (size_t)warp * (4 * L + 2 * (size_t)p.nL);
            double *lay_i = lay_r + 2 * L;
            double *pur = lay_r + 4 * L;
            double *pui = pur + p.nL;
            for (int e = lane; e < p.nL; e += 32) {
                pur[e] = 0.0;
                pui[e] = 0.0;
            }
            __syncwarp();
            for (int k = warp; k < nin; k += NW) {
                const double x = C.sx[k], y = C.sy[k], z = C.sz[k];
                const double rsq = x * x + y * y + z * z;
                const double r = sqrt(rsq);
                const double rc = C.src[k];
                // z0 = r / tan(theta0) from one sincos and one reciprocal
                double sth, cth;
                sincos((r - p.rmin0) * (p.rfac0 * kPi / (rc - p.rmin0)), &sth, &cth);
                const double z0 = r * cth / sth;
                const double r0inv = rsqrt(r * r + z0 * z0);
                const double a_r = r0inv * z0, a_i = -r0inv * z;
                const double b_r = r0inv * y, b_i = -r0inv * x;
                const double sf = sfac_of(p, r, rc) * C.sw[k];
                if (lane == 0) {
                    lay_r[0] = 1.0;
                    lay_i[0] = 0.0;
                    pur[0] += sf;
                }
                __syncwarp();
                for (int jl = 1; jl <= J; ++jl) {
                    const int cur = jl & 1, prv = cur ^ 1;
                    const int hj = jl / 2, nc = hj + 1, nel = (jl + 1) * nc;
                    const bool even = (jl & 1) == 0;
                    const double *plr = lay_r + prv * L, *pli = lay_i + prv * L;
                    double *clr = lay_r + cur * L, *cli = lay_i + cur * L;
                    const int lb = __ldg(p.lblock + jl);
                    for (int e = lane; e < nel; e += 32) {
                        const int ma = e / nc, mb = e - ma * nc;
                        if (even && mb == hj && ma > hj) continue;
                        double ur = 0.0, ui = 0.0;
                        if (ma >= 1) {
                            double vr, vi;
                            prev_elem(plr, pli, jl - 1, ma - 1, mb, vr, vi);
                            const double rq = __ldg(p.rootpq + ma * D + (jl - mb));
                            ur = -rq * (b_r * vr + b_i * vi);
                            ui = -rq * (b_r * vi - b_i * vr);
                        }
                        if (ma < jl) {
                            double vr, vi;
                            prev_elem(plr, pli, jl - 1, ma, mb, vr, vi);
                            const double rq = __ldg(p.rootpq + (jl - ma) * D + (jl - mb));
                            ur += rq * (a_r * vr + a_i * vi);
                            ui += rq * (a_r * vi - a_i * vr);
                        }
                        if (even && ma == hj && mb == hj) ui = -ui;
                        clr[e] = ur;
                        cli[e] = ui;
                        pur[lb + e] += sf * ur;
                        pui[lb + e] += sf * ui;
                    }
                    __syncwarp();
                    if (even) {
                        for (int ma = hj + 1 + lane; ma <= jl; ma += 32) {
                            const int src = (jl - ma) * nc + hj;
                            const double s = ((ma - hj) & 1) ? -1.0 : 1.0;
                            clr[ma * nc + hj] = s * clr[src];
                            cli[ma * nc + hj] = -s * cli[src];
                        }
                        __syncwarp();
                    }
                }
            }
            __syncthreads();
            // Utot left half = wself*I + sum of warp partials
            for (int e = tid; e < p.nL; e += NT) {
                const int pk = __ldg(p.lel + e);
                const int jl = pk & 0xff, ma = (pk >> 8) & 0xff, mb = (pk >> 16) & 0xff;
                const int hj = jl / 2;
                if ((jl & 1) == 0 && mb == hj && ma > hj) continue;
                double sr = (ma == mb) ? p.wself : 0.0, si = 0.0;
#pragma unroll
                for (int w = 0; w < NW; ++w) {
                    const double *q = C.scratch + (size_t)w * (4 * L + 2 * (size_t)p.nL) + 4 * L;
                    sr += q[e];
                    si += q[p.nL + e];
                }
                const int u = __ldg(p.ublock + jl) + ma * (jl + 1) + mb;
                C.utr[u] = sr;
                C.uti[u] = si;
            }
            __syncthreads();
            // right half by inversion symmetry U(j-ma, j-mb) = (-1)^(ma-mb) conj U(ma, mb)
            for (int jl = 0; jl <= J; ++jl) {
                const int hj = jl / 2, nn = (jl + 1) * (jl + 1);
                const int ub = __ldg(p.ublock + jl);
                for (int e = tid; e < nn; e += NT) {
                    const int ma = e / (jl + 1), mb = e - ma * (jl + 1);
                    const bool right = (mb > hj) || ((jl & 1) == 0 && mb == hj && ma > hj);
                    if (!right) continue;
                    const int sm_ = ub + (jl - ma) * (jl + 1) + (jl - mb);
                    const double s = ((ma - mb) & 1) ? -1.0 : 1.0;
                    C.utr[ub + e] = s * C.utr[sm_];
                    C.uti[ub + e] = -s * C.uti[sm_];
                }
            }
            __syncthreads();
        }

        // ------------------------------------------------------------ P2
        {
            double *zr = C.scratch, *zi = C.scratch + p.nZall;
            const int *toff = VJP ? p.toff_v : p.toff_f;
            const int4 *task = VJP ? p.task_v : p.task_f;
            const int t0 = __ldg(toff + tid), t1 = __ldg(toff + tid + 1);
            for (int t = t0; t < t1; ++t) {
                const int4 tk = __ldg(task + t);
                const int j1 = tk.x & 0xff, j2 = (tk.x >> 8) & 0xff, jl = (tk.x >> 16) & 0xff;
                const int ma = (tk.x >> 24) & 0xff, mb = tk.y;
                const int zidx = tk.z, cgo = tk.w;
                const int n2 = j2 + 1;
                int lo = (2 * ma - jl - j2 + j1) / 2, hi = (2 * ma - jl + j2 + j1) / 2;
                if (lo < 0) lo = 0;
                if (hi > j1) hi = j1;
                int blo = (2 * mb - jl - j2 + j1) / 2, bhi = (2 * mb - jl + j2 + j1) / 2;
                if (blo < 0) blo = 0;
                if (bhi > j1) bhi = j1;
                const int cb = (2 * mb - jl + j1 + j2) / 2;   // mb2 = cb - mb1
                const int ca = (2 * ma - jl + j1 + j2) / 2;   // ma2 = ca - ma1
                const int u1b = __ldg(p.ublock + j1), u2b = __ldg(p.ublock + j2);
                double zre = 0.0, zim = 0.0;
                for (int ma1 = lo; ma1 <= hi; ++ma1) {
                    const int ma2 = ca - ma1;
                    const double *u1r = C.utr + u1b + ma1 * (j1 + 1);
                    const double *u1i = C.uti + u1b + ma1 * (j1 + 1);
                    const double *u2r = C.utr + u2b + ma2 * n2;
                    const double *u2i = C.uti + u2b + ma2 * n2;
                    double sr = 0.0, si = 0.0;
                    for (int mb1 = blo; mb1 <= bhi; ++mb1) {
                        const int mb2 = cb - mb1;
                        const double c = __ldg(p.cg + cgo + mb1 * n2 + mb2);
                        const double ar = u1r[mb1], ai = u1i[mb1];
                        const double br = u2r[mb2], bi = u2i[mb2];
                        sr += c * (ar * br - ai * bi);
                        si += c * (ar * bi + ai * br);
                    }
                    const double cga = __ldg(p.cg + cgo + ma1 * n2 + ma2);
                    zre += sr * cga;
                    zim += si * cga;
                }
                zr[zidx] = zre;
                zi[zidx] = zim;
            }
            __syncthreads();
        }

        // ------------------------------------------------------------ P3
        {
            const double *zr = C.scratch, *zi = C.scratch + p.nZall;
            for (int o = tid; o < width; o += NT) {
                const int t = __ldg(p.otrip + o);
                if (t < 0) {   // parity-forbidden triple: constant zero output
                    if (a.desc) a.desc[(size_t)row * width + o] = 0.0;
                    if (VJP) C.beta[o] = 0.0;
                    continue;
                }
                const int4 tr = __ldg(p.trip + t);
                const int jl = tr.z, hj = jl / 2, nc = hj + 1, zo = tr.w;
                const int ub = __ldg(p.ublock + jl);
                double b = 0.0;
                for (int mb = 0; 2 * mb < jl; ++mb)
                    for (int ma = 0; ma <= jl; ++ma) {
                        const int u = ub + ma * (jl + 1) + mb, z = zo + ma * nc + mb;
                        b += C.utr[u] * zr[z] + C.uti[u] * zi[z];
                    }
                if ((jl & 1) == 0) {
                    const int mb = hj;
                    for (int ma = 0; ma < mb; ++ma) {
                        const int u = ub + ma * (jl + 1) + mb, z = zo + ma * nc + mb;
                        b += C.utr[u] * zr[z] + C.uti[u] * zi[z];
                    }
                    const int u = ub + mb * (jl + 1) + mb, z = zo + mb * nc + mb;
                    b += (C.utr[u] * zr[z] + C.uti[u] * zi[z]) * 0.5;
                }
                b *= 2.0;
                if (p.bzero_flag) b -= __ldg(p.bzero + jl);
                if (a.desc) a.desc[(size_t)row * width + o] = b;
                if (VJP) C.beta[o] = a.dE[(size_t)row * width + o];
            }
            if (VJP) {
                __syncthreads();
                for (int t = tid; t < p.ntrip; t += NT) {
                    double s = 0.0;
                    const int m0 = __ldg(p.moff + t), m1 = __ldg(p.moff + t + 1);
                    for (int m = m0; m < m1; ++m) s += __ldg(p.mcoef + m) * C.beta[__ldg(p.mo + m)];
                    C.betaj[t] = s;
                }
                __syncthreads();
                for (int e = tid; e < p.nL; e += NT) {
                    const int pk = __ldg(p.lel + e);
                    const int jl = pk & 0xff, ma = (pk >> 8) & 0xff, mb = (pk >> 16) & 0xff;
                    const int nc = jl / 2 + 1;
                    if ((jl & 1) == 0 && mb == jl / 2 && ma > jl / 2) continue;  // mirror row: unused
                    double yr = 0.0, yi = 0.0;
                    const int q0 = __ldg(p.jtoff + jl), q1 = __ldg(p.jtoff + jl + 1);
                    for (int q = q0; q < q1; ++q) {
                        const int t = __ldg(p.jtlist + q);
                        const double bj = C.betaj[t];
                        const int z = __ldg(p.trip + t).w + ma * nc + mb;
                        yr += bj * zr[z];
                        yi += bj * zi[z];
                    }
                    C.yr[e] = yr;
                    C.yi[e] = yi;
                }
                __syncthreads();
            }
        }

        // ------------------------------------------------------------ P4
        if (VJP) {
            double *Lr = C.scratch + (size_t)warp * 16 * L;   // [2][4][L]
            double *Li = Lr + 8 * L;
            double gcx = 0.0, gcy = 0.0, gcz = 0.0;
            for (int k = warp; k < nin; k += NW) {
                const double x = C.sx[k], y = C.sy[k], z = C.sz[k];
                const double rsq = x * x + y * y + z * z;
                const double r = sqrt(rsq);
                const double rc = C.src[k];
                const double c0 = p.rfac0 * kPi / (rc - p.rmin0);
                double sth, cth;
                sincos((r - p.rmin0) * c0, &sth, &cth);
                const double isth = 1.0 / sth;
                const double z0 = r * cth * isth;
                const double dz0 = cth * isth - r * c0 * isth * isth;
                const double r0inv = rsqrt(r * r + z0 * z0);
                const double dr0inv = -r0inv * r0inv * r0inv * (r + z0 * dz0);
                const double a_r = r0inv * z0, a_i = -r0inv * z;
                const double b_r = r0inv * y, b_i = -r0inv * x;
                const double rinv = 1.0 / r;
                const double u3[3] = {x * rinv, y * rinv, z * rinv};
                double dar[3], dai[3], dbr[3], dbi[3];
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    dar[d] = (dz0 * r0inv + z0 * dr0inv) * u3[d];
                    dai[d] = -(z * dr0inv * u3[d] + (d == 2 ? r0inv : 0.0));
                    dbr[d] = y * dr0inv * u3[d] + (d == 1 ? r0inv : 0.0);
                    dbi[d] = -(x * dr0inv * u3[d] + (d == 0 ? r0inv : 0.0));
                }
                double S = 0.0, V0 = 0.0, V1 = 0.0, V2 = 0.0;
                if (lane == 0) {
                    Lr[0] = 1.0;
                    Li[0] = 0.0;
#pragma unroll
                    for (int d = 1; d < 4; ++d) {
                        Lr[d * L] = 0.0;
                        Li[d * L] = 0.0;
                    }
                    S = 0.5 * C.yr[0];
                }
                __syncwarp();
                for (int jl = 1; jl <= J; ++jl) {
                    const int cur = jl & 1, prv = cur ^ 1;
                    const int hj = jl / 2, nc = hj + 1, nel = (jl + 1) * nc;
                    const bool even = (jl & 1) == 0;
                    const int lb = __ldg(p.lblock + jl);
                    for (int e = lane; e < nel; e += 32) {
                        const int ma = e / nc, mb = e - ma * nc;
                        if (even && mb == hj && ma > hj) continue;
                        double ur = 0.0, ui = 0.0, dr_[3] = {0, 0, 0}, di_[3] = {0, 0, 0};
                        if (ma >= 1) {
                            const double rq = -__ldg(p.rootpq + ma * D + (jl - mb));
                            double vr, vi;
                            prev_elem(Lr + (prv * 4) * L, Li + (prv * 4) * L, jl - 1, ma - 1, mb, vr, vi);
                            ur = rq * (b_r * vr + b_i * vi);
                            ui = rq * (b_r * vi - b_i * vr);
#pragma unroll
                            for (int d = 0; d < 3; ++d) {
                                double wr, wi;
                                prev_elem(Lr + (prv * 4 + 1 + d) * L, Li + (prv * 4 + 1 + d) * L, jl - 1,
                                          ma - 1, mb, wr, wi);
                                dr_[d] = rq * (dbr[d] * vr + dbi[d] * vi + b_r * wr + b_i * wi);
                                di_[d] = rq * (dbr[d] * vi - dbi[d] * vr + b_r * wi - b_i * wr);
                            }
                        }
                        if (ma < jl) {
                            const double rq = __ldg(p.rootpq + (jl - ma) * D + (jl - mb));
                            double vr, vi;
                            prev_elem(Lr + (prv * 4) * L, Li + (prv * 4) * L, jl - 1, ma, mb, vr, vi);
                            ur += rq * (a_r * vr + a_i * vi);
                            ui += rq * (a_r * vi - a_i * vr);
#pragma unroll
                            for (int d = 0; d < 3; ++d) {
                                double wr, wi;
                                prev_elem(Lr + (prv * 4 + 1 + d) * L, Li + (prv * 4 + 1 + d) * L, jl - 1,
                                          ma, mb, wr, wi);
                                dr_[d] += rq * (dar[d] * vr + dai[d] * vi + a_r * wr + a_i * wi);
                                di_[d] += rq * (dar[d] * vi - dai[d] * vr + a_r * wi - a_i * wr);
                            }
                        }
                        double wgt = 1.0;
                        if (even && mb == hj) {
                            if (ma == hj) {
                                ui = -ui;
#pragma unroll
                                for (int d = 0; d < 3; ++d) di_[d] = -di_[d];
                                wgt = 0.5;
                            }
                        }
                        double *cr = Lr + (cur * 4) * L, *ci = Li + (cur * 4) * L;
                        cr[e] = ur;
                        ci[e] = ui;
#pragma unroll
                        for (int d = 0; d < 3; ++d) {
                            cr[(1 + d) * L + e] = dr_[d];
                            ci[(1 + d) * L + e] = di_[d];
                        }
                        const double yr = C.yr[lb + e], yi = C.yi[lb + e];
                        S += wgt * (yr * ur + yi * ui);
                        V0 += wgt * (yr * dr_[0] + yi * di_[0]);
                        V1 += wgt * (yr * dr_[1] + yi * di_[1]);
                        V2 += wgt * (yr * dr_[2] + yi * di_[2]);
                    }
                    __syncwarp();
                    if (even) {
                        for (int ma = hj + 1 + lane; ma <= jl; ma += 32) {
                            const int src = (jl - ma) * nc + hj;
                            const double s = ((ma - hj) & 1) ? -1.0 : 1.0;
#pragma unroll
                            for (int q = 0; q < 4; ++q) {
                                double *cr = Lr + (cur * 4 + q) * L, *ci = Li + (cur * 4 + q) * L;
                                cr[ma * nc + hj] = s * cr[src];
                                ci[ma * nc + hj] = -s * ci[src];
                            }
                        }
                        __syncwarp();
                    }
                }
                S = warp_sum(S);
                V0 = warp_sum(V0);
                V1 = warp_sum(V1);
                V2 = warp_sum(V2);
                if (lane == 0) {
                    const double wk = C.sw[k];
                    const double sf = sfac_of(p, r, rc), dsf = dsfac_of(p, r, rc);
                    const double g0 = 2.0 * wk * (dsf * u3[0] * S + sf * V0);
                    const double g1 = 2.0 * wk * (dsf * u3[1] * S + sf * V1);
                    const double g2 = 2.0 * wk * (dsf * u3[2] * S + sf * V2);
                    const int nb = C.sidx[k];
                    const int tn = a.image ? a.image[nb] : nb;
                    atomicAdd(dco + 3 * (size_t)tn, g0);
                    atomicAdd(dco + 3 * (size_t)tn + 1, g1);
                    atomicAdd(dco + 3 * (size_t)tn + 2, g2);
                    gcx -= g0;
                    gcy -= g1;
                    gcz -= g2;
                }
                __syncwarp();
            }
            if (lane == 0) {
                C.gred[warp * 3] = gcx;
                C.gred[warp * 3 + 1] = gcy;
                C.gred[warp * 3 + 2] = gcz;
            }
            __syncthreads();
            if (tid < 3) {
                double s = 0.0;
#pragma unroll
                for (int w = 0; w < NW; ++w) s += C.gred[w * 3 + tid];
                const int ti = a.image ? a.image[i] : i;
                atomicAdd(dco + 3 * (size_t)ti + tid, s);
            }
        }
        __syncthreads();
    }
}

}  // namespace

size_t bs_smem_bytes(const BSDev &p, int max_neigh, bool vjp) {
    const int cap = max_neigh > 0 ? max_neigh : 1;
    size_t d = 2 * (size_t)p.nU + 6 * (size_t)cap + NW * 3 +
               scratch_doubles(p.J, p.nL, p.nZall, vjp);
    if (vjp) d += 2 * (size_t)p.nL + p.ncoeff + p.ntrip;
    size_t ints = (size_t)cap + 16;
    return d * sizeof(double) + ints * sizeof(int);
}

template <int J>
int bs2_launch_t(const BSDev &p, const RowArgs &a, cudaStream_t s);

// twojmax-specialised path (ld_bs2*.cu): per-centre kernel + pair-parallel
// gradient kernel; it needs a stream-ordered work space for Y, so the
// no-allocation entry point and the Jacobian (row remapping) use the single
// fused kernel below instead.
static int bs2_dispatch(const BSDev &p, const RowArgs &a, cudaStream_t s) {
    switch (p.J) {
    case 0: return bs2_launch_t<0>(p, a, s);
    case 1: return bs2_launch_t<1>(p, a, s);
    case 2: return bs2_launch_t<2>(p, a, s);
    case 3: return bs2_launch_t<3>(p, a, s);
    case 4: return bs2_launch_t<4>(p, a, s);
    case 5: return bs2_launch_t<5>(p, a, s);
    case 6: return bs2_launch_t<6>(p, a, s);
    case 7: return bs2_launch_t<7>(p, a, s);
    case 8: return bs2_launch_t<8>(p, a, s);
    case 9: return bs2_launch_t<9>(p, a, s);
    case 10: return bs2_launch_t<10>(p, a, s);
    }
    return fail(LD_ERR_CAPACITY, "bispectrum: twojmax outside the compiled range");
}

size_t bs_work_bytes(const BSDev &p, int n_rows, bool vjp) {
    const size_t rows = (size_t)(n_rows > 0 ? n_rows : 0);
    const size_t y = vjp ? ((sizeof(double2) * rows * p.nL + 16 + 255) & ~(size_t)255) : 0;
    // the split form's U blocks: [group of 32 rows][element][row % 32]
    const size_t ug = bs_split(p) ? ((((rows + 31) / 32) * p.nU * 32 * sizeof(double2) + 255) & ~(size_t)255) : 0;
    return y + ug + 256;
}

int bs_launch(const BSDev &p, const RowArgs &a, cudaStream_t s) {
    if (a.n_rows <= 0) return LD_OK;
    const bool vjp = a.dE != nullptr;
    if (!a.fused_only && a.row_list == nullptr && a.dc_stride == 0 && p.J <= kMaxTwoJ)
        return bs2_dispatch(p, a, s);
    const int cap = a.max_neigh > 0 ? a.max_neigh : 1;
    const size_t smem = bs_smem_bytes(p, cap, vjp);
    if (smem > 227 * 1024)
        return fail(LD_ERR_CAPACITY, "bispectrum: twojmax=" + std::to_string(p.J) + " with max_neigh=" +
                                         std::to_string(a.max_neigh) +
                                         " exceeds the per-CTA shared memory (" +
                                         std::to_string(smem) + " bytes)");
    auto kern = vjp ? bs_kernel<true> : bs_kernel<false>;
    LDB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int dev = 0, nsm = 148, per_sm = 1;
    LDB_CUDA(cudaGetDevice(&dev));
    LDB_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    LDB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NT, smem));
    if (per_sm < 1) per_sm = 1;
    long long grid = (long long)nsm * per_sm;
    if (a.n_rows < grid) grid = a.n_rows;
    if (a.in_ready) LDB_CUDA(cudaStreamWaitEvent(s, a.in_ready, 0));
    kern<<<(unsigned)grid, NT, smem, s>>>(p, a, cap);
    count_launch();
    LDB_CUDA(cudaGetLastError());
    if (a.desc_done) LDB_CUDA(cudaEventRecord(a.desc_done, s));
    return LD_OK;
}

}  // namespace ldb
