// ld_sfp.cu -- gradients of a symmetry-function loss with respect to the
// descriptor's own parameters (eta, Rs, kappa, zeta, lambda):
//   dL/dtheta = sum_i sum_o dL/dG_io * dG_io/dtheta.
// The reference differentiates Descriptor::compute with Enzyme into a shadow
// DescriptorKind and drops that shadow (src/Descriptors.cpp:165-215); here
// the partials are written out in the caller's flat parameter layout.
// Definitions as in SymmetryFunctions::compute (src/SymmetryFunctions.cpp:
// 141-259): g2 = sum_j exp(-eta (r - Rs)^2) fc, g3 = sum_j cos(kappa r) fc,
// g4 = 2^(1-zeta) sum_{j<k} (1 + lambda cos)^zeta exp(-eta S) fc fc fc with
// S = r_ij^2 + r_ik^2 + r_jk^2 (g5: without the r_jk terms); a triplet whose
// base 1 + lambda cos is not positive contributes nothing.
//
// One warp per centre row; lane l owns outputs l, l + 32, l + 64, l + 96.
// All lanes walk the row's pairs and triplets together (the geometry loads
// are warp-uniform broadcasts) and each evaluates its own outputs' partials;
// a lane keeps its outputs' sums over the rows it visits in registers and
// adds them to the result once.  This is a training-time call, written for
// clarity over speed.
#include "ld_sf_common.cuh"

namespace ldb {
namespace {
using namespace sfc;

constexpr int kMaxOutPerLane = 4;   // width <= 128 (64 two-body + 64 three-body)
constexpr double kLn2 = 0.69314718055994530942;

__global__ void __launch_bounds__(128) sf_param_kernel(const __grid_constant__ SFDev p, RowArgs a,
                                                       double *__restrict__ dparams) {
    const int lane = threadIdx.x & 31;
    const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    const int width = p.width;
    int ot[kMaxOutPerLane];
    double pv[kMaxOutPerLane][3], acc[kMaxOutPerLane][3];
    bool has2 = false, has3 = false;
#pragma unroll
    for (int m = 0; m < kMaxOutPerLane; ++m) {
        const int o = lane + 32 * m;
        ot[m] = o < width ? p.pt[o] : 0;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            pv[m][k] = o < width ? p.pv[3 * o + k] : 0.0;
            acc[m][k] = 0.0;
        }
        has2 |= ot[m] == 2 || ot[m] == 3;
        has3 |= ot[m] >= 4;
    }
    const bool any2 = __any_sync(0xffffffffu, has2), any3 = __any_sync(0xffffffffu, has3);
    for (long long row = gw; row < a.n_rows; row += nwarps) {
        const int i = (int)row;
        const long long off = a.off[row];
        const int n = (int)(a.off[row + 1] - a.off[row]);
        if (i >= a.n_total) {
            if (lane == 0) raise_status(a.status, kDevBadIndex);
            continue;
        }
        const double cix = a.coords[3 * i], ciy = a.coords[3 * i + 1], ciz = a.coords[3 * i + 2];
        const int is = a.species[i];
        double g[kMaxOutPerLane][3];
#pragma unroll
        for (int m = 0; m < kMaxOutPerLane; ++m)
#pragma unroll
            for (int k = 0; k < 3; ++k) g[m][k] = 0.0;
        // neighbour jj of the row: position, distance, cutoff; false when it
        // is outside the cutoff (or a bad index, which raises the status)
        auto nb = [&](int jj, double &x, double &y, double &z, double &r, double &rc, double &fc, int &js) {
            const int j = a.nbl[off + jj];
            if (j < 0 || j >= a.n_total) {
                if (lane == 0) raise_status(a.status, kDevBadIndex);
                return false;
            }
            js = a.species[j];
            x = a.coords[3 * j];
            y = a.coords[3 * j + 1];
            z = a.coords[3 * j + 2];
            const double rx = x - cix, ry = y - ciy, rz = z - ciz;
            r = sqrt(rx * rx + ry * ry + rz * rz);
            rc = p.rcut[is * p.ns + js];
            fc = cutc(r, rc);
            return !(r > rc);
        };
        if (any2) {
            for (int jj = 0; jj < n; ++jj) {
                double x, y, z, r, rc, fc;
                int js;
                if (!nb(jj, x, y, z, r, rc, fc, js)) continue;
#pragma unroll
                for (int m = 0; m < kMaxOutPerLane; ++m) {
                    if (ot[m] == 2) {
                        const double eta = pv[m][0], d = r - pv[m][1];
                        const double e = exp(-eta * d * d) * fc;
                        g[m][0] -= d * d * e;          // d/d eta
                        g[m][1] += 2.0 * eta * d * e;  // d/d Rs
                    } else if (ot[m] == 3) {
                        g[m][0] -= r * sin(pv[m][0] * r) * fc;   // d/d kappa
                    }
                }
            }
        }
        if (any3) {
            for (int jj = 0; jj < n - 1; ++jj) {
                double xj, yj, zj, ra, rcj, fa;
                int js;
                if (!nb(jj, xj, yj, zj, ra, rcj, fa, js)) continue;
                for (int kk = jj + 1; kk < n; ++kk) {
                    double xk, yk, zk, rb, rck, fb;
                    int ks;
                    if (!nb(kk, xk, yk, zk, rb, rck, fb, ks)) continue;
                    const double rcjk = p.rcut[js * p.ns + ks];
                    const double jkx = xk - xj, jky = yk - yj, jkz = zk - zj;
                    const double d = sqrt(jkx * jkx + jky * jky + jkz * jkz);
                    const double asq = ra * ra, bsq = rb * rb, dsq = d * d;
                    const double cth = (asq + bsq - dsq) * (0.5 / (ra * rb));
                    const double fd = d < rcjk ? 0.5 * (cos(kPi * d / rcjk) + 1.0) : 0.0;
                    const bool g4ok = !(d > rcjk);
#pragma unroll
                    for (int m = 0; m < kMaxOutPerLane; ++m) {
                        if (ot[m] < 4 || (ot[m] == 4 && !g4ok)) continue;
                        const double zeta = pv[m][0], lam = pv[m][1], eta = pv[m][2];
                        const double base = 1.0 + lam * cth;
                        if (!(base > 0.0)) continue;
                        const double S = ot[m] == 4 ? asq + bsq + dsq : asq + bsq;
                        const double F = ot[m] == 4 ? fa * fb * fd : fa * fb;
                        const double EF = exp(-eta * S) * F * exp2(1.0 - zeta);
                        const double cp = pow(base, zeta);
                        const double T = cp * EF;
                        g[m][0] += T * (log(base) - kLn2);                 // d/d zeta
                        g[m][1] += zeta * pow(base, zeta - 1.0) * cth * EF; // d/d lambda
                        g[m][2] -= S * T;                                   // d/d eta
                    }
                }
            }
        }
        const double *dEr = a.dE + (size_t)row * width;
#pragma unroll
        for (int m = 0; m < kMaxOutPerLane; ++m) {
            const int o = lane + 32 * m;
            if (o >= width) continue;
            const double w = dEr[o];
#pragma unroll
            for (int k = 0; k < 3; ++k) acc[m][k] = fma(w, g[m][k], acc[m][k]);
        }
    }
#pragma unroll
    for (int m = 0; m < kMaxOutPerLane; ++m) {
        const int o = lane + 32 * m;
        if (o >= width) continue;
        const int np = ot[m] == 2 ? 2 : ot[m] == 3 ? 1 : ot[m] >= 4 ? 3 : 0;
        const int base = p.pofs[o];
        for (int k = 0; k < np; ++k) atomicAdd(dparams + base + k, acc[m][k]);
    }
}

}  // namespace

int sf_param_launch(const SFDev &p, const RowArgs &a, double *d_params, cudaStream_t s) {
    if (p.width > 32 * kMaxOutPerLane) return fail(LD_ERR_CAPACITY, "hyperparameter gradients: width above 128");
    LDB_CUDA(cudaMemsetAsync(d_params, 0, sizeof(double) * (p.nparams > 0 ? p.nparams : 1), s));
    if (a.n_rows <= 0) return LD_OK;
    int dev = 0, nsm = 148;
    LDB_CUDA(cudaGetDevice(&dev));
    LDB_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    long long grid = ((long long)a.n_rows + 3) / 4;
    if (grid > (long long)nsm * 16) grid = (long long)nsm * 16;
    sf_param_kernel<<<(unsigned)grid, 128, 0, s>>>(p, a, d_params);
    count_launch();
    LDB_CUDA(cudaGetLastError());
    return LD_OK;
}

}  // namespace ldb
