// ld_core.cpp -- host side of the C ABI: descriptor handles, parameter and
// Clebsch-Gordan tables, the bispectrum work schedule, staging of host
// buffers, and the device-pointer entry points.
#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstring>
#include <fstream>
#include <map>
#include <cstdint>
#include <mutex>
#include <queue>
#include <set>
#include <sstream>
#include <string>
#include <vector>

#include "ld_internal.h"

// ======================================================================
// errors, launch accounting, device buffers
// ======================================================================
namespace ldb {

static thread_local std::string g_err;
static std::atomic<long long> g_launches{0};

void set_error(const std::string &msg) { g_err = msg; }
int fail(int code, const std::string &msg) {
    g_err = msg;
    return code;
}
int cuda_fail(cudaError_t e, const char *what) {
    g_err = std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e);
    if (e == cudaErrorMemoryAllocation) return LD_ERR_OOM;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return LD_ERR_NO_DEVICE;
    return LD_ERR_CUDA;
}
void count_launch(int n) { g_launches += n; }

// Device allocations of the library (grow-only buffers and the scratch
// pool), and the test hook that makes the k-th next one fail.
static std::atomic<long long> g_allocs{0};
static std::atomic<int> g_fail_in{0};
int count_alloc() {
    ++g_allocs;
    int k = g_fail_in.load();
    while (k > 0) {
        if (g_fail_in.compare_exchange_weak(k, k - 1)) {
            if (k == 1) return fail(LD_ERR_OOM, "device allocation failed (injected by ld_fail_next_allocation)");
            break;
        }
    }
    return LD_OK;
}

// Test hook: a byte (0..255) that every new device allocation of the library
// is filled with, so that a kernel reading memory nobody wrote sees garbage
// (0xff: NaN doubles) on every run; -1 leaves allocations as they come.
static std::atomic<int> g_fill{-1};
int scratch_fill() { return g_fill.load(); }

int DevBuf::ensure(size_t n) {
    if (n <= bytes && p) return LD_OK;
    release();
    size_t want = n < 256 ? 256 : n;
    if (int rc = count_alloc()) return rc;
    cudaError_t e = cudaMalloc(&p, want);
    if (e != cudaSuccess) {
        p = nullptr;
        bytes = 0;
        return cuda_fail(e, "cudaMalloc");
    }
    bytes = want;
    const int f = scratch_fill();
    if (f >= 0) LDB_CUDA(cudaMemset(p, f, want));
    return LD_OK;
}
void DevBuf::release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
}

// Packs host vectors into one device allocation (256-byte aligned slots).
struct Arena {
    std::vector<char> host;
    std::vector<std::pair<size_t, const void **>> fix;  // offset, pointer to patch
    template <class T> void add(const std::vector<T> &v, const T **dst) {
        size_t off = (host.size() + 255) & ~(size_t)255;
        host.resize(off + std::max<size_t>(v.size() * sizeof(T), 1));
        if (!v.empty()) std::memcpy(host.data() + off, v.data(), v.size() * sizeof(T));
        fix.emplace_back(off, reinterpret_cast<const void **>(dst));
    }
    int upload(DevBuf &buf) {
        int rc = buf.ensure(host.size());
        if (rc) return rc;
        LDB_CUDA(cudaMemcpy(buf.p, host.data(), host.size(), cudaMemcpyHostToDevice));
        for (auto &f : fix) *f.second = static_cast<const char *>(buf.p) + f.first;
        return LD_OK;
    }
};

// ======================================================================
// Clebsch-Gordan coefficients (Racah formula), doubled-integer arguments:
// j1, j2, j are 2*(angular momentum); m1 in 0..j1 indexes 2*m = 2*m1 - j1.
// Same definition as Bispectrum::init_clebsch_gordan (src/Bispectrum.cpp:
// 683-727); factorials are exact products in double.
// ======================================================================
static double fact(int n) {
    double f = 1.0;
    for (int k = 2; k <= n; ++k) f *= (double)k;
    return f;
}

static double clebsch_gordan(int j1, int j2, int j, int m1, int m2) {
    const int a2 = 2 * m1 - j1, b2 = 2 * m2 - j2;   // 2*m of the two inputs
    const int c2 = a2 + b2;                        // 2*m of the output
    if (c2 < -j || c2 > j) return 0.0;
    // physical combinations (all integers by the triangle/parity rules)
    const int s1 = (j1 + j2 - j) / 2, s2 = (j1 - j2 + j) / 2, s3 = (-j1 + j2 + j) / 2;
    const int top = (j1 + j2 + j) / 2 + 1;
    const int p1 = (j1 + a2) / 2, q1 = (j1 - a2) / 2;
    const int p2 = (j2 + b2) / 2, q2 = (j2 - b2) / 2;
    const int p3 = (j + c2) / 2, q3 = (j - c2) / 2;
    const int kmin = std::max(0, std::max((j2 - j - a2) / 2, (j1 - j + b2) / 2));
    const int kmax = std::min(s1, std::min(q1, p2));
    double sum = 0.0;
    for (int k = kmin; k <= kmax; ++k) {
        const double den = fact(k) * fact(s1 - k) * fact(q1 - k) * fact(p2 - k) *
                           fact((j - j2 + a2) / 2 + k) * fact((j - j1 - b2) / 2 + k);
        sum += ((k & 1) ? -1.0 : 1.0) / den;
    }
    const double tri = std::sqrt(fact(s1) * fact(s2) * fact(s3) / fact(top));
    const double mf = std::sqrt(fact(p1) * fact(q1) * fact(p2) * fact(q2) * fact(p3) * fact(q3) *
                                (double)(j + 1));
    return sum * tri * mf;
}

}  // namespace ldb

// ======================================================================
// descriptor handle
// ======================================================================
struct ld_descriptor {
    int kind = -1;
    int width = 0;
    int device = 0;
    ldb::SFDev sf;
    ldb::BSDev bs;
    ldb::DevBuf tables;
    // host-API staging (grow-only)
    ldb::DevBuf species, nbl, off, coords, desc, dE, dc, centre, list, status, tmp, work;
    cudaStream_t stream = nullptr;
    // the host API's second stream: dE's upload and the descriptors' read-back
    // overlap the kernels that do not need them
    cudaStream_t stream2 = nullptr;
    cudaEvent_t ev_in = nullptr, ev_desc = nullptr;
    int *hstatus = nullptr;   // pinned copy of the device status word
    std::mutex mu;
    // introspection
    std::vector<int> bs_out_j1, bs_out_j2, bs_out_j;
    long long bs_inner_fwd = 0, bs_inner_vjp = 0;  // CG inner iterations per centre
    int bs_tasks_fwd = 0, bs_tasks_vjp = 0;
    // launch-shape tuning (LD_TUNE_*), 0 = built-in choice
    int tune[5] = {0, 0, 0, 0, 0};
};

namespace ldb {

int handle_device(const ld_descriptor *d) { return d->device; }

static int ensure_stream(ld_descriptor *d) {
    if (d->stream) return LD_OK;
    LDB_CUDA(cudaSetDevice(d->device));
    LDB_CUDA(cudaStreamCreateWithFlags(&d->stream, cudaStreamNonBlocking));
    return LD_OK;
}

static int ensure_stream2(ld_descriptor *d) {
    if (d->stream2 && d->ev_in && d->ev_desc) return LD_OK;
    LDB_CUDA(cudaSetDevice(d->device));
    if (!d->stream2) LDB_CUDA(cudaStreamCreateWithFlags(&d->stream2, cudaStreamNonBlocking));
    if (!d->ev_in) LDB_CUDA(cudaEventCreateWithFlags(&d->ev_in, cudaEventDisableTiming));
    if (!d->ev_desc) LDB_CUDA(cudaEventCreateWithFlags(&d->ev_desc, cudaEventDisableTiming));
    return LD_OK;
}

// Drains a stream when the host API returns, on every path: a copy still
// running there must neither meet the next call's buffers nor read the
// caller's arrays after the call has returned.
struct DrainOnExit {
    cudaStream_t st = nullptr;
    ~DrainOnExit() {
        if (st) cudaStreamSynchronize(st);
    }
};

static int check_device() {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0)
        return fail(LD_ERR_NO_DEVICE, std::string("no CUDA device visible (") +
                                          (e == cudaSuccess ? "count 0" : cudaGetErrorString(e)) + ")");
    return LD_OK;
}

// ------------------------------------------------------ symmetry functions
static int build_sf(ld_descriptor *d, int ns, const double *cutoff, int n_types,
                    const int *codes, const int *sizes, const double *params) {
    if (ns <= 0 || !cutoff) return fail(LD_ERR_INVALID_ARG, "symmetry functions: n_species must be > 0");
    if (n_types < 0 || (n_types > 0 && (!codes || !sizes)))
        return fail(LD_ERR_INVALID_ARG, "symmetry functions: bad type list");
    std::vector<double> rcut(cutoff, cutoff + (size_t)ns * ns);
    std::vector<int> o2, t2, o3, t3, zi3;
    std::vector<double> a2, b2, P3, z3, l3, e3;
    struct Three { int o, t; double zeta, lam, eta; };
    std::vector<Three> three;
    std::vector<int> pt, pofs;
    std::vector<double> pv;
    int width = 0;
    size_t poff = 0;
    for (int b = 0; b < n_types; ++b) {
        const int t = codes[b], rows = sizes[2 * b], cols = sizes[2 * b + 1];
        if (t < 1 || t > 5) return fail(LD_ERR_INVALID_ARG, "symmetry functions: type code " + std::to_string(t) + " is not g1..g5");
        if (rows < 0 || cols < 0) return fail(LD_ERR_INVALID_ARG, "symmetry functions: negative block size");
        const int need = (t == 1) ? 0 : (t == 2) ? 2 : (t == 3) ? 1 : 3;
        if (rows > 0 && cols < need)
            return fail(LD_ERR_INVALID_ARG, "symmetry functions: g" + std::to_string(t) + " needs " +
                                                std::to_string(need) + " parameters per row");
        if (rows * cols > 0 && !params) return fail(LD_ERR_INVALID_ARG, "symmetry functions: params is NULL");
        for (int q = 0; q < rows; ++q) {
            const double *pp = params ? params + poff + (size_t)q * cols : nullptr;
            const int o = width + q;
            pt.push_back(t);
            pofs.push_back((int)(poff + (size_t)q * cols));
            for (int k = 0; k < 3; ++k) pv.push_back(k < need ? pp[k] : 0.0);
            if (t <= 3) {
                o2.push_back(o);
                t2.push_back(t);
                a2.push_back(cols > 0 ? pp[0] : 0.0);
                b2.push_back(cols > 1 ? pp[1] : 0.0);
            } else {
                three.push_back({o, t, pp[0], pp[1], pp[2]});
            }
        }
        poff += (size_t)rows * cols;
        width += rows;
    }
    std::stable_sort(three.begin(), three.end(), [](const Three &x, const Three &y) {
        if (x.t != y.t) return x.t < y.t;
        return x.eta < y.eta;
    });
    std::vector<int> ec3;
    {
        int prev_t = -1;
        double prev_eta = 0.0, base_eta = 0.0;
        for (auto &q : three) {
            int code = 0;
            if (q.t == prev_t && q.eta == prev_eta) {
                code = -1;
            } else if (q.t != prev_t) {
                base_eta = q.eta;   // smallest eta of the type group (sorted ascending)
                code = 0;
            } else if (base_eta > 0 && q.eta > 0) {
                const double ratio = q.eta / base_eta;
                const double k = std::floor(ratio + 0.5);
                if (k >= 2 && k <= 256 && std::fabs(ratio - k) <= 1e-9 * ratio) code = (int)k;
            }
            ec3.push_back(code);
            prev_t = q.t;
            prev_eta = q.eta;
        }
    }
    for (auto &q : three) {
        o3.push_back(q.o);
        t3.push_back(q.t);
        z3.push_back(q.zeta);
        l3.push_back(q.lam);
        e3.push_back(q.eta);
        P3.push_back(std::pow(2, 1 - q.zeta));
        const bool integral = q.zeta >= 0 && q.zeta <= 64 && std::floor(q.zeta) == q.zeta;
        zi3.push_back(integral ? (int)q.zeta : -1);
    }
    if ((int)o2.size() > 64 || (int)o3.size() > 64)
        return fail(LD_ERR_CAPACITY, "symmetry functions: at most 64 outputs of one body order are supported");
    SFDev &s = d->sf;
    // factored (grid) form for the specialised kernel, when the set has one
    {
        SFGrid g;
        bool ok = (int)o2.size() <= kSFG2;
        g.n2 = (int)o2.size();
        for (int q = 0; ok && q < g.n2; ++q) {
            g.t2[q] = t2[q];
            g.o2[q] = o2[q];
            g.a2[q] = a2[q];
            g.b2[q] = b2[q];
        }
        for (int ty = 0; ok && ty < 2; ++ty) {
            const int tcode = ty == 0 ? 4 : 5;
            std::vector<std::pair<double, double>> ang;   // (lambda, zeta), first appearance
            std::vector<double> rad;                      // ascending eta
            for (auto &q : three)
                if (q.t == tcode) {
                    if (std::find(ang.begin(), ang.end(), std::make_pair(q.lam, q.zeta)) == ang.end())
                        ang.push_back({q.lam, q.zeta});
                    if (std::find(rad.begin(), rad.end(), q.eta) == rad.end()) rad.push_back(q.eta);
                }
            std::sort(rad.begin(), rad.end());
            if ((int)ang.size() > kSFGA || (int)rad.size() > kSFGR) {
                ok = false;
                break;
            }
            g.na[ty] = (int)ang.size();
            g.nr[ty] = (int)rad.size();
            for (int a = 0; a < kSFGA; ++a)
                for (int r = 0; r < kSFGR; ++r) g.out[ty][a][r] = -1;
            for (int a = 0; a < g.na[ty]; ++a) {
                g.lam[ty][a] = ang[a].first;
                g.zeta[ty][a] = ang[a].second;
                g.P[ty][a] = std::pow(2, 1 - ang[a].second);
                const double z = ang[a].second;
                g.zi[ty][a] = (z >= 0 && z <= 64 && std::floor(z) == z) ? (int)z : -1;
            }
            for (int r = 0; r < g.nr[ty]; ++r) {
                g.eta[ty][r] = rad[r];
                int code = 0;
                if (r > 0 && rad[0] > 0 && rad[r] > 0) {
                    const double ratio = rad[r] / rad[0];
                    const double k = std::floor(ratio + 0.5);
                    if (k >= 2 && k <= 256 && std::fabs(ratio - k) <= 1e-9 * ratio) code = (int)k;
                }
                g.ec[ty][r] = code;
            }
            for (auto &q : three)
                if (q.t == tcode) {
                    const int a = (int)(std::find(ang.begin(), ang.end(), std::make_pair(q.lam, q.zeta)) - ang.begin());
                    const int r = (int)(std::find(rad.begin(), rad.end(), q.eta) - rad.begin());
                    if (g.out[ty][a][r] >= 0) {   // two outputs with identical parameters
                        ok = false;
                        break;
                    }
                    g.out[ty][a][r] = q.o;
                }
        }
        s.has_grid = ok;
        if (ok) s.grid = g;
    }
    s.ns = ns;
    s.width = width;
    s.n2 = (int)o2.size();
    s.n3 = (int)o3.size();
    Arena ar;
    ar.add(rcut, &s.rcut);
    std::vector<double> ircut(rcut.size());
    for (size_t k = 0; k < rcut.size(); ++k) ircut[k] = rcut[k] > 0.0 ? 1.0 / rcut[k] : 0.0;
    ar.add(ircut, &s.ircut);
    ar.add(o2, &s.o2);
    ar.add(t2, &s.t2);
    ar.add(a2, &s.a2);
    ar.add(b2, &s.b2);
    ar.add(o3, &s.o3);
    ar.add(t3, &s.t3);
    ar.add(P3, &s.P3);
    ar.add(z3, &s.z3);
    ar.add(l3, &s.l3);
    ar.add(e3, &s.e3);
    ar.add(zi3, &s.zi3);
    ar.add(ec3, &s.ec3);
    ar.add(pt, &s.pt);
    ar.add(pofs, &s.pofs);
    ar.add(pv, &s.pv);
    s.nparams = (int)poff;
    int rc = ar.upload(d->tables);
    if (rc) return rc;
    d->kind = LD_KIND_SYMMETRY_FUNCTIONS;
    d->width = width;
    return LD_OK;
}

// ------------------------------------------------------------- bispectrum
// Output triples per diagonal style (src/Bispectrum.cpp:84-193, 429-468).
static bool bs_outputs(int J, int style, std::vector<std::array<int, 3>> &out) {
    out.clear();
    switch (style) {
    case 0:
        for (int j1 = 0; j1 <= J; ++j1)
            for (int j2 = 0; j2 <= j1; ++j2)
                for (int j = j1 - j2; j <= std::min(J, j1 + j2); j += 2) out.push_back({j1, j2, j});
        return true;
    case 1:
        for (int j1 = 0; j1 <= J; ++j1)
            for (int j = 0; j <= std::min(J, 2 * j1); j += 2) out.push_back({j1, j1, j});
        return true;
    case 2:
        for (int j1 = 0; j1 <= J; ++j1) out.push_back({j1, j1, j1});
        return true;
    case 3:
        for (int j1 = 0; j1 <= J; ++j1)
            for (int j2 = 0; j2 <= j1; ++j2)
                for (int j = j1 - j2; j <= std::min(J, j1 + j2); j += 2)
                    if (j >= j1) out.push_back({j1, j2, j});
        return true;
    }
    return false;
}

struct BSTask {
    int t, ma, mb;
    long long cost;
};

// Longest-processing-time assignment of Z-element tasks to kBSThreads
// threads; tasks of one thread are stored contiguously, costliest first.
static void lpt_schedule(const std::vector<BSTask> &tasks_in, const std::vector<std::array<int, 4>> &trip,
                         const std::vector<int> &cgoff, std::vector<int> &toff, std::vector<int4> &packed,
                         int nt = kBSThreads) {
    std::vector<BSTask> tasks = tasks_in;
    std::stable_sort(tasks.begin(), tasks.end(), [](const BSTask &a, const BSTask &b) { return a.cost > b.cost; });
    std::vector<std::vector<BSTask>> bins(nt);
    using E = std::pair<long long, int>;
    std::priority_queue<E, std::vector<E>, std::greater<E>> heap;
    for (int b = 0; b < nt; ++b) heap.push({0, b});
    for (auto &tk : tasks) {
        E e = heap.top();
        heap.pop();
        bins[e.second].push_back(tk);
        e.first += tk.cost;
        heap.push(e);
    }
    toff.assign(nt + 1, 0);
    packed.clear();
    for (int b = 0; b < nt; ++b) {
        toff[b] = (int)packed.size();
        for (auto &tk : bins[b]) {
            const auto &tr = trip[tk.t];
            const int j = tr[2], nc = j / 2 + 1;
            int4 v;
            v.x = tr[0] | (tr[1] << 8) | (j << 16) | (tk.ma << 24);
            v.y = tk.mb;
            v.z = tr[3] + tk.ma * nc + tk.mb;
            v.w = cgoff[tk.t];
            packed.push_back(v);
        }
    }
    toff[nt] = (int)packed.size();
}

// Z tiles of the twojmax-specialised kernel: kZTileA x kZTileB outputs of
// one triple, scheduled over nt threads by longest processing time.  A tile
// made only of the middle column's mirror rows (never read) is dropped.
struct BSTile {
    int t, a0, b0, na, nb;
    long long cost;
};

static std::vector<BSTile> make_tiles(const std::set<int> &need, const std::vector<std::array<int, 4>> &trip) {
    std::vector<BSTile> tiles;
    for (int t : need) {
        const int j1 = trip[t][0], j2 = trip[t][1], j = trip[t][2], nc = j / 2 + 1;
        for (int a0 = 0; a0 <= j; a0 += kZTileA)
            for (int b0 = 0; b0 < nc; b0 += kZTileB) {
                const int na = std::min(kZTileA, j + 1 - a0), nb = std::min(kZTileB, nc - b0);
                if (j % 2 == 0 && b0 == j / 2 && 2 * a0 > j) continue;
                const int ca0 = (2 * a0 - j + j1 + j2) / 2, cb0 = (2 * b0 - j + j1 + j2) / 2;
                const int nma1 = std::min(j1, ca0 + na - 1) - std::max(0, ca0 - j2) + 1;
                const int nmb1 = std::min(j1, cb0 + nb - 1) - std::max(0, cb0 - j2) + 1;
                const long long steps = (long long)std::max(nma1, 0) * std::max(nmb1, 0);
                const long long cost = steps * (4 * kZTileA * kZTileB + 2 * kZTileA + 2 * kZTileB) +
                                       (long long)std::max(nma1, 0) * (2 * kZTileA * kZTileB + 8) + 24;
                tiles.push_back({t, a0, b0, na, nb, cost});
            }
    }
    return tiles;
}

static void lpt_tiles(const std::vector<BSTile> &tiles_in, const std::vector<std::array<int, 4>> &trip,
                      const std::vector<int> &cgoff, std::vector<int> &toff, std::vector<int4> &packed, int nt) {
    std::vector<BSTile> tiles = tiles_in;
    std::stable_sort(tiles.begin(), tiles.end(), [](const BSTile &a, const BSTile &b) { return a.cost > b.cost; });
    std::vector<std::vector<BSTile>> bins(nt);
    using E = std::pair<long long, int>;
    std::priority_queue<E, std::vector<E>, std::greater<E>> heap;
    for (int b = 0; b < nt; ++b) heap.push({0, b});
    for (auto &tk : tiles) {
        E e = heap.top();
        heap.pop();
        bins[e.second].push_back(tk);
        e.first += tk.cost;
        heap.push(e);
    }
    toff.assign(nt + 1, 0);
    packed.clear();
    for (int b = 0; b < nt; ++b) {
        toff[b] = (int)packed.size();
        for (auto &tk : bins[b]) {
            const auto &tr = trip[tk.t];
            int4 v;
            v.x = tr[0] | (tr[1] << 8) | (tr[2] << 16) | (tk.a0 << 24);
            v.y = tk.b0 | (tk.na << 8) | (tk.nb << 16);
            v.z = tr[3];
            v.w = cgoff[tk.t];
            packed.push_back(v);
        }
    }
    toff[nt] = (int)packed.size();
}

static int build_bs_impl(ld_descriptor *d, double rfac0, int J, int style, double rmin0, int switch_flag,
                         int bzero_flag, int ns, const double *cutoff, const double *weights);

static int build_bs(ld_descriptor *d, double rfac0, int J, int style, double rmin0, int switch_flag,
                    int bzero_flag, int ns, const double *cutoff, const double *weights) {
    try {
        return build_bs_impl(d, rfac0, J, style, rmin0, switch_flag, bzero_flag, ns, cutoff, weights);
    } catch (const std::exception &e) {
        return fail(LD_ERR_INVALID_ARG, std::string("bispectrum tables: ") + e.what());
    }
}

static int build_bs_impl(ld_descriptor *d, double rfac0, int J, int style, double rmin0, int switch_flag,
                         int bzero_flag, int ns, const double *cutoff, const double *weights) {
    if (J < 0 || J > kMaxTwoJ)
        return fail(J < 0 ? LD_ERR_INVALID_ARG : LD_ERR_CAPACITY,
                    "bispectrum: twojmax=" + std::to_string(J) + " outside 0.." + std::to_string(kMaxTwoJ));
    if (style < 0 || style > 3)
        return fail(LD_ERR_INVALID_ARG, "bispectrum: diagonalstyle " + std::to_string(style) + " is not a valid index");
    if (ns <= 0 || !cutoff || !weights) return fail(LD_ERR_INVALID_ARG, "bispectrum: species/cutoff/weights missing");
    const int D = J + 1;
    BSDev &b = d->bs;
    b.J = J;
    b.style = style;
    b.switch_flag = switch_flag;
    b.bzero_flag = bzero_flag;
    b.ns = ns;
    b.rfac0 = rfac0;
    b.rmin0 = rmin0;
    b.wself = 1.0;
    // cutoff of neighbour species js is element [js] of the flattened matrix
    // (the reference reads rcuts(iSpecies, jSpecies) from an Array2D whose
    // extents are never set, src/Bispectrum.cpp:271,305)
    std::vector<double> rcut_flat(cutoff, cutoff + ns);
    std::vector<double> wj(weights, weights + ns);
    std::vector<double> bzero(D, 0.0);
    if (bzero_flag)
        for (int j = 1; j <= J; ++j) bzero[j] = b.wself * b.wself * b.wself * j;
    std::vector<double> rootpq((size_t)D * D, 0.0);
    for (int p = 1; p <= J; ++p)
        for (int q = 1; q <= J; ++q) rootpq[p * D + q] = std::sqrt((double)p / q);
    std::vector<int> ublock(J + 2, 0), lblock(J + 2, 0);
    for (int j = 0; j <= J; ++j) {
        ublock[j + 1] = ublock[j] + (j + 1) * (j + 1);
        lblock[j + 1] = lblock[j] + (j + 1) * (j / 2 + 1);
    }
    b.nU = ublock[J + 1];
    b.nL = lblock[J + 1];
    std::vector<int> lel(b.nL);
    for (int j = 0; j <= J; ++j)
        for (int ma = 0; ma <= j; ++ma)
            for (int mb = 0; mb <= j / 2; ++mb) lel[lblock[j] + ma * (j / 2 + 1) + mb] = j | (ma << 8) | (mb << 16);
    // all j1 >= j2 triples
    std::vector<std::array<int, 4>> trip;  // j1, j2, j, zoff
    std::map<std::array<int, 3>, int> tindex;
    std::vector<int> cgoff;
    std::vector<double> cg;
    int zoff = 0;
    for (int j1 = 0; j1 <= J; ++j1)
        for (int j2 = 0; j2 <= j1; ++j2)
            for (int j = j1 - j2; j <= std::min(J, j1 + j2); j += 2) {
                tindex[{j1, j2, j}] = (int)trip.size();
                trip.push_back({j1, j2, j, zoff});
                zoff += (j + 1) * (j / 2 + 1);
                cgoff.push_back((int)cg.size());
                for (int m1 = 0; m1 <= j1; ++m1)
                    for (int m2 = 0; m2 <= j2; ++m2) cg.push_back(clebsch_gordan(j1, j2, j, m1, m2));
            }
    b.ntrip = (int)trip.size();
    b.nZall = zoff;
    b.ncg = (int)cg.size();
    // anti-diagonal packing: for output m of triple (j1, j2, j) the valid
    // entries are m1 + m2 = c + m, c = (j1 + j2 - j) / 2, m1 in
    // [max(0, c + m - j2), min(j1, c + m)]
    std::vector<double> cgp;
    std::vector<int> dbase, doffs;
    for (size_t t = 0; t < trip.size(); ++t) {
        const int j1 = trip[t][0], j2 = trip[t][1], j = trip[t][2], c = (j1 + j2 - j) / 2;
        doffs.push_back((int)dbase.size());
        for (int m = 0; m <= j; ++m) {
            const int sd = c + m, lo = std::max(0, sd - j2), hi = std::min(j1, sd);
            dbase.push_back((int)cgp.size() - lo);
            for (int m1 = lo; m1 <= hi; ++m1) cgp.push_back(cg[cgoff[t] + m1 * (j2 + 1) + (sd - m1)]);
        }
    }
    b.ncgp = (int)cgp.size();
    std::vector<std::array<int, 3>> outs;
    bs_outputs(J, style, outs);
    b.ncoeff = (int)outs.size();
    // An output whose (j1, j2, j) breaks the parity rule (style 2 with odd
    // j1) is never written by the reference's compute_bi, so it keeps the
    // zero its barray was allocated with (src/Bispectrum.cpp:391-427,
    // 450-454): otrip = -1 marks a constant-zero output.
    std::vector<int> otrip;
    d->bs_out_j1.clear();
    d->bs_out_j2.clear();
    d->bs_out_j.clear();
    for (auto &o : outs) {
        auto it = tindex.find(o);
        otrip.push_back(it == tindex.end() ? -1 : it->second);
        d->bs_out_j1.push_back(o[0]);
        d->bs_out_j2.push_back(o[1]);
        d->bs_out_j.push_back(o[2]);
    }
    // Gradient map.  B(a,b,c) = sum_{all ma,mb} Re(conj(U_c) Z_abc) is, by
    // the Clebsch-Gordan symmetries, also (a+1)/(c+1) sum Re(conj(U_a) Z_cba)
    // and (b+1)/(c+1) sum Re(conj(U_b) Z_cab); so dB/dU_x for each of its
    // three factors is a Z array of another triple, scaled.  betaj_t collects
    // those scaled dL/dB per triple t (first index ordered >= second, Z being
    // symmetric in its first two indices) and Y_j = sum_t betaj_t Z_t.
    std::vector<std::map<int, double>> M(trip.size());
    auto tri = [&](int x, int y, int z) { return tindex.at({std::max(x, y), std::min(x, y), z}); };
    for (int o = 0; o < (int)outs.size(); ++o) {
        if (otrip[o] < 0) continue;
        const int a = outs[o][0], bb = outs[o][1], c = outs[o][2];
        M[tri(a, bb, c)][o] += 1.0;
        M[tri(c, bb, a)][o] += (double)(c + 1) / (a + 1);
        M[tri(c, a, bb)][o] += (double)(c + 1) / (bb + 1);
    }
    std::vector<int> moff(trip.size() + 1, 0), mo;
    std::vector<double> mcoef;
    for (size_t t = 0; t < trip.size(); ++t) {
        moff[t] = (int)mo.size();
        for (auto &kv : M[t]) {
            mo.push_back(kv.first);
            mcoef.push_back(kv.second);
        }
    }
    moff[trip.size()] = (int)mo.size();
    std::vector<int> jtoff(J + 2, 0), jtlist;
    for (int j = 0; j <= J; ++j) {
        jtoff[j] = (int)jtlist.size();
        for (size_t t = 0; t < trip.size(); ++t)
            if (trip[t][2] == j && !M[t].empty()) jtlist.push_back((int)t);
    }
    jtoff[J + 1] = (int)jtlist.size();
    // Z-element tasks: (triple, ma, mb<=j/2) except the mirror rows of the
    // middle column, which neither B nor Y reads.
    std::set<int> need_f;
    for (int t : otrip)
        if (t >= 0) need_f.insert(t);
    std::set<int> need_v = need_f;
    for (size_t t = 0; t < trip.size(); ++t)
        if (!M[t].empty()) need_v.insert((int)t);
    auto make_tasks = [&](const std::set<int> &need, long long &inner) {
        std::vector<BSTask> tasks;
        inner = 0;
        for (int t : need) {
            const int j1 = trip[t][0], j2 = trip[t][1], j = trip[t][2];
            for (int mb = 0; 2 * mb <= j; ++mb)
                for (int ma = 0; ma <= j; ++ma) {
                    if (j % 2 == 0 && mb == j / 2 && ma > j / 2) continue;
                    const int na = std::min(j1, (2 * ma - j + j2 + j1) / 2) - std::max(0, (2 * ma - j - j2 + j1) / 2) + 1;
                    const int nb = std::min(j1, (2 * mb - j + j2 + j1) / 2) - std::max(0, (2 * mb - j - j2 + j1) / 2) + 1;
                    const long long c = (long long)std::max(na, 0) * std::max(nb, 0);
                    inner += c;
                    tasks.push_back({t, ma, mb, c + 2});
                }
        }
        return tasks;
    };
    std::vector<int> toff_f, toff_v, toff2_f, toff2_v;
    std::vector<int4> task_f, task_v, task2_f, task2_v;
    b.nt2 = 32 * bs2_warps(J);
    {
        auto tf = make_tasks(need_f, d->bs_inner_fwd);
        lpt_schedule(tf, trip, cgoff, toff_f, task_f);
        lpt_tiles(make_tiles(need_f, trip), trip, doffs, toff2_f, task2_f, b.nt2);
        auto tv = make_tasks(need_v, d->bs_inner_vjp);
        lpt_schedule(tv, trip, cgoff, toff_v, task_v);
        lpt_tiles(make_tiles(need_v, trip), trip, doffs, toff2_v, task2_v, b.nt2);
        d->bs_tasks_fwd = (int)tf.size();
        d->bs_tasks_vjp = (int)tv.size();
    }
    // rows-in-lanes Z schedule: one item per output row (j, ma) of a layer
    // with needed triples; its cost counts the window steps of every triple
    // of the layer; items go to the least loaded warp, largest first
    std::vector<int> oslot(outs.size(), -1), tslot(trip.size(), -1);
    b.nbslot = 0;
    for (size_t o = 0; o < outs.size(); ++o) {
        const int t = otrip[o];
        if (t < 0) continue;
        if (tslot[t] < 0) tslot[t] = b.nbslot++;
        oslot[o] = tslot[t];
    }
    // column weights by window step: G_t[mb][q] = cg(c + q - mb, mb)
    std::vector<double> zg;
    std::vector<int> gofs(trip.size(), 0);
    for (size_t t = 0; t < trip.size(); ++t) {
        const int j1 = trip[t][0], j2 = trip[t][1], j = trip[t][2], c = (j1 + j2 - j) / 2;
        const int nc = j / 2 + 1, ncp = nc + (nc & 1), nst = std::min(j2, c + nc - 1) + 1;
        gofs[t] = (int)zg.size();
        for (int mb = 0; mb < nst; ++mb)
            for (int q = 0; q < ncp; ++q) {
                const int mb1 = c + q - mb;
                zg.push_back(q < nc && mb1 >= 0 && mb1 <= j1 ? cg[cgoff[t] + mb1 * (j2 + 1) + mb] : 0.0);
            }
    }
    // with_y: every layer gets items, also layers without needed triples,
    // whose items write zero Y rows (the pair kernel reads Y of all layers)
    auto zsched = [&](const std::set<int> &need, bool with_y, std::vector<int> &zoff, std::vector<int> &zitem,
                      std::vector<int> &ztoff, std::vector<int4> &ztl) {
        ztoff.assign(J + 2, 0);
        ztl.clear();
        std::vector<std::pair<long long, int>> items;
        for (int j = 0; j <= J; ++j) {
            ztoff[j] = (int)ztl.size();
            const int nc = j / 2 + 1;
            for (int t : need) {
                if (trip[t][2] != j) continue;
                const int j1 = trip[t][0], j2 = trip[t][1], c = (j1 + j2 - j) / 2;
                ztl.push_back(make_int4(j1 | (j2 << 8) | (c << 16), gofs[t], cgoff[t], t | ((tslot[t] + 1) << 16)));
            }
            const int t0 = ztoff[j], t1 = (int)ztl.size();
            if (t1 == t0 && !with_y) continue;
            for (int ma = 0; ma <= j; ++ma) {
                long long cost = 16;
                for (int k = t0; k < t1; ++k) {
                    const int j1 = ztl[k].x & 0xff, j2 = (ztl[k].x >> 8) & 0xff, c = (ztl[k].x >> 16) & 0xff;
                    const int rows = std::min(j2, c + ma) - std::max(0, c + ma - j1) + 1;
                    const int steps = std::min(j2, c + nc - 1) + 1;
                    cost += (long long)rows * (steps * (6 * nc + 6) + 4 * nc + 16) + 8 * nc + 32;
                }
                items.push_back({cost, j | (ma << 8)});
            }
        }
        ztoff[J + 1] = (int)ztl.size();
        std::stable_sort(items.begin(), items.end(),
                         [](const std::pair<long long, int> &x, const std::pair<long long, int> &y) {
                             return x.first > y.first;
                         });
        std::vector<std::vector<int>> bins(kZWarps);
        std::vector<long long> load(kZWarps, 0);
        for (auto &it : items) {
            const int w = (int)(std::min_element(load.begin(), load.end()) - load.begin());
            bins[w].push_back(it.second);
            load[w] += it.first;
        }
        zoff.assign(kZWarps + 1, 0);
        zitem.clear();
        for (int w = 0; w < kZWarps; ++w) {
            zoff[w] = (int)zitem.size();
            zitem.insert(zitem.end(), bins[w].begin(), bins[w].end());
        }
        zoff[kZWarps] = (int)zitem.size();
    };
    std::vector<int> zoff_f, zitem_f, ztoff_f, zoff_v, zitem_v, ztoff_v;
    std::vector<int4> ztl_f, ztl_v;
    zsched(need_f, false, zoff_f, zitem_f, ztoff_f, ztl_f);
    zsched(need_v, true, zoff_v, zitem_v, ztoff_v, ztl_v);
    std::vector<int4> trip4;
    for (auto &t : trip) trip4.push_back(make_int4(t[0], t[1], t[2], t[3]));
    Arena ar;
    ar.add(rcut_flat, &b.rcut_flat);
    std::vector<double> ang_flat(ns), isw_flat(ns);
    for (int k = 0; k < ns; ++k) {
        const double span = rcut_flat[k] - rmin0;
        ang_flat[k] = span > 0.0 ? rfac0 * 3.1415926535897932 / span : 0.0;
        isw_flat[k] = span > 0.0 ? 1.0 / span : 0.0;
    }
    ar.add(ang_flat, &b.ang_flat);
    ar.add(isw_flat, &b.isw_flat);
    ar.add(wj, &b.wj);
    ar.add(bzero, &b.bzero);
    ar.add(rootpq, &b.rootpq);
    ar.add(ublock, &b.ublock);
    ar.add(lblock, &b.lblock);
    ar.add(trip4, &b.trip);
    ar.add(cgoff, &b.cgoff);
    ar.add(cgp, &b.cgp);
    ar.add(dbase, &b.dbase);
    ar.add(cg, &b.cg);
    ar.add(otrip, &b.otrip);
    ar.add(moff, &b.moff);
    ar.add(mo, &b.mo);
    ar.add(mcoef, &b.mcoef);
    ar.add(jtoff, &b.jtoff);
    ar.add(jtlist, &b.jtlist);
    ar.add(lel, &b.lel);
    ar.add(toff_f, &b.toff_f);
    ar.add(task_f, &b.task_f);
    ar.add(toff_v, &b.toff_v);
    ar.add(task_v, &b.task_v);
    ar.add(toff2_f, &b.toff2_f);
    ar.add(task2_f, &b.task2_f);
    ar.add(toff2_v, &b.toff2_v);
    ar.add(task2_v, &b.task2_v);
    ar.add(oslot, &b.oslot);
    ar.add(zg, &b.zg);
    b.nzg = (int)zg.size();
    ar.add(zoff_f, &b.zoff_f);
    ar.add(zitem_f, &b.zitem_f);
    ar.add(ztoff_f, &b.ztoff_f);
    ar.add(ztl_f, &b.ztl_f);
    ar.add(zoff_v, &b.zoff_v);
    ar.add(zitem_v, &b.zitem_v);
    ar.add(ztoff_v, &b.ztoff_v);
    ar.add(ztl_v, &b.ztl_v);
    int rc = ar.upload(d->tables);
    if (rc) return rc;
    d->kind = LD_KIND_BISPECTRUM;
    d->width = b.ncoeff;
    return LD_OK;
}

// ------------------------------------------------------------ host staging
struct HostRows {
    int n_rows = 0;
    std::vector<int> centre;   // empty: centre == row
    std::vector<long long> off;
    int maxn = 0;
    long long nnz = 0;
};

static int make_rows(int n_rows, const int *counts, HostRows &h) {
    h.n_rows = n_rows;
    h.off.assign((size_t)n_rows + 1, 0);
    h.maxn = 0;
    for (int r = 0; r < n_rows; ++r) {
        if (counts[r] < 0) return fail(LD_ERR_INVALID_ARG, "number_of_neighs[" + std::to_string(r) + "] < 0");
        h.off[r + 1] = h.off[r] + counts[r];
        h.maxn = std::max(h.maxn, counts[r]);
    }
    h.nnz = h.off[n_rows];
    return LD_OK;
}

// The shapes: centre rows inside the coordinates.
static int validate_rows(const HostRows &h, int n_total) {
    if (!h.centre.empty()) {
        for (int r = 0; r < h.n_rows; ++r)
            if (h.centre[r] < 0 || h.centre[r] >= n_total)
                return fail(LD_ERR_INVALID_ARG, "centre atom " + std::to_string(h.centre[r]) + " outside coords");
    } else if (h.n_rows > n_total) {
        return fail(LD_ERR_INVALID_ARG, "n_atoms exceeds the number of coordinates");
    }
    return LD_OK;
}

// The indices: species inside the descriptor's list, neighbours inside the
// coordinates.
static int validate_indices(const ld_descriptor *d, const HostRows &h, int n_total, const int *species,
                            const int *nbl) {
    const int ns = d->kind == LD_KIND_SYMMETRY_FUNCTIONS ? d->sf.ns : d->bs.ns;
    // an unsigned compare per value folded into one flag (no early exit, so
    // the loop vectorises); the first offender is looked for only on failure
    auto any_outside = [](const int *v, long long n, int hi) {
        unsigned bad = 0;
        for (long long q = 0; q < n; ++q) bad |= (unsigned)((unsigned)v[q] >= (unsigned)hi);
        return bad != 0;
    };
    if (any_outside(species, n_total, ns))
        for (int a = 0; a < n_total; ++a)
            if (species[a] < 0 || species[a] >= ns)
                return fail(LD_ERR_INVALID_ARG, "species[" + std::to_string(a) + "]=" + std::to_string(species[a]) +
                                                    " outside 0.." + std::to_string(ns - 1));
    if (any_outside(nbl, h.nnz, n_total))
        for (long long q = 0; q < h.nnz; ++q)
            if (nbl[q] < 0 || nbl[q] >= n_total)
                return fail(LD_ERR_INVALID_ARG, "neighbor_list[" + std::to_string(q) + "]=" +
                                                    std::to_string(nbl[q]) + " outside 0.." +
                                                    std::to_string(n_total - 1));
    return LD_OK;
}

static int validate(const ld_descriptor *d, const HostRows &h, int n_total, const int *species,
                    const int *nbl) {
    const int rc = validate_indices(d, h, n_total, species, nbl);
    return rc ? rc : validate_rows(h, n_total);
}

int launch_rows(ld_descriptor *d, const RowArgs &a0, cudaStream_t s) {
    NvtxRange range(d->kind == LD_KIND_SYMMETRY_FUNCTIONS
                        ? (a0.dE ? "ld: symmetry functions desc+VJP" : "ld: symmetry functions desc")
                        : (a0.dE ? "ld: bispectrum desc+VJP" : "ld: bispectrum desc"));
    RowArgs a = a0;
    a.sf_warps = d->tune[LD_TUNE_SF_WARPS];
    a.ctas_per_sm = d->tune[LD_TUNE_CTAS_PER_SM];
    a.pair_grid_mult = d->tune[LD_TUNE_PAIR_GRID_MULT];
    // the allocation-free entry point never takes the queue counter
    // the row queue: 1 always, 2 never, 0 (built-in) for batches of at least
    // 8192 rows, whose rows of uneven cost balance better when claimed from a
    // counter than in grid-stride order
    const int dq = d->tune[LD_TUNE_DYNAMIC_QUEUE];
    a.dynamic_queue = a0.fused_only ? 0 : (dq == 1 ? 1 : dq == 2 ? 0 : (a0.n_rows >= 8192 ? 1 : 0));
    a.force_generic = d->tune[LD_TUNE_SF_GENERIC] != 0;
    if (d->kind == LD_KIND_SYMMETRY_FUNCTIONS) {
        // one fused pass: dE is read from the first kernel on, and the
        // descriptors are final with the last
        if (a.in_ready) LDB_CUDA(cudaStreamWaitEvent(s, a.in_ready, 0));
        const int rc = sf_launch(d->sf, a, s);
        if (rc == LD_OK && a.desc_done) LDB_CUDA(cudaEventRecord(a.desc_done, s));
        return rc;
    }
    return bs_launch(d->bs, a, s);
}

static int status_error(ld_descriptor *d, cudaStream_t s, int st) {
    if (st != 0) {
        LDB_CUDA(cudaMemsetAsync(d->status.p, 0, sizeof(int), s));
        LDB_CUDA(cudaStreamSynchronize(s));
        if (st == kDevCapacity) return fail(LD_ERR_CAPACITY, "a centre has more neighbours than max_neigh");
        if (st == kDevTimeout) return fail(LD_ERR_TIMEOUT, "a kernel's bounded wait for its shared-memory tile ran out");
        return fail(LD_ERR_INVALID_ARG, "a neighbour or centre index lies outside the coordinates");
    }
    return LD_OK;
}

static int read_status(ld_descriptor *d, cudaStream_t s) {
    if (!d->status.p) return LD_OK;
    int st = 0;
    LDB_CUDA(cudaMemcpyAsync(&st, d->status.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    LDB_CUDA(cudaStreamSynchronize(s));
    return status_error(d, s, st);
}

static int ensure_status(ld_descriptor *d) {
    if (d->status.p) return LD_OK;
    int rc = d->status.ensure(sizeof(int) * 4);
    if (rc) return rc;
    LDB_CUDA(cudaMemset(d->status.p, 0, sizeof(int) * 4));
    // a pinned copy of the word, read back with a call's results (no pinned
    // memory: read_status's own round trip instead)
    if (!d->hstatus && cudaHostAlloc((void **)&d->hstatus, 64, cudaHostAllocDefault) != cudaSuccess) {
        cudaGetLastError();
        d->hstatus = nullptr;
    }
    return LD_OK;
}

// Generic host-buffer pass: stage, launch, copy back.  dE == nullptr means
// forward only.  dcoords (n_total*3) and desc are overwritten when given.
// jac_width > 0 turns rows into (centre, component) pairs of a Jacobian.
static int host_pass_impl(ld_descriptor *d, HostRows &h, int n_total, const int *species, const int *nbl,
                          const double *coords, const double *dE, double *dcoords, double *desc,
                          int jac_width);

static int host_pass(ld_descriptor *d, HostRows &h, int n_total, const int *species, const int *nbl,
                     const double *coords, const double *dE, double *dcoords, double *desc,
                     int jac_width = 0) {
    NvtxRange range("ld: host-buffer call (stage, launch, read back)");
    try {
        return host_pass_impl(d, h, n_total, species, nbl, coords, dE, dcoords, desc, jac_width);
    } catch (const std::bad_alloc &) {
        return fail(LD_ERR_OOM, "host allocation failed");
    } catch (const std::exception &e) {
        return fail(LD_ERR_INVALID_ARG, e.what());
    }
}

static int host_pass_impl(ld_descriptor *d, HostRows &h, int n_total, const int *species, const int *nbl,
                          const double *coords, const double *dE, double *dcoords, double *desc,
                          int jac_width) {
    if (!d) return fail(LD_ERR_INVALID_ARG, "descriptor handle is NULL");
    if (h.n_rows < 0 || n_total < 0) return fail(LD_ERR_INVALID_ARG, "negative size");
    if (h.n_rows > 0 && (!species || !coords || (h.nnz > 0 && !nbl)))
        return fail(LD_ERR_INVALID_ARG, "NULL input array");
    if (dE && h.n_rows > 0 && !dcoords) return fail(LD_ERR_INVALID_ARG, "d_coords is NULL");
    if (!dE && h.n_rows > 0 && !desc) return fail(LD_ERR_INVALID_ARG, "desc is NULL");
    int rc = validate_rows(h, n_total);
    if (rc) return rc;
    if (h.n_rows == 0 && !dE) return validate_indices(d, h, n_total, species, nbl);
    std::lock_guard<std::mutex> lk(d->mu);
    if ((rc = ensure_stream(d)) || (rc = ensure_status(d))) return rc;
    cudaStream_t s = d->stream;
    const int W = d->width;
    const int rows = jac_width > 0 ? h.n_rows * jac_width : h.n_rows;
    if ((rc = d->species.ensure(sizeof(int) * std::max(n_total, 1))) || (rc = d->nbl.ensure(sizeof(int) * std::max<long long>(h.nnz, 1))) ||
        (rc = d->off.ensure(sizeof(long long) * (h.n_rows + 1))) || (rc = d->coords.ensure(sizeof(double) * 3 * std::max(n_total, 1))))
        return rc;
    // from the first upload on, every return waits for the handle's stream:
    // an error return must not leave copies from the caller's arrays running
    DrainOnExit drain_s;
    drain_s.st = s;
    LDB_CUDA(cudaMemcpyAsync(d->species.p, species, sizeof(int) * n_total, cudaMemcpyHostToDevice, s));
    if (h.nnz) LDB_CUDA(cudaMemcpyAsync(d->nbl.p, nbl, sizeof(int) * h.nnz, cudaMemcpyHostToDevice, s));
    LDB_CUDA(cudaMemcpyAsync(d->off.p, h.off.data(), sizeof(long long) * (h.n_rows + 1), cudaMemcpyHostToDevice, s));
    LDB_CUDA(cudaMemcpyAsync(d->coords.p, coords, sizeof(double) * 3 * n_total, cudaMemcpyHostToDevice, s));
    RowArgs a;
    a.n_rows = rows;
    a.species = d->species.as<int>();
    a.nbl = d->nbl.as<int>();
    a.off = d->off.as<long long>();
    a.max_neigh = std::max(h.maxn, 1);
    a.coords = d->coords.as<double>();
    a.n_total = n_total;
    a.status = d->status.as<int>();
    std::vector<int> centre, list;
    if (jac_width > 0) {
        centre.resize(rows);
        list.resize(rows);
        for (int r = 0; r < rows; ++r) {
            const int base = r / jac_width;
            list[r] = base;
            centre[r] = h.centre.empty() ? base : h.centre[base];
        }
    } else if (!h.centre.empty()) {
        centre = h.centre;
    }
    if (!centre.empty()) {
        if ((rc = d->centre.ensure(sizeof(int) * rows))) return rc;
        LDB_CUDA(cudaMemcpyAsync(d->centre.p, centre.data(), sizeof(int) * rows, cudaMemcpyHostToDevice, s));
        a.row_centre = d->centre.as<int>();
    }
    if (!list.empty()) {
        if ((rc = d->list.ensure(sizeof(int) * rows))) return rc;
        LDB_CUDA(cudaMemcpyAsync(d->list.p, list.data(), sizeof(int) * rows, cudaMemcpyHostToDevice, s));
        a.row_list = d->list.as<int>();
    }
    std::vector<double> onehot;
    DrainOnExit drain;
    if (desc || !dE) {
        if ((rc = d->desc.ensure(sizeof(double) * std::max<size_t>((size_t)rows * W, 1)))) return rc;
        a.desc = d->desc.as<double>();
    }
    if (dE) {
        const size_t ndc = jac_width > 0 ? (size_t)rows * 3 * n_total : (size_t)3 * n_total;
        if ((rc = d->dE.ensure(sizeof(double) * std::max<size_t>((size_t)rows * W, 1))) ||
            (rc = d->dc.ensure(sizeof(double) * std::max<size_t>(ndc, 1))))
            return rc;
        if (jac_width > 0) {
            onehot.assign((size_t)rows * W, 0.0);
            for (int r = 0; r < rows; ++r) onehot[(size_t)r * W + (r % jac_width)] = 1.0;
            LDB_CUDA(cudaMemcpyAsync(d->dE.p, onehot.data(), sizeof(double) * onehot.size(), cudaMemcpyHostToDevice, s));
            a.dc_stride = 3LL * n_total;
        } else if (rows > 0) {
            if ((rc = ensure_stream2(d))) return rc;
            drain.st = d->stream2;
            LDB_CUDA(cudaMemcpyAsync(d->dE.p, dE, sizeof(double) * (size_t)rows * W, cudaMemcpyHostToDevice,
                                     d->stream2));
            LDB_CUDA(cudaEventRecord(d->ev_in, d->stream2));
            a.in_ready = d->ev_in;
        }
        LDB_CUDA(cudaMemsetAsync(d->dc.p, 0, sizeof(double) * ndc, s));
        a.dE = d->dE.as<double>();
        a.dcoords = d->dc.as<double>();
        if (jac_width > 0) a.desc = nullptr;
    }
    // the indices are checked on the host while the uploads run; no kernel
    // is launched before they pass (the guards above drain both streams on
    // this and every other error return)
    if ((rc = validate_indices(d, h, n_total, species, nbl))) return rc;
    if (rows > 0) {
        // the kernels' work space lives in a grow-only buffer of the handle,
        // so repeated calls allocate nothing
        size_t wb = 0;
        if ((rc = ld_rows_work_bytes(d, rows, dE ? 1 : 0, &wb))) return rc;
        if ((rc = d->work.ensure(wb))) return rc;
        a.work = d->work.p;
        a.work_bytes = wb;
        // with a gradient, the descriptors are read back on the second stream
        // as soon as they are final (issued before the gradient's copy, which
        // blocks the host when its destination is pageable)
        const bool early_desc = desc && a.desc && a.in_ready;
        if (early_desc) a.desc_done = d->ev_desc;
        if ((rc = launch_rows(d, a, s))) return rc;
        if (early_desc) {
            LDB_CUDA(cudaStreamWaitEvent(d->stream2, d->ev_desc, 0));
            LDB_CUDA(cudaMemcpyAsync(desc, d->desc.p, sizeof(double) * (size_t)rows * W, cudaMemcpyDeviceToHost,
                                     d->stream2));
            desc = nullptr;
        }
    }
    if (dE) {
        const size_t ndc = jac_width > 0 ? (size_t)rows * 3 * n_total : (size_t)3 * n_total;
        LDB_CUDA(cudaMemcpyAsync(dcoords, d->dc.p, sizeof(double) * ndc, cudaMemcpyDeviceToHost, s));
    }
    if (desc && a.desc && rows > 0)
        LDB_CUDA(cudaMemcpyAsync(desc, d->desc.p, sizeof(double) * (size_t)rows * W, cudaMemcpyDeviceToHost, s));
    if (!d->hstatus) {
        LDB_CUDA(cudaStreamSynchronize(s));
        drain_s.st = nullptr;
        if (drain.st) LDB_CUDA(cudaStreamSynchronize(drain.st));
        return read_status(d, s);
    }
    // the status word travels with the results: one synchronisation
    LDB_CUDA(cudaMemcpyAsync(d->hstatus, d->status.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    LDB_CUDA(cudaStreamSynchronize(s));
    drain_s.st = nullptr;
    if (drain.st) LDB_CUDA(cudaStreamSynchronize(drain.st));
    return status_error(d, s, *d->hstatus);
}

static void batch_centres(int n_configs, const int *n_atoms, const int *config_ptr, std::vector<int> &c) {
    c.clear();
    for (int k = 0; k < n_configs; ++k)
        for (int j = 0; j < n_atoms[k]; ++j) c.push_back(j + config_ptr[k]);
}

// ------------------------------------------------------- parameter files
// FileIOUtils semantics (include/file_io_utils.hpp): data lines skip blank
// lines and lines whose first character is '#'; numbers are read from the
// whitespace tokens that parse as numbers (a leading numeric prefix counts).
struct LineReader {
    std::ifstream f;
    bool next(std::string &line) {
        line.clear();
        while (line.empty() || line[0] == '#') {
            if (!std::getline(f, line)) return false;
        }
        return true;
    }
};
static bool tok_ints(const std::string &line, int n, std::vector<int> &out) {
    std::stringstream ss(line);
    std::string t;
    out.clear();
    while ((int)out.size() < n && (ss >> t)) {
        try {
            out.push_back(std::stoi(t));
        } catch (...) {
        }
    }
    return (int)out.size() == n;
}
static bool tok_doubles(const std::string &line, int n, std::vector<double> &out) {
    std::stringstream ss(line);
    std::string t;
    out.clear();
    while ((int)out.size() < n && (ss >> t)) {
        try {
            out.push_back(std::stod(t));
        } catch (...) {
        }
    }
    return (int)out.size() == n;
}
static bool tok_strings(const std::string &line, int n, std::vector<std::string> &out) {
    std::stringstream ss(line);
    std::string t;
    out.clear();
    while ((int)out.size() < n && (ss >> t)) out.push_back(t);
    return (int)out.size() == n;
}

// Species block shared by both formats: n_species lines "A B rcut".  The
// reference reads exactly n_species such lines and orders species names
// as a sorted set (src/SymmetryFunctions.cpp:302-324).
static int parse_species(LineReader &lr, int n_species, std::vector<std::string> &species,
                         std::vector<double> &cutoff) {
    std::map<std::pair<std::string, std::string>, double> pc;
    std::set<std::string> names;
    std::string line;
    std::vector<std::string> s;
    std::vector<double> v;
    for (int k = 0; k < n_species; ++k) {
        if (!lr.next(line) || !tok_strings(line, 2, s) || !tok_doubles(line, 1, v))
            return fail(LD_ERR_PARSE, "parameter file: bad species cutoff line");
        names.insert(s[0]);
        names.insert(s[1]);
        pc[{s[0], s[1]}] = v[0];
        pc[{s[1], s[0]}] = v[0];
    }
    species.assign(names.begin(), names.end());
    const int ns = n_species;
    cutoff.assign((size_t)ns * ns, 0.0);
    for (int a = 0; a < ns; ++a)
        for (int b = 0; b < ns; ++b) {
            if (a >= (int)species.size() || b >= (int)species.size()) continue;
            auto it = pc.find({species[a], species[b]});
            cutoff[(size_t)a * ns + b] = it == pc.end() ? 0.0 : it->second;
        }
    return LD_OK;
}

// What a parameter file defines, before any device table is built.
struct ParsedFile {
    int kind = -1, ns = 0;
    std::vector<std::string> species;
    std::vector<double> cutoff;                 // ns x ns
    std::vector<int> codes, sizes;              // symmetry functions
    std::vector<double> params;
    double rfac0 = 0, rmin0 = 0;                // bispectrum
    int twojmax = 0, style = 0, sw = 0, bz = 0;
    std::vector<double> weights;
};

static int parse_file_impl(ParsedFile &pf, const char *path, int kind);

static int parse_file(ParsedFile &pf, const char *path, int kind) {
    try {
        return parse_file_impl(pf, path, kind);
    } catch (const std::exception &e) {
        return fail(LD_ERR_PARSE, std::string("parameter file: ") + e.what());
    }
}

static int parse_file_impl(ParsedFile &pf, const char *path, int kind) {
    if (!path) return fail(LD_ERR_INVALID_ARG, "path is NULL");
    if (kind != LD_KIND_SYMMETRY_FUNCTIONS && kind != LD_KIND_BISPECTRUM)
        return fail(LD_ERR_INVALID_KIND, "descriptor kind " + std::to_string(kind) +
                                             " is not supported (SOAP and Xi are out of scope)");
    LineReader lr;
    lr.f.open(path);
    if (!lr.f.is_open()) return fail(LD_ERR_PARSE, std::string("Could not open file: ") + path);
    std::string line;
    std::vector<int> iv;
    std::vector<double> dv;
    std::vector<std::string> sv;
    if (!lr.next(line) || !tok_strings(line, 1, sv)) return fail(LD_ERR_PARSE, "parameter file: cutoff type");
    if (!lr.next(line) || !tok_ints(line, 1, iv) || iv[0] <= 0) return fail(LD_ERR_PARSE, "parameter file: number of species");
    pf.kind = kind;
    pf.ns = iv[0];
    int rc = parse_species(lr, pf.ns, pf.species, pf.cutoff);
    if (rc) return rc;
    if (kind == LD_KIND_SYMMETRY_FUNCTIONS) {
        // src/SymmetryFunctions.cpp:326-406.  The parameter vector is shared
        // across types and never cleared, and each type's block is read from
        // the START of that vector -- reproduced as is.
        if (!lr.next(line) || !tok_ints(line, 1, iv)) return fail(LD_ERR_PARSE, "parameter file: number of types");
        const int nt = iv[0];
        std::vector<std::string> names;
        std::vector<double> acc;
        std::map<std::string, std::vector<double>> per_type;
        std::map<std::string, std::pair<int, int>> type_sizes;
        for (int t = 0; t < nt; ++t) {
            if (!lr.next(line) || !tok_strings(line, 1, sv) || !tok_ints(line, 2, iv))
                return fail(LD_ERR_PARSE, "parameter file: symmetry-function type line");
            names.push_back(sv[0]);
            type_sizes[sv[0]] = {iv[0], iv[1]};
            for (int r = 0; r < iv[0]; ++r) {
                if (!lr.next(line) || !tok_doubles(line, iv[1], dv)) return fail(LD_ERR_PARSE, "parameter file: parameter row");
                acc.insert(acc.end(), dv.begin(), dv.end());
                per_type[sv[0]] = acc;
            }
        }
        if (!lr.next(line)) return fail(LD_ERR_PARSE, "parameter file: normalize flag");
        if (!lr.next(line) || !tok_ints(line, 1, iv)) return fail(LD_ERR_PARSE, "parameter file: descriptor size");
        for (auto &nm : names) {
            int code = 0;
            if (nm == "g1") code = 1;
            else if (nm == "g2") code = 2;
            else if (nm == "g3") code = 3;
            else if (nm == "g4") code = 4;
            else if (nm == "g5") code = 5;
            if (!code) return fail(LD_ERR_PARSE, "parameter file: unknown symmetry function " + nm);
            const auto sz = type_sizes[nm];
            pf.codes.push_back(code);
            pf.sizes.push_back(sz.first);
            pf.sizes.push_back(sz.second);
            const auto &src = per_type[nm];
            const size_t need = (size_t)sz.first * sz.second;
            if (src.size() < need) return fail(LD_ERR_PARSE, "parameter file: too few parameters");
            pf.params.insert(pf.params.end(), src.begin(), src.begin() + need);
        }
        return LD_OK;
    }
    // src/Bispectrum.cpp:909-1006: jmax (doubled), rfac0, diagonalstyle,
    // rmin0, switch flag, bzero flag, one weight per species
    if (!lr.next(line) || !tok_ints(line, 1, iv)) return fail(LD_ERR_PARSE, "parameter file: jmax");
    pf.twojmax = 2 * iv[0];
    if (!lr.next(line) || !tok_doubles(line, 1, dv)) return fail(LD_ERR_PARSE, "parameter file: rfac0");
    pf.rfac0 = dv[0];
    if (!lr.next(line) || !tok_ints(line, 1, iv)) return fail(LD_ERR_PARSE, "parameter file: diagonalstyle");
    pf.style = iv[0];
    if (!lr.next(line) || !tok_doubles(line, 1, dv)) return fail(LD_ERR_PARSE, "parameter file: rmin0");
    pf.rmin0 = dv[0];
    if (!lr.next(line) || !tok_ints(line, 1, iv)) return fail(LD_ERR_PARSE, "parameter file: switch flag");
    pf.sw = iv[0];
    if (!lr.next(line) || !tok_ints(line, 1, iv)) return fail(LD_ERR_PARSE, "parameter file: bzero flag");
    pf.bz = iv[0];
    if (!lr.next(line) || !tok_doubles(line, (int)pf.species.size(), dv)) return fail(LD_ERR_PARSE, "parameter file: weights");
    pf.weights.assign(pf.ns, 0.0);
    for (int k = 0; k < pf.ns && k < (int)dv.size(); ++k) pf.weights[k] = dv[k];
    return LD_OK;
}

static int build_parsed(ld_descriptor *d, const ParsedFile &pf) {
    if (pf.kind == LD_KIND_SYMMETRY_FUNCTIONS)
        return build_sf(d, pf.ns, pf.cutoff.data(), (int)pf.codes.size(), pf.codes.data(), pf.sizes.data(),
                        pf.params.data());
    return build_bs(d, pf.rfac0, pf.twojmax, pf.style, pf.rmin0, pf.sw, pf.bz, pf.ns, pf.cutoff.data(),
                    pf.weights.data());
}

// "key = values" text of a parsed file (ld_describe_parameter_file)
static std::string describe_parsed(const ParsedFile &pf) {
    std::ostringstream o;
    o.precision(17);
    auto list = [&o](const char *key, const auto &v) {
        o << key << " =";
        for (const auto &x : v) o << ' ' << x;
        o << '\n';
    };
    o << "kind = " << pf.kind << '\n' << "n_species = " << pf.ns << '\n';
    list("species", pf.species);
    list("cutoff_matrix", pf.cutoff);
    if (pf.kind == LD_KIND_SYMMETRY_FUNCTIONS) {
        list("type_codes", pf.codes);
        list("sizes", pf.sizes);
        list("params", pf.params);
    } else {
        o << "rfac0 = " << pf.rfac0 << '\n' << "twojmax = " << pf.twojmax << '\n' << "diagonalstyle = " << pf.style
          << '\n' << "rmin0 = " << pf.rmin0 << '\n' << "switch_flag = " << pf.sw << '\n' << "bzero_flag = " << pf.bz
          << '\n';
        list("weights", pf.weights);
    }
    return o.str();
}

}  // namespace ldb

// ======================================================================
// C ABI
// ======================================================================
using namespace ldb;

extern "C" {

const char *ld_error_message(void) { return g_err.c_str(); }
int ld_version(void) { return 10000 * 0 + 100 * 1 + 0; }
long long ld_launch_count(void) { return g_launches.load(); }
long long ld_alloc_count(void) { return g_allocs.load(); }
int ld_debug_fill_scratch(int byte) {
    if (byte < -1 || byte > 255) return fail(LD_ERR_INVALID_ARG, "ld_debug_fill_scratch: byte outside -1..255");
    g_fill.store(byte);
    return LD_OK;
}

int ld_fail_next_allocation(int k) {
    if (k < 0) return fail(LD_ERR_INVALID_ARG, "ld_fail_next_allocation: k < 0");
    g_fail_in.store(k);
    return LD_OK;
}

namespace {
// Pinned result blocks: sizes by pointer, released blocks by size.  The pool
// lives on the heap and is never destroyed, so a block released during
// process exit (a result array freed late) finds it intact.
struct PinPool {
    std::mutex mu;
    std::map<void *, size_t> size;
    std::multimap<size_t, void *> idle;
    size_t kept = 0;   // bytes of idle blocks
    size_t out = 0;    // bytes handed out and not yet released
};
PinPool &pin_pool() {
    static PinPool *pool = new PinPool;
    return *pool;
}
constexpr size_t kPinRound = 64u << 10, kPinKeep = 256u << 20, kPinOut = 512u << 20;
}  // namespace

int ld_host_alloc(size_t bytes, void **p) {
    if (!p) return fail(LD_ERR_INVALID_ARG, "p is NULL");
    *p = nullptr;
    const size_t want = ((bytes ? bytes : 1) + kPinRound - 1) / kPinRound * kPinRound;
    PinPool &pool = pin_pool();
    {
        std::lock_guard<std::mutex> lk(pool.mu);
        auto it = pool.idle.lower_bound(want);
        if (it != pool.idle.end() && it->first / 2 <= want) {
            *p = it->second;
            pool.kept -= it->first;
            pool.out += it->first;
            pool.idle.erase(it);
            return LD_OK;
        }
        // callers that keep their results release nothing: past this bound
        // each new block would be a fresh page-locking allocation, dearer
        // than the pageable copy it saves
        if (pool.out + want > kPinOut)
            return fail(LD_ERR_CAPACITY, "pinned result blocks: 512 MiB handed out and not released");
        // reserved before the allocation, so concurrent callers cannot pass
        // the bound together
        pool.out += want;
    }
    void *q = nullptr;
    const cudaError_t e = cudaHostAlloc(&q, want, cudaHostAllocPortable);
    std::lock_guard<std::mutex> lk(pool.mu);
    if (e != cudaSuccess) {
        pool.out -= want;
        cudaGetLastError();
        return cuda_fail(e, "cudaHostAlloc");
    }
    pool.size[q] = want;
    *p = q;
    return LD_OK;
}

void ld_host_free(void *p) {
    if (!p) return;
    PinPool &pool = pin_pool();
    {
        std::lock_guard<std::mutex> lk(pool.mu);
        auto it = pool.size.find(p);
        if (it == pool.size.end()) return;
        pool.out -= it->second;
        if (pool.kept + it->second <= kPinKeep) {
            pool.idle.emplace(it->second, p);
            pool.kept += it->second;
            return;
        }
        pool.size.erase(it);
    }
    cudaFreeHost(p);
    cudaGetLastError();
}

static int new_handle(ld_descriptor **out) {
    if (!out) return fail(LD_ERR_INVALID_ARG, "out is NULL");
    *out = nullptr;
    int rc = check_device();
    if (rc) return rc;
    auto *d = new (std::nothrow) ld_descriptor;
    if (!d) return fail(LD_ERR_OOM, "host allocation failed");
    cudaGetDevice(&d->device);
    *out = d;
    return LD_OK;
}

int ld_create_symmetry_functions(ld_descriptor **out, int n_species, const double *cutoff_matrix, int n_types,
                                 const int *type_codes, const int *sizes, const double *params) {
    int rc = new_handle(out);
    if (rc) return rc;
    rc = build_sf(*out, n_species, cutoff_matrix, n_types, type_codes, sizes, params);
    if (rc) {
        delete *out;
        *out = nullptr;
    }
    return rc;
}

int ld_create_bispectrum(ld_descriptor **out, double rfac0, int twojmax, int diagonalstyle, int use_shared_arrays,
                         double rmin0, int switch_flag, int bzero_flag, int n_species, const double *cutoff_matrix,
                         const double *weights) {
    (void)use_shared_arrays;
    int rc = new_handle(out);
    if (rc) return rc;
    rc = build_bs(*out, rfac0, twojmax, diagonalstyle, rmin0, switch_flag, bzero_flag, n_species, cutoff_matrix,
                  weights);
    if (rc) {
        delete *out;
        *out = nullptr;
    }
    return rc;
}

int ld_create_from_file(ld_descriptor **out, const char *path, int kind) {
    if (!out) return fail(LD_ERR_INVALID_ARG, "out is NULL");
    *out = nullptr;
    ParsedFile pf;
    int rc = parse_file(pf, path, kind);
    if (rc) return rc;
    rc = new_handle(out);
    if (rc) return rc;
    try {
        rc = build_parsed(*out, pf);
    } catch (const std::bad_alloc &) {
        rc = fail(LD_ERR_OOM, "host allocation failed");
    }
    if (rc) {
        delete *out;
        *out = nullptr;
    }
    return rc;
}

int ld_describe_parameter_file(const char *path, int kind, char *text, size_t capacity, size_t *length) {
    ParsedFile pf;
    int rc = parse_file(pf, path, kind);
    if (rc) return rc;
    const std::string t = describe_parsed(pf);
    if (length) *length = t.size() + 1;
    if (text && capacity > 0) {
        const size_t n = std::min(capacity - 1, t.size());
        std::memcpy(text, t.data(), n);
        text[n] = '\0';
        if (n < t.size()) return fail(LD_ERR_CAPACITY, "ld_describe_parameter_file: text buffer too small");
    }
    return LD_OK;
}

int ld_destroy(ld_descriptor *d) {
    if (!d) return LD_OK;
    if (d->stream) cudaStreamDestroy(d->stream);
    if (d->stream2) cudaStreamDestroy(d->stream2);
    if (d->ev_in) cudaEventDestroy(d->ev_in);
    if (d->ev_desc) cudaEventDestroy(d->ev_desc);
    if (d->hstatus) cudaFreeHost(d->hstatus);
    delete d;
    return LD_OK;
}

int ld_width(const ld_descriptor *d, int *width) {
    if (!d || !width) return fail(LD_ERR_INVALID_ARG, "NULL argument");
    *width = d->width;
    return LD_OK;
}

int ld_kind(const ld_descriptor *d, int *kind) {
    if (!d || !kind) return fail(LD_ERR_INVALID_ARG, "NULL argument");
    *kind = d->kind;
    return LD_OK;
}

int ld_compute(ld_descriptor *d, int n_atoms, int n_total, const int *species, const int *neighbor_list,
               const int *number_of_neighs, const double *coords, double *desc) {
    if (n_atoms < 0 || (n_atoms > 0 && !number_of_neighs)) return fail(LD_ERR_INVALID_ARG, "bad n_atoms / counts");
    HostRows h;
    int rc = make_rows(n_atoms, number_of_neighs, h);
    if (rc) return rc;
    return host_pass(d, h, n_total, species, neighbor_list, coords, nullptr, nullptr, desc);
}

int ld_gradient(ld_descriptor *d, int n_atoms, int n_total, const int *species, const int *neighbor_list,
                const int *number_of_neighs, const double *coords, const double *dE_ddesc, double *d_coords,
                double *desc_out) {
    if (n_atoms < 0 || (n_atoms > 0 && (!number_of_neighs || !dE_ddesc)))
        return fail(LD_ERR_INVALID_ARG, "bad n_atoms / counts / dE_ddesc");
    HostRows h;
    int rc = make_rows(n_atoms, number_of_neighs, h);
    if (rc) return rc;
    static const double dummy = 0.0;
    return host_pass(d, h, n_total, species, neighbor_list, coords, dE_ddesc ? dE_ddesc : &dummy, d_coords, desc_out);
}

static int gradient_params_impl(ld_descriptor *d, int n_atoms, int n_total, const int *species,
                                const int *neighbor_list, const int *number_of_neighs, const double *coords,
                                const double *dE_ddesc, double *d_params, int n_params) {
    if (!d) return fail(LD_ERR_INVALID_ARG, "descriptor handle is NULL");
    const bool bs = d->kind == LD_KIND_BISPECTRUM;
    const int np_have = bs ? 1 : d->sf.nparams;
    if (n_params != np_have)
        return fail(LD_ERR_INVALID_ARG, "n_params=" + std::to_string(n_params) + " but the descriptor has " +
                                            std::to_string(np_have) + " parameters");
    if (bs && d->bs.J > kMaxTwoJ)
        return fail(LD_ERR_CAPACITY, "the rfac0 gradient needs twojmax <= " + std::to_string(kMaxTwoJ));
    if (n_atoms < 0 || n_total < 0 || (n_atoms > 0 && (!number_of_neighs || !dE_ddesc || !species || !coords)))
        return fail(LD_ERR_INVALID_ARG, "bad n_atoms / NULL input array");
    if (n_params > 0 && !d_params) return fail(LD_ERR_INVALID_ARG, "d_params is NULL");
    HostRows h;
    int rc = make_rows(n_atoms, number_of_neighs, h);
    if (rc) return rc;
    if (h.nnz > 0 && !neighbor_list) return fail(LD_ERR_INVALID_ARG, "neighbor_list is NULL");
    if ((rc = validate(d, h, n_total, species, neighbor_list))) return rc;
    std::lock_guard<std::mutex> lk(d->mu);
    if ((rc = ensure_stream(d)) || (rc = ensure_status(d))) return rc;
    cudaStream_t s = d->stream;
    const int W = d->width;
    if ((rc = d->species.ensure(sizeof(int) * std::max(n_total, 1))) ||
        (rc = d->nbl.ensure(sizeof(int) * std::max<long long>(h.nnz, 1))) ||
        (rc = d->off.ensure(sizeof(long long) * (h.n_rows + 1))) ||
        (rc = d->coords.ensure(sizeof(double) * 3 * std::max(n_total, 1))) ||
        (rc = d->dE.ensure(sizeof(double) * std::max<size_t>((size_t)n_atoms * W, 1))) ||
        (rc = d->dc.ensure(sizeof(double) * (std::max(n_params, 1) + (bs ? 3 * (size_t)std::max(n_total, 1) : 0)))))
        return rc;
    DrainOnExit drain_s;   // no copy from the caller's arrays outlives an error return
    drain_s.st = s;
    if (n_total) LDB_CUDA(cudaMemcpyAsync(d->species.p, species, sizeof(int) * n_total, cudaMemcpyHostToDevice, s));
    if (h.nnz) LDB_CUDA(cudaMemcpyAsync(d->nbl.p, neighbor_list, sizeof(int) * h.nnz, cudaMemcpyHostToDevice, s));
    LDB_CUDA(cudaMemcpyAsync(d->off.p, h.off.data(), sizeof(long long) * (h.n_rows + 1), cudaMemcpyHostToDevice, s));
    if (n_total) LDB_CUDA(cudaMemcpyAsync(d->coords.p, coords, sizeof(double) * 3 * n_total, cudaMemcpyHostToDevice, s));
    if (n_atoms) LDB_CUDA(cudaMemcpyAsync(d->dE.p, dE_ddesc, sizeof(double) * n_atoms * W, cudaMemcpyHostToDevice, s));
    RowArgs a;
    a.n_rows = n_atoms;
    a.species = d->species.as<int>();
    a.nbl = d->nbl.as<int>();
    a.off = d->off.as<long long>();
    a.max_neigh = std::max(h.maxn, 1);
    a.coords = d->coords.as<double>();
    a.n_total = n_total;
    a.dE = d->dE.as<double>();
    a.status = d->status.as<int>();
    if (bs) {
        // the regular desc + VJP pass (coordinate gradient into scratch) with
        // the pair kernel also summing dL/d rfac0
        double *dp = d->dc.as<double>();
        LDB_CUDA(cudaMemsetAsync(dp, 0, sizeof(double) * (1 + 3 * (size_t)std::max(n_total, 1)), s));
        a.dcoords = dp + 1;
        a.d_rfac0 = dp;
        if (n_atoms > 0) {
            size_t wb = 0;
            if ((rc = ld_rows_work_bytes(d, n_atoms, 1, &wb))) return rc;
            if ((rc = d->work.ensure(wb))) return rc;
            a.work = d->work.p;
            a.work_bytes = wb;
            if ((rc = launch_rows(d, a, s))) return rc;
        }
    } else if ((rc = sf_param_launch(d->sf, a, d->dc.as<double>(), s))) {
        return rc;
    }
    if (n_params) LDB_CUDA(cudaMemcpyAsync(d_params, d->dc.p, sizeof(double) * n_params, cudaMemcpyDeviceToHost, s));
    return read_status(d, s);
}

int ld_gradient_params(ld_descriptor *d, int n_atoms, int n_total, const int *species, const int *neighbor_list,
                       const int *number_of_neighs, const double *coords, const double *dE_ddesc, double *d_params,
                       int n_params) {
    try {
        return gradient_params_impl(d, n_atoms, n_total, species, neighbor_list, number_of_neighs, coords, dE_ddesc,
                                    d_params, n_params);
    } catch (const std::bad_alloc &) {
        return fail(LD_ERR_OOM, "host allocation failed");
    }
}

int ld_num_params(const ld_descriptor *d, int *n_params) {
    if (!d || !n_params) return fail(LD_ERR_INVALID_ARG, "ld_num_params: bad arguments");
    *n_params = d->kind == LD_KIND_SYMMETRY_FUNCTIONS ? d->sf.nparams : 1;
    return LD_OK;
}

int ld_compute_batch(ld_descriptor *d, int n_configs, const int *n_atoms, const int *config_ptr, int n_total,
                     const int *species, const int *neighbor_list, const int *number_of_neighs, const double *coords,
                     double *desc) {
    if (n_configs < 0 || (n_configs > 0 && (!n_atoms || !config_ptr)))
        return fail(LD_ERR_INVALID_ARG, "bad configuration arrays");
    HostRows h;
    batch_centres(n_configs, n_atoms, config_ptr, h.centre);
    const int rows = (int)h.centre.size();
    if (rows > 0 && !number_of_neighs) return fail(LD_ERR_INVALID_ARG, "number_of_neighs is NULL");
    std::vector<int> keep = h.centre;
    int rc = make_rows(rows, number_of_neighs, h);
    if (rc) return rc;
    h.centre = keep;
    return host_pass(d, h, n_total, species, neighbor_list, coords, nullptr, nullptr, desc);
}

int ld_gradient_batch(ld_descriptor *d, int n_configs, const int *n_atoms, const int *config_ptr, int n_total,
                      const int *species, const int *neighbor_list, const int *number_of_neighs, const double *coords,
                      const double *dE_ddesc, double *d_coords, double *desc_out) {
    if (n_configs < 0 || (n_configs > 0 && (!n_atoms || !config_ptr)))
        return fail(LD_ERR_INVALID_ARG, "bad configuration arrays");
    HostRows h;
    batch_centres(n_configs, n_atoms, config_ptr, h.centre);
    const int rows = (int)h.centre.size();
    if (rows > 0 && (!number_of_neighs || !dE_ddesc)) return fail(LD_ERR_INVALID_ARG, "NULL counts / dE_ddesc");
    std::vector<int> keep = h.centre;
    int rc = make_rows(rows, number_of_neighs, h);
    if (rc) return rc;
    h.centre = keep;
    static const double dummy = 0.0;
    return host_pass(d, h, n_total, species, neighbor_list, coords, dE_ddesc ? dE_ddesc : &dummy, d_coords, desc_out);
}

int ld_compute_single_atom(ld_descriptor *d, int index, int n_total, const int *species, const int *neighbors,
                           int n_neigh, const double *coords, double *desc) {
    if (n_neigh < 0) return fail(LD_ERR_INVALID_ARG, "n_neigh < 0");
    HostRows h;
    int rc = make_rows(1, &n_neigh, h);
    if (rc) return rc;
    h.centre = {index};
    return host_pass(d, h, n_total, species, neighbors, coords, nullptr, nullptr, desc);
}

int ld_gradient_single_atom(ld_descriptor *d, int index, int n_total, const int *species, const int *neighbors,
                            int n_neigh, const double *coords, const double *dE_ddesc, double *d_coords,
                            double *desc_out) {
    if (n_neigh < 0 || !dE_ddesc) return fail(LD_ERR_INVALID_ARG, "bad n_neigh / dE_ddesc");
    HostRows h;
    int rc = make_rows(1, &n_neigh, h);
    if (rc) return rc;
    h.centre = {index};
    return host_pass(d, h, n_total, species, neighbors, coords, dE_ddesc, d_coords, desc_out);
}

int ld_jacobian(ld_descriptor *d, int n_atoms, int n_total, const int *species, const int *neighbor_list,
                const int *number_of_neighs, const double *coords, double *J) {
    if (!d) return fail(LD_ERR_INVALID_ARG, "descriptor handle is NULL");
    if (n_atoms < 0 || (n_atoms > 0 && (!number_of_neighs || !J))) return fail(LD_ERR_INVALID_ARG, "bad arguments");
    HostRows h;
    int rc = make_rows(n_atoms, number_of_neighs, h);
    if (rc) return rc;
    static const double dummy = 0.0;
    return host_pass(d, h, n_total, species, neighbor_list, coords, &dummy, J, nullptr, d->width);
}

int ld_neighbor_offsets_dev(ld_descriptor *d, int n_rows, const int *number_of_neighs, long long *neigh_offsets,
                            int *max_neigh, ld_stream stream) {
    if (!d || n_rows < 0 || !neigh_offsets || (n_rows > 0 && !number_of_neighs))
        return fail(LD_ERR_INVALID_ARG, "ld_neighbor_offsets_dev: bad arguments");
    std::lock_guard<std::mutex> lk(d->mu);
    cudaStream_t s = (cudaStream_t)stream;
    // the max lands right after the CUB scratch: keep it 256-byte aligned
    size_t tb = (offsets_tmp_bytes(std::max(n_rows, 1)) + 255) & ~(size_t)255;
    int rc = d->tmp.ensure(tb + 256);
    if (rc) return rc;
    int *dmax = max_neigh ? reinterpret_cast<int *>(static_cast<char *>(d->tmp.p) + tb) : nullptr;
    rc = offsets_launch(n_rows, number_of_neighs, neigh_offsets, dmax, d->tmp.p, tb, s);
    if (rc) return rc;
    if (max_neigh) {
        LDB_CUDA(cudaMemcpyAsync(max_neigh, dmax, sizeof(int), cudaMemcpyDeviceToHost, s));
        LDB_CUDA(cudaStreamSynchronize(s));
    }
    return LD_OK;
}

static int dev_pass(ld_descriptor *d, int n_rows, const int *row_centre, const int *species, const int *nbl,
                    const long long *off, int max_neigh, const double *coords, double *desc, const double *dE,
                    double *dcoords, const int *image, ld_stream stream, const long long *nbl_begin = nullptr,
                    void *work = nullptr, size_t work_bytes = 0) {
    if (!d) return fail(LD_ERR_INVALID_ARG, "descriptor handle is NULL");
    if (n_rows < 0 || max_neigh < 0) return fail(LD_ERR_INVALID_ARG, "negative size");
    if (n_rows == 0) return LD_OK;
    if (!species || !off || !coords || (!nbl && max_neigh > 0)) return fail(LD_ERR_INVALID_ARG, "NULL device array");
    if (dE && !dcoords) return fail(LD_ERR_INVALID_ARG, "d_coords is NULL");
    if (!dE && !desc) return fail(LD_ERR_INVALID_ARG, "desc is NULL");
    int rc = ensure_status(d);
    if (rc) return rc;
    RowArgs a;
    a.n_rows = n_rows;
    a.row_centre = row_centre;
    a.species = species;
    a.nbl = nbl;
    a.off = off;
    a.max_neigh = std::max(max_neigh, 1);
    a.coords = coords;
    a.desc = desc;
    a.dE = dE;
    a.dcoords = dcoords;
    a.image = image;
    a.status = d->status.as<int>();
    a.nbl_begin = nbl_begin;
    if (work) {
        if (reinterpret_cast<std::uintptr_t>(work) & 255)
            return fail(LD_ERR_INVALID_ARG, "work space must start on a 256-byte boundary");
        size_t need = 0;
        int rc2 = ld_rows_work_bytes(d, n_rows, dE ? 1 : 0, &need);
        if (rc2) return rc2;
        if (work_bytes < need)
            return fail(LD_ERR_INVALID_ARG, "work space of " + std::to_string(work_bytes) + " bytes < " +
                                                std::to_string(need) + " needed");
        a.work = work;
        a.work_bytes = work_bytes;
    }
    return launch_rows(d, a, (cudaStream_t)stream);
}

int ld_rows_work_bytes(const ld_descriptor *d, int n_rows, int vjp, size_t *bytes) {
    if (!d || !bytes || n_rows < 0) return fail(LD_ERR_INVALID_ARG, "ld_rows_work_bytes: bad arguments");
    *bytes = d->kind == LD_KIND_SYMMETRY_FUNCTIONS ? sf_work_bytes(d->sf, n_rows, vjp != 0)
                                                   : bs_work_bytes(d->bs, n_rows, vjp != 0);
    return LD_OK;
}

int ld_compute_rows_dev(ld_descriptor *d, int n_rows, const int *row_centre, const long long *nbl_begin,
                        const int *species, const int *neighbor_list, const long long *neigh_offsets,
                        int max_neigh, const double *coords, double *desc, void *work, size_t work_bytes,
                        ld_stream stream) {
    if (n_rows > 0 && (!row_centre || !nbl_begin))
        return fail(LD_ERR_INVALID_ARG, "ld_compute_rows_dev: row_centre and nbl_begin are required");
    return dev_pass(d, n_rows, row_centre, species, neighbor_list, neigh_offsets, max_neigh, coords, desc, nullptr,
                    nullptr, nullptr, stream, nbl_begin, work, work_bytes);
}

int ld_gradient_rows_dev(ld_descriptor *d, int n_rows, const int *row_centre, const long long *nbl_begin,
                         const int *species, const int *neighbor_list, const long long *neigh_offsets,
                         int max_neigh, const double *coords, const double *dE_ddesc, double *d_coords,
                         double *desc_out, const int *image, void *work, size_t work_bytes, ld_stream stream) {
    if (n_rows > 0 && (!row_centre || !nbl_begin))
        return fail(LD_ERR_INVALID_ARG, "ld_gradient_rows_dev: row_centre and nbl_begin are required");
    if (n_rows > 0 && !dE_ddesc) return fail(LD_ERR_INVALID_ARG, "dE_ddesc is NULL");
    return dev_pass(d, n_rows, row_centre, species, neighbor_list, neigh_offsets, max_neigh, coords, desc_out,
                    dE_ddesc, d_coords, image, stream, nbl_begin, work, work_bytes);
}

int ld_set_tuning(ld_descriptor *d, int key, int value) {
    if (!d) return fail(LD_ERR_INVALID_ARG, "descriptor handle is NULL");
    if (key < 0 || key > LD_TUNE_SF_GENERIC) return fail(LD_ERR_INVALID_ARG, "unknown tuning key");
    if (value < 0) value = 0;
    if (key == LD_TUNE_SF_WARPS && value != 0 && value != 1 && value != 2 && value != 4)
        return fail(LD_ERR_INVALID_ARG, "LD_TUNE_SF_WARPS must be 1, 2 or 4");
    if (key == LD_TUNE_DYNAMIC_QUEUE && value > 2)
        return fail(LD_ERR_INVALID_ARG, "LD_TUNE_DYNAMIC_QUEUE must be 0 (built-in), 1 (on) or 2 (off)");
    if (key == LD_TUNE_SF_GENERIC) value = value ? 1 : 0;
    std::lock_guard<std::mutex> lk(d->mu);
    d->tune[key] = value;
    return LD_OK;
}

int ld_get_tuning(const ld_descriptor *d, int key, int *value) {
    if (!d || !value) return fail(LD_ERR_INVALID_ARG, "NULL argument");
    if (key < 0 || key > LD_TUNE_SF_GENERIC) return fail(LD_ERR_INVALID_ARG, "unknown tuning key");
    *value = d->tune[key];
    return LD_OK;
}

int ld_compute_dev(ld_descriptor *d, int n_rows, const int *row_centre, const int *species, const int *neighbor_list,
                   const long long *neigh_offsets, int max_neigh, const double *coords, double *desc,
                   ld_stream stream) {
    return dev_pass(d, n_rows, row_centre, species, neighbor_list, neigh_offsets, max_neigh, coords, desc, nullptr,
                    nullptr, nullptr, stream);
}

int ld_gradient_dev(ld_descriptor *d, int n_rows, const int *row_centre, const int *species,
                    const int *neighbor_list, const long long *neigh_offsets, int max_neigh, const double *coords,
                    const double *dE_ddesc, double *d_coords, double *desc_out, const int *image, ld_stream stream) {
    if (n_rows > 0 && !dE_ddesc) return fail(LD_ERR_INVALID_ARG, "dE_ddesc is NULL");
    return dev_pass(d, n_rows, row_centre, species, neighbor_list, neigh_offsets, max_neigh, coords, desc_out,
                    dE_ddesc, d_coords, image, stream);
}

int ld_sync_status(ld_descriptor *d, ld_stream stream) {
    if (!d) return fail(LD_ERR_INVALID_ARG, "descriptor handle is NULL");
    cudaStream_t s = (cudaStream_t)stream;
    LDB_CUDA(cudaStreamSynchronize(s));
    return read_status(d, s);
}

// introspection for tests and the roofline accounting (not in the public
// header: declared by the Python binding only)
int ld_bs_info(const ld_descriptor *d, long long *inner_fwd, long long *inner_vjp, int *tasks_fwd, int *tasks_vjp,
               int *nU, int *nL, int *ntrip, int *nZ) {
    if (!d || d->kind != LD_KIND_BISPECTRUM) return fail(LD_ERR_INVALID_KIND, "not a bispectrum descriptor");
    if (inner_fwd) *inner_fwd = d->bs_inner_fwd;
    if (inner_vjp) *inner_vjp = d->bs_inner_vjp;
    if (tasks_fwd) *tasks_fwd = d->bs_tasks_fwd;
    if (tasks_vjp) *tasks_vjp = d->bs_tasks_vjp;
    if (nU) *nU = d->bs.nU;
    if (nL) *nL = d->bs.nL;
    if (ntrip) *ntrip = d->bs.ntrip;
    if (nZ) *nZ = d->bs.nZall;
    return LD_OK;
}

}  // extern "C"
