// ld_serve.cpp -- host side of the serving runtime: staging of one request.
//
// A served request arrives as host arrays in the reference's call layout
// with local indices (coordinate rows 0..n_total-1, master rows
// 0..n_atoms-1).  Admission assigns it slots in the resident device rings:
// rows [row0, row0 + n_atoms), atoms [atom0, atom0 + n_total), neighbour
// entries [entry0, entry0 + nnz).  ld_stage_request writes the inputs, with
// every index rebased to those slots, into pinned staging memory and
// enqueues one upload per field on the given stream: after it the rows can
// join any batch launched through ld_gradient_rows_dev on the rings.
#include <cstdint>
#include <cstring>
#include <string>
#include <thread>
#include <vector>
#include <algorithm>

#include "ld_internal.h"

namespace {

constexpr size_t kAlign = 256;

size_t up(size_t b) { return (b + kAlign - 1) & ~(kAlign - 1); }

struct StageLayout {
    size_t off[8];
    size_t total;
};

StageLayout layout(int n, int nt, long long nnz, int width) {
    const size_t sz[8] = {(size_t)nt * 24, (size_t)nt * 4, (size_t)nt * 4, (size_t)nnz * 4,
                          (size_t)n * 4,   (size_t)n * 8,  (size_t)n * 4,  (size_t)n * width * 8};
    StageLayout L{};
    size_t t = 0;
    for (int i = 0; i < 8; ++i) {
        L.off[i] = t;
        t += up(sz[i]);
    }
    L.total = t;
    return L;
}

}  // namespace

extern "C" int ld_stage_bytes(int n_atoms, int n_total, long long nnz, int width, size_t *bytes) {
    using namespace ldb;
    if (!bytes || n_atoms < 0 || n_total < n_atoms || nnz < 0 || width <= 0)
        return fail(LD_ERR_INVALID_ARG, "ld_stage_bytes: bad sizes");
    *bytes = layout(n_atoms, n_total, nnz, width).total;
    return LD_OK;
}

extern "C" int ld_stage_request(int n_atoms, int n_total, long long nnz, int width, int row0, int atom0,
                                long long entry0, const double *coords, const int *species, const int *image,
                                const int *neighbor_list, const int *number_of_neighs, const double *dE_ddesc,
                                void *staging, size_t staging_bytes, double *d_coords, int *d_species,
                                int *d_image, int *d_nbl, int *d_centre, long long *d_begin, int *d_counts,
                                double *d_dE, ld_stream stream) {
    using namespace ldb;
    if (n_atoms <= 0 || n_total < n_atoms || nnz < 0 || width <= 0 || row0 < 0 || atom0 < 0 || entry0 < 0)
        return fail(LD_ERR_INVALID_ARG, "ld_stage_request: bad sizes or slots");
    if (!coords || !species || !image || !number_of_neighs || !dE_ddesc || (nnz > 0 && !neighbor_list) ||
        !staging || !d_coords || !d_species || !d_image || (nnz > 0 && !d_nbl) || !d_centre || !d_begin ||
        !d_counts || !d_dE)
        return fail(LD_ERR_INVALID_ARG, "ld_stage_request: NULL array");
    if (reinterpret_cast<std::uintptr_t>(staging) % kAlign)
        return fail(LD_ERR_INVALID_ARG, "ld_stage_request: staging must be 256-byte aligned");
    const StageLayout L = layout(n_atoms, n_total, nnz, width);
    if (staging_bytes < L.total)
        return fail(LD_ERR_INVALID_ARG, "ld_stage_request: staging of " + std::to_string(staging_bytes) +
                                            " bytes < " + std::to_string(L.total) + " needed");
    char *b = static_cast<char *>(staging);
    double *s_coords = reinterpret_cast<double *>(b + L.off[0]);
    int *s_species = reinterpret_cast<int *>(b + L.off[1]);
    int *s_image = reinterpret_cast<int *>(b + L.off[2]);
    int *s_nbl = reinterpret_cast<int *>(b + L.off[3]);
    int *s_centre = reinterpret_cast<int *>(b + L.off[4]);
    long long *s_begin = reinterpret_cast<long long *>(b + L.off[5]);
    int *s_counts = reinterpret_cast<int *>(b + L.off[6]);
    double *s_dE = reinterpret_cast<double *>(b + L.off[7]);

    // row arrays (sequential prefix) + count check
    long long pos = entry0;
    for (int j = 0; j < n_atoms; ++j) {
        const int c = number_of_neighs[j];
        if (c < 0) return fail(LD_ERR_INVALID_ARG, "negative neighbour count");
        s_centre[j] = atom0 + j;
        s_begin[j] = pos;
        pos += c;
    }
    if (pos - entry0 != nnz) return fail(LD_ERR_INVALID_ARG, "neighbour counts do not add up to nnz");

    // bulk fields in chunks: plain copies and rebased index copies (with
    // their range checks), spread over host threads for large requests
    struct Job {
        char *dst;
        const char *src;
        long long count;   // bytes (copy) or ints (rebase)
        int add, hi;       // rebase: dst = src + add, src in [0, hi)
        bool rebase;
    };
    Job jobs[6] = {
        {(char *)s_coords, (const char *)coords, (long long)n_total * 24, 0, 0, false},
        {(char *)s_species, (const char *)species, (long long)n_total * 4, 0, 0, false},
        {(char *)s_counts, (const char *)number_of_neighs, (long long)n_atoms * 4, 0, 0, false},
        {(char *)s_dE, (const char *)dE_ddesc, (long long)n_atoms * width * 8, 0, 0, false},
        {(char *)s_image, (const char *)image, (long long)n_total, row0, n_atoms, true},
        {(char *)s_nbl, (const char *)neighbor_list, nnz, atom0, n_total, true},
    };
    constexpr long long kChunkBytes = 1 << 20;
    struct Piece {
        int job;
        long long lo, hi;
    };
    std::vector<Piece> pieces;
    long long total = 0;
    for (int k = 0; k < 6; ++k) {
        const long long unit = jobs[k].rebase ? 4 : 1;
        const long long step = kChunkBytes / unit;
        for (long long lo = 0; lo < jobs[k].count; lo += step)
            pieces.push_back({k, lo, std::min(jobs[k].count, lo + step)});
        total += jobs[k].count * unit;
    }
    int bad = 0;
    const int np = (int)pieces.size();
    // one host thread per MiB of copying, up to the cores (at most 16)
    static const int kCores = std::max(1, std::min(16, (int)std::thread::hardware_concurrency()));
    const int nthr = (int)std::max(1LL, std::min<long long>(kCores, total / kChunkBytes));
#pragma omp parallel for num_threads(nthr) schedule(dynamic, 1) reduction(| : bad) if (nthr > 1)
    for (int i = 0; i < np; ++i) {
        const Piece &pc = pieces[i];
        const Job &jb = jobs[pc.job];
        if (!jb.rebase) {
            std::memcpy(jb.dst + pc.lo, jb.src + pc.lo, (size_t)(pc.hi - pc.lo));
        } else {
            const int *src = reinterpret_cast<const int *>(jb.src);
            int *dst = reinterpret_cast<int *>(jb.dst);
            int local_bad = 0;
            for (long long e = pc.lo; e < pc.hi; ++e) {
                const int v = src[e];
                local_bad |= (v < 0) | (v >= jb.hi);
                dst[e] = v + jb.add;
            }
            bad |= local_bad;
        }
    }
    if (bad) return fail(LD_ERR_INVALID_ARG, "an image or neighbour index lies outside the request's atoms");

    cudaStream_t s = (cudaStream_t)stream;
    const auto h2d = cudaMemcpyHostToDevice;
    LDB_CUDA(cudaMemcpyAsync(d_coords + 3 * (size_t)atom0, s_coords, (size_t)n_total * 24, h2d, s));
    LDB_CUDA(cudaMemcpyAsync(d_species + atom0, s_species, (size_t)n_total * 4, h2d, s));
    LDB_CUDA(cudaMemcpyAsync(d_image + atom0, s_image, (size_t)n_total * 4, h2d, s));
    if (nnz > 0) LDB_CUDA(cudaMemcpyAsync(d_nbl + entry0, s_nbl, (size_t)nnz * 4, h2d, s));
    LDB_CUDA(cudaMemcpyAsync(d_centre + row0, s_centre, (size_t)n_atoms * 4, h2d, s));
    LDB_CUDA(cudaMemcpyAsync(d_begin + row0, s_begin, (size_t)n_atoms * 8, h2d, s));
    LDB_CUDA(cudaMemcpyAsync(d_counts + row0, s_counts, (size_t)n_atoms * 4, h2d, s));
    LDB_CUDA(cudaMemcpyAsync(d_dE + (size_t)row0 * width, s_dE, (size_t)n_atoms * width * 8, h2d, s));
    return LD_OK;
}
