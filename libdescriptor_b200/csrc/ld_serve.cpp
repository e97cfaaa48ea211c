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
// ld_stage_pack_fields / ld_stage_upload_fields do the same for requests
// admitted together into consecutive slots: each request's fields go to its
// place in one block laid out field by field, uploaded with one copy per
// field for the whole block.
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

namespace {

struct Fields {
    double *coords;
    int *species, *image, *nbl, *centre;
    long long *begin;
    int *counts;
    double *dE;
};

Fields fields(void *staging, const StageLayout &L) {
    char *b = static_cast<char *>(staging);
    return {reinterpret_cast<double *>(b + L.off[0]), reinterpret_cast<int *>(b + L.off[1]),
            reinterpret_cast<int *>(b + L.off[2]),    reinterpret_cast<int *>(b + L.off[3]),
            reinterpret_cast<int *>(b + L.off[4]),    reinterpret_cast<long long *>(b + L.off[5]),
            reinterpret_cast<int *>(b + L.off[6]),    reinterpret_cast<double *>(b + L.off[7])};
}

int check_staging(void *staging, size_t staging_bytes, const StageLayout &L, const char *who) {
    using namespace ldb;
    if (!staging) return fail(LD_ERR_INVALID_ARG, std::string(who) + ": staging is NULL");
    if (reinterpret_cast<std::uintptr_t>(staging) % kAlign)
        return fail(LD_ERR_INVALID_ARG, std::string(who) + ": staging must be 256-byte aligned");
    if (staging_bytes < L.total)
        return fail(LD_ERR_INVALID_ARG, std::string(who) + ": staging of " + std::to_string(staging_bytes) +
                                            " bytes < " + std::to_string(L.total) + " needed");
    return LD_OK;
}

int stage_pack_fields(int n_atoms, int n_total, long long nnz, int width, int row0, int atom0, long long entry0,
                      const double *coords, const int *species, const int *image, const int *neighbor_list,
                      const int *number_of_neighs, const double *dE_ddesc, const Fields &F, int max_threads);

// The host half of staging: every field of the request into the staging
// layout (see stage_pack_fields).
int stage_pack(int n_atoms, int n_total, long long nnz, int width, int row0, int atom0, long long entry0,
               const double *coords, const int *species, const int *image, const int *neighbor_list,
               const int *number_of_neighs, const double *dE_ddesc, void *staging, size_t staging_bytes,
               int max_threads, const char *who) {
    using namespace ldb;
    if (n_atoms <= 0 || n_total < n_atoms || nnz < 0 || width <= 0 || row0 < 0 || atom0 < 0 || entry0 < 0)
        return fail(LD_ERR_INVALID_ARG, std::string(who) + ": bad sizes or slots");
    if (!coords || !species || !image || !number_of_neighs || !dE_ddesc || (nnz > 0 && !neighbor_list))
        return fail(LD_ERR_INVALID_ARG, std::string(who) + ": NULL array");
    const StageLayout L = layout(n_atoms, n_total, nnz, width);
    if (int rc = check_staging(staging, staging_bytes, L, who)) return rc;
    return stage_pack_fields(n_atoms, n_total, nnz, width, row0, atom0, entry0, coords, species, image,
                             neighbor_list, number_of_neighs, dE_ddesc, fields(staging, L), max_threads);
}

// Every field of one request written at the given host pointers, indices
// rebased to the slots and range-checked.  max_threads 0: one host thread
// per MiB of copying, up to the cores (at most 16); 1: this thread.
int stage_pack_fields(int n_atoms, int n_total, long long nnz, int width, int row0, int atom0, long long entry0,
                      const double *coords, const int *species, const int *image, const int *neighbor_list,
                      const int *number_of_neighs, const double *dE_ddesc, const Fields &F, int max_threads) {
    using namespace ldb;
    // row arrays (sequential prefix) + count check
    long long pos = entry0;
    for (int j = 0; j < n_atoms; ++j) {
        const int c = number_of_neighs[j];
        if (c < 0) return fail(LD_ERR_INVALID_ARG, "negative neighbour count");
        F.centre[j] = atom0 + j;
        F.begin[j] = pos;
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
        {(char *)F.coords, (const char *)coords, (long long)n_total * 24, 0, 0, false},
        {(char *)F.species, (const char *)species, (long long)n_total * 4, 0, 0, false},
        {(char *)F.counts, (const char *)number_of_neighs, (long long)n_atoms * 4, 0, 0, false},
        {(char *)F.dE, (const char *)dE_ddesc, (long long)n_atoms * width * 8, 0, 0, false},
        {(char *)F.image, (const char *)image, (long long)n_total, row0, n_atoms, true},
        {(char *)F.nbl, (const char *)neighbor_list, nnz, atom0, n_total, true},
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
    static const int kCores = std::max(1, std::min(16, (int)std::thread::hardware_concurrency()));
    const int cap = max_threads > 0 ? std::min(max_threads, kCores) : kCores;
    const int nthr = (int)std::max(1LL, std::min<long long>(cap, total / kChunkBytes));
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
    return LD_OK;
}

// The device half: one upload per field of a packed staging area.
int stage_upload(int n_atoms, int n_total, long long nnz, int width, int row0, int atom0, long long entry0,
                 void *staging, size_t staging_bytes, double *d_coords, int *d_species, int *d_image, int *d_nbl,
                 int *d_centre, long long *d_begin, int *d_counts, double *d_dE, ld_stream stream,
                 const char *who) {
    using namespace ldb;
    if (n_atoms <= 0 || n_total < n_atoms || nnz < 0 || width <= 0 || row0 < 0 || atom0 < 0 || entry0 < 0)
        return fail(LD_ERR_INVALID_ARG, std::string(who) + ": bad sizes or slots");
    if (!d_coords || !d_species || !d_image || (nnz > 0 && !d_nbl) || !d_centre || !d_begin || !d_counts || !d_dE)
        return fail(LD_ERR_INVALID_ARG, std::string(who) + ": NULL device array");
    const StageLayout L = layout(n_atoms, n_total, nnz, width);
    if (int rc = check_staging(staging, staging_bytes, L, who)) return rc;
    const Fields F = fields(staging, L);
    cudaStream_t s = (cudaStream_t)stream;
    const auto h2d = cudaMemcpyHostToDevice;
    LDB_CUDA(cudaMemcpyAsync(d_coords + 3 * (size_t)atom0, F.coords, (size_t)n_total * 24, h2d, s));
    LDB_CUDA(cudaMemcpyAsync(d_species + atom0, F.species, (size_t)n_total * 4, h2d, s));
    LDB_CUDA(cudaMemcpyAsync(d_image + atom0, F.image, (size_t)n_total * 4, h2d, s));
    if (nnz > 0) LDB_CUDA(cudaMemcpyAsync(d_nbl + entry0, F.nbl, (size_t)nnz * 4, h2d, s));
    LDB_CUDA(cudaMemcpyAsync(d_centre + row0, F.centre, (size_t)n_atoms * 4, h2d, s));
    LDB_CUDA(cudaMemcpyAsync(d_begin + row0, F.begin, (size_t)n_atoms * 8, h2d, s));
    LDB_CUDA(cudaMemcpyAsync(d_counts + row0, F.counts, (size_t)n_atoms * 4, h2d, s));
    LDB_CUDA(cudaMemcpyAsync(d_dE + (size_t)row0 * width, F.dE, (size_t)n_atoms * width * 8, h2d, s));
    return LD_OK;
}

}  // namespace

extern "C" int ld_stage_request(int n_atoms, int n_total, long long nnz, int width, int row0, int atom0,
                                long long entry0, const double *coords, const int *species, const int *image,
                                const int *neighbor_list, const int *number_of_neighs, const double *dE_ddesc,
                                void *staging, size_t staging_bytes, double *d_coords, int *d_species,
                                int *d_image, int *d_nbl, int *d_centre, long long *d_begin, int *d_counts,
                                double *d_dE, ld_stream stream) {
    using namespace ldb;
    if (!d_coords || !d_species || !d_image || (nnz > 0 && !d_nbl) || !d_centre || !d_begin || !d_counts || !d_dE)
        return fail(LD_ERR_INVALID_ARG, "ld_stage_request: NULL array");
    int rc = stage_pack(n_atoms, n_total, nnz, width, row0, atom0, entry0, coords, species, image, neighbor_list,
                        number_of_neighs, dE_ddesc, staging, staging_bytes, 0, "ld_stage_request");
    if (rc) return rc;
    return stage_upload(n_atoms, n_total, nnz, width, row0, atom0, entry0, staging, staging_bytes, d_coords,
                        d_species, d_image, d_nbl, d_centre, d_begin, d_counts, d_dE, stream, "ld_stage_request");
}

extern "C" int ld_stage_pack(int n_atoms, int n_total, long long nnz, int width, int row0, int atom0,
                             long long entry0, const double *coords, const int *species, const int *image,
                             const int *neighbor_list, const int *number_of_neighs, const double *dE_ddesc,
                             void *staging, size_t staging_bytes) {
    return stage_pack(n_atoms, n_total, nnz, width, row0, atom0, entry0, coords, species, image, neighbor_list,
                      number_of_neighs, dE_ddesc, staging, staging_bytes, 1, "ld_stage_pack");
}

extern "C" int ld_stage_pack_fields(int n_atoms, int n_total, long long nnz, int width, int row0, int atom0,
                                    long long entry0, const double *coords, const int *species, const int *image,
                                    const int *neighbor_list, const int *number_of_neighs, const double *dE_ddesc,
                                    double *coords_out, int *species_out, int *image_out, int *nbl_out,
                                    int *centre_out, long long *begin_out, int *counts_out, double *dE_out) {
    using namespace ldb;
    if (n_atoms <= 0 || n_total < n_atoms || nnz < 0 || width <= 0 || row0 < 0 || atom0 < 0 || entry0 < 0)
        return fail(LD_ERR_INVALID_ARG, "ld_stage_pack_fields: bad sizes or slots");
    if (!coords || !species || !image || !number_of_neighs || !dE_ddesc || (nnz > 0 && !neighbor_list))
        return fail(LD_ERR_INVALID_ARG, "ld_stage_pack_fields: NULL array");
    if (!coords_out || !species_out || !image_out || (nnz > 0 && !nbl_out) || !centre_out || !begin_out ||
        !counts_out || !dE_out)
        return fail(LD_ERR_INVALID_ARG, "ld_stage_pack_fields: NULL output field");
    const Fields F{coords_out, species_out, image_out, nbl_out, centre_out, begin_out, counts_out, dE_out};
    return stage_pack_fields(n_atoms, n_total, nnz, width, row0, atom0, entry0, coords, species, image,
                             neighbor_list, number_of_neighs, dE_ddesc, F, 1);
}

extern "C" int ld_stage_upload_fields(int n_fields, const void *const *src, void *const *dst, const size_t *bytes,
                                      ld_stream stream) {
    using namespace ldb;
    if (n_fields < 0 || n_fields > 64 || (n_fields > 0 && (!src || !dst || !bytes)))
        return fail(LD_ERR_INVALID_ARG, "ld_stage_upload_fields: bad field list");
    for (int i = 0; i < n_fields; ++i)
        if (bytes[i] > 0 && (!src[i] || !dst[i]))
            return fail(LD_ERR_INVALID_ARG, "ld_stage_upload_fields: NULL field pointer");
    cudaStream_t s = (cudaStream_t)stream;
    for (int i = 0; i < n_fields; ++i)
        if (bytes[i] > 0) LDB_CUDA(cudaMemcpyAsync(dst[i], src[i], bytes[i], cudaMemcpyHostToDevice, s));
    return LD_OK;
}

extern "C" int ld_stage_upload(int n_atoms, int n_total, long long nnz, int width, int row0, int atom0,
                               long long entry0, void *staging, size_t staging_bytes, double *d_coords,
                               int *d_species, int *d_image, int *d_nbl, int *d_centre, long long *d_begin,
                               int *d_counts, double *d_dE, ld_stream stream) {
    return stage_upload(n_atoms, n_total, nnz, width, row0, atom0, entry0, staging, staging_bytes, d_coords,
                        d_species, d_image, d_nbl, d_centre, d_begin, d_counts, d_dE, stream, "ld_stage_upload");
}
