/*
 * libdescriptor_b200.h -- C ABI of the B200 (sm_100a) descriptor library.
 *
 * A drop-in for libdescriptor's per-atom descriptor hot path: Behler
 * symmetry functions and the SNAP-style bispectrum, their forward pass and
 * the reverse-mode gradient (vector-Jacobian product) w.r.t. coordinates.
 * All arithmetic is FP64.  Plain pointers and sizes only; every entry point
 * returns an int status (LD_OK == 0) and sets a thread-local message that
 * ld_error_message() returns.
 *
 * Input layout is the reference's (src/Descriptors.cpp:121-163):
 *   coords[n_total*3]        contributing atoms first, then ghost images
 *   species[n_total]         species code 0..n_species-1
 *   number_of_neighs[rows]   neighbour count of each centre row
 *   neighbor_list[sum]       neighbour indices (into coords), rows in order
 *   desc[rows*width]         one row per centre
 * Batches concatenate configurations: centre of row (c, j) is
 * j + config_ptr[c]; neighbour indices are global.
 */
#ifndef LIBDESCRIPTOR_B200_H_
#define LIBDESCRIPTOR_B200_H_

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LD_OK 0
#define LD_ERR_INVALID_KIND 1     /* descriptor kind not supported        */
#define LD_ERR_INVALID_ARG 2      /* bad size, pointer or index           */
#define LD_ERR_CAPACITY 3         /* a fixed capacity of the kernels      */
#define LD_ERR_OOM 4              /* device or host allocation failed     */
#define LD_ERR_CUDA 5             /* CUDA runtime error                   */
#define LD_ERR_TIMEOUT 6          /* a bounded device wait ran out        */
#define LD_ERR_NO_DEVICE 7        /* no CUDA device visible               */
#define LD_ERR_PARSE 8            /* descriptor parameter file malformed  */

/* Descriptor kinds, numbered as the reference's AvailableDescriptor enum
 * (include/Descriptors.hpp:21-26). */
#define LD_KIND_SYMMETRY_FUNCTIONS 0
#define LD_KIND_BISPECTRUM 1
#define LD_KIND_SOAP 2
#define LD_KIND_XI 3

typedef struct ld_descriptor ld_descriptor; /* opaque, owns device tables */
typedef void *ld_stream;                    /* a cudaStream_t (0 = legacy) */

/* Last error of the calling thread ("" if none). */
const char *ld_error_message(void);
/* Library version as 10000*major + 100*minor + patch. */
int ld_version(void);

/* ---------------- creation (DescriptorKind::initDescriptor) ---------------- */

/* Symmetry functions.  Replaces DescriptorKind::initDescriptor(kind, species,
 * cutoff_function, cutoff, types, sizes, params) (include/Descriptors.hpp:250-254,
 * src/Descriptors.cpp:579-590; SymmetryFunctions ctor
 * src/SymmetryFunctions.cpp:429-451).  type_codes[t] in 1..5 (g1..g5);
 * sizes[2t], sizes[2t+1] = rows, params per row of block t; params is the
 * concatenation of the row-major blocks; cutoff_matrix is n_species^2
 * row-major (the reference's direct init fills it with cutoff[0]). */
int ld_create_symmetry_functions(ld_descriptor **out, int n_species,
                                 const double *cutoff_matrix, int n_types,
                                 const int *type_codes, const int *sizes,
                                 const double *params);

/* Bispectrum.  Replaces DescriptorKind::initDescriptor(kind, rfac0, twojmax,
 * diagonalstyle, use_shared_arrays, rmin0, switch_flag, bzero_flag, cutoff,
 * species, weights) (include/Descriptors.hpp:257-260,
 * src/Descriptors.cpp:592-607; Bispectrum ctor src/Bispectrum.cpp:44-82).
 * twojmax <= 10.  use_shared_arrays is accepted and ignored (memory layout
 * is the library's own). */
int ld_create_bispectrum(ld_descriptor **out, double rfac0, int twojmax,
                         int diagonalstyle, int use_shared_arrays, double rmin0,
                         int switch_flag, int bzero_flag, int n_species,
                         const double *cutoff_matrix, const double *weights);

/* Parameter-file init.  Replaces DescriptorKind::initDescriptor(file, kind)
 * (include/Descriptors.hpp:201-202; SymmetryFunctions::initFromFile
 * src/SymmetryFunctions.cpp:266-407, Bispectrum::initFromFile
 * src/Bispectrum.cpp:852-1007). */
int ld_create_from_file(ld_descriptor **out, const char *path, int kind);

/* Reads and checks a parameter file on the host only (no device, no
 * tables): writes what the file defines, with the reference's reading
 * quirks applied, as "key = values" lines into text[capacity] (NUL
 * terminated; *length = bytes needed including the NUL).  Keys: kind,
 * n_species, species, cutoff_matrix, then type_codes, sizes, params
 * (symmetry functions) or rfac0, twojmax, diagonalstyle, rmin0,
 * switch_flag, bzero_flag, weights (bispectrum).  No reference counterpart
 * (its initFromFile builds the descriptor directly); lets a caller validate
 * a file without a GPU.  LD_ERR_PARSE on a malformed file, LD_ERR_CAPACITY
 * when text is too small (it then holds a truncated copy). */
int ld_describe_parameter_file(const char *path, int kind, char *text, size_t capacity,
                               size_t *length);

int ld_destroy(ld_descriptor *d);
int ld_width(const ld_descriptor *d, int *width);   /* DescriptorKind::width */
int ld_kind(const ld_descriptor *d, int *kind);     /* DescriptorKind::descriptor_kind */

/* ---------------- host-pointer API (staging through the device) ----------- */

/* Descriptor::compute (src/Descriptors.cpp:121-136).  desc[n_atoms*width]
 * is overwritten. */
int ld_compute(ld_descriptor *d, int n_atoms, int n_total, const int *species,
               const int *neighbor_list, const int *number_of_neighs,
               const double *coords, double *desc);

/* Descriptor::gradient (src/Descriptors.cpp:165-260) for the coordinates:
 * d_coords[n_total*3] = sum_{i,k} dE_ddesc[i,k] d desc[i,k] / d coords
 * (overwritten, ghost rows unfolded, as the reference returns them).
 * desc_out (nullable) receives the forward descriptors of the same pass. */
int ld_gradient(ld_descriptor *d, int n_atoms, int n_total, const int *species,
                const int *neighbor_list, const int *number_of_neighs,
                const double *coords, const double *dE_ddesc, double *d_coords,
                double *desc_out);

/* Gradient of a loss with respect to the descriptor's parameters, the part
 * of the reference's Enzyme gradient that it computes into a shadow
 * DescriptorKind and then discards (src/Descriptors.cpp:165-215):
 * d_params[k] = sum_{i,o} dE_ddesc[i,o] d desc[i,o] / d params[k].
 * Symmetry functions: in the layout of the flat parameter vector given at
 * init (g2 rows (eta, Rs), g3 (kappa), g4/g5 (zeta, lambda, eta); extra
 * columns of a row get 0).  Bispectrum: one value, dL/d rfac0.
 * n_params must equal ld_num_params. */
int ld_gradient_params(ld_descriptor *d, int n_atoms, int n_total, const int *species,
                       const int *neighbor_list, const int *number_of_neighs,
                       const double *coords, const double *dE_ddesc, double *d_params,
                       int n_params);

/* Number of values ld_gradient_params returns: the length of the flat
 * parameter vector of a symmetry-function descriptor, 1 (rfac0) for the
 * bispectrum. */
int ld_num_params(const ld_descriptor *d, int *n_params);

/* Descriptor::compute_batch (src/Descriptors.cpp:138-163). */
int ld_compute_batch(ld_descriptor *d, int n_configs, const int *n_atoms,
                     const int *config_ptr, int n_total, const int *species,
                     const int *neighbor_list, const int *number_of_neighs,
                     const double *coords, double *desc);

/* Descriptor::gradient_batch (src/Descriptors.cpp:263-352). */
int ld_gradient_batch(ld_descriptor *d, int n_configs, const int *n_atoms,
                      const int *config_ptr, int n_total, const int *species,
                      const int *neighbor_list, const int *number_of_neighs,
                      const double *coords, const double *dE_ddesc,
                      double *d_coords, double *desc_out);

/* Descriptor::compute_single_atom (src/Descriptors.cpp:355-365):
 * desc[width] of centre `index` with its own neighbour list. */
int ld_compute_single_atom(ld_descriptor *d, int index, int n_total,
                           const int *species, const int *neighbors, int n_neigh,
                           const double *coords, double *desc);

/* Descriptor::gradient_single_atom (src/Descriptors.cpp:368-452):
 * d_coords[n_total*3] = dE_ddesc . d desc_index / d coords (overwritten). */
int ld_gradient_single_atom(ld_descriptor *d, int index, int n_total,
                            const int *species, const int *neighbors, int n_neigh,
                            const double *coords, const double *dE_ddesc,
                            double *d_coords, double *desc_out);

/* Descriptor::jacobian (src/Descriptors.cpp:454-486): J[(width*n_atoms) x
 * (n_total*3)], row r = d desc_flat[r] / d coords_flat (overwritten). */
int ld_jacobian(ld_descriptor *d, int n_atoms, int n_total, const int *species,
                const int *neighbor_list, const int *number_of_neighs,
                const double *coords, double *J);

/* ---------------- device-pointer API (stream ordered) ---------------------- */
/* All array arguments are device pointers.  neigh_offsets[n_rows+1] is the
 * exclusive prefix sum of number_of_neighs (see ld_neighbor_offsets_dev);
 * row_centre[n_rows] (nullable: centre == row) maps rows to centre atoms.
 * Nothing is synchronised; errors raised inside kernels are reported by the
 * next ld_sync_status() on this descriptor. */

/* Exclusive prefix sum of number_of_neighs into neigh_offsets[n_rows+1];
 * when max_neigh != NULL it also returns max(number_of_neighs) (this
 * synchronises the stream). */
int ld_neighbor_offsets_dev(ld_descriptor *d, int n_rows, const int *number_of_neighs,
                            long long *neigh_offsets, int *max_neigh, ld_stream stream);

/* desc[n_rows*width] overwritten.  max_neigh bounds every row's neighbour
 * count (it sizes on-chip staging); a row above it raises LD_ERR_CAPACITY
 * through ld_sync_status and its outputs are set to NaN. */
int ld_compute_dev(ld_descriptor *d, int n_rows, const int *row_centre,
                   const int *species, const int *neighbor_list,
                   const long long *neigh_offsets, int max_neigh,
                   const double *coords, double *desc, ld_stream stream);

/* d_coords is ACCUMULATED into (the caller zeroes it), like the reference's
 * gradient shadow.  image (nullable, device int[n_total]) folds each ghost
 * row onto its contributing master row image[g] (the reference's
 * assemble_forces, python_package/libdescriptor/neighbor.py:227-263), in
 * which case d_coords has n_atoms rows where n_atoms > max(image).
 * desc_out (nullable) receives the forward descriptors. */
int ld_gradient_dev(ld_descriptor *d, int n_rows, const int *row_centre,
                    const int *species, const int *neighbor_list,
                    const long long *neigh_offsets, int max_neigh,
                    const double *coords,
                    const double *dE_ddesc, double *d_coords, double *desc_out,
                    const int *image, ld_stream stream);

/* Batched / served form of ld_compute_dev and ld_gradient_dev (no
 * counterpart in the reference; its compute_batch / gradient_batch,
 * src/Descriptors.cpp:138-163 and 190-215, loop over configurations on the
 * host).  Row r's neighbours are neighbor_list[nbl_begin[r] ..
 * nbl_begin[r] + (neigh_offsets[r+1] - neigh_offsets[r])): the rows of
 * many configurations held anywhere in one resident neighbour arena are
 * batched into one launch without copying their lists.  neigh_offsets is
 * the exclusive prefix sum of the rows' neighbour counts in batch order;
 * row_centre (required here) holds the rows' centre atoms in the same
 * coordinate arena that the neighbour indices address. */
int ld_compute_rows_dev(ld_descriptor *d, int n_rows, const int *row_centre,
                        const long long *nbl_begin, const int *species,
                        const int *neighbor_list, const long long *neigh_offsets,
                        int max_neigh, const double *coords, double *desc,
                        void *work, size_t work_bytes, ld_stream stream);
int ld_gradient_rows_dev(ld_descriptor *d, int n_rows, const int *row_centre,
                         const long long *nbl_begin, const int *species,
                         const int *neighbor_list, const long long *neigh_offsets,
                         int max_neigh, const double *coords,
                         const double *dE_ddesc, double *d_coords, double *desc_out,
                         const int *image, void *work, size_t work_bytes,
                         ld_stream stream);

/* Device work space (bytes, 256-byte aligned start required) that one
 * ld_compute_rows_dev (vjp = 0) or ld_gradient_rows_dev (vjp = 1) call over
 * n_rows rows needs when the caller passes `work`.  With work == NULL those
 * calls take it by stream-ordered allocation; a caller-owned work space keeps
 * the calls free of allocations (CUDA-graph capture, serving arenas).  One
 * work space serves one call in flight at a time. */
int ld_rows_work_bytes(const ld_descriptor *d, int n_rows, int vjp, size_t *bytes);

/* Launch-shape tuning of one descriptor (no counterpart in the reference).
 * Values <= 0 restore the built-in choice.  Results do not depend on the
 * tuning except for the order of floating-point atomic additions. */
#define LD_TUNE_SF_WARPS 0        /* symmetry functions: warps per CTA (1, 2, 4) */
#define LD_TUNE_CTAS_PER_SM 1     /* per-centre kernels: resident CTA cap per SM */
#define LD_TUNE_PAIR_GRID_MULT 2  /* bispectrum pair kernel: grid cap / (SMs x occupancy) */
#define LD_TUNE_DYNAMIC_QUEUE 3   /* centres claimed from an atomic counter: 1 on,
                                     2 off, 0 (built-in) on for 8192+ rows     */
#define LD_TUNE_SF_GENERIC 4      /* 1: table-driven symmetry-function kernel even
                                     when the parameter set has a factored form */
int ld_set_tuning(ld_descriptor *d, int key, int value);
int ld_get_tuning(const ld_descriptor *d, int key, int *value);

/* Serving runtime (no counterpart in the reference): staging of one request
 * into resident device rings.  The request's arrays are host arrays in the
 * reference's layout with local indices (coords[n_total*3], species and
 * image[n_total] with image = master row in 0..n_atoms-1,
 * number_of_neighs[n_atoms], neighbor_list[nnz] into 0..n_total-1,
 * dE_ddesc[n_atoms*width]).  ld_stage_request checks the indices, writes the
 * fields into `staging` (pinned host memory, 256-byte aligned, at least
 * ld_stage_bytes) with every index rebased to the ring slots row0 / atom0 /
 * entry0, and enqueues the uploads on `stream`:
 *   d_coords[atom0..], d_species[atom0..], d_image[atom0..] (= row0 + image),
 *   d_nbl[entry0..] (= atom0 + neighbour), d_centre[row0..] (= atom0 + j),
 *   d_begin[row0..] (= entry0 + exclusive prefix of the counts),
 *   d_counts[row0..], d_dE[row0*width..].
 * The staging memory may be reused once the stream has passed the uploads.
 * The staged rows then join batches of ld_gradient_rows_dev over the rings
 * (row_centre = d_centre, nbl_begin = d_begin, image = d_image). */
int ld_stage_bytes(int n_atoms, int n_total, long long nnz, int width, size_t *bytes);
int ld_stage_request(int n_atoms, int n_total, long long nnz, int width,
                     int row0, int atom0, long long entry0,
                     const double *coords, const int *species, const int *image,
                     const int *neighbor_list, const int *number_of_neighs,
                     const double *dE_ddesc, void *staging, size_t staging_bytes,
                     double *d_coords, int *d_species, int *d_image, int *d_nbl,
                     int *d_centre, long long *d_begin, int *d_counts, double *d_dE,
                     ld_stream stream);

/* The two halves of ld_stage_request, for a runtime that packs several
 * requests on host threads at once and then enqueues their uploads in
 * admission order (no reference counterpart).  ld_stage_pack writes the
 * request into `staging` exactly as ld_stage_request does (indices rebased
 * and checked) on the calling thread only and touches no device: calls for
 * different requests and staging areas may run concurrently.
 * ld_stage_upload enqueues the uploads of a packed staging area on
 * `stream`, with the same slots and sizes as its ld_stage_pack. */
int ld_stage_pack(int n_atoms, int n_total, long long nnz, int width,
                  int row0, int atom0, long long entry0,
                  const double *coords, const int *species, const int *image,
                  const int *neighbor_list, const int *number_of_neighs,
                  const double *dE_ddesc, void *staging, size_t staging_bytes);
int ld_stage_upload(int n_atoms, int n_total, long long nnz, int width,
                    int row0, int atom0, long long entry0, void *staging, size_t staging_bytes,
                    double *d_coords, int *d_species, int *d_image, int *d_nbl,
                    int *d_centre, long long *d_begin, int *d_counts, double *d_dE,
                    ld_stream stream);

/* Staging by chunk (no reference counterpart): requests admitted together
 * into consecutive ring slots share one staging block laid out field by field
 * (all their coordinates, then all species, ... in admission order), so the
 * block uploads with one copy per field instead of one per field and request.
 * ld_stage_pack_fields writes one request's fields at the given host pointers
 * -- the request's place inside each field's run -- with indices rebased to
 * the slots and checked exactly as ld_stage_pack does; it touches no device
 * and calls for different requests may run concurrently.
 * ld_stage_upload_fields enqueues n_fields host-to-device copies
 * (dst[i] <- src[i], bytes[i]; zero-byte entries are skipped) on `stream`. */
int ld_stage_pack_fields(int n_atoms, int n_total, long long nnz, int width,
                         int row0, int atom0, long long entry0,
                         const double *coords, const int *species, const int *image,
                         const int *neighbor_list, const int *number_of_neighs,
                         const double *dE_ddesc, double *coords_out, int *species_out,
                         int *image_out, int *nbl_out, int *centre_out, long long *begin_out,
                         int *counts_out, double *dE_out);
int ld_stage_upload_fields(int n_fields, const void *const *src, void *const *dst,
                           const size_t *bytes, ld_stream stream);

/* Descriptor + VJP pass that allocates no device memory (no counterpart in
 * the reference; it serves callers that cannot call cudaMalloc while they
 * evaluate forces, e.g. engines whose device memory is owned by their own
 * pool or loops with a no-allocation rule).  Same arguments as
 * ld_gradient_dev, except that it takes number_of_neighs (device, n_rows)
 * instead of neigh_offsets: the row offsets, the prefix-sum work space and
 * the status word live in a fixed 4 MiB array of the library's own device
 * memory, held by every GPU that loads the library until the process exits.
 * Limit: n_rows <= 262144 per call (larger requests return LD_ERR_CAPACITY).
 * d_coords is accumulated into; the call waits for `stream` and returns any
 * device-side status (LD_ERR_CAPACITY when a row exceeds max_neigh).  All
 * calls share the array: calls that overlap on the GPU race on it.  The
 * current device must be the descriptor's (else LD_ERR_INVALID_ARG), and, as
 * with ld_gradient_dev, the caller keeps every index inside the coordinates:
 * the number of coordinate rows is not passed, so no device-side index check
 * runs. */
int ld_gradient_counts_dev_noalloc(ld_descriptor *d, int n_rows, const int *row_centre,
                                   const int *species, const int *neighbor_list,
                                   const int *number_of_neighs, int max_neigh,
                                   const double *coords, const double *dE_ddesc,
                                   double *d_coords, double *desc_out, const int *image,
                                   ld_stream stream);

/* Wait for `stream` and return the first device-side error status raised by
 * this descriptor's kernels since the last call (then clear it). */
int ld_sync_status(ld_descriptor *d, ld_stream stream);

/* ---------------- neighbour lists (python_bindings/neighbor) -------------- */

/* nbl_create_paddings (python_bindings/neighbor/neighbor_list.cpp:283-418):
 * ghost images of `coords` within `cutoff` of the periodic cell faces.
 * Call with pad_* == NULL to get *n_pad, then again with buffers of that
 * size (pad_coords n_pad*3, pad_species n_pad, pad_image n_pad). */
int ld_create_paddings(double cutoff, const double *cell, const int *pbc,
                       const double *coords, const int *species, int n_atoms,
                       int *n_pad, double *pad_coords, int *pad_species,
                       int *pad_image);

/* nbl_build (neighbor_list.cpp:78-243) with one cutoff, flattened to the
 * (number_of_neighs, neighbor_list) layout of the rows 0..n_query-1.  Call
 * with neighbor_list == NULL to get *nnz (counts are filled), then again. */
int ld_build_neighbor_list(const double *coords, int n_total, double cutoff,
                           const int *need_neigh, int n_query,
                           int *number_of_neighs, int *neighbor_list,
                           long long *nnz);

/* Device forms of the two calls above (same ghosts in the same order with
 * the same coordinates, and the same lists in the same order; every product
 * and sum rounded as on the host).  coords, species, need_neigh and all
 * outputs are device arrays; cell (9) and pbc (3) are host arrays.
 *
 * ld_create_paddings_dev: *n_pad receives the ghost count; with all of
 * pad_coords / pad_species / pad_image NULL it only counts, otherwise it
 * writes them (capacity max_pad ghosts, LD_ERR_CAPACITY beyond).
 *
 * ld_build_neighbor_list_dev: fills number_of_neighs[n_query] and the CSR
 * offsets neigh_offsets[n_query+1] (the form ld_gradient_dev takes), and
 * *nnz, *max_neigh (nullable); with neighbor_list NULL it stops there,
 * otherwise it writes the list (capacity max_nnz, LD_ERR_CAPACITY beyond).
 * Both wait for `stream` before returning (the counts are read back). */
int ld_create_paddings_dev(double cutoff, const double *cell, const int *pbc,
                           const double *coords, const int *species, int n_atoms,
                           int max_pad, double *pad_coords, int *pad_species,
                           int *pad_image, int *n_pad, ld_stream stream);
int ld_build_neighbor_list_dev(const double *coords, int n_total, double cutoff,
                               const int *need_neigh, int n_query,
                               int *number_of_neighs, long long *neigh_offsets,
                               long long max_nnz, int *neighbor_list,
                               long long *nnz, int *max_neigh, ld_stream stream);

/* ---------------- measurement helpers ------------------------------------- */

/* Run `iters` rounds of FP64 fused multiply-adds on the device and report
 * the achieved FP64 rate (TFLOP/s, FMA = 2 flops).  Used as the roofline
 * denominator of the FP64-bound kernels. */
int ld_measure_fp64_peak(int iters, double *tflops);

/* Cost of one FP64 library call in FP64-pipe flops at the rate
 * fp64_tflops (from ld_measure_fp64_peak): op 0 exp, 1 sincos, 2 sqrt,
 * 3 divide, 4 tan, 5 pow, 6 cos.  Weights transcendental calls in the
 * algorithmic flop counts of the roofline. */
int ld_measure_fp64_op_cost(int op, int iters, double fp64_tflops, double *flop_equiv);

/* Number of this library's kernel launches issued so far (all descriptors). */
long long ld_launch_count(void);

/* Number of device allocations this library has requested so far: growth of
 * a handle's buffers (cudaMalloc) and stream-ordered scratch taken from the
 * library's per-device pool.  No reference counterpart (the reference
 * allocates host memory only); lets a caller check that a call allocated
 * nothing. */
long long ld_alloc_count(void);

/* Fault injection for tests of the out-of-memory path (no reference
 * counterpart): the k-th device allocation from now (k >= 1) fails with
 * LD_ERR_OOM, as a failed cudaMalloc would; k = 0 disarms.  Host-side only:
 * nothing is asked of the device, and the handle stays usable afterwards. */
int ld_fail_next_allocation(int k);

/* Test hook (no reference counterpart): from now on every new device
 * allocation of the library -- grow-only buffers and scratch-pool blocks -- is
 * filled with `byte` (0..255; 0xff makes every double a NaN) before use, so
 * that a read of memory no kernel wrote shows on every run instead of
 * depending on what the memory held before; -1 (the default) switches it
 * off.  Costs one memset per allocation while on. */
int ld_debug_fill_scratch(int byte);

/* Self-test of the kernels' bounded waits (no reference counterpart): one
 * CTA arms a shared-memory barrier for a bulk copy that is never issued and
 * waits for it at most limit_ns nanoseconds of device time (1 .. 1e9), the
 * same wait the Z kernel uses for its bulk-copied U tile.  Returns
 * LD_ERR_TIMEOUT when the wait ran out -- the expected outcome -- with the
 * device left usable; LD_OK would mean the wait never gave up. */
int ld_debug_bulk_wait_timeout(long long limit_ns);

/* Pinned (page-locked) host memory for results: the device writes into it at
 * the link's rate, where a copy into fresh pageable memory runs several
 * times slower.  Blocks are rounded up to 64 KiB; a released block is kept
 * for reuse (up to 256 MiB in all) and handed out again for requests of
 * between half its size and its size.  While 512 MiB are handed out and not
 * released, a request that no kept block serves fails with LD_ERR_CAPACITY
 * (callers then use pageable memory).  No reference counterpart: the
 * reference computes on the host.  ld_host_alloc sets *p to NULL on failure;
 * ld_host_free(NULL) and pointers that did not come from ld_host_alloc are
 * ignored.  Both are thread-safe. */
int ld_host_alloc(size_t bytes, void **p);
void ld_host_free(void *p);

#ifdef __cplusplus
}
#endif
#endif /* LIBDESCRIPTOR_B200_H_ */
