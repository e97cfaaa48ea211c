/*
 * ld_oracle.h -- CPU oracle for the descriptor hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (libdescriptor_b200/)
 * links, imports or calls this code; only tests/, __graft_entry__.smoke()
 * and bench.py's cpu_baseline / --impl reference legs use it, as the checker.
 *
 * A plain-C restatement of libdescriptor's per-atom descriptor algorithms
 * (reference files cited per function in ld_oracle.c) plus an independent
 * analytic reverse-mode gradient (the reference differentiates with Enzyme,
 * which cannot be built offline).  Parity of the forward restatement is
 * pinned against the reference's own C++ compiled from source
 * (oracle/Makefile -> oracle/_ref/libldref.so) and against committed golden
 * fixtures (tests/golden/).  The gradient is pinned by finite differences of
 * the reference forward (8th-order stencil of the reference's
 * include/finite_difference.hpp).
 */
#ifndef LD_ORACLE_H_
#define LD_ORACLE_H_

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ */
/* Symmetry functions (Behler G1..G5)                                   */
/* ------------------------------------------------------------------ */
typedef struct ldo_sf ldo_sf;

/* types[b] in {1..5} (g1..g5); rows[b] parameter sets, cols[b] params per
 * set; params = concatenation of row-major blocks.  rcut = n_species^2
 * row-major cutoff matrix. */
ldo_sf *ldo_sf_new(int n_species, const double *rcut, int n_blocks,
                   const int *types, const int *rows, const int *cols,
                   const double *params);
void ldo_sf_free(ldo_sf *sf);
int ldo_sf_width(const ldo_sf *sf);

/* desc[width] += descriptor of centre `index` (reference accumulate rule). */
void ldo_sf_atom(const ldo_sf *sf, int index, const int *species,
                 const int *nbl, int n_neigh, const double *coords,
                 double *desc);
/* dcoords[n_total*3] += sum_d dE[d] * d desc[d] / d coords. */
void ldo_sf_atom_vjp(const ldo_sf *sf, int index, const int *species,
                     const int *nbl, int n_neigh, const double *coords,
                     const double *dE, double *dcoords);

/* ------------------------------------------------------------------ */
/* Bispectrum (SNAP-style U -> Z -> B)                                   */
/* ------------------------------------------------------------------ */
typedef struct ldo_bs ldo_bs;

ldo_bs *ldo_bs_new(double rfac0, int twojmax, int diagonalstyle, double rmin0,
                   int switch_flag, int bzero_flag, int n_species,
                   const double *rcut, const double *weights);
void ldo_bs_free(ldo_bs *bs);
int ldo_bs_width(const ldo_bs *bs);
/* output triple (j1,j2,j) of component `c` */
void ldo_bs_triple(const ldo_bs *bs, int c, int *j1, int *j2, int *j);

/* desc[width] = bispectrum of centre `index`.  When dE != NULL also
 * dcoords[n_total*3] += VJP (analytic, independent reverse mode). */
void ldo_bs_atom(const ldo_bs *bs, int index, const int *species,
                 const int *nbl, int n_neigh, const double *coords,
                 double *desc, const double *dE, double *dcoords);

/* ------------------------------------------------------------------ */
/* Whole-configuration drivers (reference Descriptor::compute /        */
/* compute_batch layout), threaded over centre atoms with pthreads.     */
/* kind: 0 = symmetry functions, 1 = bispectrum.                       */
/* Batch layout: n_configs==0 means a single configuration whose       */
/* centres are 0..n_atoms[0]-1; otherwise centre (c, j) is             */
/* j + config_ptr[c].  Neighbour rows are consumed in centre order.    */
/* dE/dcoords may be NULL (forward only).  desc is overwritten,        */
/* dcoords (n_total*3) is overwritten.                                  */
/* ------------------------------------------------------------------ */
int ldo_run(int kind, const void *obj, int n_configs, const int *n_atoms,
            const int *config_ptr, const int *species, const int *nbl,
            const int *counts, const double *coords, int n_total,
            double *desc, const double *dE, double *dcoords, int n_threads);

/* Finite-difference VJP of the oracle forward w.r.t. the listed flat
 * coordinate indices: out[q] = sum dE * d desc / d x.  step > 0 uses the
 * 2-point central difference with that step; step <= 0 the reference's
 * 8th-order stencil and step (include/finite_difference.hpp:60-143). */
int ldo_fd_vjp(int kind, const void *obj, int n_atoms, const int *species,
               const int *nbl, const int *counts, const double *coords,
               int n_total, const double *dE, int n_idx, const int *idx,
               double *out, double step, int n_threads);

#ifdef __cplusplus
}
#endif
#endif
