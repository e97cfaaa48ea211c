/*
 * ld_oracle.c -- CPU oracle (TEST INFRASTRUCTURE ONLY; see ld_oracle.h).
 *
 * Forward restatements follow the reference algorithms step by step so that
 * rounding stays close to the reference's own CPU results:
 *   symmetry functions : src/SymmetryFunctions.cpp:67-259 (cut_cos, sym_g1..g5,
 *                        SymmetryFunctions::compute)
 *   bispectrum         : src/Bispectrum.cpp:229-297 (compute), :314-343
 *                        (compute_ui), :345-389 (compute_zi), :391-427
 *                        (compute_bi), :429-468 (copy_bi2bvec), :490-554
 *                        (compute_uarray), :556-586 (add_uarraytot,
 *                        compute_sfac), :683-735 (Clebsch-Gordan, rootpq)
 *   drivers            : src/Descriptors.cpp:121-163 (compute, compute_batch)
 *   finite differences : include/finite_difference.hpp:46-143
 *
 * The gradients are NOT restatements (the reference has no gradient code of
 * its own; Enzyme generates it).  They are an independent analytic reverse
 * mode written from the mathematics:
 *   - symmetry functions: per-term partial derivatives w.r.t. the three
 *     interatomic distances, chained to Cartesian coordinates;
 *   - bispectrum: reverse sweep through B and Z (bilinear CG contraction)
 *     to dL/dUtot over the FULL (ma,mb) matrices, then forward-mode dual
 *     numbers through the U recursion of every neighbour.
 * This deliberately differs from the GPU method (adjoint "Y" arrays from the
 * bispectrum symmetry identity and half-matrix contraction), so the two
 * cross-check each other.
 */
#include "ld_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#define LDO_PI 3.1415926535897932

/* ================================================================== */
/* Symmetry functions                                                  */
/* ================================================================== */
struct ldo_sf {
    int ns;
    double *rcut;
    int nb;
    int *type, *rows, *cols, *start;
    double *par;     /* concatenated blocks */
    int *par_off;    /* offset of block b in par */
    int width;
    int has3;
};

/* cut_cos, src/SymmetryFunctions.cpp:67-69 */
static double ldo_cutc(double r, double rc) {
    return (r < rc) ? 0.5 * (cos(LDO_PI * r / rc) + 1.0) : 0.0;
}
static double ldo_dcutc(double r, double rc) {
    return (r < rc) ? -0.5 * sin(LDO_PI * r / rc) * (LDO_PI / rc) : 0.0;
}

ldo_sf *ldo_sf_new(int n_species, const double *rcut, int n_blocks,
                   const int *types, const int *rows, const int *cols,
                   const double *params) {
    ldo_sf *sf = (ldo_sf *)calloc(1, sizeof(ldo_sf));
    sf->ns = n_species;
    sf->rcut = (double *)malloc(sizeof(double) * n_species * n_species);
    memcpy(sf->rcut, rcut, sizeof(double) * n_species * n_species);
    sf->nb = n_blocks;
    sf->type = (int *)malloc(sizeof(int) * n_blocks);
    sf->rows = (int *)malloc(sizeof(int) * n_blocks);
    sf->cols = (int *)malloc(sizeof(int) * n_blocks);
    sf->start = (int *)malloc(sizeof(int) * n_blocks);
    sf->par_off = (int *)malloc(sizeof(int) * n_blocks);
    int np = 0, w = 0;
    for (int b = 0; b < n_blocks; ++b) {
        sf->type[b] = types[b];
        sf->rows[b] = rows[b];
        sf->cols[b] = cols[b];
        sf->start[b] = w;          /* add_descriptor: starting_index_ */
        sf->par_off[b] = np;
        np += rows[b] * cols[b];
        w += rows[b];
        if (types[b] == 4 || types[b] == 5) sf->has3 = 1;
    }
    sf->par = (double *)malloc(sizeof(double) * (np > 0 ? np : 1));
    if (np) memcpy(sf->par, params, sizeof(double) * np);
    sf->width = w;
    return sf;
}

void ldo_sf_free(ldo_sf *sf) {
    if (!sf) return;
    free(sf->rcut); free(sf->type); free(sf->rows); free(sf->cols);
    free(sf->start); free(sf->par); free(sf->par_off); free(sf);
}

int ldo_sf_width(const ldo_sf *sf) { return sf->width; }

/* sym_g4 / sym_g5, src/SymmetryFunctions.cpp:75-127; r = {rij, rik, rjk} */
static double ldo_g45(int type, double zeta, double lambda, double eta,
                      const double *r, const double *rc) {
    const double rij = r[0], rik = r[1], rjk = r[2];
    if (type == 4) {
        if (rij > rc[0] || rik > rc[1] || rjk > rc[2]) return 0.0;
    } else {
        if (rij > rc[0] || rik > rc[1]) return 0.0;
    }
    const double rijsq = rij * rij, riksq = rik * rik, rjksq = rjk * rjk;
    const double cos_ijk = (rijsq + riksq - rjksq) / (2 * rij * rik);
    const double base = 1.0 + lambda * cos_ijk;
    const double costerm = (base <= 0) ? 0.0 : pow(base, zeta);
    if (type == 4) {
        const double eterm = exp(-eta * (rijsq + riksq + rjksq));
        return pow(2, 1 - zeta) * costerm * eterm * ldo_cutc(rij, rc[0]) *
               ldo_cutc(rik, rc[1]) * ldo_cutc(rjk, rc[2]);
    }
    const double eterm = exp(-eta * (rijsq + riksq));
    return pow(2, 1 - zeta) * costerm * eterm * ldo_cutc(rij, rc[0]) *
           ldo_cutc(rik, rc[1]);
}

/* value + partials w.r.t. (rij, rik, rjk) of g4/g5 (analytic) */
static void ldo_g45_grad(int type, double zeta, double lambda, double eta,
                         const double *r, const double *rc, double *dr) {
    dr[0] = dr[1] = dr[2] = 0.0;
    const double a = r[0], b = r[1], d = r[2];
    if (type == 4) {
        if (a > rc[0] || b > rc[1] || d > rc[2]) return;
    } else {
        if (a > rc[0] || b > rc[1]) return;
    }
    const double cth = (a * a + b * b - d * d) / (2 * a * b);
    const double c = 1.0 + lambda * cth;
    if (c <= 0) return;
    const double P = pow(2, 1 - zeta);
    const double cz = pow(c, zeta);
    const double dcz = zeta * pow(c, zeta - 1.0) * lambda; /* d c^z / d cos */
    const double dcos_da = (a * a - b * b + d * d) / (2 * a * a * b);
    const double dcos_db = (b * b - a * a + d * d) / (2 * a * b * b);
    const double dcos_dd = -d / (a * b);
    const double fa = ldo_cutc(a, rc[0]), fb = ldo_cutc(b, rc[1]);
    const double dfa = ldo_dcutc(a, rc[0]), dfb = ldo_dcutc(b, rc[1]);
    if (type == 4) {
        const double fd = ldo_cutc(d, rc[2]), dfd = ldo_dcutc(d, rc[2]);
        const double E = exp(-eta * (a * a + b * b + d * d));
        const double F = fa * fb * fd;
        dr[0] = P * E * (dcz * dcos_da * F + cz * (-2 * eta * a) * F + cz * dfa * fb * fd);
        dr[1] = P * E * (dcz * dcos_db * F + cz * (-2 * eta * b) * F + cz * fa * dfb * fd);
        dr[2] = P * E * (dcz * dcos_dd * F + cz * (-2 * eta * d) * F + cz * fa * fb * dfd);
    } else {
        const double E = exp(-eta * (a * a + b * b));
        const double F = fa * fb;
        dr[0] = P * E * (dcz * dcos_da * F + cz * (-2 * eta * a) * F + cz * dfa * fb);
        dr[1] = P * E * (dcz * dcos_db * F + cz * (-2 * eta * b) * F + cz * fa * dfb);
        dr[2] = P * E * (dcz * dcos_dd * F);
    }
}

/* two-body value, src/SymmetryFunctions.cpp:129-139 */
static double ldo_g123(int type, const double *p, double r, double rc) {
    if (type == 1) return ldo_cutc(r, rc);
    if (type == 2) return exp(-p[0] * (r - p[1]) * (r - p[1])) * ldo_cutc(r, rc);
    return cos(p[0] * r) * ldo_cutc(r, rc);
}
static double ldo_g123_grad(int type, const double *p, double r, double rc) {
    if (type == 1) return ldo_dcutc(r, rc);
    if (type == 2) {
        const double e = exp(-p[0] * (r - p[1]) * (r - p[1]));
        return e * (-2 * p[0] * (r - p[1]) * ldo_cutc(r, rc) + ldo_dcutc(r, rc));
    }
    return -p[0] * sin(p[0] * r) * ldo_cutc(r, rc) + cos(p[0] * r) * ldo_dcutc(r, rc);
}

/* SymmetryFunctions::compute, src/SymmetryFunctions.cpp:141-259 */
void ldo_sf_atom(const ldo_sf *sf, int index, const int *species,
                 const int *nbl, int n, const double *coords, double *desc) {
    const int is = species[index];
    const double *ci = coords + 3 * index;
    for (int jj = 0; jj < n; ++jj) {
        const int j = nbl[jj];
        const int js = species[j];
        const double rcij = sf->rcut[is * sf->ns + js];
        double rij[3];
        for (int d = 0; d < 3; ++d) rij[d] = coords[3 * j + d] - ci[d];
        const double rijsq = rij[0] * rij[0] + rij[1] * rij[1] + rij[2] * rij[2];
        const double rijmag = sqrt(rijsq);
        if (rijmag > rcij) continue;
        for (int p = 0; p < sf->nb; ++p) {
            const int t = sf->type[p];
            if (t > 3) continue;
            int idx = sf->start[p];
            for (int q = 0; q < sf->rows[p]; ++q) {
                const double *pp = sf->par + sf->par_off[p] + q * sf->cols[p];
                desc[idx] += ldo_g123(t, pp, rijmag, rcij);
                ++idx;
            }
        }
        if (!sf->has3) continue;
        for (int kk = jj + 1; kk < n; ++kk) {
            const int k = nbl[kk];
            const int ks = species[k];
            const double rcik = sf->rcut[is * sf->ns + ks];
            const double rcjk = sf->rcut[js * sf->ns + ks];
            double rik[3], rjk[3];
            for (int d = 0; d < 3; ++d) {
                rik[d] = coords[3 * k + d] - ci[d];
                rjk[d] = coords[3 * k + d] - coords[3 * j + d];
            }
            const double riksq = rik[0] * rik[0] + rik[1] * rik[1] + rik[2] * rik[2];
            const double rjksq = rjk[0] * rjk[0] + rjk[1] * rjk[1] + rjk[2] * rjk[2];
            const double rikmag = sqrt(riksq);
            const double rjkmag = sqrt(rjksq);
            if (rikmag > rcik) continue;
            const double rv[3] = {rijmag, rikmag, rjkmag};
            const double rcv[3] = {rcij, rcik, rcjk};
            for (int p = 0; p < sf->nb; ++p) {
                const int t = sf->type[p];
                if (t != 4 && t != 5) continue;
                int idx = sf->start[p];
                for (int q = 0; q < sf->rows[p]; ++q) {
                    const double *pp = sf->par + sf->par_off[p] + q * sf->cols[p];
                    desc[idx] += ldo_g45(t, pp[0], pp[1], pp[2], rv, rcv);
                    ++idx;
                }
            }
        }
    }
}

void ldo_sf_atom_vjp(const ldo_sf *sf, int index, const int *species,
                     const int *nbl, int n, const double *coords,
                     const double *dE, double *dcoords) {
    const int is = species[index];
    const double *ci = coords + 3 * index;
    for (int jj = 0; jj < n; ++jj) {
        const int j = nbl[jj];
        const int js = species[j];
        const double rcij = sf->rcut[is * sf->ns + js];
        double rij[3];
        for (int d = 0; d < 3; ++d) rij[d] = coords[3 * j + d] - ci[d];
        const double rijmag = sqrt(rij[0] * rij[0] + rij[1] * rij[1] + rij[2] * rij[2]);
        if (rijmag > rcij) continue;
        double ga = 0.0;
        for (int p = 0; p < sf->nb; ++p) {
            const int t = sf->type[p];
            if (t > 3) continue;
            for (int q = 0; q < sf->rows[p]; ++q) {
                const double *pp = sf->par + sf->par_off[p] + q * sf->cols[p];
                ga += dE[sf->start[p] + q] * ldo_g123_grad(t, pp, rijmag, rcij);
            }
        }
        for (int d = 0; d < 3; ++d) {
            const double g = ga * rij[d] / rijmag;
            dcoords[3 * j + d] += g;
            dcoords[3 * index + d] -= g;
        }
        if (!sf->has3) continue;
        for (int kk = jj + 1; kk < n; ++kk) {
            const int k = nbl[kk];
            const int ks = species[k];
            const double rcik = sf->rcut[is * sf->ns + ks];
            const double rcjk = sf->rcut[js * sf->ns + ks];
            double rik[3], rjk[3];
            for (int d = 0; d < 3; ++d) {
                rik[d] = coords[3 * k + d] - ci[d];
                rjk[d] = coords[3 * k + d] - coords[3 * j + d];
            }
            const double rikmag = sqrt(rik[0] * rik[0] + rik[1] * rik[1] + rik[2] * rik[2]);
            const double rjkmag = sqrt(rjk[0] * rjk[0] + rjk[1] * rjk[1] + rjk[2] * rjk[2]);
            if (rikmag > rcik) continue;
            const double rv[3] = {rijmag, rikmag, rjkmag};
            const double rcv[3] = {rcij, rcik, rcjk};
            double gd[3] = {0, 0, 0};
            for (int p = 0; p < sf->nb; ++p) {
                const int t = sf->type[p];
                if (t != 4 && t != 5) continue;
                for (int q = 0; q < sf->rows[p]; ++q) {
                    const double *pp = sf->par + sf->par_off[p] + q * sf->cols[p];
                    double dr[3];
                    ldo_g45_grad(t, pp[0], pp[1], pp[2], rv, rcv, dr);
                    const double g = dE[sf->start[p] + q];
                    gd[0] += g * dr[0];
                    gd[1] += g * dr[1];
                    gd[2] += g * dr[2];
                }
            }
            for (int d = 0; d < 3; ++d) {
                const double uij = rij[d] / rijmag, uik = rik[d] / rikmag;
                const double ujk = rjkmag > 0 ? rjk[d] / rjkmag : 0.0;
                dcoords[3 * j + d] += gd[0] * uij - gd[2] * ujk;
                dcoords[3 * k + d] += gd[1] * uik + gd[2] * ujk;
                dcoords[3 * index + d] -= gd[0] * uij + gd[1] * uik;
            }
        }
    }
}

/* ================================================================== */
/* Bispectrum                                                          */
/* ================================================================== */
struct ldo_bs {
    int J, style, switch_flag, bzero_flag, ns, ncoeff;
    double rfac0, rmin0, wself;
    double *rcut, *wj;
    int *oj1, *oj2, *oj;
    double *cg;      /* [(j1*D + j2)*D + j][m1*D + m2], D = J+1 */
    double *rootpq;  /* [p*(J+1) + q] = sqrt(p/q) */
    double *bzero;   /* [J+1] */
};

#define D1(bs) ((bs)->J + 1)
#define CGI(bs, j1, j2, j, m1, m2) \
    (((((j1) * D1(bs) + (j2)) * D1(bs) + (j)) * D1(bs) + (m1)) * D1(bs) + (m2))
#define UI(bs, j, ma, mb) ((((j) * D1(bs)) + (ma)) * D1(bs) + (mb))

static double ldo_fact(int n) {
    double f = 1.0;
    for (int i = 2; i <= n; ++i) f *= (double)i;
    return f;
}

/* Racah formula; same definition as Bispectrum::init_clebsch_gordan
 * (src/Bispectrum.cpp:677-727), doubled-integer convention. */
static void ldo_bs_init_cg(ldo_bs *bs) {
    const int J = bs->J;
    for (int j1 = 0; j1 <= J; ++j1)
        for (int j2 = 0; j2 <= J; ++j2)
            for (int j = abs(j1 - j2); j <= (J < j1 + j2 ? J : j1 + j2); j += 2)
                for (int m1 = 0; m1 <= j1; ++m1) {
                    const int aa2 = 2 * m1 - j1;
                    for (int m2 = 0; m2 <= j2; ++m2) {
                        const int bb2 = 2 * m2 - j2;
                        const int m = (aa2 + bb2 + j) / 2;
                        if (m < 0 || m > j) continue;
                        int zlo = 0;
                        if (-(j - j2 + aa2) / 2 > zlo) zlo = -(j - j2 + aa2) / 2;
                        if (-(j - j1 - bb2) / 2 > zlo) zlo = -(j - j1 - bb2) / 2;
                        int zhi = (j1 + j2 - j) / 2;
                        if ((j1 - aa2) / 2 < zhi) zhi = (j1 - aa2) / 2;
                        if ((j2 + bb2) / 2 < zhi) zhi = (j2 + bb2) / 2;
                        double sum = 0.0;
                        for (int z = zlo; z <= zhi; ++z) {
                            const double sgn = (z % 2) ? -1.0 : 1.0;
                            sum += sgn / (ldo_fact(z) * ldo_fact((j1 + j2 - j) / 2 - z) *
                                          ldo_fact((j1 - aa2) / 2 - z) *
                                          ldo_fact((j2 + bb2) / 2 - z) *
                                          ldo_fact((j - j2 + aa2) / 2 + z) *
                                          ldo_fact((j - j1 - bb2) / 2 + z));
                        }
                        const int cc2 = 2 * m - j;
                        const double dcg = sqrt(ldo_fact((j1 + j2 - j) / 2) *
                                                ldo_fact((j1 - j2 + j) / 2) *
                                                ldo_fact((-j1 + j2 + j) / 2) /
                                                ldo_fact((j1 + j2 + j) / 2 + 1));
                        const double sfaccg = sqrt(
                            ldo_fact((j1 + aa2) / 2) * ldo_fact((j1 - aa2) / 2) *
                            ldo_fact((j2 + bb2) / 2) * ldo_fact((j2 - bb2) / 2) *
                            ldo_fact((j + cc2) / 2) * ldo_fact((j - cc2) / 2) * (j + 1));
                        bs->cg[CGI(bs, j1, j2, j, m1, m2)] = sum * dcg * sfaccg;
                    }
                }
}

/* output triples per diagonal style, src/Bispectrum.cpp:429-468 */
static int ldo_bs_outputs(ldo_bs *bs, int fill) {
    const int J = bs->J;
    int n = 0;
#define EMIT(a, b, c)                                     \
    do {                                                  \
        if (fill) { bs->oj1[n] = a; bs->oj2[n] = b; bs->oj[n] = c; } \
        ++n;                                              \
    } while (0)
    switch (bs->style) {
    case 0:
        for (int j1 = 0; j1 <= J; ++j1)
            for (int j2 = 0; j2 <= j1; ++j2)
                for (int j = j1 - j2; j <= (J < j1 + j2 ? J : j1 + j2); j += 2) EMIT(j1, j2, j);
        break;
    case 1:
        for (int j1 = 0; j1 <= J; ++j1)
            for (int j = 0; j <= (J < 2 * j1 ? J : 2 * j1); j += 2) EMIT(j1, j1, j);
        break;
    case 2:
        for (int j1 = 0; j1 <= J; ++j1) EMIT(j1, j1, j1);
        break;
    case 3:
        for (int j1 = 0; j1 <= J; ++j1)
            for (int j2 = 0; j2 <= j1; ++j2)
                for (int j = j1 - j2; j <= (J < j1 + j2 ? J : j1 + j2); j += 2)
                    if (j >= j1) EMIT(j1, j2, j);
        break;
    default:
        return -1;
    }
#undef EMIT
    return n;
}

ldo_bs *ldo_bs_new(double rfac0, int twojmax, int diagonalstyle, double rmin0,
                   int switch_flag, int bzero_flag, int n_species,
                   const double *rcut, const double *weights) {
    if (twojmax < 0 || diagonalstyle < 0 || diagonalstyle > 3) return NULL;
    ldo_bs *bs = (ldo_bs *)calloc(1, sizeof(ldo_bs));
    bs->J = twojmax;
    bs->style = diagonalstyle;
    bs->rfac0 = rfac0;
    bs->rmin0 = rmin0;
    bs->switch_flag = switch_flag;
    bs->bzero_flag = bzero_flag;
    bs->wself = 1.0;
    bs->ns = n_species;
    bs->rcut = (double *)malloc(sizeof(double) * n_species * n_species);
    memcpy(bs->rcut, rcut, sizeof(double) * n_species * n_species);
    bs->wj = (double *)malloc(sizeof(double) * n_species);
    memcpy(bs->wj, weights, sizeof(double) * n_species);
    const int D = twojmax + 1;
    bs->cg = (double *)calloc((size_t)D * D * D * D * D, sizeof(double));
    ldo_bs_init_cg(bs);
    bs->rootpq = (double *)calloc((size_t)D * D, sizeof(double));
    for (int p = 1; p <= twojmax; ++p)
        for (int q = 1; q <= twojmax; ++q)
            bs->rootpq[p * D + q] = sqrt((double)p / q);
    bs->bzero = (double *)calloc(D, sizeof(double));
    if (bzero_flag) {
        const double www = bs->wself * bs->wself * bs->wself;
        for (int j = 1; j <= twojmax; ++j) bs->bzero[j] = www * j;
    }
    bs->ncoeff = ldo_bs_outputs(bs, 0);
    bs->oj1 = (int *)malloc(sizeof(int) * (bs->ncoeff + 1));
    bs->oj2 = (int *)malloc(sizeof(int) * (bs->ncoeff + 1));
    bs->oj = (int *)malloc(sizeof(int) * (bs->ncoeff + 1));
    ldo_bs_outputs(bs, 1);
    return bs;
}

void ldo_bs_free(ldo_bs *bs) {
    if (!bs) return;
    free(bs->rcut); free(bs->wj); free(bs->oj1); free(bs->oj2); free(bs->oj);
    free(bs->cg); free(bs->rootpq); free(bs->bzero); free(bs);
}

int ldo_bs_width(const ldo_bs *bs) { return bs->ncoeff; }

void ldo_bs_triple(const ldo_bs *bs, int c, int *j1, int *j2, int *j) {
    *j1 = bs->oj1[c]; *j2 = bs->oj2[c]; *j = bs->oj[c];
}

/* ---- dual numbers with three tangent directions (x, y, z) ---- */
typedef struct { double v, d[3]; } dual3;

static dual3 dconst(double v) { dual3 r = {v, {0, 0, 0}}; return r; }
static dual3 dadd(dual3 a, dual3 b) {
    dual3 r = {a.v + b.v, {a.d[0] + b.d[0], a.d[1] + b.d[1], a.d[2] + b.d[2]}};
    return r;
}
static dual3 dsub(dual3 a, dual3 b) {
    dual3 r = {a.v - b.v, {a.d[0] - b.d[0], a.d[1] - b.d[1], a.d[2] - b.d[2]}};
    return r;
}
static dual3 dmul(dual3 a, dual3 b) {
    dual3 r;
    r.v = a.v * b.v;
    for (int k = 0; k < 3; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
    return r;
}
static dual3 dscale(dual3 a, double s) {
    dual3 r = {a.v * s, {a.d[0] * s, a.d[1] * s, a.d[2] * s}};
    return r;
}
static dual3 ddiv(dual3 a, dual3 b) {
    dual3 r;
    r.v = a.v / b.v;
    for (int k = 0; k < 3; ++k) r.d[k] = (a.d[k] * b.v - a.v * b.d[k]) / (b.v * b.v);
    return r;
}
static dual3 dsqrt(dual3 a) {
    dual3 r;
    r.v = sqrt(a.v);
    for (int k = 0; k < 3; ++k) r.d[k] = a.d[k] / (2.0 * r.v);
    return r;
}
static dual3 dtan(dual3 a) {
    dual3 r;
    r.v = tan(a.v);
    const double c = cos(a.v);
    for (int k = 0; k < 3; ++k) r.d[k] = a.d[k] / (c * c);
    return r;
}
static dual3 dcos(dual3 a) {
    dual3 r;
    r.v = cos(a.v);
    const double s = -sin(a.v);
    for (int k = 0; k < 3; ++k) r.d[k] = a.d[k] * s;
    return r;
}

typedef struct {
    double *ur, *ui;       /* per-neighbour U, (J+1)^3 */
    double *utr, *uti;     /* Utot */
    double *zr, *zi;       /* Z, (J+1)^5 */
    double *b;             /* B, (J+1)^3 */
    double *gur, *gui;     /* dL/dUtot, (J+1)^3 */
    double *gb;            /* dL/dB, (J+1)^3 */
    dual3 *dur, *dui;      /* dual U, (J+1)^3 */
    int cap;
    double *rij;           /* cap x 3 */
    double *w, *rc;
    int *inside;
} ldo_bs_work;

static void ldo_bs_work_init(const ldo_bs *bs, ldo_bs_work *w, int cap) {
    const size_t D = bs->J + 1;
    const size_t n3 = D * D * D, n5 = D * D * D * D * D;
    w->ur = (double *)calloc(n3, sizeof(double));
    w->ui = (double *)calloc(n3, sizeof(double));
    w->utr = (double *)calloc(n3, sizeof(double));
    w->uti = (double *)calloc(n3, sizeof(double));
    w->zr = (double *)calloc(n5, sizeof(double));
    w->zi = (double *)calloc(n5, sizeof(double));
    w->b = (double *)calloc(n3, sizeof(double));
    w->gur = (double *)calloc(n3, sizeof(double));
    w->gui = (double *)calloc(n3, sizeof(double));
    w->gb = (double *)calloc(n3, sizeof(double));
    w->dur = (dual3 *)calloc(n3, sizeof(dual3));
    w->dui = (dual3 *)calloc(n3, sizeof(dual3));
    w->cap = cap > 0 ? cap : 1;
    w->rij = (double *)malloc(sizeof(double) * 3 * w->cap);
    w->w = (double *)malloc(sizeof(double) * w->cap);
    w->rc = (double *)malloc(sizeof(double) * w->cap);
    w->inside = (int *)malloc(sizeof(int) * w->cap);
}

static void ldo_bs_work_free(ldo_bs_work *w) {
    free(w->ur); free(w->ui); free(w->utr); free(w->uti); free(w->zr);
    free(w->zi); free(w->b); free(w->gur); free(w->gui); free(w->gb);
    free(w->dur); free(w->dui); free(w->rij); free(w->w); free(w->rc);
    free(w->inside);
}

/* compute_uarray, src/Bispectrum.cpp:490-554 (VMK 4.8.2 recursion,
 * then the inversion-symmetry copy VMK 4.4(2)). */
static void ldo_bs_uarray(const ldo_bs *bs, ldo_bs_work *w, double x, double y,
                          double z, double z0, double r) {
    const int J = bs->J, D = J + 1;
    double *ur = w->ur, *ui = w->ui;
    const double r0inv = 1.0 / sqrt(r * r + z0 * z0);
    const double a_r = r0inv * z0, a_i = -r0inv * z;
    const double b_r = r0inv * y, b_i = -r0inv * x;
    ur[UI(bs, 0, 0, 0)] = 1.0;
    ui[UI(bs, 0, 0, 0)] = 0.0;
    for (int j = 1; j <= J; ++j) {
        for (int mb = 0; 2 * mb <= j; ++mb) {
            ur[UI(bs, j, 0, mb)] = 0.0;
            ui[UI(bs, j, 0, mb)] = 0.0;
            for (int ma = 0; ma < j; ++ma) {
                const double pr = ur[UI(bs, j - 1, ma, mb)], pi = ui[UI(bs, j - 1, ma, mb)];
                double rq = bs->rootpq[(j - ma) * D + (j - mb)];
                ur[UI(bs, j, ma, mb)] += rq * (a_r * pr + a_i * pi);
                ui[UI(bs, j, ma, mb)] += rq * (a_r * pi - a_i * pr);
                rq = bs->rootpq[(ma + 1) * D + (j - mb)];
                ur[UI(bs, j, ma + 1, mb)] = -rq * (b_r * pr + b_i * pi);
                ui[UI(bs, j, ma + 1, mb)] = -rq * (b_r * pi - b_i * pr);
            }
        }
        int mbpar = -1;
        for (int mb = 0; 2 * mb <= j; ++mb) {
            mbpar = -mbpar;
            int mapar = -mbpar;
            for (int ma = 0; ma <= j; ++ma) {
                mapar = -mapar;
                const int s = UI(bs, j, ma, mb), t = UI(bs, j, j - ma, j - mb);
                if (mapar == 1) {
                    ur[t] = ur[s];
                    ui[t] = -ui[s];
                } else {
                    ur[t] = -ur[s];
                    ui[t] = ui[s];
                }
            }
        }
    }
}

/* same recursion on dual numbers (value + d/dx, d/dy, d/dz) */
static void ldo_bs_uarray_dual(const ldo_bs *bs, ldo_bs_work *w, dual3 x,
                               dual3 y, dual3 z, dual3 z0, dual3 r) {
    const int J = bs->J, D = J + 1;
    dual3 *ur = w->dur, *ui = w->dui;
    const dual3 r0inv = ddiv(dconst(1.0), dsqrt(dadd(dmul(r, r), dmul(z0, z0))));
    const dual3 a_r = dmul(r0inv, z0), a_i = dscale(dmul(r0inv, z), -1.0);
    const dual3 b_r = dmul(r0inv, y), b_i = dscale(dmul(r0inv, x), -1.0);
    ur[UI(bs, 0, 0, 0)] = dconst(1.0);
    ui[UI(bs, 0, 0, 0)] = dconst(0.0);
    for (int j = 1; j <= J; ++j) {
        for (int mb = 0; 2 * mb <= j; ++mb) {
            ur[UI(bs, j, 0, mb)] = dconst(0.0);
            ui[UI(bs, j, 0, mb)] = dconst(0.0);
            for (int ma = 0; ma < j; ++ma) {
                const dual3 pr = ur[UI(bs, j - 1, ma, mb)], pi = ui[UI(bs, j - 1, ma, mb)];
                double rq = bs->rootpq[(j - ma) * D + (j - mb)];
                ur[UI(bs, j, ma, mb)] = dadd(ur[UI(bs, j, ma, mb)],
                                             dscale(dadd(dmul(a_r, pr), dmul(a_i, pi)), rq));
                ui[UI(bs, j, ma, mb)] = dadd(ui[UI(bs, j, ma, mb)],
                                             dscale(dsub(dmul(a_r, pi), dmul(a_i, pr)), rq));
                rq = bs->rootpq[(ma + 1) * D + (j - mb)];
                ur[UI(bs, j, ma + 1, mb)] = dscale(dadd(dmul(b_r, pr), dmul(b_i, pi)), -rq);
                ui[UI(bs, j, ma + 1, mb)] = dscale(dsub(dmul(b_r, pi), dmul(b_i, pr)), -rq);
            }
        }
        int mbpar = -1;
        for (int mb = 0; 2 * mb <= j; ++mb) {
            mbpar = -mbpar;
            int mapar = -mbpar;
            for (int ma = 0; ma <= j; ++ma) {
                mapar = -mapar;
                const int s = UI(bs, j, ma, mb), t = UI(bs, j, j - ma, j - mb);
                if (mapar == 1) {
                    ur[t] = ur[s];
                    ui[t] = dscale(ui[s], -1.0);
                } else {
                    ur[t] = dscale(ur[s], -1.0);
                    ui[t] = ui[s];
                }
            }
        }
    }
}

/* compute_sfac, src/Bispectrum.cpp:572-586 */
static double ldo_bs_sfac(const ldo_bs *bs, double r, double rc) {
    if (bs->switch_flag == 0) return 1.0;
    if (bs->switch_flag == 1) {
        if (r <= bs->rmin0) return 1.0;
        if (r > rc) return 0.0;
        return 0.5 * (cos((r - bs->rmin0) * LDO_PI / (rc - bs->rmin0)) + 1.0);
    }
    return 0.0;
}

static dual3 ldo_bs_sfac_dual(const ldo_bs *bs, dual3 r, double rc) {
    if (bs->switch_flag == 0) return dconst(1.0);
    if (bs->switch_flag == 1) {
        if (r.v <= bs->rmin0) return dconst(1.0);
        if (r.v > rc) return dconst(0.0);
        dual3 t = dscale(dsub(r, dconst(bs->rmin0)), LDO_PI / (rc - bs->rmin0));
        return dscale(dadd(dcos(t), dconst(1.0)), 0.5);
    }
    return dconst(0.0);
}

static int ldo_bs_half_weight2(int j, int ma, int mb, double *wt) {
    /* weight of element (ma, mb) in compute_bi's half-matrix sum */
    if (2 * mb < j) { *wt = 1.0; return 1; }
    if (j % 2 == 0 && mb == j / 2) {
        if (ma < mb) { *wt = 1.0; return 1; }
        if (ma == mb) { *wt = 0.5; return 1; }
    }
    *wt = 0.0;
    return 0;
}

static void ldo_bs_atom_w(const ldo_bs *bs, ldo_bs_work *w, int index,
                          const int *species, const int *nbl, int n,
                          const double *coords, double *desc, const double *dE,
                          double *dcoords) {
    const int J = bs->J, D = J + 1;
    const int is = species[index];
    (void)is;
    const double *ci = coords + 3 * index;
    if (n > w->cap) {
        free(w->rij); free(w->w); free(w->rc); free(w->inside);
        w->cap = n;
        w->rij = (double *)malloc(sizeof(double) * 3 * n);
        w->w = (double *)malloc(sizeof(double) * n);
        w->rc = (double *)malloc(sizeof(double) * n);
        w->inside = (int *)malloc(sizeof(int) * n);
    }
    /* Bispectrum::compute, src/Bispectrum.cpp:255-286.  The cutoff is
     * looked up as rcuts(iSpecies, jSpecies) on an Array2D filled by
     * push_back with zero extents, i.e. flat element [jSpecies]. */
    int nin = 0;
    for (int jj = 0; jj < n; ++jj) {
        const int j = nbl[jj];
        const int js = species[j];
        double rv[3];
        for (int d = 0; d < 3; ++d) rv[d] = coords[3 * j + d] - ci[d];
        const double rsq = rv[0] * rv[0] + rv[1] * rv[1] + rv[2] * rv[2];
        const double rmag = sqrt(rsq);
        const double rc = bs->rcut[js];
        if (rmag < rc && rmag > 1e-10) {
            w->rij[3 * nin + 0] = rv[0];
            w->rij[3 * nin + 1] = rv[1];
            w->rij[3 * nin + 2] = rv[2];
            w->inside[nin] = j;
            w->w[nin] = bs->wj[js];
            w->rc[nin] = rc;
            ++nin;
        }
    }
    /* compute_ui */
    const size_t n3 = (size_t)D * D * D;
    memset(w->utr, 0, n3 * sizeof(double));
    memset(w->uti, 0, n3 * sizeof(double));
    for (int j = 0; j <= J; ++j)
        for (int ma = 0; ma <= j; ++ma) {
            w->utr[UI(bs, j, ma, ma)] = bs->wself;
            w->uti[UI(bs, j, ma, ma)] = 0.0;
        }
    for (int k = 0; k < nin; ++k) {
        const double x = w->rij[3 * k], y = w->rij[3 * k + 1], z = w->rij[3 * k + 2];
        const double rsq = x * x + y * y + z * z;
        const double r = sqrt(rsq);
        const double theta0 = (r - bs->rmin0) * bs->rfac0 * LDO_PI / (w->rc[k] - bs->rmin0);
        const double z0 = r / tan(theta0);
        ldo_bs_uarray(bs, w, x, y, z, z0, r);
        double sfac = ldo_bs_sfac(bs, r, w->rc[k]);
        sfac *= w->w[k];
        for (int j = 0; j <= J; ++j)
            for (int ma = 0; ma <= j; ++ma)
                for (int mb = 0; mb <= j; ++mb) {
                    w->utr[UI(bs, j, ma, mb)] += sfac * w->ur[UI(bs, j, ma, mb)];
                    w->uti[UI(bs, j, ma, mb)] += sfac * w->ui[UI(bs, j, ma, mb)];
                }
    }
    /* compute_zi: all j1 >= j2 triples */
#define ZI(j1, j2, j, ma, mb) CGI(bs, j1, j2, j, ma, mb)
    for (int j1 = 0; j1 <= J; ++j1)
        for (int j2 = 0; j2 <= j1; ++j2)
            for (int j = j1 - j2; j <= (J < j1 + j2 ? J : j1 + j2); j += 2)
                for (int mb = 0; 2 * mb <= j; ++mb)
                    for (int ma = 0; ma <= j; ++ma) {
                        double zr = 0.0, zi = 0.0;
                        int lo = (2 * ma - j - j2 + j1) / 2;
                        int hi = (2 * ma - j + j2 + j1) / 2;
                        if (lo < 0) lo = 0;
                        if (hi > j1) hi = j1;
                        for (int ma1 = lo; ma1 <= hi; ++ma1) {
                            double sr = 0.0, si = 0.0;
                            const int ma2 = (2 * ma - j - (2 * ma1 - j1) + j2) / 2;
                            int blo = (2 * mb - j - j2 + j1) / 2;
                            int bhi = (2 * mb - j + j2 + j1) / 2;
                            if (blo < 0) blo = 0;
                            if (bhi > j1) bhi = j1;
                            for (int mb1 = blo; mb1 <= bhi; ++mb1) {
                                const int mb2 = (2 * mb - j - (2 * mb1 - j1) + j2) / 2;
                                const double c = bs->cg[CGI(bs, j1, j2, j, mb1, mb2)];
                                const double u1r = w->utr[UI(bs, j1, ma1, mb1)];
                                const double u1i = w->uti[UI(bs, j1, ma1, mb1)];
                                const double u2r = w->utr[UI(bs, j2, ma2, mb2)];
                                const double u2i = w->uti[UI(bs, j2, ma2, mb2)];
                                sr += c * (u1r * u2r - u1i * u2i);
                                si += c * (u1r * u2i + u1i * u2r);
                            }
                            zr += sr * bs->cg[CGI(bs, j1, j2, j, ma1, ma2)];
                            zi += si * bs->cg[CGI(bs, j1, j2, j, ma1, ma2)];
                        }
                        w->zr[ZI(j1, j2, j, ma, mb)] = zr;
                        w->zi[ZI(j1, j2, j, ma, mb)] = zi;
                    }
    /* compute_bi */
    for (int j1 = 0; j1 <= J; ++j1)
        for (int j2 = 0; j2 <= j1; ++j2)
            for (int j = j1 - j2; j <= (J < j1 + j2 ? J : j1 + j2); j += 2) {
                double b = 0.0;
                for (int mb = 0; 2 * mb < j; ++mb)
                    for (int ma = 0; ma <= j; ++ma)
                        b += w->utr[UI(bs, j, ma, mb)] * w->zr[ZI(j1, j2, j, ma, mb)] +
                             w->uti[UI(bs, j, ma, mb)] * w->zi[ZI(j1, j2, j, ma, mb)];
                if (j % 2 == 0) {
                    const int mb = j / 2;
                    for (int ma = 0; ma < mb; ++ma)
                        b += w->utr[UI(bs, j, ma, mb)] * w->zr[ZI(j1, j2, j, ma, mb)] +
                             w->uti[UI(bs, j, ma, mb)] * w->zi[ZI(j1, j2, j, ma, mb)];
                    b += (w->utr[UI(bs, j, mb, mb)] * w->zr[ZI(j1, j2, j, mb, mb)] +
                          w->uti[UI(bs, j, mb, mb)] * w->zi[ZI(j1, j2, j, mb, mb)]) * 0.5;
                }
                b *= 2.0;
                if (bs->bzero_flag) b -= bs->bzero[j];
                w->b[UI(bs, j1, j2, j)] = b;
            }
    for (int c = 0; c < bs->ncoeff; ++c)
        desc[c] = w->b[UI(bs, bs->oj1[c], bs->oj2[c], bs->oj[c])];
    if (!dE) return;

    /* ---------------- reverse mode ---------------- */
    memset(w->gb, 0, n3 * sizeof(double));
    memset(w->gur, 0, n3 * sizeof(double));
    memset(w->gui, 0, n3 * sizeof(double));
    for (int c = 0; c < bs->ncoeff; ++c)
        w->gb[UI(bs, bs->oj1[c], bs->oj2[c], bs->oj[c])] += dE[c];
    for (int j1 = 0; j1 <= J; ++j1)
        for (int j2 = 0; j2 <= j1; ++j2)
            for (int j = j1 - j2; j <= (J < j1 + j2 ? J : j1 + j2); j += 2) {
                const double gB = w->gb[UI(bs, j1, j2, j)];
                if (gB == 0.0) continue;
                for (int mb = 0; 2 * mb <= j; ++mb)
                    for (int ma = 0; ma <= j; ++ma) {
                        double wt;
                        if (!ldo_bs_half_weight2(j, ma, mb, &wt)) continue;
                        const double f = 2.0 * gB * wt;
                        /* explicit U_j factor of B */
                        w->gur[UI(bs, j, ma, mb)] += f * w->zr[ZI(j1, j2, j, ma, mb)];
                        w->gui[UI(bs, j, ma, mb)] += f * w->zi[ZI(j1, j2, j, ma, mb)];
                        /* dL/dZ(ma,mb) */
                        const double gzr = f * w->utr[UI(bs, j, ma, mb)];
                        const double gzi = f * w->uti[UI(bs, j, ma, mb)];
                        int lo = (2 * ma - j - j2 + j1) / 2;
                        int hi = (2 * ma - j + j2 + j1) / 2;
                        if (lo < 0) lo = 0;
                        if (hi > j1) hi = j1;
                        for (int ma1 = lo; ma1 <= hi; ++ma1) {
                            const int ma2 = (2 * ma - j - (2 * ma1 - j1) + j2) / 2;
                            const double ca = bs->cg[CGI(bs, j1, j2, j, ma1, ma2)];
                            int blo = (2 * mb - j - j2 + j1) / 2;
                            int bhi = (2 * mb - j + j2 + j1) / 2;
                            if (blo < 0) blo = 0;
                            if (bhi > j1) bhi = j1;
                            for (int mb1 = blo; mb1 <= bhi; ++mb1) {
                                const int mb2 = (2 * mb - j - (2 * mb1 - j1) + j2) / 2;
                                const double cc = ca * bs->cg[CGI(bs, j1, j2, j, mb1, mb2)];
                                const int i1 = UI(bs, j1, ma1, mb1), i2 = UI(bs, j2, ma2, mb2);
                                const double u1r = w->utr[i1], u1i = w->uti[i1];
                                const double u2r = w->utr[i2], u2i = w->uti[i2];
                                /* g_U1 += cc * gZ * conj(U2); g_U2 += cc * gZ * conj(U1) */
                                w->gur[i1] += cc * (gzr * u2r + gzi * u2i);
                                w->gui[i1] += cc * (gzi * u2r - gzr * u2i);
                                w->gur[i2] += cc * (gzr * u1r + gzi * u1i);
                                w->gui[i2] += cc * (gzi * u1r - gzr * u1i);
                            }
                        }
                    }
            }
    /* per neighbour: forward-mode tangents of sfac * w * U, contracted with
     * dL/dUtot over every (j, ma, mb) element */
    for (int k = 0; k < nin; ++k) {
        dual3 x = {w->rij[3 * k], {1, 0, 0}};
        dual3 y = {w->rij[3 * k + 1], {0, 1, 0}};
        dual3 z = {w->rij[3 * k + 2], {0, 0, 1}};
        const dual3 r = dsqrt(dadd(dadd(dmul(x, x), dmul(y, y)), dmul(z, z)));
        const dual3 theta0 = dscale(dsub(r, dconst(bs->rmin0)),
                                    bs->rfac0 * LDO_PI / (w->rc[k] - bs->rmin0));
        const dual3 z0 = ddiv(r, dtan(theta0));
        ldo_bs_uarray_dual(bs, w, x, y, z, z0, r);
        const dual3 sf = dscale(ldo_bs_sfac_dual(bs, r, w->rc[k]), w->w[k]);
        double g[3] = {0, 0, 0};
        for (int j = 0; j <= J; ++j)
            for (int ma = 0; ma <= j; ++ma)
                for (int mb = 0; mb <= j; ++mb) {
                    const int e = UI(bs, j, ma, mb);
                    const dual3 tr = dmul(sf, w->dur[e]), ti = dmul(sf, w->dui[e]);
                    for (int d = 0; d < 3; ++d)
                        g[d] += w->gur[e] * tr.d[d] + w->gui[e] * ti.d[d];
                }
        const int nb = w->inside[k];
        for (int d = 0; d < 3; ++d) {
            dcoords[3 * nb + d] += g[d];
            dcoords[3 * index + d] -= g[d];
        }
    }
#undef ZI
}

void ldo_bs_atom(const ldo_bs *bs, int index, const int *species,
                 const int *nbl, int n, const double *coords, double *desc,
                 const double *dE, double *dcoords) {
    ldo_bs_work w;
    ldo_bs_work_init(bs, &w, n);
    ldo_bs_atom_w(bs, &w, index, species, nbl, n, coords, desc, dE, dcoords);
    ldo_bs_work_free(&w);
}

/* ================================================================== */
/* Drivers                                                             */
/* ================================================================== */
typedef struct {
    int kind;
    const void *obj;
    int width;
    const int *centre;      /* centre index per row */
    const long long *off;   /* neighbour row offsets */
    const int *counts, *species, *nbl;
    const double *coords;
    int n_total;
    double *desc;
    const double *dE;
    double *dc;             /* private gradient buffer (n_total*3) */
    int r0, r1;
} ldo_task;

static void *ldo_worker(void *arg) {
    ldo_task *t = (ldo_task *)arg;
    ldo_bs_work w;
    if (t->kind == 1) ldo_bs_work_init((const ldo_bs *)t->obj, &w, 64);
    for (int r = t->r0; r < t->r1; ++r) {
        const int i = t->centre[r];
        const int *nb = t->nbl + t->off[r];
        const int n = t->counts[r];
        double *d = t->desc + (size_t)r * t->width;
        if (t->kind == 0) {
            const ldo_sf *sf = (const ldo_sf *)t->obj;
            memset(d, 0, sizeof(double) * t->width);
            ldo_sf_atom(sf, i, t->species, nb, n, t->coords, d);
            if (t->dE)
                ldo_sf_atom_vjp(sf, i, t->species, nb, n, t->coords,
                                t->dE + (size_t)r * t->width, t->dc);
        } else {
            ldo_bs_atom_w((const ldo_bs *)t->obj, &w, i, t->species, nb, n,
                          t->coords, d, t->dE ? t->dE + (size_t)r * t->width : NULL,
                          t->dc);
        }
    }
    if (t->kind == 1) ldo_bs_work_free(&w);
    return NULL;
}

static int ldo_centres(int n_configs, const int *n_atoms, const int *config_ptr,
                       int **centre_out) {
    int nrows = 0;
    if (n_configs <= 0) {
        nrows = n_atoms[0];
        int *c = (int *)malloc(sizeof(int) * (nrows > 0 ? nrows : 1));
        for (int i = 0; i < nrows; ++i) c[i] = i;
        *centre_out = c;
        return nrows;
    }
    for (int c = 0; c < n_configs; ++c) nrows += n_atoms[c];
    int *cen = (int *)malloc(sizeof(int) * (nrows > 0 ? nrows : 1));
    int r = 0;
    for (int c = 0; c < n_configs; ++c)
        for (int j = 0; j < n_atoms[c]; ++j) cen[r++] = j + config_ptr[c];
    *centre_out = cen;
    return nrows;
}

int ldo_run(int kind, const void *obj, int n_configs, const int *n_atoms,
            const int *config_ptr, const int *species, const int *nbl,
            const int *counts, const double *coords, int n_total,
            double *desc, const double *dE, double *dcoords, int n_threads) {
    int *centre = NULL;
    const int nrows = ldo_centres(n_configs, n_atoms, config_ptr, &centre);
    long long *off = (long long *)malloc(sizeof(long long) * (nrows + 1));
    off[0] = 0;
    for (int r = 0; r < nrows; ++r) off[r + 1] = off[r] + counts[r];
    const int width = kind == 0 ? ldo_sf_width((const ldo_sf *)obj)
                                : ldo_bs_width((const ldo_bs *)obj);
    if (n_threads < 1) n_threads = 1;
    if (n_threads > nrows) n_threads = nrows > 0 ? nrows : 1;
    ldo_task *tasks = (ldo_task *)calloc(n_threads, sizeof(ldo_task));
    pthread_t *th = (pthread_t *)calloc(n_threads, sizeof(pthread_t));
    for (int t = 0; t < n_threads; ++t) {
        ldo_task *k = &tasks[t];
        k->kind = kind; k->obj = obj; k->width = width; k->centre = centre;
        k->off = off; k->counts = counts; k->species = species; k->nbl = nbl;
        k->coords = coords; k->n_total = n_total; k->desc = desc; k->dE = dE;
        k->dc = dE ? (double *)calloc((size_t)n_total * 3, sizeof(double)) : NULL;
        k->r0 = (int)((long long)nrows * t / n_threads);
        k->r1 = (int)((long long)nrows * (t + 1) / n_threads);
        if (n_threads > 1) pthread_create(&th[t], NULL, ldo_worker, k);
    }
    if (n_threads == 1) ldo_worker(&tasks[0]);
    else
        for (int t = 0; t < n_threads; ++t) pthread_join(th[t], NULL);
    if (dE) {
        memset(dcoords, 0, sizeof(double) * (size_t)n_total * 3);
        for (int t = 0; t < n_threads; ++t) {
            for (size_t q = 0; q < (size_t)n_total * 3; ++q) dcoords[q] += tasks[t].dc[q];
            free(tasks[t].dc);
        }
    }
    free(tasks); free(th); free(off); free(centre);
    return 0;
}

/* ---- finite differences (reference stencil) ---- */
typedef struct {
    int kind;
    const void *obj;
    int width, n_atoms;
    const int *species, *nbl, *counts;
    const long long *off;
    const double *coords;
    int n_total;
    const double *dE;
    const int *idx;
    double *out;
    int q0, q1;
    const int *aff_off, *aff;  /* affected centres per atom */
    double step;               /* > 0: 2-point central difference step */
} ldo_fd_task;

/* make_xph_representable, include/finite_difference.hpp:46-57 */
static double ldo_xph(double x, double h) {
    volatile double temp = x + h;
    h = temp - x;
    if (h == 0) h = nextafter(x, 1.7976931348623157e308) - x;
    return h;
}

static double ldo_fd_eval(ldo_fd_task *t, double *x, int a, double *buf,
                          ldo_bs_work *w) {
    /* sum over affected centres of dE . desc */
    double s = 0.0;
    for (int q = t->aff_off[a]; q < t->aff_off[a + 1]; ++q) {
        const int i = t->aff[q];
        memset(buf, 0, sizeof(double) * t->width);
        if (t->kind == 0)
            ldo_sf_atom((const ldo_sf *)t->obj, i, t->species, t->nbl + t->off[i],
                        t->counts[i], x, buf);
        else
            ldo_bs_atom_w((const ldo_bs *)t->obj, w, i, t->species, t->nbl + t->off[i],
                          t->counts[i], x, buf, NULL, NULL);
        for (int d = 0; d < t->width; ++d) s += t->dE[(size_t)i * t->width + d] * buf[d];
    }
    return s;
}

static void *ldo_fd_worker(void *arg) {
    ldo_fd_task *t = (ldo_fd_task *)arg;
    double *x = (double *)malloc(sizeof(double) * 3 * (size_t)t->n_total);
    memcpy(x, t->coords, sizeof(double) * 3 * (size_t)t->n_total);
    double *buf = (double *)malloc(sizeof(double) * (t->width > 0 ? t->width : 1));
    ldo_bs_work w;
    if (t->kind == 1) ldo_bs_work_init((const ldo_bs *)t->obj, &w, 64);
    const double eps = 2.220446049250313e-16;
    for (int q = t->q0; q < t->q1; ++q) {
        const int pos = t->idx[q];
        const int a = pos / 3;
        const double x0 = t->coords[pos];
        if (t->step > 0) {
            x[pos] = x0 + t->step;
            const double fp = ldo_fd_eval(t, x, a, buf, &w);
            x[pos] = x0 - t->step;
            const double fm = ldo_fd_eval(t, x, a, buf, &w);
            x[pos] = x0;
            t->out[q] = (fp - fm) / (2.0 * t->step);
            continue;
        }
        double h = pow(551.25 * eps, 1.0 / 9.0);
        h = ldo_xph(x0, h);
        double f[9];
        for (int s = -4; s <= 4; ++s) {
            if (s == 0) continue;
            x[pos] = x0 + s * h;
            f[s + 4] = ldo_fd_eval(t, x, a, buf, &w);
        }
        x[pos] = x0;
        const double y1 = f[5] - f[3];
        const double y2 = f[2] - f[6];
        const double y3 = f[7] - f[1];
        const double y4 = f[0] - f[8];
        t->out[q] = ((3 * y4 / 8 + 4 * y3) + (21 * y2 + 84 * y1)) / (105 * h);
    }
    if (t->kind == 1) ldo_bs_work_free(&w);
    free(x); free(buf);
    return NULL;
}

int ldo_fd_vjp(int kind, const void *obj, int n_atoms, const int *species,
               const int *nbl, const int *counts, const double *coords,
               int n_total, const double *dE, int n_idx, const int *idx,
               double *out, double step, int n_threads) {
    long long *off = (long long *)malloc(sizeof(long long) * (n_atoms + 1));
    off[0] = 0;
    for (int r = 0; r < n_atoms; ++r) off[r + 1] = off[r] + counts[r];
    /* affected centres of each atom: itself (if contributing) + every centre
     * listing it as a neighbour */
    int *cnt = (int *)calloc(n_total + 1, sizeof(int));
    for (int i = 0; i < n_atoms; ++i) {
        cnt[i]++;
        for (long long q = off[i]; q < off[i + 1]; ++q) cnt[nbl[q]]++;
    }
    int *aoff = (int *)malloc(sizeof(int) * (n_total + 1));
    aoff[0] = 0;
    for (int a = 0; a < n_total; ++a) aoff[a + 1] = aoff[a] + cnt[a];
    int *aff = (int *)malloc(sizeof(int) * (aoff[n_total] > 0 ? aoff[n_total] : 1));
    int *fill = (int *)calloc(n_total, sizeof(int));
    for (int i = 0; i < n_atoms; ++i) {
        /* keep each centre at most once per atom */
        aff[aoff[i] + fill[i]++] = i;
        for (long long q = off[i]; q < off[i + 1]; ++q) {
            const int a = nbl[q];
            int dup = 0;
            for (int s = aoff[a]; s < aoff[a] + fill[a]; ++s)
                if (aff[s] == i) { dup = 1; break; }
            if (!dup) aff[aoff[a] + fill[a]++] = i;
        }
    }
    /* compact */
    int *aoff2 = (int *)malloc(sizeof(int) * (n_total + 1));
    int *aff2 = (int *)malloc(sizeof(int) * (aoff[n_total] > 0 ? aoff[n_total] : 1));
    aoff2[0] = 0;
    for (int a = 0; a < n_total; ++a) {
        memcpy(aff2 + aoff2[a], aff + aoff[a], sizeof(int) * fill[a]);
        aoff2[a + 1] = aoff2[a] + fill[a];
    }
    const int width = kind == 0 ? ldo_sf_width((const ldo_sf *)obj)
                                : ldo_bs_width((const ldo_bs *)obj);
    if (n_threads < 1) n_threads = 1;
    if (n_threads > n_idx) n_threads = n_idx > 0 ? n_idx : 1;
    ldo_fd_task *tasks = (ldo_fd_task *)calloc(n_threads, sizeof(ldo_fd_task));
    pthread_t *th = (pthread_t *)calloc(n_threads, sizeof(pthread_t));
    for (int t = 0; t < n_threads; ++t) {
        ldo_fd_task *k = &tasks[t];
        k->kind = kind; k->obj = obj; k->width = width; k->n_atoms = n_atoms;
        k->species = species; k->nbl = nbl; k->counts = counts; k->off = off;
        k->coords = coords; k->n_total = n_total; k->dE = dE; k->idx = idx;
        k->out = out; k->aff_off = aoff2; k->aff = aff2; k->step = step;
        k->q0 = (int)((long long)n_idx * t / n_threads);
        k->q1 = (int)((long long)n_idx * (t + 1) / n_threads);
        if (n_threads > 1) pthread_create(&th[t], NULL, ldo_fd_worker, k);
    }
    if (n_threads == 1) ldo_fd_worker(&tasks[0]);
    else
        for (int t = 0; t < n_threads; ++t) pthread_join(th[t], NULL);
    free(tasks); free(th); free(off); free(cnt); free(aoff); free(aff);
    free(fill); free(aoff2); free(aff2);
    return 0;
}
