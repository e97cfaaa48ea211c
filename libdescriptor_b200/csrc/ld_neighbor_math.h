// ld_neighbor_math.h -- small host geometry helpers shared by the host and
// device neighbour builders (same arithmetic order as the reference's
// helper.hpp, python_bindings/neighbor/neighbor_list.cpp).
#pragma once

#include <cmath>

namespace ldnb {

constexpr double kTol = 1.0e-10;

inline double vdot(const double *a, const double *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
inline double vnorm(const double *a) { return std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]); }
inline void vcross(const double *a, const double *b, double *c) {
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}
inline double minor2(double a, double b, double c, double d) { return (a * d) - (b * c); }

// inverse by cofactors / determinant; returns false when |det| < 1e-10
inline bool invert3(const double *m, double *inv) {
    inv[0] = minor2(m[4], m[5], m[7], m[8]);
    inv[1] = minor2(m[2], m[1], m[8], m[7]);
    inv[2] = minor2(m[1], m[2], m[4], m[5]);
    inv[3] = minor2(m[5], m[3], m[8], m[6]);
    inv[4] = minor2(m[0], m[2], m[6], m[8]);
    inv[5] = minor2(m[2], m[0], m[5], m[3]);
    inv[6] = minor2(m[3], m[4], m[6], m[7]);
    inv[7] = minor2(m[1], m[0], m[7], m[6]);
    inv[8] = minor2(m[0], m[1], m[3], m[4]);
    const double det = m[0] * m[4] * m[8] - m[0] * m[5] * m[7] - m[1] * m[3] * m[8] + m[1] * m[5] * m[6] +
                       m[2] * m[3] * m[7] - m[2] * m[4] * m[6];
    if (std::abs(det) < kTol) return false;
    for (int k = 0; k < 9; ++k) inv[k] /= det;
    return true;
}


// Padding geometry of a cell: transposed cell (rows = Cartesian components),
// its inverse (fractional coordinates) and, per lattice direction, the number
// of image shells and the slack of the outermost shell.
struct PadGeom {
    double tcell[9], fcell[9];
    int size[3];
    double slack[3];
};

inline bool pad_geometry(double cutoff, const double *cell, PadGeom &g) {
    const double t[9] = {cell[0], cell[3], cell[6], cell[1], cell[4], cell[7], cell[2], cell[5], cell[8]};
    for (int k = 0; k < 9; ++k) g.tcell[k] = t[k];
    if (!invert3(g.tcell, g.fcell)) return false;
    double xp[3];
    vcross(cell + 3, cell + 6, xp);
    const double volume = std::abs(vdot(cell, xp));
    double dist[3];
    vcross(cell + 3, cell + 6, xp);
    dist[0] = volume / vnorm(xp);
    vcross(cell + 6, cell + 0, xp);
    dist[1] = volume / vnorm(xp);
    vcross(cell, cell + 3, xp);
    dist[2] = volume / vnorm(xp);
    const double ratio[3] = {cutoff / dist[0], cutoff / dist[1], cutoff / dist[2]};
    for (int d = 0; d < 3; ++d) {
        g.size[d] = (int)std::ceil(ratio[d]);
        g.slack[d] = (double)g.size[d] - ratio[d];
    }
    return true;
}

}  // namespace ldnb
