// ld_fd.h -- 8th-order central finite difference used by the
// num_gradient_single_atom entry points (Python module and C++ shim).
#pragma once

#include <cmath>
#include <limits>
#include <vector>

namespace ldb {

// Derivative of the vector function f (f(x, y) writes y[width]) with respect
// to x[pos]: the stencil and step of the reference's
// include/finite_difference.hpp:60-143 (used by its num_gradient_single_atom,
// src/Descriptors.cpp:488-518).  x is restored on return.
template <class F>
void fd8(F &&f, std::vector<double> &x, int pos, int width, std::vector<double> &out) {
    const double eps = std::numeric_limits<double>::epsilon();
    double h = std::pow(551.25 * eps, 1.0 / 9.0);
    {
        volatile double t = x[pos] + h;
        h = t - x[pos];
        if (h == 0) h = std::nextafter(x[pos], std::numeric_limits<double>::max()) - x[pos];
    }
    const double x0 = x[pos];
    std::vector<std::vector<double>> y(9, std::vector<double>(width, 0.0));
    for (int s = -4; s <= 4; ++s) {
        if (!s) continue;
        x[pos] = x0 + s * h;
        f(x.data(), y[s + 4].data());
    }
    x[pos] = x0;
    out.assign(width, 0.0);
    for (int c = 0; c < width; ++c) {
        const double y1 = y[5][c] - y[3][c], y2 = y[2][c] - y[6][c];
        const double y3 = y[7][c] - y[1][c], y4 = y[0][c] - y[8][c];
        out[c] = ((3 * y4 / 8 + 4 * y3) + (21 * y2 + 84 * y1)) / (105 * h);
    }
}

}  // namespace ldb
