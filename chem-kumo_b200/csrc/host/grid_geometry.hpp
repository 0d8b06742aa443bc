#pragma once
// Grid validation and point numbering: the rules of chem-kumo's
// src/grid_geometry.hpp:30-86 (Field order, k fastest).
#include "chem/kumo/density.hpp"

#include <cmath>
#include <limits>
#include <stdexcept>

namespace chem::kumo::detail {

inline double det3(const double a[3], const double b[3], const double c[3]) {
    return a[0] * (b[1] * c[2] - b[2] * c[1]) - b[0] * (a[1] * c[2] - a[2] * c[1]) + c[0] * (a[1] * b[2] - a[2] * b[1]);
}

inline std::size_t validated_point_count(const Grid& g) {
    std::size_t count = 1;
    for (int a = 0; a < 3; ++a) {
        const int n = g.counts[a];
        if (n <= 0 || static_cast<std::size_t>(n) > std::numeric_limits<std::size_t>::max() / count)
            throw std::invalid_argument("invalid or oversized grid");
        count *= static_cast<std::size_t>(n);
    }
    for (double v : g.origin)
        if (!std::isfinite(v)) throw std::invalid_argument("invalid grid geometry: nonfinite origin or step");
    for (double v : g.steps.m)
        if (!std::isfinite(v)) throw std::invalid_argument("invalid grid geometry: nonfinite origin or step");
    double dir[3][3];
    for (int a = 0; a < 3; ++a) {
        const double len = std::sqrt(g.steps(0, a) * g.steps(0, a) + g.steps(1, a) * g.steps(1, a) +
                                     g.steps(2, a) * g.steps(2, a));
        if (!std::isfinite(len) || len <= 0.0) throw std::invalid_argument("invalid grid geometry: zero step vector");
        for (int r = 0; r < 3; ++r) dir[a][r] = g.steps(r, a) / len;
    }
    if (std::abs(det3(dir[0], dir[1], dir[2])) < 1e-12)
        throw std::invalid_argument("invalid grid geometry: linearly dependent axes");
    return count;
}

}  // namespace chem::kumo::detail
