#pragma once
// Grid validation and point numbering: the rules of chem-kumo's
// src/grid_geometry.hpp:30-86 (Field order, k fastest).
#include "chem/kumo/density.hpp"

#include <cmath>
#include <cstdlib>
#include <limits>
#include <stdexcept>
#include <vector>

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

// Compact tiles of 128 points over a grid, as the mixed form evaluates grids
// (kumo_dev::GridTiles): extents 2^sa x 2^sb x 2^sc (sa + sb + sc = 7) along
// i, j, k; the shape that leaves the fewest padding points and, among those,
// spans the shortest diagonal.  Tiles are numbered with k fastest and i
// slowest, points inside a tile with k fastest.
struct TileShape {
    int sa = 0, sb = 0, sc = 0;
    long long tnx = 0, tny = 0, tnz = 0;  // tiles along i, j, k
    long long padded() const { return tnx * tny * tnz * 128; }
};

inline TileShape choose_tiles(const Grid& g) {
    double len[3];
    for (int a = 0; a < 3; ++a)
        len[a] = std::sqrt(g.steps(0, a) * g.steps(0, a) + g.steps(1, a) * g.steps(1, a) + g.steps(2, a) * g.steps(2, a));
    TileShape best;
    double best_diag = 0.0;
    bool first = true;
    for (int sa = 0; sa <= 7; ++sa)
        for (int sb = 0; sa + sb <= 7; ++sb) {
            const int sc = 7 - sa - sb;
            TileShape t{sa, sb, sc, (g.counts[0] + (1ll << sa) - 1) >> sa, (g.counts[1] + (1ll << sb) - 1) >> sb,
                        (g.counts[2] + (1ll << sc) - 1) >> sc};
            const double da = len[0] * double(1 << sa), db = len[1] * double(1 << sb), dc = len[2] * double(1 << sc);
            const double diag = da * da + db * db + dc * dc;
            if (first || t.padded() < best.padded() || (t.padded() == best.padded() && diag < best_diag * (1.0 - 1e-12))) {
                best = t;
                best_diag = diag;
                first = false;
            }
        }
    return best;
}

// Whether the mixed form evaluates a grid with screening blocks of
// `block_size` points as tiles: blocks of 128 points or more (CTAs take 128),
// unless KUMO_MIXED_TILES=0.
inline bool mixed_grid_tiles(std::size_t block_size) {
    const char* e = std::getenv("KUMO_MIXED_TILES");
    return block_size >= 128 && !(e && e[0] == '0');
}

// Grid index of each evaluation index of a tiled grid (t.padded() entries),
// -1 for padding.
inline void tile_order(const Grid& g, const TileShape& t, std::vector<long long>& grid_index) {
    grid_index.assign(static_cast<std::size_t>(t.padded()), -1);
    const long long ny = g.counts[1], nz = g.counts[2];
    std::size_t e = 0;
    for (long long ti = 0; ti < t.tnx; ++ti)
        for (long long tj = 0; tj < t.tny; ++tj)
            for (long long tk = 0; tk < t.tnz; ++tk)
                for (int w = 0; w < 128; ++w, ++e) {
                    const long long i = (ti << t.sa) + (w >> (t.sb + t.sc));
                    const long long j = (tj << t.sb) + ((w >> t.sc) & ((1 << t.sb) - 1));
                    const long long k = (tk << t.sc) + (w & ((1 << t.sc) - 1));
                    if (i < g.counts[0] && j < ny && k < nz) grid_index[e] = (i * ny + j) * nz + k;
                }
}

}  // namespace chem::kumo::detail
