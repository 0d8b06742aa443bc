// Device-side data layout of a molecule and of the grid-block evaluation.
//
// A molecule lives in HBM as structure-of-arrays tables, uploaded once:
//  - AO blocks (shells after splitting SP shells, src/basis_math.cpp:27-66):
//    origin + squared cutoff radius, angular momentum, primitive range,
//    weight range, AO offset, pure flag;
//  - primitive exponents and weights (contraction coefficient times
//    primitive normalisation, ncart x nprim per block, row-major);
//  - occupied MO coefficients transposed to [AO][MO] (MO contiguous, padded
//    to a multiple of 8) so that a kept AO row is one contiguous load;
//  - the density matrices P_total / P_spin (n x n).
// Cartesian-to-pure matrices for l = 2..4 travel in the kernel parameters
// (constant bank).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace kumo_dev {

constexpr int kBlockPoints = 128;  // points per CTA of the AO build (screening block)
constexpr int kMaxL = 4;           // largest angular momentum of the device kernels
constexpr int kMaxPrim = 16;       // largest number of primitives per shell
constexpr int kMaxBlocksPerWave = 1 << 20;

// Panel sets stored in the AO scratch (mask panels are always those of the
// reference's AO order: 1, 4 or 10).
enum PanelMode : int {
    kPanelsValue = 1,      // value
    kPanelsGradient = 4,   // value, x, y, z
    kPanelsLaplacian = 5,  // value, x, y, z, xx + yy + zz
    kPanelsFull = 10,      // value, x, y, z, xx, xy, xz, yy, yz, zz
};

struct DevBasis {
    int nblocks = 0;
    int nao = 0;
    int max_l = 0;
    int max_count = 0;               // largest number of AOs of one block
    const double4* origin_r2 = nullptr;  // x, y, z, cutoff radius squared
    const int4* info = nullptr;          // l | pure << 8 | nprim << 16, prim offset, weight offset, ao offset
    const double* exps = nullptr;
    const double* weights = nullptr;
    const float* exps_f = nullptr;
    const float* weights_f = nullptr;
    const int* ao_block = nullptr;       // per AO: its block index * 32 + its component within the block
};

// Compact tiles of a grid.  With `on`, evaluation index e does not follow the
// grid's linear order: block e / 128 is tile number e / 128 of ta x tb x tc
// points (ta = 2^sa along i, tb = 2^sb along j, tc = 2^sc along k, product
// 128), tiles numbered with k fastest and i slowest, and e % 128 numbers the
// points inside the tile with k fastest.  Indices of a partial tile that fall
// outside the grid are padding: no point, nothing stored.  The mixed form
// evaluates grids this way, so that each 128-point block is a small box whose
// largest AO rows dominate at all of its points.
struct GridTiles {
    int on = 0;
    int sa = 0, sb = 0, sc = 0;
    long long nx = 0, ny = 0, nz = 0;  // grid counts
    long long tny = 0, tnz = 0;        // tiles along j and k
};

// Source of the evaluation points: a regular grid (generated in the kernel)
// or an explicit 3 x N array (x, y, z per point).
struct PointSource {
    const double* points = nullptr;  // device, 3 * count, or null for a grid
    double origin[3] = {0, 0, 0};
    double steps[9] = {0};           // column a = step vector of axis a
    long long ny = 1, nz = 1;
    long long count = 0;             // evaluation indices (tiles * 128 when tiled)
    GridTiles tiles;
};

#ifdef __CUDACC__
// Linear grid index of evaluation index e of a tiled grid; false for padding.
__device__ __forceinline__ bool tile_to_linear(const GridTiles& t, long long e, long long& q) {
    const long long tile = e >> 7;
    const int w = static_cast<int>(e & 127);
    long long tk, tj, ti;
    if (tile < 0xffffffffll && t.tnz < 0xffffffffll && t.tny < 0xffffffffll) {
        // 32-bit quotients (a fraction of the 64-bit division's instructions).
        const unsigned u = static_cast<unsigned>(tile), nz = static_cast<unsigned>(t.tnz),
                       ny = static_cast<unsigned>(t.tny);
        const unsigned rest = u / nz;
        tk = u - rest * nz;
        ti = rest / ny;
        tj = rest - static_cast<unsigned>(ti) * ny;
    } else {
        tk = tile % t.tnz;
        const long long rest = tile / t.tnz;
        tj = rest % t.tny;
        ti = rest / t.tny;
    }
    const int wk = w & ((1 << t.sc) - 1), wj = (w >> t.sc) & ((1 << t.sb) - 1), wi = w >> (t.sb + t.sc);
    const long long i = (ti << t.sa) + wi, j = (tj << t.sb) + wj, k = (tk << t.sc) + wk;
    if (i >= t.nx || j >= t.ny || k >= t.nz) return false;
    q = (i * t.ny + j) * t.nz + k;
    return true;
}

// Whether evaluation index q is a point (not past the end, not tile padding).
__device__ __forceinline__ bool point_exists(const PointSource& s, long long q) {
    if (q >= s.count) return false;
    if (!s.tiles.on) return true;
    long long lin;
    return tile_to_linear(s.tiles, q, lin);
}

// Points of CTA `blk` of a wave whose first point is `first` (the start of a
// screening block).  Screening blocks have `screen` points (0: `chunk`); a
// CTA takes at most `chunk` (<= 128) points, so a larger screening block is
// split into ceil(screen / chunk) chunks and CTA blk takes chunk
// blk % chunks of screening block blk / chunks.  On return [start, start + n)
// are the CTA's points (n <= 0 past the last point) and sblock is the
// screening block's index in the wave.
__device__ __forceinline__ void cta_points(long long first, long long chunk, long long screen, long long count, int blk,
                                           long long& start, long long& n, int& sblock) {
    if (screen <= chunk) {
        sblock = blk;
        start = first + static_cast<long long>(blk) * chunk;
        n = count - start < chunk ? count - start : chunk;
        return;
    }
    const long long per = (screen + chunk - 1) / chunk;
    const long long b = blk / per, c = blk - b * per;
    sblock = static_cast<int>(b);
    start = first + b * screen + c * chunk;
    long long m = screen - c * chunk;
    if (m > chunk) m = chunk;
    if (m > count - start) m = count - start;
    n = m;
}

// Coordinates of evaluation index q (a point: see point_exists).
__device__ __forceinline__ void point_at(const PointSource& s, long long q, double& x, double& y,
                                         double& z) {
    if (s.tiles.on) {
        long long lin = 0;
        (void)tile_to_linear(s.tiles, q, lin);
        q = lin;
    }
    if (s.points) {
        x = s.points[3 * q];
        y = s.points[3 * q + 1];
        z = s.points[3 * q + 2];
        return;
    }
    // src/grid_geometry.hpp:59-68: linear = (i * ny + j) * nz + k.
    long long i, j, k;
    if (q < 0xffffffffll && s.nz < 0xffffffffll && s.ny < 0xffffffffll) {
        const unsigned u = static_cast<unsigned>(q), nz = static_cast<unsigned>(s.nz), ny = static_cast<unsigned>(s.ny);
        const unsigned r = u / nz;
        k = u - r * nz;
        i = r / ny;
        j = r - static_cast<unsigned>(i) * ny;
    } else {
        i = q / (s.ny * s.nz);
        j = (q / s.nz) % s.ny;
        k = q % s.nz;
    }
    const double di = (double)i, dj = (double)j, dk = (double)k;
    x = __dadd_rn(s.origin[0], __dadd_rn(__dadd_rn(__dmul_rn(s.steps[0], di), __dmul_rn(s.steps[3], dj)),
                                         __dmul_rn(s.steps[6], dk)));
    y = __dadd_rn(s.origin[1], __dadd_rn(__dadd_rn(__dmul_rn(s.steps[1], di), __dmul_rn(s.steps[4], dj)),
                                         __dmul_rn(s.steps[7], dk)));
    z = __dadd_rn(s.origin[2], __dadd_rn(__dadd_rn(__dmul_rn(s.steps[2], di), __dmul_rn(s.steps[5], dj)),
                                         __dmul_rn(s.steps[8], dk)));
}
#endif

// AO scratch of one wave of point blocks.  Block b of the wave holds its
// kept AO rows, compacted in AO order:
//   panels[(b * npanel + c) * row_stride + slot) * 128 + j]
// with kept[b * row_stride + slot] the AO index of the slot and nkept[b]
// the number of slots.  T is double (FP64 path) or float (mixed path).
template <typename T>
struct AoScratch {
    T* panels = nullptr;
    int* kept = nullptr;
    int* nkept = nullptr;
    int row_stride = 0;   // >= nao
    int npanel = 0;
    float* rowmax = nullptr;  // optional: block maximum |value| of each kept row
};

// Parameters of the AO build of one wave.
template <typename T>
struct AoBuildParams {
    DevBasis basis;
    PointSource src;
    long long first_point = 0;     // first point of the wave
    long long block_size = 128;    // points per screening block (<= 128)
    int nblocks = 0;               // blocks in this wave
    double threshold = 1e-12;      // screening threshold (0 keeps every AO)
    // With threshold 0: keep every AO of the shells whose cutoff sphere reaches
    // the block's bounding box (the other AOs are cutoff zeros at every point
    // of the block), instead of every AO of the basis.
    int keep_reaching = 0;
    AoScratch<T> out;
    T pure[3][135];                // Cartesian-to-pure matrices, l = 2..4, row-major
    // Screening blocks larger than the `block_size` points of a CTA (see
    // cta_points): screen_block points each (0: block_size).  Such a block
    // is screened in two launches: mask_pass 1 stores nothing but raises
    // block_max[sblock * nao + ao] to the largest |value| of each AO over the
    // CTA's points (all panels of the AO order; block_max zeroed before);
    // mask_pass 2 builds the panels and keeps the AOs whose block_max is
    // above the threshold (src/ao_screening.hpp:35-50 over the whole block).
    long long screen_block = 0;
    int mask_pass = 0;
    double* block_max = nullptr;
};

template <typename T>
void launch_ao_build(const AoBuildParams<T>& p, int order, int npanel, cudaStream_t stream);

}  // namespace kumo_dev
