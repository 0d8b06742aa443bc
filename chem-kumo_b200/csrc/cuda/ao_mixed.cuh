// AO build of the mixed-precision form: FP32 AO values and derivatives of
// one 128-point block per CTA, written as rows of the AO blocks whose cutoff
// sphere reaches the block's bounding box (in AO order), with the per-warp
// maximum |value| of each row for the contraction's screening and K order.
//
// The contraction of each AO block factorises: its primitive weights are
// W[k][p] = u_p g_k (src/basis_math.cpp normalisation: u_p = c_p
// (2a_p/pi)^(3/4) (4a_p)^(l/2), g_k = ((2x-1)!!(2y-1)!!(2z-1)!!)^(-1/2)), so
// with e(r) = sum_p u_p exp(-a_p r^2) and the radial sums R0 = sum u_p e_p,
// R1' = -2 sum u_p a_p e_p, R2' = 4 sum u_p a_p^2 e_p, a Cartesian component
// with monomial M gives
//   value  M R0
//   d_i    M_i R0 + x_i M R1'
//   d_ij   M_ij R0 + (M_i x_j + M_j x_i) R1' + M (delta_ij R1' + x_i x_j R2')
//   lapl.  lap(M) R0 + M ((2l+3) R1' + r^2 R2')        (r.grad M = l M)
// and a pure AO applies the same formulas to the solid-harmonic polynomial
// sum_k T[m][k] g_k M_k, whose Laplacian is zero.  Exponentials take an FP64
// argument reduction (a r^2 log2 e = n - f) so each factor keeps FP32
// relative accuracy.
#pragma once

#include "kumo_device.cuh"

namespace kumo_dev {

struct MixPrim {
    double al2;   // exponent * log2(e)
    float alpha;  // exponent
    float u;      // contraction coefficient * radial normalisation * (4 alpha)^(l/2)
};

struct AoMixedParams {
    DevBasis basis;
    const MixPrim* prims = nullptr;  // indexed like DevBasis::exps
    PointSource src;
    long long first_point = 0;
    long long block_size = 128;
    int nblocks = 0;
    // panels[((b * npanel + c) * row_stride + row) * 128 + j], kept[b * row_stride + row],
    // nkept[b], rowmax[(b * row_stride + row) * 4 + warp].
    AoScratch<float> out;
    float tpure[3][135] = {};  // T[m][k] * g_k, l = 2..4, row-major (m, k)
    float gcart[5][15] = {};   // g_k of Cartesian components, l = 0..4
};

void launch_ao_mixed(const AoMixedParams& p, int npanel, cudaStream_t stream);

// Whether T[m][k] of the Cartesian-to-pure transform of src/basis_evaluator
// (Schlegel-Frisch, Gaussian order; m index 0, +1, -1, +2, -2, ...) can be
// nonzero: the integer conditions of its sum (the coefficients themselves
// are uploaded).
__host__ __device__ constexpr bool solid_harmonic_nonzero(int l, int mi, int lx, int ly) {
    const int m = mi == 0 ? 0 : ((mi & 1) ? (mi + 1) / 2 : -(mi / 2));
    const int lz = l - lx - ly;
    const int am = m < 0 ? -m : m;
    if (am > l || lz < 0) return false;
    const int rest = l - am - lz;
    if (rest < 0 || (rest & 1)) return false;
    const int half = rest / 2;
    for (int i = 0; i <= (l - am) / 2; ++i) {
        if (half > i) continue;
        for (int k = 0; k <= half; ++k) {
            const int e = lx - 2 * k;
            if (e < 0 || e > am) continue;
            const int d = am - lx < 0 ? lx - am : am - lx;
            if (m == 0 && lx % 2 == 0) return true;
            if (m > 0 && d % 2 == 0) return true;
            if (m < 0 && d % 2 == 1) return true;
        }
    }
    return false;
}

}  // namespace kumo_dev
