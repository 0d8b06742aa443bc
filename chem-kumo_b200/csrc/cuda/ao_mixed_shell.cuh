// Device pieces of the mixed-precision AO build shared by ao_mixed_kernel and
// the fused AO-MO contraction: the FP32 exponential with FP64 argument
// reduction and the panels of one AO block at one point (see ao_mixed.cuh).
#pragma once

#include "ao_common.cuh"
#include "ao_mixed.cuh"

namespace kumo_dev {
namespace {

// exp(-a r^2) given al2 = a log2(e): FP64 argument reduction t = n - f with
// |f| <= 1/2, FP32 2^f, scaling by 2^-n as two products by normal powers of
// two (2^-h, h = n/2, exact; then 2^-(n-h), the only rounding, which also
// gives the subnormal results exactly as ldexpf does); 0 below the FP32 range.
__device__ __forceinline__ float exp_neg(double al2, double r2) {
    const double t = al2 * r2;
    if (!(t < 149.0)) return 0.0f;
    // n = rint(t) by adding and removing 1.5 * 2^52 (round to nearest even,
    // as rint), its integer read from the low word: FP64 adds instead of a
    // rounding and a conversion instruction.
    const double tb = t + 6755399441055744.0;
    const double n = tb - 6755399441055744.0;
    const int ni = __double2loint(tb), h = ni >> 1;
    const float s1 = __int_as_float((127 - h) << 23), s2 = __int_as_float((127 - (ni - h)) << 23);
    return (exp2f(static_cast<float>(n - t)) * s1) * s2;
}

template <int L, bool PURE, int P, bool ROWMAX = true>
__device__ __forceinline__ void mixed_shell(const AoMixedParams& prm, float x, float y, float z, float r2, float R0,
                                            float R1p, float R2p, float q, float* dst, size_t pstride, float* rmax,
                                            int lane) {
    constexpr int NC = Cart<L>::NC;
    constexpr int NOUT = PURE ? 2 * L + 1 : NC;
    constexpr bool LAPM = P == 5 && !PURE;  // Cartesian Laplacian of the monomials
    float xp[L + 1], yp[L + 1], zp[L + 1];
    xp[0] = yp[0] = zp[0] = 1.0f;
#pragma unroll
    for (int n = 1; n <= L; ++n) {
        xp[n] = xp[n - 1] * x;
        yp[n] = yp[n - 1] * y;
        zp[n] = zp[n - 1] * z;
    }
    float pm[NOUT], pg[3][NOUT], ph[6][NOUT], pl[NOUT];
#pragma unroll
    for (int m = 0; m < NOUT; ++m) {
        pm[m] = pl[m] = 0.0f;
#pragma unroll
        for (int i = 0; i < 3; ++i) pg[i][m] = 0.0f;
#pragma unroll
        for (int h = 0; h < 6; ++h) ph[h][m] = 0.0f;
    }
    static_for<NC>([&](auto kc) {
        constexpr int k = decltype(kc)::value;
        constexpr int a = cart_power(L, k, 0), b = cart_power(L, k, 1), c = cart_power(L, k, 2);
        const float M = xp[a] * yp[b] * zp[c];
        [[maybe_unused]] float Mi[3] = {0.0f, 0.0f, 0.0f};
        [[maybe_unused]] float Mh[6] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
        if constexpr (P >= 4) {
            if constexpr (a > 0) Mi[0] = (float)a * xp[a > 0 ? a - 1 : 0] * yp[b] * zp[c];
            if constexpr (b > 0) Mi[1] = (float)b * xp[a] * yp[b > 0 ? b - 1 : 0] * zp[c];
            if constexpr (c > 0) Mi[2] = (float)c * xp[a] * yp[b] * zp[c > 0 ? c - 1 : 0];
        }
        if constexpr (P == 10 || LAPM) {
            if constexpr (a > 1) Mh[0] = (float)(a * (a - 1)) * xp[a > 1 ? a - 2 : 0] * yp[b] * zp[c];
            if constexpr (b > 1) Mh[3] = (float)(b * (b - 1)) * xp[a] * yp[b > 1 ? b - 2 : 0] * zp[c];
            if constexpr (c > 1) Mh[5] = (float)(c * (c - 1)) * xp[a] * yp[b] * zp[c > 1 ? c - 2 : 0];
        }
        if constexpr (P == 10) {
            if constexpr (a > 0 && b > 0) Mh[1] = (float)(a * b) * xp[a > 0 ? a - 1 : 0] * yp[b > 0 ? b - 1 : 0] * zp[c];
            if constexpr (a > 0 && c > 0) Mh[2] = (float)(a * c) * xp[a > 0 ? a - 1 : 0] * yp[b] * zp[c > 0 ? c - 1 : 0];
            if constexpr (b > 0 && c > 0) Mh[4] = (float)(b * c) * xp[a] * yp[b > 0 ? b - 1 : 0] * zp[c > 0 ? c - 1 : 0];
        }
        if constexpr (PURE) {
            static_for<NOUT>([&](auto mc) {
                constexpr int m = decltype(mc)::value;
                if constexpr (solid_harmonic_nonzero(L, m, a, b)) {
                    const float t = prm.tpure[L - 2][m * NC + k];
                    pm[m] += t * M;
                    if constexpr (P >= 4)
#pragma unroll
                        for (int i = 0; i < 3; ++i) pg[i][m] += t * Mi[i];
                    if constexpr (P == 10)
#pragma unroll
                        for (int h = 0; h < 6; ++h) ph[h][m] += t * Mh[h];
                }
            });
        } else {
            const float g = prm.gcart[L][k];
            pm[k] = g * M;
            if constexpr (P >= 4)
#pragma unroll
                for (int i = 0; i < 3; ++i) pg[i][k] = g * Mi[i];
            if constexpr (P == 10)
#pragma unroll
                for (int h = 0; h < 6; ++h) ph[h][k] = g * Mh[h];
            if constexpr (LAPM) pl[k] = g * (Mh[0] + Mh[3] + Mh[5]);
        }
    });
    const float r[3] = {x, y, z};
    // q = (2L+3) R1' + r^2 R2' comes from the caller, formed in FP64.
#pragma unroll
    for (int m = 0; m < NOUT; ++m) {
        float* d = dst + m * kBlockPoints;
        const float v = pm[m] * R0;
        d[0] = v;
        float mx = fabsf(v);
        if constexpr (P >= 4) {
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const float gi = pg[i][m] * R0 + r[i] * pm[m] * R1p;
                d[(1 + i) * pstride] = gi;
                mx = fmaxf(mx, fabsf(gi));
            }
        }
        if constexpr (P == 5) {
            const float lap = (LAPM ? pl[m] * R0 : 0.0f) + pm[m] * q;
            d[4 * pstride] = lap;
            mx = fmaxf(mx, fabsf(lap));
        }
        if constexpr (P == 10) {
            constexpr int hi[6] = {0, 0, 0, 1, 1, 2}, hj[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
            for (int h = 0; h < 6; ++h) {
                const int i = hi[h], j = hj[h];
                const float hv = ph[h][m] * R0 + (pg[i][m] * r[j] + pg[j][m] * r[i]) * R1p +
                                 pm[m] * ((i == j ? R1p : 0.0f) + r[i] * r[j] * R2p);
                d[(4 + h) * pstride] = hv;
                mx = fmaxf(mx, fabsf(hv));
            }
        }
        if constexpr (ROWMAX) {
            // Non-negative floats order like their bit patterns: one warp
            // reduction instruction.
            mx = __uint_as_float(__reduce_max_sync(0xffffffffu, __float_as_uint(mx)));
            if (lane == 0) rmax[m * 4] = mx;
        }
    }
}


}  // namespace
}  // namespace kumo_dev
