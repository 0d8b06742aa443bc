// AO build kernel: AO values and first/second Cartesian derivatives on one
// screening block of points per CTA, with the reference's shell cutoff and
// block screening fused in, writing only the kept AO rows (compacted, in AO
// order) to the wave's scratch.
//
// Arithmetic follows BasisEvaluator::evaluate_derivatives_batch
// (src/basis_evaluator.cpp:552-642) for orders 1 and 2 and
// BasisEvaluator::evaluate_into_impl (src/basis_evaluator.cpp:425-487) for
// order 0, operation by operation; the FP64 instantiation is compiled with
// -fmad=false so that every product and sum is rounded as written.  The
// Cartesian-to-pure transform sums the Cartesian components in index order.
// Screening follows significant_aos (src/ao_screening.hpp:35-50): an AO row is
// kept if max |value| over every panel of the reference's AO order and every
// point of the block exceeds the threshold (threshold 0 keeps every row).
//
// Thread j of the CTA owns point j of the block; the CTA walks the AO blocks
// in order, stages each block's exponents and weights in shared memory,
// computes its panels into a shared staging tile, reduces the per-AO maxima
// over the block, and copies the kept rows out with coalesced stores.
#pragma once

#include "kumo_device.cuh"

#include <utility>

namespace kumo_dev {

template <int L>
struct Cart {
    static constexpr int NC = (L + 1) * (L + 2) / 2;
};

// Gaussian Cartesian order (src/basis_evaluator.cpp:135-152) as a constexpr table.
__host__ __device__ constexpr int cart_power(int l, int k, int axis) {
    constexpr int d[6][3] = {{2, 0, 0}, {0, 2, 0}, {0, 0, 2}, {1, 1, 0}, {1, 0, 1}, {0, 1, 1}};
    constexpr int f[10][3] = {{3, 0, 0}, {0, 3, 0}, {0, 0, 3}, {1, 2, 0}, {2, 1, 0},
                              {2, 0, 1}, {1, 0, 2}, {0, 1, 2}, {0, 2, 1}, {1, 1, 1}};
    if (l == 0) return 0;
    if (l == 1) return k == axis ? 1 : 0;
    if (l == 2) return d[k][axis];
    if (l == 3) return f[k][axis];
    // l >= 4: lexicographic in (lx, ly)
    int n = 0;
    for (int lx = 0; lx <= l; ++lx)
        for (int ly = 0; ly <= l - lx; ++ly) {
            if (n == k) return axis == 0 ? lx : (axis == 1 ? ly : l - lx - ly);
            ++n;
        }
    return 0;
}

template <typename T>
struct MathOf;
template <>
struct MathOf<double> {
    __device__ static double ex(double x) { return exp(x); }
};
template <>
struct MathOf<float> {
    __device__ static float ex(float x) { return expf(x); }
};

// 1D factors of src/basis_evaluator.cpp:594-603 for power m:
// f0 = x^m, f1 = m x^(m-1) - 2 a x x^m,
// f2 = m (m-1) x^(m-2) - 2 a (2m+1) x^m + 4 a^2 x^2 x^m.
template <typename T, int M>
__device__ __forceinline__ T factor1(const T* xp, T a, T x) {
    const T t1 = M ? (T)M * xp[M > 0 ? M - 1 : 0] : (T)0;
    return t1 - (T)2 * a * x * xp[M];
}
template <typename T, int M>
__device__ __forceinline__ T factor2(const T* xp, T a, T x) {
    const T t1 = M >= 2 ? (T)(M * (M - 1)) * xp[M >= 2 ? M - 2 : 0] : (T)0;
    return t1 - (T)2 * a * (T)(2 * M + 1) * xp[M] + (T)4 * a * a * x * x * xp[M];
}

template <int... Is, typename Fn>
__device__ __forceinline__ void static_for_impl(std::integer_sequence<int, Is...>, Fn&& fn) {
    (fn(std::integral_constant<int, Is>{}), ...);
}
template <int N, typename Fn>
__device__ __forceinline__ void static_for(Fn&& fn) {
    static_for_impl(std::make_integer_sequence<int, N>{}, fn);
}

// Stage layout: stage[(m * P + c) * 128 + j].
template <typename T, int L, bool PURE, int ORDER, int P>
__device__ __forceinline__ void shell_panels(const T (&pure)[3][135], const T* s_w, const T* s_exps,
                                             const T* s_rad, int nprim, T rx, T ry, T rz, bool inside,
                                             T* stage, T (&maxabs)[15]) {
    constexpr int NC = Cart<L>::NC;
    constexpr int NOUT = PURE ? 2 * L + 1 : NC;
    constexpr int TL = L >= 2 ? L - 2 : 0;
    const int j = threadIdx.x;
    T xp[L + 1], yp[L + 1], zp[L + 1];
    xp[0] = yp[0] = zp[0] = (T)1;
#pragma unroll
    for (int n = 1; n <= L; ++n) {
        xp[n] = xp[n - 1] * rx;
        yp[n] = yp[n - 1] * ry;
        zp[n] = zp[n - 1] * rz;
    }
#pragma unroll
    for (int m = 0; m < NOUT; ++m) maxabs[m] = (T)0;

    if constexpr (ORDER == 0) {
        // evaluate_into_impl: cart[k] = ((x^px y^py) z^pz) * sum_p W_kp e^(-a_p r^2)
        T acc[NOUT];
#pragma unroll
        for (int m = 0; m < NOUT; ++m) acc[m] = (T)0;
        static_for<NC>([&](auto kc) {
            constexpr int k = decltype(kc)::value;
            constexpr int px = cart_power(L, k, 0), py = cart_power(L, k, 1), pz = cart_power(L, k, 2);
            const T polynomial = (xp[px] * yp[py]) * zp[pz];
            T radial_sum = (T)0;
            for (int p = 0; p < nprim; ++p)
                radial_sum = radial_sum + s_w[k * nprim + p] * s_rad[p * kBlockPoints + j];
            const T cart = polynomial * radial_sum;
            if constexpr (PURE) {
#pragma unroll
                for (int m = 0; m < NOUT; ++m) {
                    const T t = pure[TL][m * NC + k];
                    if (t != (T)0) acc[m] = acc[m] + t * cart;
                }
            } else {
                acc[k] = cart;
            }
        });
#pragma unroll
        for (int m = 0; m < NOUT; ++m) {
            const T v = inside ? acc[m] : (T)0;
            stage[(m * P + 0) * kBlockPoints + j] = v;
            maxabs[m] = v < 0 ? -v : v;
        }
        return;
    } else {
        // Group 0: value and gradient panels.
        {
            T acc[NOUT][4];
#pragma unroll
            for (int m = 0; m < NOUT; ++m)
#pragma unroll
                for (int c = 0; c < 4; ++c) acc[m][c] = (T)0;
            static_for<NC>([&](auto kc) {
                constexpr int k = decltype(kc)::value;
                constexpr int px = cart_power(L, k, 0), py = cart_power(L, k, 1), pz = cart_power(L, k, 2);
                T s0 = 0, s1 = 0, s2 = 0, s3 = 0;
                for (int p = 0; p < nprim; ++p) {
                    const T a = s_exps[p];
                    const T weight = s_w[k * nprim + p] * s_rad[p * kBlockPoints + j];
                    const T fx0 = xp[px], fy0 = yp[py], fz0 = zp[pz];
                    const T fx1 = factor1<T, px>(xp, a, rx);
                    const T fy1 = factor1<T, py>(yp, a, ry);
                    const T fz1 = factor1<T, pz>(zp, a, rz);
                    s0 = s0 + weight * fx0 * fy0 * fz0;
                    s1 = s1 + weight * fx1 * fy0 * fz0;
                    s2 = s2 + weight * fx0 * fy1 * fz0;
                    s3 = s3 + weight * fx0 * fy0 * fz1;
                }
                if constexpr (PURE) {
#pragma unroll
                    for (int m = 0; m < NOUT; ++m) {
                        const T t = pure[TL][m * NC + k];
                        if (t != (T)0) {
                            acc[m][0] = acc[m][0] + t * s0;
                            acc[m][1] = acc[m][1] + t * s1;
                            acc[m][2] = acc[m][2] + t * s2;
                            acc[m][3] = acc[m][3] + t * s3;
                        }
                    }
                } else {
                    acc[k][0] = s0;
                    acc[k][1] = s1;
                    acc[k][2] = s2;
                    acc[k][3] = s3;
                }
            });
#pragma unroll
            for (int m = 0; m < NOUT; ++m) {
                T mx = (T)0;
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    const T v = inside ? acc[m][c] : (T)0;
                    const T av = v < 0 ? -v : v;
                    mx = av > mx ? av : mx;
                    if (c < P) stage[(m * P + c) * kBlockPoints + j] = v;
                }
                maxabs[m] = mx;
            }
        }
        if constexpr (ORDER == 2) {
            // Group 1: second-derivative panels xx, xy, xz, yy, yz, zz.
            T acc[NOUT][6];
#pragma unroll
            for (int m = 0; m < NOUT; ++m)
#pragma unroll
                for (int c = 0; c < 6; ++c) acc[m][c] = (T)0;
            static_for<NC>([&](auto kc) {
                constexpr int k = decltype(kc)::value;
                constexpr int px = cart_power(L, k, 0), py = cart_power(L, k, 1), pz = cart_power(L, k, 2);
                T s[6] = {0, 0, 0, 0, 0, 0};
                for (int p = 0; p < nprim; ++p) {
                    const T a = s_exps[p];
                    const T weight = s_w[k * nprim + p] * s_rad[p * kBlockPoints + j];
                    const T fx0 = xp[px], fy0 = yp[py], fz0 = zp[pz];
                    const T fx1 = factor1<T, px>(xp, a, rx);
                    const T fy1 = factor1<T, py>(yp, a, ry);
                    const T fz1 = factor1<T, pz>(zp, a, rz);
                    const T fx2 = factor2<T, px>(xp, a, rx);
                    const T fy2 = factor2<T, py>(yp, a, ry);
                    const T fz2 = factor2<T, pz>(zp, a, rz);
                    s[0] = s[0] + weight * fx2 * fy0 * fz0;
                    s[1] = s[1] + weight * fx1 * fy1 * fz0;
                    s[2] = s[2] + weight * fx1 * fy0 * fz1;
                    s[3] = s[3] + weight * fx0 * fy2 * fz0;
                    s[4] = s[4] + weight * fx0 * fy1 * fz1;
                    s[5] = s[5] + weight * fx0 * fy0 * fz2;
                }
                if constexpr (PURE) {
#pragma unroll
                    for (int m = 0; m < NOUT; ++m) {
                        const T t = pure[TL][m * NC + k];
                        if (t != (T)0) {
#pragma unroll
                            for (int c = 0; c < 6; ++c) acc[m][c] = acc[m][c] + t * s[c];
                        }
                    }
                } else {
#pragma unroll
                    for (int c = 0; c < 6; ++c) acc[k][c] = s[c];
                }
            });
#pragma unroll
            for (int m = 0; m < NOUT; ++m) {
                T mx = maxabs[m];
                T h[6];
#pragma unroll
                for (int c = 0; c < 6; ++c) {
                    h[c] = inside ? acc[m][c] : (T)0;
                    const T av = h[c] < 0 ? -h[c] : h[c];
                    mx = av > mx ? av : mx;
                    if constexpr (P == kPanelsFull) stage[(m * P + 4 + c) * kBlockPoints + j] = h[c];
                }
                if constexpr (P == kPanelsLaplacian) stage[(m * P + 4) * kBlockPoints + j] = (h[0] + h[3]) + h[5];
                maxabs[m] = mx;
            }
        }
    }
}

template <typename T>
__device__ __forceinline__ T warp_max(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const T w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w > v ? w : v;
    }
    return v;
}

// One CTA per screening block.  Dynamic shared memory: the staging tile
// (max_count * P * 128 values of T) followed by the radial factors
// (kMaxPrim * 128 values).
template <typename T, int ORDER, int P>
__global__ void __launch_bounds__(kBlockPoints) ao_build_kernel(const __grid_constant__ AoBuildParams<T> prm) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* stage = reinterpret_cast<T*>(smem_raw);
    T* s_rad = stage + (size_t)prm.basis.max_count * P * kBlockPoints;
    __shared__ T s_exps[kMaxPrim];
    __shared__ T s_w[15 * kMaxPrim];
    __shared__ T s_red[kBlockPoints / 32][16];
    __shared__ int s_keep[16];

    const int blk = blockIdx.x;
    if (blk >= prm.nblocks) return;
    const int j = threadIdx.x;
    const long long start = prm.first_point + (long long)blk * prm.block_size;
    long long b = prm.src.count - start;
    if (b > prm.block_size) b = prm.block_size;
    const bool valid = j < b;
    double px = 0, py = 0, pz = 0;
    if (valid) point_at(prm.src, start + j, px, py, pz);

    const DevBasis& B = prm.basis;
    const AoScratch<T>& out = prm.out;
    T* panels = out.panels + (size_t)blk * P * out.row_stride * kBlockPoints;
    int* kept = out.kept + (size_t)blk * out.row_stride;
    const bool keep_all = prm.threshold == 0.0;
    const T thr = (T)prm.threshold;
    int nk = 0;

    for (int s = 0; s < B.nblocks; ++s) {
        const double4 o = B.origin_r2[s];
        const int4 inf = B.info[s];
        const int l = inf.x & 0xff;
        const bool pure = (inf.x >> 8) & 1;
        const int nprim = inf.x >> 16;
        const int count = pure ? 2 * l + 1 : (l + 1) * (l + 2) / 2;
        const int ncart = (l + 1) * (l + 2) / 2;
        // Displacement and squared distance in FP64 (the cutoff test is FP64 in
        // both precisions, so the cutoff zeros are those of the reference).
        const double dx = px - o.x, dy = py - o.y, dz = pz - o.z;
        const double r2d = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
        const bool inside = valid && (r2d <= o.w);
        const int any_inside = __syncthreads_or(inside);
        if (!any_inside && !keep_all) continue;
        // Stage this block's exponents and weights.
        const T* gexp = sizeof(T) == 8 ? (const T*)B.exps : (const T*)B.exps_f;
        const T* gw = sizeof(T) == 8 ? (const T*)B.weights : (const T*)B.weights_f;
        if (j < nprim) s_exps[j] = gexp[inf.y + j];
        for (int q = j; q < ncart * nprim; q += kBlockPoints) s_w[q] = gw[inf.z + q];
        __syncthreads();
        const T r2 = sizeof(T) == 8 ? (T)r2d : (T)((T)dx * (T)dx + (T)dy * (T)dy + (T)dz * (T)dz);
        if (inside)
            for (int p = 0; p < nprim; ++p) s_rad[p * kBlockPoints + j] = MathOf<T>::ex(-s_exps[p] * r2);
        T maxabs[15];
        const T rx = (T)dx, ry = (T)dy, rz = (T)dz;
        // Each thread only reads its own radial factors, so no barrier is needed here.
        switch (l | (pure ? 16 : 0)) {
#define KUMO_SHELL(LL, PP)                                                                        \
    case (LL) | ((PP) ? 16 : 0):                                                                 \
        shell_panels<T, LL, PP, ORDER, P>(prm.pure, s_w, s_exps, s_rad, nprim, rx, ry, rz, inside, stage, \
                                          maxabs);                                                        \
        break;
            KUMO_SHELL(0, false) KUMO_SHELL(1, false) KUMO_SHELL(2, false) KUMO_SHELL(3, false)
            KUMO_SHELL(4, false) KUMO_SHELL(2, true) KUMO_SHELL(3, true) KUMO_SHELL(4, true)
#undef KUMO_SHELL
            default: break;
        }
        // Block-wide maximum per AO of the shell.
        const int warp = j >> 5, lane = j & 31;
#pragma unroll
        for (int m = 0; m < 15; ++m) {
            if (m < count) {
                const T w = warp_max(maxabs[m]);
                if (lane == 0) s_red[warp][m] = w;
            }
        }
        __syncthreads();
        if (j < count) {
            T mx = s_red[0][j];
#pragma unroll
            for (int w = 1; w < kBlockPoints / 32; ++w) mx = s_red[w][j] > mx ? s_red[w][j] : mx;
            s_keep[j] = keep_all || mx > thr;
        }
        __syncthreads();
        for (int m = 0; m < count; ++m) {
            if (!s_keep[m]) continue;
#pragma unroll
            for (int c = 0; c < P; ++c)
                panels[((size_t)c * out.row_stride + nk) * kBlockPoints + j] = stage[(m * P + c) * kBlockPoints + j];
            if (j == 0) kept[nk] = (inf.w) + m;
            ++nk;
        }
        __syncthreads();
    }
    if (j == 0) out.nkept[blk] = nk;
}

}  // namespace kumo_dev
