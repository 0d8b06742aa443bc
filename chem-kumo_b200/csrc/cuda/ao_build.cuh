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
// Thread j of the CTA owns point j of the block.  The CTA first bounds its
// points with a box and lists, in AO order, the AO blocks whose cutoff sphere
// reaches the box (the others give exact zeros everywhere and, with a
// positive threshold, no kept row); it then walks that list with each
// block's exponents and weights staged in shared memory (double-buffered),
// computes the panels into a shared staging tile, reduces the per-AO maxima
// over the block and copies the kept rows out with coalesced stores.
#pragma once

#include <utility>

#include "ao_common.cuh"
#include "kumo_device.cuh"

namespace kumo_dev {

// exp(-a r^2) for a radial factor: FP64 as the reference; in FP32 the
// argument is reduced in FP64 (-a r^2 log2 e = n + f, |f| <= 1/2) so that the
// factor keeps FP32 relative accuracy for large a r^2.
template <typename T>
struct RadialExp;
template <>
struct RadialExp<double> {
    __device__ static double of(double a, double r2) { return exp(-a * r2); }
};
template <>
struct RadialExp<float> {
    __device__ static float of(double a, double r2) {
        const double t = -a * r2 * 1.4426950408889634;  // log2(e)
        const double n = rint(t);
        if (n < -149.0) return 0.0f;
        return ldexpf(exp2f(static_cast<float>(t - n)), static_cast<int>(n));
    }
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

// Largest angular momentum whose panels are summed primitives-outer (more
// accumulators live at once: f shells spill a few bytes and are still
// faster that way, 104 -> 91 ms per FP64 step of the 740-AO workload; g
// shells would spill far more).
constexpr int kPOuterMaxL = 3;

// Panels of one shell for the thread's point into stage[(m * P + c) * 128 + j],
// with maxabs[m] the largest |value| over the panels of the AO order.
template <typename T, int L, bool PURE, int ORDER, int P, int NMAX>
__device__ __forceinline__ void shell_panels(const T (&pure)[3][135], const T* s_w, const T* s_exps,
                                             const T* s_rad, int nprim, T rx, T ry, T rz, bool inside,
                                             T* stage, T (&maxabs)[NMAX]) {
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
            if constexpr (L <= kPOuterMaxL) {
                // Primitives outer, components inner: the sums of every
                // component advance together (independent chains), and each
                // 1D factor is formed once per primitive and power.  Every
                // sum still adds its primitives in order and every product
                // is formed as in the components-outer form, so the values
                // are the same bits.
                T s[NC][4];
#pragma unroll
                for (int k = 0; k < NC; ++k)
#pragma unroll
                    for (int c = 0; c < 4; ++c) s[k][c] = (T)0;
                for (int p = 0; p < nprim; ++p) {
                    const T a = s_exps[p];
                    const T rad = s_rad[p * kBlockPoints + j];
                    T f1x[L + 1], f1y[L + 1], f1z[L + 1];
                    static_for<L + 1>([&](auto nc) {
                        constexpr int n = decltype(nc)::value;
                        f1x[n] = factor1<T, n>(xp, a, rx);
                        f1y[n] = factor1<T, n>(yp, a, ry);
                        f1z[n] = factor1<T, n>(zp, a, rz);
                    });
                    static_for<NC>([&](auto kc) {
                        constexpr int k = decltype(kc)::value;
                        constexpr int px = cart_power(L, k, 0), py = cart_power(L, k, 1), pz = cart_power(L, k, 2);
                        const T weight = s_w[k * nprim + p] * rad;
                        const T fx0 = xp[px], fy0 = yp[py], fz0 = zp[pz];
                        s[k][0] = s[k][0] + weight * fx0 * fy0 * fz0;
                        s[k][1] = s[k][1] + weight * f1x[px] * fy0 * fz0;
                        s[k][2] = s[k][2] + weight * fx0 * f1y[py] * fz0;
                        s[k][3] = s[k][3] + weight * fx0 * fy0 * f1z[pz];
                    });
                }
                static_for<NC>([&](auto kc) {
                    constexpr int k = decltype(kc)::value;
                    if constexpr (PURE) {
#pragma unroll
                        for (int m = 0; m < NOUT; ++m) {
                            const T t = pure[TL][m * NC + k];
                            if (t != (T)0) {
#pragma unroll
                                for (int c = 0; c < 4; ++c) acc[m][c] = acc[m][c] + t * s[k][c];
                            }
                        }
                    } else {
#pragma unroll
                        for (int c = 0; c < 4; ++c) acc[k][c] = s[k][c];
                    }
                });
            } else static_for<NC>([&](auto kc) {
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
            // Second-derivative panels in two halves (xx, xy, xz), (yy, yz, zz)
            // to bound the live accumulators; each panel's sum over primitives
            // is independent, so the halves give the same values as one pass.
            static_for<2>([&](auto hc) {
                constexpr int H = decltype(hc)::value;
                T acc[NOUT][3];
#pragma unroll
                for (int m = 0; m < NOUT; ++m)
#pragma unroll
                    for (int c = 0; c < 3; ++c) acc[m][c] = (T)0;
                if constexpr (L <= kPOuterMaxL) {
                    // Primitives outer, as for group 0 (same bits).
                    T s[NC][3];
#pragma unroll
                    for (int k = 0; k < NC; ++k)
#pragma unroll
                        for (int c = 0; c < 3; ++c) s[k][c] = (T)0;
                    for (int p = 0; p < nprim; ++p) {
                        const T a = s_exps[p];
                        const T rad = s_rad[p * kBlockPoints + j];
                        T f1x[L + 1], f1y[L + 1], f1z[L + 1], f2a[L + 1], f2b[L + 1];
                        static_for<L + 1>([&](auto nc) {
                            constexpr int n = decltype(nc)::value;
                            f1y[n] = factor1<T, n>(yp, a, ry);
                            f1z[n] = factor1<T, n>(zp, a, rz);
                            if constexpr (H == 0) {
                                f1x[n] = factor1<T, n>(xp, a, rx);
                                f2a[n] = factor2<T, n>(xp, a, rx);
                            } else {
                                f2a[n] = factor2<T, n>(yp, a, ry);
                                f2b[n] = factor2<T, n>(zp, a, rz);
                            }
                        });
                        static_for<NC>([&](auto kc) {
                            constexpr int k = decltype(kc)::value;
                            constexpr int px = cart_power(L, k, 0), py = cart_power(L, k, 1), pz = cart_power(L, k, 2);
                            const T weight = s_w[k * nprim + p] * rad;
                            const T fx0 = xp[px], fy0 = yp[py], fz0 = zp[pz];
                            if constexpr (H == 0) {
                                s[k][0] = s[k][0] + weight * f2a[px] * fy0 * fz0;
                                s[k][1] = s[k][1] + weight * f1x[px] * f1y[py] * fz0;
                                s[k][2] = s[k][2] + weight * f1x[px] * fy0 * f1z[pz];
                            } else {
                                s[k][0] = s[k][0] + weight * fx0 * f2a[py] * fz0;
                                s[k][1] = s[k][1] + weight * fx0 * f1y[py] * f1z[pz];
                                s[k][2] = s[k][2] + weight * fx0 * fy0 * f2b[pz];
                            }
                        });
                    }
                    static_for<NC>([&](auto kc) {
                        constexpr int k = decltype(kc)::value;
                        if constexpr (PURE) {
#pragma unroll
                            for (int m = 0; m < NOUT; ++m) {
                                const T t = pure[TL][m * NC + k];
                                if (t != (T)0) {
#pragma unroll
                                    for (int c = 0; c < 3; ++c) acc[m][c] = acc[m][c] + t * s[k][c];
                                }
                            }
                        } else {
#pragma unroll
                            for (int c = 0; c < 3; ++c) acc[k][c] = s[k][c];
                        }
                    });
                } else static_for<NC>([&](auto kc) {
                    constexpr int k = decltype(kc)::value;
                    constexpr int px = cart_power(L, k, 0), py = cart_power(L, k, 1), pz = cart_power(L, k, 2);
                    T s[3] = {0, 0, 0};
                    for (int p = 0; p < nprim; ++p) {
                        const T a = s_exps[p];
                        const T weight = s_w[k * nprim + p] * s_rad[p * kBlockPoints + j];
                        const T fx0 = xp[px], fy0 = yp[py], fz0 = zp[pz];
                        const T fy1 = factor1<T, py>(yp, a, ry);
                        const T fz1 = factor1<T, pz>(zp, a, rz);
                        if constexpr (H == 0) {
                            const T fx1 = factor1<T, px>(xp, a, rx);
                            const T fx2 = factor2<T, px>(xp, a, rx);
                            s[0] = s[0] + weight * fx2 * fy0 * fz0;
                            s[1] = s[1] + weight * fx1 * fy1 * fz0;
                            s[2] = s[2] + weight * fx1 * fy0 * fz1;
                        } else {
                            const T fy2 = factor2<T, py>(yp, a, ry);
                            const T fz2 = factor2<T, pz>(zp, a, rz);
                            s[0] = s[0] + weight * fx0 * fy2 * fz0;
                            s[1] = s[1] + weight * fx0 * fy1 * fz1;
                            s[2] = s[2] + weight * fx0 * fy0 * fz2;
                        }
                    }
                    if constexpr (PURE) {
#pragma unroll
                        for (int m = 0; m < NOUT; ++m) {
                            const T t = pure[TL][m * NC + k];
                            if (t != (T)0) {
#pragma unroll
                                for (int c = 0; c < 3; ++c) acc[m][c] = acc[m][c] + t * s[c];
                            }
                        }
                    } else {
#pragma unroll
                        for (int c = 0; c < 3; ++c) acc[k][c] = s[c];
                    }
                });
#pragma unroll
                for (int m = 0; m < NOUT; ++m) {
                    T mx = maxabs[m];
                    T h[3];
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        h[c] = inside ? acc[m][c] : (T)0;
                        const T av = h[c] < 0 ? -h[c] : h[c];
                        mx = av > mx ? av : mx;
                        if constexpr (P == kPanelsFull) stage[(m * P + 4 + 3 * H + c) * kBlockPoints + j] = h[c];
                    }
                    if constexpr (P == kPanelsLaplacian) {
                        // Laplacian panel (xx + yy) + zz.
                        T* lap = &stage[(m * P + 4) * kBlockPoints + j];
                        if constexpr (H == 0)
                            *lap = h[0];
                        else
                            *lap = (*lap + h[0]) + h[2];
                    }
                    maxabs[m] = mx;
                }
            });
        }
    }
}

// One CTA per screening block.  Dynamic shared memory: the staging tile
// (max_count * P * 128 values of T), the radial factors (kMaxPrim * 128
// values of T) and the list of AO blocks within reach (nblocks ints).
template <typename T, int ORDER, int P, int MAXL>
__global__ void __launch_bounds__(kBlockPoints, sizeof(T) == 8 ? 3 : 5) ao_build_kernel(const __grid_constant__ AoBuildParams<T> prm) {
    constexpr int NW = kBlockPoints / 32;
    constexpr int NMAX = MaxOut<MAXL>::v;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* stage = reinterpret_cast<T*>(smem_raw);
    T* s_rad = stage + (size_t)prm.basis.max_count * P * kBlockPoints;
    int* s_list = reinterpret_cast<int*>(s_rad + (size_t)kMaxPrim * kBlockPoints);
    __shared__ T s_exps[2][kMaxPrim];
    __shared__ T s_w[2][15 * kMaxPrim];
    __shared__ T s_red[2][NW][16];
    __shared__ double s_box[NW][6];
    __shared__ int s_count[NW];

    const int blk = blockIdx.x;
    if (blk >= prm.nblocks) return;
    const int j = threadIdx.x, warp = j >> 5, lane = j & 31;
    long long start, b;
    int sblock;
    cta_points(prm.first_point, prm.block_size, prm.screen_block, prm.src.count, blk, start, b, sblock);
    const bool valid = j < b;
    double px = 0, py = 0, pz = 0;
    if (valid) point_at(prm.src, start + j, px, py, pz);

    const DevBasis& B = prm.basis;
    const AoScratch<T>& out = prm.out;
    T* panels = out.panels + (size_t)blk * P * out.row_stride * kBlockPoints;
    int* kept = out.kept + (size_t)blk * out.row_stride;
    const bool keep_all = prm.threshold == 0.0;
    const T thr = (T)prm.threshold;

    const int nlist = block_shell_list(B, valid, px, py, pz, keep_all && !prm.keep_reaching, s_list, s_box, s_count);

    const T* gexp = sizeof(T) == 8 ? (const T*)B.exps : (const T*)B.exps_f;
    const T* gw = sizeof(T) == 8 ? (const T*)B.weights : (const T*)B.weights_f;
    const double* gexp64 = B.exps;
    int nk = 0;
    for (int it = 0; it < nlist; ++it) {
        const int buf = it & 1;
        const int s = s_list[it];
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
        // Stage this block's exponents and weights (double-buffered, so one
        // barrier per block suffices).
        if (j < nprim) s_exps[buf][j] = gexp[inf.y + j];
        for (int q = j; q < ncart * nprim; q += kBlockPoints) s_w[buf][q] = gw[inf.z + q];
        __syncthreads();
        if (inside)
            for (int p = 0; p < nprim; ++p) s_rad[p * kBlockPoints + j] = RadialExp<T>::of(gexp64[inf.y + p], r2d);
        T maxabs[NMAX];
        const T rx = (T)dx, ry = (T)dy, rz = (T)dz;
        // Each thread only reads its own radial factors, so no barrier is needed here.
        switch (l | (pure ? 16 : 0)) {
#define KUMO_SHELL(LL, PP)                                                                                \
    case (LL) | ((PP) ? 16 : 0):                                                                          \
        if constexpr (LL <= MAXL)                                                                         \
            shell_panels<T, (LL <= MAXL ? LL : 0), PP, ORDER, P, NMAX>(prm.pure, s_w[buf], s_exps[buf], s_rad, \
                                                                      nprim, rx, ry, rz, inside, stage, maxabs); \
        break;
            KUMO_SHELL(0, false) KUMO_SHELL(1, false) KUMO_SHELL(2, false) KUMO_SHELL(3, false)
            KUMO_SHELL(4, false) KUMO_SHELL(2, true) KUMO_SHELL(3, true) KUMO_SHELL(4, true)
#undef KUMO_SHELL
            default: break;
        }
        // Block-wide maximum per AO of the shell.
#pragma unroll
        for (int m = 0; m < NMAX; ++m) {
            if (m < count) {
                const T w = warp_max(maxabs[m]);
                if (lane == 0) s_red[buf][warp][m] = w;
            }
        }
        __syncthreads();
        for (int m = 0; m < count; ++m) {
            T mx = s_red[buf][0][m];
#pragma unroll
            for (int w = 1; w < NW; ++w) mx = s_red[buf][w][m] > mx ? s_red[buf][w][m] : mx;
            if (prm.mask_pass == 1) {
                // Non-negative doubles order like their bit patterns.
                if (j == 0 && mx > (T)0)
                    atomicMax(reinterpret_cast<unsigned long long*>(prm.block_max) +
                                  (size_t)sblock * B.nao + inf.w + m,
                              static_cast<unsigned long long>(__double_as_longlong(static_cast<double>(mx))));
                continue;
            }
            if (prm.mask_pass == 2) mx = (T)prm.block_max[(size_t)sblock * B.nao + inf.w + m];
            if (!(keep_all || mx > thr)) continue;
#pragma unroll
            for (int c = 0; c < P; ++c)
                panels[((size_t)c * out.row_stride + nk) * kBlockPoints + j] = stage[(m * P + c) * kBlockPoints + j];
            if (j == 0) {
                kept[nk] = inf.w + m;
                if (out.rowmax) out.rowmax[(size_t)blk * out.row_stride + nk] = static_cast<float>(mx);
            }
            ++nk;
        }
    }
    if (j == 0) out.nkept[blk] = nk;
}

}  // namespace kumo_dev
