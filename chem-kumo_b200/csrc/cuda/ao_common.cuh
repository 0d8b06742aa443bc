// Device helpers shared by the AO build kernels: Gaussian Cartesian order,
// compile-time loops, warp reductions, and the list of AO blocks whose cutoff
// sphere reaches a point block's bounding box.
#pragma once

#include <utility>

#include "kumo_device.cuh"

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

template <int... Is, typename Fn>
__device__ __forceinline__ void static_for_impl(std::integer_sequence<int, Is...>, Fn&& fn) {
    (fn(std::integral_constant<int, Is>{}), ...);
}
template <int N, typename Fn>
__device__ __forceinline__ void static_for(Fn&& fn) {
    static_for_impl(std::make_integer_sequence<int, N>{}, fn);
}

template <int MAXL>
struct MaxOut {
    static constexpr int v = (MAXL + 1) * (MAXL + 2) / 2;
};

template <typename T>
__device__ __forceinline__ T warp_max(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const T w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w > v ? w : v;
    }
    return v;
}

__device__ __forceinline__ double warp_min_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ double warp_max_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Bounding box of the block's points (thread j owns point j; invalid points
// do not count) and the AO blocks within reach of it, in AO order, written to
// s_list; returns their number.  With keep_all every AO block is listed.  A
// block is left out only if the box is farther than its cutoff radius by a
// relative margin that covers the rounding of both distances, so every point
// it leaves out is also outside the cutoff in the reference's arithmetic.
// s_box and s_count are shared scratch of kBlockPoints / 32 entries.
__device__ inline int block_shell_list(const DevBasis& B, bool valid, double px, double py, double pz, bool keep_all,
                                       int* s_list, double (*s_box)[6], int* s_count) {
    constexpr int NW = kBlockPoints / 32;
    const int j = threadIdx.x, warp = j >> 5, lane = j & 31;
    {
        const double big = 1.0e300;
        double lo[3] = {valid ? px : big, valid ? py : big, valid ? pz : big};
        double hi[3] = {valid ? px : -big, valid ? py : -big, valid ? pz : -big};
        for (int a = 0; a < 3; ++a) {
            lo[a] = warp_min_d(lo[a]);
            hi[a] = warp_max_d(hi[a]);
        }
        if (lane == 0)
            for (int a = 0; a < 3; ++a) {
                s_box[warp][a] = lo[a];
                s_box[warp][3 + a] = hi[a];
            }
    }
    __syncthreads();
    double lo[3], hi[3];
    for (int a = 0; a < 3; ++a) {
        lo[a] = s_box[0][a];
        hi[a] = s_box[0][3 + a];
        for (int w = 1; w < NW; ++w) {
            lo[a] = fmin(lo[a], s_box[w][a]);
            hi[a] = fmax(hi[a], s_box[w][3 + a]);
        }
    }
    int nlist = 0;
    for (int c0 = 0; c0 < B.nblocks; c0 += kBlockPoints) {
        const int s = c0 + j;
        bool reach = false;
        if (s < B.nblocks) {
            if (keep_all) {
                reach = true;
            } else {
                const double4 o = B.origin_r2[s];
                const double ox[3] = {o.x, o.y, o.z};
                double d2 = 0.0;
                for (int a = 0; a < 3; ++a) {
                    const double d = fmax(0.0, fmax(lo[a] - ox[a], ox[a] - hi[a]));
                    d2 += d * d;
                }
                reach = !(d2 > o.w * (1.0 + 1e-10) + 1e-300);
            }
        }
        const unsigned ballot = __ballot_sync(0xffffffffu, reach);
        if (lane == 0) s_count[warp] = __popc(ballot);
        __syncthreads();
        int before = nlist;
        for (int w = 0; w < warp; ++w) before += s_count[w];
        if (reach) s_list[before + __popc(ballot & ((1u << lane) - 1u))] = s;
        int total = 0;
        for (int w = 0; w < NW; ++w) total += s_count[w];
        __syncthreads();
        nlist += total;
    }
    return nlist;
}

}  // namespace kumo_dev
