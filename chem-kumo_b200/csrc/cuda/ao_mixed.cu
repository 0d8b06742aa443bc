// FP32 AO build of the mixed-precision form (factorised radial sums; see
// ao_mixed.cuh).  One CTA of 128 threads per point block, thread j owns point
// j.  For each AO block within reach of the block's bounding box, a warp
// whose 32 points all lie outside the block's cutoff radius writes zeros
// without arithmetic; otherwise each thread forms the three radial sums of
// its point and the polynomial terms of the block's components, and stores
// the P panels of each AO row with coalesced 128-point rows.
#include "ao_common.cuh"
#include "ao_mixed.cuh"

namespace kumo_dev {
namespace {

// exp(-a r^2) given al2 = a log2(e): FP64 argument reduction t = n - f with
// |f| <= 1/2, FP32 2^f, exact scaling by 2^-n; 0 below the FP32 range.
__device__ __forceinline__ float exp_neg(double al2, double r2) {
    const double t = al2 * r2;
    if (!(t < 149.0)) return 0.0f;
    const double n = rint(t);
    return ldexpf(exp2f(static_cast<float>(n - t)), -static_cast<int>(n));
}

template <int L, bool PURE, int P>
__device__ __forceinline__ void mixed_shell(const AoMixedParams& prm, float x, float y, float z, float r2, float R0,
                                            float R1p, float R2p, float* dst, size_t pstride, float* rmax, int lane) {
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
    const float q = (float)(2 * L + 3) * R1p + r2 * R2p;
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
        mx = warp_max(mx);
        if (lane == 0) rmax[m * 4] = mx;
    }
}

template <int P, int MAXL>
__global__ void __launch_bounds__(kBlockPoints, 4) ao_mixed_kernel(const __grid_constant__ AoMixedParams prm) {
    constexpr int NW = kBlockPoints / 32;
    extern __shared__ int s_list[];
    __shared__ double s_box[NW][6];
    __shared__ int s_count[NW];

    const int blk = blockIdx.x;
    if (blk >= prm.nblocks) return;
    const int j = threadIdx.x, warp = j >> 5, lane = j & 31;
    const long long start = prm.first_point + static_cast<long long>(blk) * prm.block_size;
    long long bcount = prm.src.count - start;
    if (bcount > prm.block_size) bcount = prm.block_size;
    const bool valid = j < bcount;
    double px = 0, py = 0, pz = 0;
    if (valid) point_at(prm.src, start + j, px, py, pz);

    const DevBasis& B = prm.basis;
    const int nlist = block_shell_list(B, valid, px, py, pz, false, s_list, s_box, s_count);

    const AoScratch<float>& out = prm.out;
    const size_t pstride = static_cast<size_t>(out.row_stride) * kBlockPoints;
    float* pan = out.panels + static_cast<size_t>(blk) * P * pstride + j;
    int* kept = out.kept + static_cast<size_t>(blk) * out.row_stride;
    float* rmx = out.rowmax + static_cast<size_t>(blk) * out.row_stride * 4 + warp;
    int row = 0;
    for (int it = 0; it < nlist; ++it) {
        const int s = s_list[it];
        const double4 o = B.origin_r2[s];
        const int4 inf = B.info[s];
        const int l = inf.x & 0xff;
        const bool pure = (inf.x >> 8) & 1;
        const int nprim = inf.x >> 16;
        const int count = pure ? 2 * l + 1 : (l + 1) * (l + 2) / 2;
        const double dx = px - o.x, dy = py - o.y, dz = pz - o.z;
        const double r2d = dx * dx + dy * dy + dz * dz;
        const bool inside = valid && r2d <= o.w;
        float* dst = pan + static_cast<size_t>(row) * kBlockPoints;
        if (__any_sync(0xffffffffu, inside)) {
            float R0 = 0.0f, R1 = 0.0f, R2 = 0.0f;
            if (inside) {
                for (int p = 0; p < nprim; ++p) {
                    const MixPrim pr = prm.prims[inf.y + p];
                    const float ue = pr.u * exp_neg(pr.al2, r2d);
                    R0 += ue;
                    R1 += ue * pr.alpha;
                    R2 += ue * pr.alpha * pr.alpha;
                }
            }
            const float x = static_cast<float>(dx), y = static_cast<float>(dy), z = static_cast<float>(dz);
            const float r2 = static_cast<float>(r2d);
            const float R1p = -2.0f * R1, R2p = 4.0f * R2;
            float* rm = rmx + static_cast<size_t>(row) * 4;
            switch (l | (pure ? 16 : 0)) {
#define KUMO_MIXED(LL, PP)                                                                                   \
    case (LL) | ((PP) ? 16 : 0):                                                                             \
        if constexpr (LL <= MAXL)                                                                            \
            mixed_shell<(LL <= MAXL ? LL : 0), PP, P>(prm, x, y, z, r2, R0, R1p, R2p, dst, pstride, rm, lane); \
        break;
                KUMO_MIXED(0, false) KUMO_MIXED(1, false) KUMO_MIXED(2, false) KUMO_MIXED(3, false)
                KUMO_MIXED(4, false) KUMO_MIXED(2, true) KUMO_MIXED(3, true) KUMO_MIXED(4, true)
#undef KUMO_MIXED
                default: break;
            }
        } else {
            for (int m = 0; m < count; ++m) {
#pragma unroll
                for (int c = 0; c < P; ++c) dst[c * pstride + m * kBlockPoints] = 0.0f;
                if (lane == 0) rmx[static_cast<size_t>(row + m) * 4] = 0.0f;
            }
        }
        if (j < count) kept[row + j] = inf.w + j;
        row += count;
    }
    if (j == 0) out.nkept[blk] = row;
}

template <int P, int MAXL>
void launch(const AoMixedParams& p, cudaStream_t stream) {
    const size_t smem = sizeof(int) * static_cast<size_t>(p.basis.nblocks > 0 ? p.basis.nblocks : 1);
    if (smem > 48 * 1024)
        cudaFuncSetAttribute(ao_mixed_kernel<P, MAXL>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    ao_mixed_kernel<P, MAXL><<<p.nblocks, kBlockPoints, smem, stream>>>(p);
}

template <int P>
void dispatch_l(const AoMixedParams& p, cudaStream_t stream) {
    if (p.basis.max_l <= 2)
        launch<P, 2>(p, stream);
    else if (p.basis.max_l == 3)
        launch<P, 3>(p, stream);
    else
        launch<P, 4>(p, stream);
}

}  // namespace

void launch_ao_mixed(const AoMixedParams& p, int npanel, cudaStream_t stream) {
    if (p.nblocks <= 0) return;
    switch (npanel) {
        case 1: dispatch_l<1>(p, stream); break;
        case 4: dispatch_l<4>(p, stream); break;
        case 5: dispatch_l<5>(p, stream); break;
        case 10: dispatch_l<10>(p, stream); break;
        default: break;
    }
}

}  // namespace kumo_dev
