// FP32 AO build of the mixed-precision form (factorised radial sums; see
// ao_mixed.cuh).  One CTA of 128 threads per point block, thread j owns point
// j.  For each AO block within reach of the block's bounding box, a warp
// whose 32 points all lie outside the block's cutoff radius writes zeros
// without arithmetic; otherwise each thread forms the three radial sums of
// its point and the polynomial terms of the block's components, and stores
// the P panels of each AO row with coalesced 128-point rows.
#include "func_attr.cuh"
#include "ao_common.cuh"
#include "ao_mixed.cuh"
#include "ao_mixed_shell.cuh"

namespace kumo_dev {
namespace {

template <int P, int MAXL>
__global__ void __launch_bounds__(kBlockPoints, (P == 10 || MAXL >= 4) ? 6 : 8) ao_mixed_kernel(const __grid_constant__ AoMixedParams prm) {
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
    const bool valid = j < bcount && point_exists(prm.src, start + j);
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
    // The next listed block's centre and table entry are loaded one iteration
    // ahead (read-only tables), so their latency overlaps this block's work.
    double4 o_next = make_double4(0.0, 0.0, 0.0, -1.0);
    int4 inf_next = make_int4(0, 0, 0, 0);
    if (nlist > 0) {
        o_next = B.origin_r2[s_list[0]];
        inf_next = B.info[s_list[0]];
    }
    for (int it = 0; it < nlist; ++it) {
        const double4 o = o_next;
        const int4 inf = inf_next;
        if (it + 1 < nlist) {
            const int sn = s_list[it + 1];
            o_next = B.origin_r2[sn];
            inf_next = B.info[sn];
        }
        const int l = inf.x & 0xff;
        const bool pure = (inf.x >> 8) & 1;
        const int nprim = inf.x >> 16;
        const int count = pure ? 2 * l + 1 : (l + 1) * (l + 2) / 2;
        const double dx = px - o.x, dy = py - o.y, dz = pz - o.z;
        const double r2d = dx * dx + dy * dy + dz * dz;
        const bool inside = valid && r2d <= o.w;
        float* dst = pan + static_cast<size_t>(row) * kBlockPoints;
        if (__any_sync(0xffffffffu, inside)) {
            // Radial sums in FP64 of the FP32 products u e (a and a^2 times
            // them are exact in FP64), and the Laplacian's radial factor
            // q = (2l+3) R1' + r^2 R2', whose terms partly cancel, formed in
            // FP64: each factor is rounded to FP32 once.
            double R0 = 0.0, R1 = 0.0, R2 = 0.0;
            if (inside) {
                for (int p = 0; p < nprim; ++p) {
                    const MixPrim pr = prm.prims[inf.y + p];
                    const double ue = static_cast<double>(pr.u * exp_neg(pr.al2, r2d));
                    const double a = pr.al2 * 0.6931471805599453;  // the exponent (ln 2 = 1 / log2 e)
                    R0 += ue;
                    R1 += ue * a;
                    R2 += ue * (a * a);
                }
            }
            const float x = static_cast<float>(dx), y = static_cast<float>(dy), z = static_cast<float>(dz);
            const float r2 = static_cast<float>(r2d);
            const float R1p = static_cast<float>(-2.0 * R1), R2p = static_cast<float>(4.0 * R2);
            const float q = static_cast<float>(static_cast<double>(2 * l + 3) * (-2.0 * R1) + r2d * (4.0 * R2));
            float* rm = rmx + static_cast<size_t>(row) * 4;
            switch (l | (pure ? 16 : 0)) {
#define KUMO_MIXED(LL, PP)                                                                                   \
    case (LL) | ((PP) ? 16 : 0):                                                                             \
        if constexpr (LL <= MAXL)                                                                            \
            mixed_shell<(LL <= MAXL ? LL : 0), PP, P>(prm, x, y, z, r2, static_cast<float>(R0), R1p, R2p, q, dst, \
                                                      pstride, rm, lane);                                   \
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
    KUMO_REGISTER_KERNEL(ao_mixed_kernel<P, MAXL>);
    const size_t smem = sizeof(int) * static_cast<size_t>(p.basis.nblocks > 0 ? p.basis.nblocks : 1);
    if (smem > 48 * 1024)
        ensure_dynamic_smem(reinterpret_cast<const void*>(ao_mixed_kernel<P, MAXL>), static_cast<int>(smem));
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
