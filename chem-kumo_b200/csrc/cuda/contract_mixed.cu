// Mixed-precision AO-MO contraction (CUDA-core form): one CTA per 32 points
// of a block, 8 warps; FP32 products accumulated in FP32 within each K tile of
// 16 AOs and folded into FP64 accumulators after every tile, so the FP32
// rounding error grows with the tile length, not with the number of AOs.
#include "mixed.cuh"

namespace kumo_dev {
namespace {

__device__ __forceinline__ void cp_async16f(void* smem, const void* gmem, bool valid) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    const int n = valid ? 16 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(n));
}

template <int P>
struct NQm {
    static constexpr int v = P == 1 ? 1 : P == 4 ? 7 : P == 5 ? 8 : 19;
};

template <int P, int MPT>
__device__ __forceinline__ void fold(const double (&acc)[P][MPT], double (&q)[NQm<P>::v]) {
#pragma unroll
    for (int t = 0; t < MPT; ++t) {
        q[0] += acc[0][t] * acc[0][t];
        if constexpr (P >= 4) {
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                q[1 + a] += acc[0][t] * acc[1 + a][t];
                q[4 + a] += acc[1 + a][t] * acc[1 + a][t];
            }
        }
        if constexpr (P == 5) q[7] += acc[0][t] * acc[4][t];
        if constexpr (P == 10) {
            constexpr int pa[6] = {0, 0, 0, 1, 1, 2}, pc[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
            for (int h = 0; h < 6; ++h) {
                q[7 + h] += acc[0][t] * acc[4 + h][t];
                q[13 + h] += acc[1 + pa[h]][t] * acc[1 + pc[h]][t];
            }
        }
    }
}

template <int P>
__device__ __forceinline__ void record(const double* f, int ao_order, DevDD& d) {
    dd_zero(d);
    d.value = f[0];
    if (ao_order == 0 || P == 1) return;
    for (int a = 0; a < 3; ++a) {
        d.grad[a] = 2.0 * f[1 + a];
        d.tau_axes[a] = 0.5 * f[4 + a];
        d.tau += d.tau_axes[a];
    }
    if (ao_order < 2) return;
    if constexpr (P == 10) {
        for (int h = 0; h < 6; ++h) d.hess[h] = 2.0 * (f[7 + h] + f[13 + h]);
        d.lap = (d.hess[0] + d.hess[3]) + d.hess[5];
    } else if constexpr (P == 5) {
        d.lap = 2.0 * f[7] + 2.0 * ((f[4] + f[5]) + f[6]);
    }
}

template <int P, int MPT, int KT>
__global__ void __launch_bounds__(256, 1) contract_mixed_kernel(const __grid_constant__ ContractMixedParams prm) {
    constexpr int MOC = 8 * MPT;
    constexpr int Q = NQm<P>::v;
    extern __shared__ __align__(16) unsigned char smraw[];
    float* phs = reinterpret_cast<float*>(smraw);            // [2][KT][P][32]
    float* cs = phs + 2 * KT * P * 32;                        // [2][KT][MOC]
    double* red = reinterpret_cast<double*>(cs + 2 * KT * MOC);  // [8][Q][32]
    double* fin = red + 8 * Q * 32;                           // [2][Q][32]

    const int blk = blockIdx.x >> 2;
    const int j0 = (blockIdx.x & 3) * 32;
    const long long start = prm.first_point + (long long)blk * prm.block_size;
    long long b = prm.count - start;
    if (b > prm.block_size) b = prm.block_size;
    if (j0 >= b) return;
    const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
    const AoScratch<float>& scr = prm.scr;
    const int nk = scr.nkept[blk];
    const float* pbase = scr.panels + (size_t)blk * P * scr.row_stride * kBlockPoints + j0;
    const int* kept = scr.kept + (size_t)blk * scr.row_stride;

    for (int ci = 0; ci < prm.nchannels; ++ci) {
        const MoChannelF ch = prm.ch[ci];
        double q[Q];
#pragma unroll
        for (int i = 0; i < Q; ++i) q[i] = 0.0;
        for (int mo0 = 0; mo0 < ch.nocc; mo0 += MOC) {
            double acc[P][MPT];
#pragma unroll
            for (int c = 0; c < P; ++c)
#pragma unroll
                for (int t = 0; t < MPT; ++t) acc[c][t] = 0.0;
            const int ntiles = (nk + KT - 1) / KT;
            auto load_tile = [&](int tile, int buf) {
                const int k0 = tile * KT;
                float* ph = phs + buf * KT * P * 32;
                for (int c = tid; c < KT * P * 8; c += 256) {
                    const int kk = c / (P * 8), rem = c % (P * 8), cc = rem / 8, jj = (rem % 8) * 4;
                    const bool ok = k0 + kk < nk;
                    const float* src = pbase + ((size_t)cc * scr.row_stride + (ok ? k0 + kk : 0)) * kBlockPoints + jj;
                    cp_async16f(ph + (kk * P + cc) * 32 + jj, src, ok);
                }
                float* cb = cs + buf * KT * MOC;
                for (int c = tid; c < KT * MOC / 4; c += 256) {
                    const int kk = c / (MOC / 4), col = (c % (MOC / 4)) * 4;
                    const bool ok = (k0 + kk < nk) && (mo0 + col < ch.ldc);
                    const float* src = ch.ct + (size_t)(ok ? kept[k0 + kk] : 0) * ch.ldc + (ok ? mo0 + col : 0);
                    cp_async16f(cb + kk * MOC + col, src, ok);
                }
                asm volatile("cp.async.commit_group;\n" ::);
            };
            if (ntiles > 0) load_tile(0, 0);
            for (int t = 0; t < ntiles; ++t) {
                if (t + 1 < ntiles) {
                    load_tile(t + 1, (t + 1) & 1);
                    asm volatile("cp.async.wait_group 1;\n" ::);
                } else {
                    asm volatile("cp.async.wait_group 0;\n" ::);
                }
                __syncthreads();
                const float* ph = phs + (t & 1) * KT * P * 32;
                const float* cb = cs + (t & 1) * KT * MOC + w * MPT;
                float part[P][MPT];
#pragma unroll
                for (int c = 0; c < P; ++c)
#pragma unroll
                    for (int tt = 0; tt < MPT; ++tt) part[c][tt] = 0.f;
#pragma unroll 4
                for (int kk = 0; kk < KT; ++kk) {
                    float phi[P];
#pragma unroll
                    for (int c = 0; c < P; ++c) phi[c] = ph[(kk * P + c) * 32 + lane];
                    float cv[MPT];
#pragma unroll
                    for (int t4 = 0; t4 < MPT / 4; ++t4) {
                        const float4 v = reinterpret_cast<const float4*>(cb + kk * MOC)[t4];
                        cv[4 * t4] = v.x;
                        cv[4 * t4 + 1] = v.y;
                        cv[4 * t4 + 2] = v.z;
                        cv[4 * t4 + 3] = v.w;
                    }
#pragma unroll
                    for (int c = 0; c < P; ++c)
#pragma unroll
                        for (int tt = 0; tt < MPT; ++tt) part[c][tt] = fmaf(phi[c], cv[tt], part[c][tt]);
                }
#pragma unroll
                for (int c = 0; c < P; ++c)
#pragma unroll
                    for (int tt = 0; tt < MPT; ++tt) acc[c][tt] += (double)part[c][tt];
                __syncthreads();
            }
            fold<P, MPT>(acc, q);
        }
#pragma unroll
        for (int i = 0; i < Q; ++i) red[(w * Q + i) * 32 + lane] = q[i];
        __syncthreads();
        for (int i = tid; i < Q * 32; i += 256) {
            const int qi = i / 32, l = i % 32;
            double s = red[qi * 32 + l];
#pragma unroll
            for (int ww = 1; ww < 8; ++ww) s += red[(ww * Q + qi) * 32 + l];
            fin[(ci * Q + qi) * 32 + l] = s;
        }
        __syncthreads();
    }
    if (w != 0 || j0 + lane >= b) return;
    double f[Q];
    DevDD alpha, beta, comp[4];
    dd_zero(alpha);
    dd_zero(beta);
    for (int ci = 0; ci < prm.nchannels; ++ci) {
        for (int i = 0; i < Q; ++i) f[i] = fin[(ci * Q + i) * 32 + lane];
        record<P>(f, prm.ao_order, prm.ch[ci].role == 1 ? alpha : beta);
    }
    if (prm.beta_is_alpha) beta = alpha;
    const bool full = P == 10 && prm.ao_order == 2;
    comp[1] = alpha;
    comp[2] = beta;
    comp[0] = dd_combine(alpha, beta, 1.0, 1.0, full);
    comp[3] = dd_combine(alpha, beta, -1.0, 1.0, full);
    store_point(prm.spec, comp, start + j0 + lane);
}

template <int P, int MPT, int KT>
void launch(const ContractMixedParams& p, cudaStream_t stream) {
    constexpr int MOC = 8 * MPT;
    constexpr int Q = NQm<P>::v;
    const size_t smem = sizeof(float) * (size_t)(2 * KT * P * 32 + 2 * KT * MOC) + sizeof(double) * (size_t)(8 * Q * 32 + 2 * Q * 32);
    cudaFuncSetAttribute(contract_mixed_kernel<P, MPT, KT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    contract_mixed_kernel<P, MPT, KT><<<p.nblocks * 4, 256, smem, stream>>>(p);
}

}  // namespace

void launch_contract_mixed(const ContractMixedParams& p, int npanel, cudaStream_t stream) {
    switch (npanel) {
        case 1: launch<1, 16, 16>(p, stream); break;
        case 4: launch<4, 16, 16>(p, stream); break;
        case 5: launch<5, 16, 16>(p, stream); break;
        case 10: launch<10, 8, 16>(p, stream); break;
        default: break;
    }
}

}  // namespace kumo_dev
