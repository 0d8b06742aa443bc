// Mixed-precision AO-MO contraction on the tcgen05 tensor cores.
//
// One CTA (8 warps) per 128-point screening block computes, for every AO
// panel c and occupied MO i, X_c[point][i] = sum_k phi_c[k][point] C[k][i]
// over the block's kept AO rows k, as an M=128 (points) x N (MOs) x K (AOs)
// product per panel with the accumulators in tensor memory (column c*N + i,
// lane = point).  Each FP32 AO value a and each coefficient b is written as
// three BF16 pieces (a = a0 + a1 + a2 exactly, each piece the BF16 rounding
// of what the previous ones leave); the six products a_i b_j with i + j <= 2
// give the product to about 2^-24 relative, the same as one FP32 product.
//
// Pipeline per K step of 16 AO rows: all threads load the FP32 panel rows,
// split them into the three pieces and store them in shared memory in the
// MN-major no-swizzle core-matrix layout (8 points x 8 AO rows of 16 bytes);
// the coefficient pieces (split once at upload) are gathered by cp.async;
// one thread issues the 6 x npanel MMAs and commits them to the stage's
// mbarrier.  Stages are reused once that mbarrier reports the MMAs done, so
// the loads and splits of step t+1 overlap the MMAs of step t.  After the
// last step the 8 warps read the accumulators (tcgen05.ld, 32 lanes per warp,
// warps w and w+4 sharing lanes and splitting the MOs), fold them into the
// per-point FP64 sums of src/density.cpp:275-325 and the fields are stored.
//
// Every wait on an mbarrier is bounded; a wait that runs out sets *status,
// stores NaN for the block's points, and the CTA waits (bounded again) for
// its MMAs before it frees tensor memory and returns.
#include "func_attr.cuh"
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <stdexcept>
#include <string>

#include "ao_mixed_shell.cuh"
#include "mixed.cuh"
#include "tc_common.cuh"

namespace kumo_dev {
namespace {

// Threads that issue a step's MMAs (the first lane of each of the first
// kIssuers warps, panels dealt round-robin), and the arrivals on a stage's
// barrier.
template <int P>
constexpr int kIssuers = P < 8 ? P : 8;

template <int P>
struct NQm {
    static constexpr int v = P == 1 ? 1 : P == 4 ? 7 : P == 5 ? 8 : 19;
};

// Per-point sums over MOs of products of panel values (the order of
// src/density.cpp:292-318): q0 = sum X0^2, q[1+a] = sum X0 Xa, q[4+a] = sum
// Xa^2, then X0 Xlap (P = 5) or X0 H_h and the gradient products (P = 10).
template <int P, int MG>
__device__ __forceinline__ void fold(const double (&xs)[P][MG], double (&q)[NQm<P>::v], int nvalid) {
#pragma unroll
    for (int t = 0; t < MG; ++t) {
        if (t >= nvalid) break;
        double x[P];
#pragma unroll
        for (int c = 0; c < P; ++c) x[c] = xs[c][t];
        q[0] += x[0] * x[0];
        if constexpr (P >= 4) {
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                q[1 + a] += x[0] * x[1 + a];
                q[4 + a] += x[1 + a] * x[1 + a];
            }
        }
        if constexpr (P == 5) q[7] += x[0] * x[4];
        if constexpr (P == 10) {
            constexpr int pa[6] = {0, 0, 0, 1, 1, 2}, pc[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
            for (int h = 0; h < 6; ++h) {
                q[7 + h] += x[0] * x[4 + h];
                q[13 + h] += x[1 + pa[h]] * x[1 + pc[h]];
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

// Shared memory of one CTA: S stages of AO pieces, SB = S + 1 stages of
// coefficient pieces (fetched two K steps ahead), the cross-warp sums, the
// row order and the AO index of each K row in that order.
template <int P, int S>
struct Smem {
    static constexpr int Q = NQm<P>::v;
    static constexpr int SB = S + 1;
    static constexpr unsigned a_bytes = 3u * P * kATile;  // one stage of A pieces
    __host__ __device__ static unsigned b_bytes(int ncols) { return 3u * 32u * static_cast<unsigned>(ncols); }
    static size_t total(int ncols) {
        return S * static_cast<size_t>(a_bytes) + SB * static_cast<size_t>(b_bytes(ncols)) +
               sizeof(double) * Q * 128 + (sizeof(int) + 1 + sizeof(std::uint16_t)) * kSortCap +
               sizeof(int) * (kBuckets + 4) + 16 * S + 16;
    }
};

// With two or more AO stages the CTA has a ninth warp that only issues the
// MMAs: the eight producer warps split the AO rows and fetch coefficients and
// arrive (without waiting) on the stage's "full" mbarrier; the MMA warp waits
// on it, issues the step's MMAs and commits them to the stage's "empty"
// mbarrier, which the producers wait on before they reuse the stage.  The MMA
// issue, which waits while the tensor pipe is full, is off the producers'
// path, and every wait is bounded.
template <int S>
constexpr bool kMmaWarp = S >= 2;
template <int S>
constexpr int kCtaThreads = kMmaWarp<S> ? kThreads + 32 : kThreads;

template <int P, int S>
__global__ void __launch_bounds__(kCtaThreads<S>, 1) contract_mixed_kernel(const __grid_constant__ ContractMixedParams prm) {
    using L = Smem<P, S>;
    constexpr int Q = L::Q;
    constexpr int SB = L::SB;
    extern __shared__ __align__(1024) unsigned char sm[];
    const int N = prm.ncols;
    const unsigned b_bytes = L::b_bytes(N);
    unsigned char* a_st = sm;
    unsigned char* b_st = sm + S * L::a_bytes;
    double* red = reinterpret_cast<double*>(b_st + SB * b_bytes);
    int* perm = reinterpret_cast<int*>(red + Q * 128);
    int* bucket_start = perm + kSortCap;
    std::uint16_t* aoidx = reinterpret_cast<std::uint16_t*>(bucket_start + kBuckets + 4);
    unsigned char* keys = reinterpret_cast<unsigned char*>(aoidx + kSortCap);
    unsigned long long* bar = reinterpret_cast<unsigned long long*>(keys + kSortCap);  // empty: MMAs done
    unsigned long long* full = bar + S;                                                // full: stage written
    unsigned* tslot = reinterpret_cast<unsigned*>(full + S);

    const int blk = blockIdx.x;
    const long long start = prm.first_point + static_cast<long long>(blk) * prm.block_size;
    long long bcount = prm.count - start;
    if (bcount > prm.block_size) bcount = prm.block_size;
    const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
    const AoScratch<float>& scr = prm.scr;
    int nk = scr.nkept[blk];
    const float* pbase = scr.panels + static_cast<size_t>(blk) * P * scr.row_stride * kBlockPoints;
    const int* kept = scr.kept + static_cast<size_t>(blk) * scr.row_stride;

    constexpr bool kSpec = kMmaWarp<S>;
    const bool producer = !kSpec || tid < kThreads;
    if (tid == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(&bar[s], kSpec ? 1 : kIssuers<P>);
            mbar_init(&full[s], kThreads);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (w == 0) tmem_alloc(tslot, static_cast<unsigned>(prm.tmem_cols));
    // K order: rows in ascending order of their block maximum (a stable
    // counting sort on the FP32 exponent), so that the accumulators are small
    // while most rows are added and the largest terms come last.
    bool sorted = false;
    nk = block_row_order(scr.rowmax ? scr.rowmax + static_cast<size_t>(blk) * scr.row_stride * 4 : nullptr, nk,
                         prm.threshold, perm, bucket_start, keys, sorted);
    // The rows kept above the threshold (read back by the profiler).
    if (threadIdx.x == 0) scr.nkept[blk] = nk;
    // AO index of each K row, in K order, so that the coefficient gathers
    // need no dependent global load (blocks of up to kSortCap rows and
    // bases below 65536 functions; others read the kept list).
    const bool have_idx = nk <= kSortCap && scr.row_stride <= 65535;
    if (have_idx)
        for (int k = tid; producer && k < nk; k += kThreads) aoidx[k] = static_cast<std::uint16_t>(kept[sorted ? perm[k] : k]);
    // The last nx rows of the K order (largest block maxima) are added in FP64
    // in the epilogue, as in contract_bulk_kernel; at most what the idle
    // stages hold (AO values: S * 3 * P * 4096 bytes = 24 * S rows of P * 512;
    // coefficients: (S + 1) * 96 * N bytes = 12 * (S + 1) rows of N doubles),
    // and only when the rows are in K order with their AO indices at hand.
    constexpr int kExactCap = 24 * S < 12 * SB ? 24 * S : 12 * SB;
    int nx = (sorted && have_idx) ? (prm.exact_rows < nk ? prm.exact_rows : nk) : 0;
    if (nx > kExactCap) nx = kExactCap;
    const int nkt = nk - nx;
    const int ntiles = (nkt + 15) / 16;
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const unsigned tmem = *tslot;
    const int G = prm.groups;
    const unsigned gcols = static_cast<unsigned>(P * N);  // columns of one accumulator group

    // This thread's A unit: AO row kh*8 + k8 of each K step, points 8g..8g+7.
    const int k8 = tid & 7, g = (tid >> 3) & 15, kh = tid >> 7;
    const unsigned a_off = static_cast<unsigned>(g * 128 + kh * 2048 + k8 * 16);
    const unsigned idesc = instr_desc(N);
    // Descriptors of stage 0, piece 0, panel 0; the start-address field (in
    // 16-byte units) is advanced by plain addition.
    const unsigned long long a_desc0 = smem_desc(smem_u32(a_st), 2048u, 128u);
    const unsigned long long b_desc0 = smem_desc(smem_u32(b_st), static_cast<unsigned>(N * 16), 128u);
    // Gather of the coefficient chunks: chunk v = ((piece * 2 + rh) * N/8 + ng) * 8 + r8;
    // division by N/8 (< 64) as a multiply-shift, exact for v / 8 < 2^10.
    const unsigned nb8 = static_cast<unsigned>(N / 8);
    const unsigned nb8_mul = (65536u + nb8 - 1u) / nb8;
    const int quarter = w & 3, half = w >> 2;
    const int point = quarter * 32 + lane;

    bool failed = false;
    long long gtile = 0;  // K steps issued so far (all passes)
    DevDD chan_dd[2];
    dd_zero(chan_dd[0]);
    dd_zero(chan_dd[1]);

    for (int ci = 0; ci < prm.nchannels && !failed; ++ci) {
        const MoChannelTC ch = prm.ch[ci];
        double q[Q];
#pragma unroll
        for (int i = 0; i < Q; ++i) q[i] = 0.0;
        for (int n0 = 0; n0 < ch.nocc && !failed; n0 += N) {
            float4 ra[P][2];
            auto load_a = [&](int t) {
                const int k = t * 16 + kh * 8 + k8;
                const bool ok = k < nkt;
                const int row = ok ? (sorted ? perm[k] : k) : 0;
#pragma unroll
                for (int c = 0; c < P; ++c) {
                    if (ok) {
                        const float4* src = reinterpret_cast<const float4*>(
                            pbase + (static_cast<size_t>(c) * scr.row_stride + row) * kBlockPoints + g * 8);
                        ra[c][0] = __ldcs(src);
                        ra[c][1] = __ldcs(src + 1);
                    } else {
                        ra[c][0] = ra[c][1] = make_float4(0.f, 0.f, 0.f, 0.f);
                    }
                }
            };
            // Coefficient pieces of step t into stage `stage`: 3 pieces x 16 rows x
            // N/8 chunks of 16 B, one cp.async group.
            auto load_b = [&](int t, int stage) {
                const unsigned bst = smem_u32(b_st + stage * b_bytes);
                const int nchunk = 3 * 16 * (N / 8);
                for (int v = tid; v < nchunk; v += kThreads) {
                    const int r8 = v & 7;
                    const unsigned rest = static_cast<unsigned>(v) >> 3;
                    const unsigned rest2 = (rest * nb8_mul) >> 16;
                    const int ng = static_cast<int>(rest - rest2 * nb8);
                    const int rh = static_cast<int>(rest2 & 1u), piece = static_cast<int>(rest2 >> 1);
                    const int k = t * 16 + rh * 8 + r8;
                    const int col = n0 + ng * 8;
                    const bool ok = k < nkt && col < ch.ldn;
                    const int ao = ok ? (have_idx ? static_cast<int>(aoidx[k]) : kept[sorted ? perm[k] : k]) : 0;
                    const std::uint16_t* src =
                        ch.cs + (ok ? piece * ch.piece_stride + static_cast<long long>(ao) * ch.ldn + col : 0);
                    cp_async16(bst + static_cast<unsigned>(piece * 32 * N + ng * 128 + rh * (N * 16) + r8 * 16), src,
                               ok);
                }
                asm volatile("cp.async.commit_group;" ::: "memory");
            };
            // Step t+1's AO stage is released by the MMAs of step t+1-S, which
            // are waited for at the end of step t.  Coefficient pieces run two
            // steps ahead in SB = S + 1 stages: step t+2's stage was last read
            // by the MMAs of step t+2-SB = t+1-S, complete by then too.
            if (ntiles > 0 && producer) {
                load_a(0);
                load_b(0, static_cast<int>(gtile % SB));
                if (ntiles > 1) load_b(1, static_cast<int>((gtile + 1) % SB));
            }
            const unsigned bpiece = (32u * static_cast<unsigned>(N)) >> 4;
            // The six MMAs of panel c of K step t (stage s, coefficient stage sb).
            auto issue_panel = [&](int t, int s, int sb, int c) {
                const unsigned long long as = a_desc0 + ((static_cast<unsigned>(s) * L::a_bytes) >> 4);
                const unsigned long long bs = b_desc0 + ((static_cast<unsigned>(sb) * b_bytes) >> 4);
                // K steps go round-robin to G accumulator groups.
                const unsigned dg = tmem + static_cast<unsigned>(t % G) * gcols;
#pragma unroll
                for (int e = 0; e < 6; ++e) {
                    const unsigned long long ad = as + static_cast<unsigned>(((piece_a(e) * P + c) * kATile) >> 4);
                    const unsigned long long bd = bs + static_cast<unsigned>(piece_b(e)) * bpiece;
                    tc_mma(dg + static_cast<unsigned>(c * N), ad, bd, idesc, (t >= G || e > 0) ? 1u : 0u);
                }
            };
            for (int t = 0; t < ntiles; ++t, ++gtile) {
                const int s = static_cast<int>(gtile % S);
                const int sb = static_cast<int>(gtile % SB);
                if constexpr (kSpec) {
                    if (!producer) {
                        // Stage s holds step t once all producers arrived on
                        // full[s] for its (gtile / S)-th use.
                        if (lane == 0) {
                            if (!mbar_wait(&full[s], static_cast<unsigned>((gtile / S) & 1), prm.wait_ns)) failed = true;
                            tc_fence_after();
#pragma unroll
                            for (int c = 0; c < P; ++c) issue_panel(t, s, sb, c);
                            tc_commit(&bar[s]);
                        }
                        __syncwarp();
                        continue;
                    }
                    unsigned char* ast = a_st + s * L::a_bytes;
#pragma unroll
                    for (int c = 0; c < P; ++c) {
                        uint4 p0, p1, p2;
                        split8(ra[c][0], ra[c][1], p0, p1, p2);
                        *reinterpret_cast<uint4*>(ast + (0 * P + c) * kATile + a_off) = p0;
                        *reinterpret_cast<uint4*>(ast + (1 * P + c) * kATile + a_off) = p1;
                        *reinterpret_cast<uint4*>(ast + (2 * P + c) * kATile + a_off) = p2;
                    }
                    if (t + 1 < ntiles) load_a(t + 1);
                    if (t + 1 < ntiles)
                        asm volatile("cp.async.wait_group 1;" ::: "memory");
                    else
                        asm volatile("cp.async.wait_group 0;" ::: "memory");
                    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                    mbar_arrive(&full[s]);
                    if (t + 1 < ntiles) {
                        // Step t+1's AO stage and step t+2's coefficient stage
                        // were last read by the MMAs of step t+1-S.
                        const long long wv = gtile + 1 - S;
                        if (wv >= 0 && !mbar_wait(&bar[wv % S], static_cast<unsigned>((wv / S) & 1), prm.wait_ns)) failed = true;
                        if (t + 2 < ntiles) load_b(t + 2, static_cast<int>((gtile + 2) % SB));
                    }
                    continue;
                }
                // One AO stage: all warps split, then the first lanes of
                // kIssuers<P> warps issue the panels' MMAs.
                unsigned char* ast = a_st + s * L::a_bytes;
#pragma unroll
                for (int c = 0; c < P; ++c) {
                    uint4 p0, p1, p2;
                    split8(ra[c][0], ra[c][1], p0, p1, p2);
                    *reinterpret_cast<uint4*>(ast + (0 * P + c) * kATile + a_off) = p0;
                    *reinterpret_cast<uint4*>(ast + (1 * P + c) * kATile + a_off) = p1;
                    *reinterpret_cast<uint4*>(ast + (2 * P + c) * kATile + a_off) = p2;
                }
                if (t + 1 < ntiles) load_a(t + 1);
                if (t + 1 < ntiles)
                    asm volatile("cp.async.wait_group 1;" ::: "memory");
                else
                    asm volatile("cp.async.wait_group 0;" ::: "memory");
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                if (__syncthreads_or(failed)) {
                    failed = true;
                    break;
                }
                if (lane == 0 && w < kIssuers<P>) {
                    tc_fence_after();
                    for (int c = w; c < P; c += kIssuers<P>) issue_panel(t, s, sb, c);
                    tc_commit(&bar[s]);
                }
                if (t + 1 < ntiles) {
                    const long long wv = gtile + 1 - S;
                    if (wv >= 0 && !mbar_wait(&bar[wv % S], static_cast<unsigned>((wv / S) & 1), prm.wait_ns)) failed = true;
                    if (t + 2 < ntiles) load_b(t + 2, static_cast<int>((gtile + 2) % SB));
                }
            }
            if (ntiles == 0 && nx == 0) continue;
            if constexpr (kSpec) {
                // Producers' timeouts become every thread's before the pass ends.
                if (__syncthreads_or(failed)) {
                    failed = true;
                    break;
                }
            } else if (failed) {
                continue;
            }
            // Accumulators of this pass complete once the last step's commit arrives.
            const long long last = gtile - 1;
            if (ntiles > 0 && !mbar_wait(&bar[last % S], static_cast<unsigned>((last / S) & 1), prm.wait_ns)) failed = true;
            if (__syncthreads_or(failed)) {
                failed = true;
                break;
            }
            tc_fence_after();
            // Stage the exact rows in the stages no MMA reads any more: AO
            // values [row][panel][point] (FP32) and this pass's coefficient
            // columns [row][column] (FP64, zero past the padded row).
            float* xs_phi = reinterpret_cast<float*>(a_st);
            double* xs_c = reinterpret_cast<double*>(b_st);
            if (nx > 0) {
                for (int v = tid; v < nx * P * 32; v += static_cast<int>(blockDim.x)) {
                    const int r = v / (P * 32), rem = v - r * (P * 32), c = rem >> 5, q4 = rem & 31;
                    const int slot = perm[nkt + r];
                    const float4 f = *reinterpret_cast<const float4*>(
                        pbase + (static_cast<size_t>(c) * scr.row_stride + slot) * kBlockPoints + q4 * 4);
                    *reinterpret_cast<float4*>(xs_phi + (r * P + c) * kBlockPoints + q4 * 4) = f;
                }
                const int half_n = N / 2;
                for (int v = tid; v < nx * half_n; v += static_cast<int>(blockDim.x)) {
                    const int r = v / half_n, j = v - r * half_n;
                    const int col = n0 + 2 * j;
                    double2 cv = make_double2(0.0, 0.0);
                    if (col < ch.ld64)
                        cv = *reinterpret_cast<const double2*>(ch.c64 + static_cast<long long>(aoidx[nkt + r]) * ch.ld64 + col);
                    *reinterpret_cast<double2*>(xs_c + r * N + 2 * j) = cv;
                }
                __syncthreads();
            }
            const int nvalid = ch.nocc - n0 < N ? ch.nocc - n0 : N;
            const int i_lo = half * (N / 2), i_hi = min(nvalid, (half + 1) * (N / 2));
            const unsigned lane_addr = tmem + (static_cast<unsigned>(quarter * 32) << 16);
            const int ng = ntiles < G ? ntiles : G;
            constexpr int MG = 4;
            for (int i0 = i_lo; i0 < i_hi; i0 += MG) {
                // tcgen05.ld is warp-collective: the trip count depends on the
                // half only; columns past the last MO are read and ignored.
                double x[P][MG];
#pragma unroll
                for (int c = 0; c < P; ++c)
#pragma unroll
                    for (int u = 0; u < MG; ++u) x[c][u] = 0.0;
                for (int gi = 0; gi < ng; ++gi) {
                    unsigned v[P][MG];
#pragma unroll
                    for (int c = 0; c < P; ++c)
                        tmem_ld<MG>(lane_addr + static_cast<unsigned>(gi) * gcols + static_cast<unsigned>(c * N + i0), v[c]);
                    tmem_wait_ld();
#pragma unroll
                    for (int c = 0; c < P; ++c) {
                        reg_fence<MG>(v[c]);
#pragma unroll
                        for (int u = 0; u < MG; ++u) x[c][u] += static_cast<double>(__uint_as_float(v[c][u]));
                    }
                }
                // The exact rows, from the staged copies, in FP64.
                for (int r = 0; r < nx; ++r) {
                    const double* crow = xs_c + r * N + i0;
                    double cv[MG];
#pragma unroll
                    for (int u = 0; u < MG; ++u) cv[u] = crow[u];
#pragma unroll
                    for (int c = 0; c < P; ++c) {
                        const double f = static_cast<double>(xs_phi[(r * P + c) * kBlockPoints + point]);
#pragma unroll
                        for (int u = 0; u < MG; ++u) x[c][u] += f * cv[u];
                    }
                }
                fold<P, MG>(x, q, i_hi - i0);
            }
            tc_fence_before();
            __syncthreads();
        }
        if (failed) break;
        // Sum the two halves' partial sums of this channel.
        if (half == 1)
#pragma unroll
            for (int i = 0; i < Q; ++i) red[i * 128 + point] = q[i];
        __syncthreads();
        if (half == 0) {
#pragma unroll
            for (int i = 0; i < Q; ++i) q[i] += red[i * 128 + point];
            record<P>(q, prm.ao_order, ch.role == 1 ? chan_dd[0] : chan_dd[1]);
        }
        __syncthreads();
    }

    if (failed) {
        asm volatile("cp.async.wait_group 0;" ::: "memory");  // no copy in flight at exit
        if (tid == 0) atomicOr(prm.status, 1u);
        // Let the MMAs already issued finish before tensor memory is freed.
        for (int s = 0; s < S; ++s) {
            const long long last = gtile - 1 - ((gtile - 1 - s) % S + S) % S;
            if (last >= 0) (void)mbar_wait(&bar[last % S], static_cast<unsigned>((last / S) & 1));
        }
    }
    tc_fence_before();
    __syncthreads();
    if (w == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, static_cast<unsigned>(prm.tmem_cols));
    }
    if (half != 0 || point >= bcount) return;
    DevDD comp[4];
    if (failed) {
        const double nan = __longlong_as_double(0x7ff8000000000000ll);
        DevDD d;
        d.value = d.lap = d.tau = nan;
        for (int i = 0; i < 3; ++i) d.grad[i] = d.tau_axes[i] = nan;
        for (int i = 0; i < 6; ++i) d.hess[i] = nan;
        comp[0] = comp[1] = comp[2] = comp[3] = d;
    } else {
        DevDD alpha = chan_dd[0], beta = chan_dd[1];
        if (prm.beta_is_alpha) beta = alpha;
        const bool full = P == 10 && prm.ao_order == 2;
        comp[1] = alpha;
        comp[2] = beta;
        comp[0] = dd_combine(alpha, beta, 1.0, 1.0, full);
        comp[3] = dd_combine(alpha, beta, -1.0, 1.0, full);
    }
    store_point(prm.spec, comp, start + point);
}

// ---------------------------------------------------------------------------
// FP64 AO rows of the exact rows (the largest rows of a block, added in FP64
// in the epilogue of the bulk-copy kernel).

__device__ __forceinline__ double ipow(double x, int n) {
    double r = 1.0;
    for (int i = 0; i < n; ++i) r *= x;
    return r;
}

// FP64 normalisation tables of the exact rows (the same for every basis;
// upload_exact_tables copies them once per device): g_k of each Cartesian
// component in Gaussian order, 1/g of the first component of each order, and
// T[m][k] g_k of the Cartesian-to-pure transforms of l = 2..4 (row-major m, k).
__constant__ double c_exact_g[kMaxL + 1][15];
__constant__ double c_exact_ig0[kMaxL + 1];
__constant__ double c_exact_tg[3][135];

// Radial sums of the factorised weights W[k][p] = u_p g_k at squared distance
// r2: S_n = sum_p u_p a_p^n exp(-a_p r2), n = 0, 1, 2, with u_p = W[0][p] / g_0
// (one FP64 exponential per primitive for all components of the shell).
__device__ __forceinline__ void exact_radial(const DevBasis& B, int4 inf, int l, double r2, double& S0, double& S1,
                                             double& S2) {
    const int nprim = inf.x >> 16;
    const double* W0 = B.weights + inf.z;
    const double* A = B.exps + inf.y;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
#pragma unroll 4
    for (int q = 0; q < nprim; ++q) {
        const double a = A[q];
        const double we = W0[q] * exp(-a * r2);
        s0 += we;
        s1 += we * a;
        s2 += we * (a * a);
    }
    const double ig0 = c_exact_ig0[l];
    S0 = s0 * ig0;
    S1 = s1 * ig0;
    S2 = s2 * ig0;
}

// FP64 AO values of the exact rows of one AO block (shell) s at one point,
// offset (dx, dy, dz) from the shell's centre.  With R0 = S_0, R1' = -2 S_1,
// R2' = 4 S_2 and the polynomial P_m = sum_k T[m][k] g_k M_k of output m (M_k
// the monomial of Cartesian component k; T the identity for Cartesian
// shells): value P_m R0, d/dx_i dP_m/dx_i R0 + x_i P_m R1', Laplacian
// lap(P_m) R0 + P_m ((2L+3) R1' + r^2 R2') (lap(P_m) = 0 for solid
// harmonics) -- the functions of the reference's evaluate_derivatives_batch
// (src/basis_evaluator.cpp:512-643), rounded differently; zero beyond the
// shell's cutoff radius, as there.  Bit m of `mask` marks an exact output m;
// its staging row is slots[number of mask bits below m].  Values for P = 1
// (value), 4 (+ gradient) or 5 (+ Laplacian) go to out[(row * P + c) * ld +
// col].  The zero entries of the pure transforms are skipped at compile time.
template <int L, bool PURE, int P>
__device__ void exact_shell(const DevBasis& B, double4 o, int4 inf, double dx, double dy, double dz, unsigned mask,
                            const int* slots, double* out, int ld, int col) {
    constexpr int NC = (L + 1) * (L + 2) / 2;
    constexpr int NOUT = PURE ? 2 * L + 1 : NC;
    const double r2 = dx * dx + dy * dy + dz * dz;
    auto row_of = [&](int m) { return slots[__popc(mask & ((1u << m) - 1u))]; };
    if (r2 > o.w) {
        static_for<NOUT>([&](auto mc) {
            constexpr int m = decltype(mc)::value;
            if ((mask >> m) & 1u) {
                const int r = row_of(m);
#pragma unroll
                for (int c = 0; c < P; ++c) out[(r * P + c) * ld + col] = 0.0;
            }
        });
        return;
    }
    double S0, S1, S2;
    exact_radial(B, inf, L, r2, S0, S1, S2);
    const double R1p = -2.0 * S1, R2p = 4.0 * S2;
    const double qf = (2.0 * L + 3.0) * R1p + r2 * R2p;
    double xp[L + 1], yp[L + 1], zp[L + 1];
    xp[0] = yp[0] = zp[0] = 1.0;
#pragma unroll
    for (int n = 1; n <= L; ++n) {
        xp[n] = xp[n - 1] * dx;
        yp[n] = yp[n - 1] * dy;
        zp[n] = zp[n - 1] * dz;
    }
    const double d[3] = {dx, dy, dz};
    if constexpr (PURE) {
        double pm[NOUT], pg[3][NOUT];
#pragma unroll
        for (int m = 0; m < NOUT; ++m) pm[m] = pg[0][m] = pg[1][m] = pg[2][m] = 0.0;
        static_for<NC>([&](auto kc) {
            constexpr int k = decltype(kc)::value;
            constexpr int a = cart_power(L, k, 0), b = cart_power(L, k, 1), c = cart_power(L, k, 2);
            const double M = xp[a] * yp[b] * zp[c];
            [[maybe_unused]] double Mi[3] = {0.0, 0.0, 0.0};
            if constexpr (P >= 4) {
                if constexpr (a > 0) Mi[0] = a * xp[a > 0 ? a - 1 : 0] * yp[b] * zp[c];
                if constexpr (b > 0) Mi[1] = b * xp[a] * yp[b > 0 ? b - 1 : 0] * zp[c];
                if constexpr (c > 0) Mi[2] = c * xp[a] * yp[b] * zp[c > 0 ? c - 1 : 0];
            }
            static_for<NOUT>([&](auto mc) {
                constexpr int m = decltype(mc)::value;
                if constexpr (solid_harmonic_nonzero(L, m, a, b)) {
                    const double t = c_exact_tg[L - 2][m * NC + k];
                    pm[m] += t * M;
                    if constexpr (P >= 4)
#pragma unroll
                        for (int i = 0; i < 3; ++i) pg[i][m] += t * Mi[i];
                }
            });
        });
        static_for<NOUT>([&](auto mc) {
            constexpr int m = decltype(mc)::value;
            if ((mask >> m) & 1u) {
                double* dst = out + static_cast<long long>(row_of(m)) * P * ld + col;
                dst[0] = pm[m] * S0;
                if constexpr (P >= 4)
#pragma unroll
                    for (int i = 0; i < 3; ++i) dst[(1 + i) * ld] = pg[i][m] * S0 + d[i] * pm[m] * R1p;
                if constexpr (P == 5) dst[4 * ld] = pm[m] * qf;
            }
        });
    } else {
        static_for<NC>([&](auto kc) {
            constexpr int k = decltype(kc)::value;
            if ((mask >> k) & 1u) {
                constexpr int a = cart_power(L, k, 0), b = cart_power(L, k, 1), c = cart_power(L, k, 2);
                const double g = c_exact_g[L][k];
                const double M = g * (xp[a] * yp[b] * zp[c]);
                double* dst = out + static_cast<long long>(row_of(k)) * P * ld + col;
                dst[0] = M * S0;
                if constexpr (P >= 4) {
                    const double mx = a > 0 ? g * (a * xp[a > 0 ? a - 1 : 0] * yp[b] * zp[c]) : 0.0;
                    const double my = b > 0 ? g * (b * xp[a] * yp[b > 0 ? b - 1 : 0] * zp[c]) : 0.0;
                    const double mz = c > 0 ? g * (c * xp[a] * yp[b] * zp[c > 0 ? c - 1 : 0]) : 0.0;
                    dst[ld] = mx * S0 + dx * M * R1p;
                    dst[2 * ld] = my * S0 + dy * M * R1p;
                    dst[3 * ld] = mz * S0 + dz * M * R1p;
                }
                if constexpr (P == 5) {
                    const double lap = (a > 1 ? a * (a - 1) * xp[a > 1 ? a - 2 : 0] * yp[b] * zp[c] : 0.0) +
                                       (b > 1 ? b * (b - 1) * xp[a] * yp[b > 1 ? b - 2 : 0] * zp[c] : 0.0) +
                                       (c > 1 ? c * (c - 1) * xp[a] * yp[b] * zp[c > 1 ? c - 2 : 0] : 0.0);
                    dst[4 * ld] = g * lap * S0 + M * qf;
                }
            }
        });
    }
}

// The same with runtime loops over components and outputs (the radial sums
// still formed once): g shells, whose templated form would not fit the
// registers.
template <int P>
__device__ void exact_shell_loops(const DevBasis& B, double4 o, int4 inf, double dx, double dy, double dz,
                                  unsigned mask, const int* slots, double* out, int ld, int col) {
    const double r2 = dx * dx + dy * dy + dz * dz;
    const int l = inf.x & 0xff;
    const bool is_pure = ((inf.x >> 8) & 1) && l >= 2;
    const int nc = (l + 1) * (l + 2) / 2, nout = is_pure ? 2 * l + 1 : nc;
    const bool inside = !(r2 > o.w);
    double S0 = 0.0, S1 = 0.0, S2 = 0.0;
    if (inside) exact_radial(B, inf, l, r2, S0, S1, S2);
    const double R1p = -2.0 * S1, R2p = 4.0 * S2;
    const double qf = (2.0 * l + 3.0) * R1p + r2 * R2p;
    for (int m = 0; m < nout; ++m) {
        if (!((mask >> m) & 1u)) continue;
        double v[P];
#pragma unroll
        for (int c = 0; c < P; ++c) v[c] = 0.0;
        if (inside) {
            double pm = 0.0, pg[3] = {0.0, 0.0, 0.0}, pl = 0.0;
            for (int k = 0; k < nc; ++k) {
                const double t = is_pure ? c_exact_tg[l - 2][m * nc + k] : (k == m ? c_exact_g[l][k] : 0.0);
                if (t == 0.0) continue;
                const int a = cart_power(l, k, 0), b = cart_power(l, k, 1), c = cart_power(l, k, 2);
                const double xa = ipow(dx, a), yb = ipow(dy, b), zc = ipow(dz, c);
                pm += t * (xa * yb * zc);
                if constexpr (P >= 4) {
                    pg[0] += a ? t * (a * ipow(dx, a - 1) * yb * zc) : 0.0;
                    pg[1] += b ? t * (b * xa * ipow(dy, b - 1) * zc) : 0.0;
                    pg[2] += c ? t * (c * xa * yb * ipow(dz, c - 1)) : 0.0;
                }
                if (P == 5 && !is_pure)
                    pl += t * ((a > 1 ? a * (a - 1) * ipow(dx, a - 2) * yb * zc : 0.0) +
                               (b > 1 ? b * (b - 1) * xa * ipow(dy, b - 2) * zc : 0.0) +
                               (c > 1 ? c * (c - 1) * xa * yb * ipow(dz, c - 2) : 0.0));
            }
            v[0] = pm * S0;
            if constexpr (P >= 4) {
                v[1] = pg[0] * S0 + dx * pm * R1p;
                v[2] = pg[1] * S0 + dy * pm * R1p;
                v[3] = pg[2] * S0 + dz * pm * R1p;
            }
            if constexpr (P == 5) v[4] = pl * S0 + pm * qf;
        }
        const int r = slots[__popc(mask & ((1u << m) - 1u))];
#pragma unroll
        for (int c = 0; c < P; ++c) out[(r * P + c) * ld + col] = v[c];
    }
}

template <int P>
__device__ void exact_shell_any(const DevBasis& B, double4 o, int4 inf, double dx, double dy, double dz,
                                unsigned mask, const int* slots, double* out, int ld, int col) {
    const int l = inf.x & 0xff;
    const bool pure_shell = ((inf.x >> 8) & 1) && l >= 2;
    switch (l | (pure_shell ? 16 : 0)) {
#define KUMO_EXACT(LL, PP) \
    case (LL) | ((PP) ? 16 : 0): exact_shell<LL, PP, P>(B, o, inf, dx, dy, dz, mask, slots, out, ld, col); break;
        KUMO_EXACT(0, false) KUMO_EXACT(1, false) KUMO_EXACT(2, false) KUMO_EXACT(3, false)
        KUMO_EXACT(2, true) KUMO_EXACT(3, true)
#undef KUMO_EXACT
        default: exact_shell_loops<P>(B, o, inf, dx, dy, dz, mask, slots, out, ld, col); break;
    }
}

// ---------------------------------------------------------------------------
// Bulk-copy form (P = 1, 4, 5; two AO stages): a tenth warp fetches the FP32
// rows of each K step into shared memory with the tensor-memory-access unit
// (one tiled copy per kept row of a 4-D map [block][panel][row][point] with a
// box of one row's P panels; completion counted in bytes on the stage's
// "loaded" mbarrier) F - 1 steps ahead of the split.  The eight producer warps read
// the rows from shared memory, arrive on the stage's "read" mbarrier, split
// them into the BF16 pieces and fetch the coefficient pieces as above; the
// MMA warp is the same.  No FP32 row occupies registers while it is in
// flight, so the bytes in flight per SM are set by F.  The eight threads of
// a quarter-warp take eight different rows, point groups of four different
// residues mod 4 and both halves of the 32-byte group in turn, so their
// shared-memory reads and stores each fall in eight different bank groups.
constexpr int kBulkThreads = kThreads + 64;  // producers, MMA warp, loader warp
constexpr unsigned kBulkRowBytes = kBlockPoints * 4u;  // one panel row

template <int P>
struct BulkSmem {
    static constexpr int Q = NQm<P>::v;
    static constexpr unsigned a_bytes = 3u * P * kATile;
    static constexpr unsigned f_slot = P * kBulkRowBytes;  // one K row's P panel rows (a copy's box)
    static constexpr unsigned f_bytes = 16u * f_slot;
    static_assert(sizeof(double) * Q * 128 <= 2u * a_bytes, "cross-warp sums must fit in the AO stages");
    __host__ __device__ static unsigned b_bytes(int ncols) { return 3u * 32u * static_cast<unsigned>(ncols); }
    __host__ __device__ static unsigned cap16(int rows) { return (static_cast<unsigned>(rows) + 15u) & ~15u; }
    static size_t total(int ncols, int F, int SB, int rows) {
        return 2 * static_cast<size_t>(a_bytes) + F * static_cast<size_t>(f_bytes) +
               SB * static_cast<size_t>(b_bytes(ncols)) + 4u * cap16(rows) + 8u * (4 + 2 * F) + 16;
    }
    // Row indices held as 16-bit values; the sort keys share the AO stages.
    static bool rows_fit(int rows) {
        return rows <= 65535 && sizeof(int) * (kBuckets + 4) + cap16(rows) <= 2u * a_bytes;
    }
};

template <int P, int F, int SB>
__global__ void __launch_bounds__(kBulkThreads, 1)
    contract_bulk_kernel(const __grid_constant__ ContractMixedParams prm, const __grid_constant__ CUtensorMap rows) {
    using L = BulkSmem<P>;
    constexpr int Q = L::Q;
    constexpr int S = 2;
    extern __shared__ __align__(1024) unsigned char sm[];
    const int N = prm.ncols;
    const unsigned b_bytes = L::b_bytes(N);
    const AoScratch<float>& scr = prm.scr;
    const unsigned cap = L::cap16(scr.row_stride);
    unsigned char* a_st = sm;
    unsigned char* f_st = sm + 2 * L::a_bytes;
    unsigned char* b_st = f_st + F * L::f_bytes;
    // The AO stages double as the sort scratch (prologue) and the cross-warp
    // sums (between passes, when no MMA reads them).
    double* red = reinterpret_cast<double*>(sm);
    int* bucket_start = reinterpret_cast<int*>(sm);
    unsigned char* keys = sm + sizeof(int) * (kBuckets + 4);
    std::uint16_t* perm = reinterpret_cast<std::uint16_t*>(b_st + SB * b_bytes);
    std::uint16_t* aoidx = perm + cap;
    unsigned long long* a_empty = reinterpret_cast<unsigned long long*>(aoidx + cap);  // MMAs of the stage done
    unsigned long long* a_full = a_empty + S;                                          // stage's pieces written
    unsigned long long* f_full = a_full + S;                                           // stage's rows landed
    unsigned long long* f_empty = f_full + F;                                          // stage's rows read
    unsigned* tslot = reinterpret_cast<unsigned*>(f_empty + F);

    const int blk = blockIdx.x;
    const long long start = prm.first_point + static_cast<long long>(blk) * prm.block_size;
    long long bcount = prm.count - start;
    if (bcount > prm.block_size) bcount = prm.block_size;
    const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
    int nk = scr.nkept[blk];
    const int* kept = scr.kept + static_cast<size_t>(blk) * scr.row_stride;
    const bool producer = tid < kThreads;
    const bool mma_warp = w == kThreads / 32;
    const bool loader = w == kThreads / 32 + 1;

    if (tid == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(&a_empty[s], 1);
            mbar_init(&a_full[s], kThreads);
        }
        for (int u = 0; u < F; ++u) {
            mbar_init(&f_full[u], 1);
            mbar_init(&f_empty[u], kThreads);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (w == 0) tmem_alloc(tslot, static_cast<unsigned>(prm.tmem_cols));
    bool sorted = false;
    const int nk_listed = nk;
    nk = block_row_order(scr.rowmax ? scr.rowmax + static_cast<size_t>(blk) * scr.row_stride * 4 : nullptr, nk,
                         prm.threshold, perm, bucket_start, keys, sorted, static_cast<int>(cap));
    // The rows kept above the threshold (read back by the profiler).
    if (threadIdx.x == 0) scr.nkept[blk] = nk;
    // Rows that may be exact: those whose block maximum reaches exact_min
    // (to the sort's power-of-two buckets); a block far from the nuclei, all
    // of whose rows are small, keeps every row on the tensor cores.
    int nbig = nk;
    if (prm.exact_min > 0.0f && sorted) {
        int emin = static_cast<int>((__float_as_uint(prm.exact_min) >> 23) & 0xffu) - 127 + kBuckets / 2;
        emin = emin < 0 ? 0 : (emin >= kBuckets ? kBuckets - 1 : emin);
        int* count = bucket_start + kBuckets + 2;  // spare slot of the sort's bucket array
        if (tid == 0) *count = 0;
        __syncthreads();
        int mine = 0;
        for (int k = tid; k < nk_listed; k += kBulkThreads) mine += (keys[k] != 0xffu && keys[k] >= emin) ? 1 : 0;
        if (mine) atomicAdd(count, mine);
        __syncthreads();
        nbig = *count;
        __syncthreads();
    }
    for (int k = tid; producer && k < nk; k += kThreads) aoidx[k] = static_cast<std::uint16_t>(kept[sorted ? perm[k] : k]);
    // The last nx rows of the K order (the largest block maxima) are added in
    // FP64 in the epilogue instead of on the tensor cores, with AO values
    // computed there in FP64: the truncation of each MMA's FP32 sum is
    // relative to its largest product and FP32 AO values carry 2^-24 relative
    // errors, so taking the largest terms out of both lowers the error of
    // every output.  The epilogue stages them in the idle stages (AO, row and
    // coefficient stages, one contiguous region): the pass's coefficient
    // columns [row][N] and the AO values [row][panel][point] of the points of
    // one phase (128, 64 or 32 points: as many as fit).
    const unsigned xs_bytes = 2u * L::a_bytes + F * L::f_bytes + SB * b_bytes;
    // Per exact row: its coefficients (N doubles), its AO values at the
    // phase's points (P * ph doubles), six ints of row tables and (for at most
    // as many shell groups) a group's centre, table entry and row mask.
    auto xs_need = [&](int rows, int ph) {
        return 8u * static_cast<unsigned>(rows) * (N + P * ph) + 76u * static_cast<unsigned>(rows) + 16u;
    };
    int nx = prm.exact_rows < nbig ? prm.exact_rows : nbig;
    while (nx > 0 && xs_need(nx, 32) > xs_bytes) --nx;
    const int ph_points = xs_need(nx, 128) <= xs_bytes ? 128 : (xs_need(nx, 64) <= xs_bytes ? 64 : 32);
    const int nkt = nk - nx;
    const int ntiles = (nkt + 15) / 16;
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const unsigned tmem = *tslot;
    const int G = prm.groups;
    const unsigned gcols = static_cast<unsigned>(P * N);

    // This thread's A unit: AO row kh*8 + k8 of each K step, points 8g..8g+7,
    // read half hf first.
    const int k8 = tid & 7, jq = (tid >> 3) & 15, kh = (tid >> 7) & 1;
    const int g = 4 * (jq >> 2) + ((k8 + jq) & 3);
    const int hf = (k8 >> 2) & 1;
    const unsigned a_off = static_cast<unsigned>(g * 128 + kh * 2048 + k8 * 16);
    const unsigned f_off = static_cast<unsigned>((kh * 8 + k8) * L::f_slot + g * 32 + hf * 16);
    const unsigned idesc = instr_desc(N);
    const unsigned long long a_desc0 = smem_desc(smem_u32(a_st), 2048u, 128u);
    const unsigned long long b_desc0 = smem_desc(smem_u32(b_st), static_cast<unsigned>(N * 16), 128u);
    const unsigned nb8 = static_cast<unsigned>(N / 8);
    const unsigned nb8_mul = (65536u + nb8 - 1u) / nb8;
    const int quarter = w & 3, half = w >> 2;
    const int point = quarter * 32 + lane;

    bool failed = false;
    long long gtile = 0;  // K steps of this thread's role so far (all passes)
    // Records of the two spin channels (kept in local memory through the
    // passes: in registers they would crowd the K loop's).
    DevDD chan_dd[2];
    dd_zero(chan_dd[0]);
    dd_zero(chan_dd[1]);

    for (int ci = 0; ci < prm.nchannels && !failed; ++ci) {
        const MoChannelTC ch = prm.ch[ci];
        double q[Q];
#pragma unroll
        for (int i = 0; i < Q; ++i) q[i] = 0.0;
        for (int n0 = 0; n0 < ch.nocc && !failed; n0 += N) {
            auto load_b = [&](int t, int stage) {
                const unsigned bst = smem_u32(b_st + stage * b_bytes);
                const int nchunk = 3 * 16 * (N / 8);
                for (int v = tid; v < nchunk; v += kThreads) {
                    const int r8 = v & 7;
                    const unsigned rest = static_cast<unsigned>(v) >> 3;
                    const unsigned rest2 = (rest * nb8_mul) >> 16;
                    const int ng = static_cast<int>(rest - rest2 * nb8);
                    const int rh = static_cast<int>(rest2 & 1u), piece = static_cast<int>(rest2 >> 1);
                    const int k = t * 16 + rh * 8 + r8;
                    const int col = n0 + ng * 8;
                    const bool ok = k < nkt && col < ch.ldn;
                    const int ao = ok ? static_cast<int>(aoidx[k]) : 0;
                    const std::uint16_t* src =
                        ch.cs + (ok ? piece * ch.piece_stride + static_cast<long long>(ao) * ch.ldn + col : 0);
                    cp_async16(bst + static_cast<unsigned>(piece * 32 * N + ng * 128 + rh * (N * 16) + r8 * 16), src,
                               ok);
                }
                asm volatile("cp.async.commit_group;" ::: "memory");
            };
            const unsigned bpiece = (32u * static_cast<unsigned>(N)) >> 4;
            auto issue_panel = [&](int t, int s, int sb, int c) {
                const unsigned long long as = a_desc0 + ((static_cast<unsigned>(s) * L::a_bytes) >> 4);
                const unsigned long long bs = b_desc0 + ((static_cast<unsigned>(sb) * b_bytes) >> 4);
                const unsigned dg = tmem + static_cast<unsigned>(t % G) * gcols;
#pragma unroll
                for (int e = 0; e < 6; ++e) {
                    const unsigned long long ad = as + static_cast<unsigned>(((piece_a(e) * P + c) * kATile) >> 4);
                    const unsigned long long bd = bs + static_cast<unsigned>(piece_b(e)) * bpiece;
                    tc_mma(dg + static_cast<unsigned>(c * N), ad, bd, idesc, (t >= G || e > 0) ? 1u : 0u);
                }
            };
            if (mma_warp) {
                for (int t = 0; t < ntiles; ++t, ++gtile) {
                    const int s = static_cast<int>(gtile % S);
                    const int sb = static_cast<int>(gtile % SB);
                    bool ok = true;
                    if (lane == 0) {
                        ok = mbar_wait(&a_full[s], static_cast<unsigned>((gtile / S) & 1), prm.wait_ns);
                        if (ok) {
                            tc_fence_after();
#pragma unroll
                            for (int c = 0; c < P; ++c) issue_panel(t, s, sb, c);
                            tc_commit(&a_empty[s]);
                        }
                    }
                    if (!__shfl_sync(0xffffffffu, ok ? 1 : 0, 0)) {
                        failed = true;  // gtile = commits issued
                        break;
                    }
                }
            } else if (loader) {
                for (int t = 0; t < ntiles; ++t, ++gtile) {
                    const int u = static_cast<int>(gtile % F);
                    const int nv = nkt - t * 16 < 16 ? nkt - t * 16 : 16;
                    bool ok = true;
                    if (lane == 0) {
                        // The stage's previous rows (step gtile - F) have been read.
                        const long long prev = gtile - F;
                        if (prev >= 0) ok = mbar_wait(&f_empty[u], static_cast<unsigned>((prev / F) & 1), prm.wait_ns);
                        if (ok) mbar_arrive_expect_tx(&f_full[u], static_cast<unsigned>(nv * P) * (kBlockPoints * 4u));
                    }
                    if (!__shfl_sync(0xffffffffu, ok ? 1 : 0, 0)) {
                        failed = true;  // gtile = stages issued
                        break;
                    }
                    if (lane < nv) {
                        const int k = t * 16 + lane;
                        const int row = sorted ? static_cast<int>(perm[k]) : k;
                        tma_load_4d(smem_u32(f_st + u * L::f_bytes + lane * L::f_slot), &rows, 0, row, 0, blk, &f_full[u]);
                    }
                }
            } else {
                if (ntiles > 0) {
                    load_b(0, static_cast<int>(gtile % SB));
                    if (SB > 2 && ntiles > 1) load_b(1, static_cast<int>((gtile + 1) % SB));
                }
                for (int t = 0; t < ntiles; ++t, ++gtile) {
                    const int s = static_cast<int>(gtile % S);
                    const int u = static_cast<int>(gtile % F);
                    // Stage s was released (MMAs of step gtile - S) at the end of
                    // the previous step; wait for this step's rows.
                    if (!mbar_wait(&f_full[u], static_cast<unsigned>((gtile / F) & 1), prm.wait_ns)) {
                        failed = true;
                        break;
                    }
                    const int k = t * 16 + kh * 8 + k8;
                    float4 ra[P][2];
                    if (k < nkt) {
                        const unsigned fs = smem_u32(f_st + u * L::f_bytes);
#pragma unroll
                        for (int c = 0; c < P; ++c) {
                            // Half hf first: the quarter-warp's two loads each touch
                            // eight different bank groups.
                            const float4 x0 = lds128(fs + c * kBulkRowBytes + f_off);
                            const float4 x1 = lds128(fs + c * kBulkRowBytes + (f_off ^ 16u));
                            ra[c][0] = hf ? x1 : x0;
                            ra[c][1] = hf ? x0 : x1;
                        }
                    } else {
#pragma unroll
                        for (int c = 0; c < P; ++c) ra[c][0] = ra[c][1] = make_float4(0.f, 0.f, 0.f, 0.f);
                    }
                    mbar_arrive(&f_empty[u]);
                    unsigned char* ast = a_st + s * L::a_bytes;
#pragma unroll
                    for (int c = 0; c < P; ++c) {
                        uint4 p0, p1, p2;
                        split8(ra[c][0], ra[c][1], p0, p1, p2);
                        *reinterpret_cast<uint4*>(ast + (0 * P + c) * kATile + a_off) = p0;
                        *reinterpret_cast<uint4*>(ast + (1 * P + c) * kATile + a_off) = p1;
                        *reinterpret_cast<uint4*>(ast + (2 * P + c) * kATile + a_off) = p2;
                    }
                    // Coefficient pieces of this step: the groups committed after
                    // it (at most SB - 2) may stay in flight.
                    if (SB > 2 && t + 1 < ntiles)
                        asm volatile("cp.async.wait_group 1;" ::: "memory");
                    else
                        asm volatile("cp.async.wait_group 0;" ::: "memory");
                    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                    mbar_arrive(&a_full[s]);
                    if (t + 1 < ntiles) {
                        // Step t+1's AO stage and step t+SB-1's coefficient stage
                        // were last read by the MMAs of step gtile - 1.
                        const long long wv = gtile + 1 - S;
                        if (wv >= 0 && !mbar_wait(&a_empty[wv % S], static_cast<unsigned>((wv / S) & 1), prm.wait_ns)) {
                            failed = true;
                            break;
                        }
                        if (t + SB - 1 < ntiles) load_b(t + SB - 1, static_cast<int>((gtile + SB - 1) % SB));
                    }
                }
            }
            if (ntiles == 0 && nx == 0) continue;
            // A role's timeout becomes every thread's before the pass ends.
            if (__syncthreads_or(failed)) {
                failed = true;
                break;
            }
            const long long last = gtile - 1;
            if (ntiles > 0 && !mbar_wait(&a_empty[last % S], static_cast<unsigned>((last / S) & 1), prm.wait_ns)) failed = true;
            if (__syncthreads_or(failed)) {
                failed = true;
                break;
            }
            tc_fence_after();
            const int nvalid = ch.nocc - n0 < N ? ch.nocc - n0 : N;
            // Warps 8 and 9 (half 2) read no accumulators.
            const int i_lo = half * (N / 2), i_hi = min(nvalid, (half + 1) * (N / 2));
            const unsigned lane_addr = tmem + (static_cast<unsigned>(quarter * 32) << 16);
            const int ng = ntiles < G ? ntiles : G;
            // Eight MO columns per register block: each exact row's P AO
            // values are read once from shared memory for 8 P FP64 products
            // (with four columns the shared-memory reads, not the FP64 pipe,
            // set the epilogue's rate).
            constexpr int MG = 8;
            double* xs_c = reinterpret_cast<double*>(sm);
            double* xs_phi = xs_c + nx * N;
            // Row tables: shell and component of each exact row, the rows
            // grouped by shell (grp_rows, group j spans grp_first[j] ..
            // grp_first[j + 1]) and the groups' shells.
            // Per group: its shell's centre and table entry, and the mask of
            // its exact components.
            double4* xs_go = reinterpret_cast<double4*>(xs_phi + nx * P * ph_points);
            int4* xs_gi = reinterpret_cast<int4*>(xs_go + nx);
            unsigned* xs_gmask = reinterpret_cast<unsigned*>(xs_gi + nx);
            int* xs_shell = reinterpret_cast<int*>(xs_gmask + nx);
            int* xs_m = xs_shell + nx;
            int* grp_rows = xs_m + nx;
            int* grp_m = grp_rows + nx;
            int* grp_first = grp_m + nx;  // nx + 2 entries; [nx + 1] holds the group count
            if (nx > 0) {
                const int half_n = N / 2;
                for (int v = tid; v < nx * half_n; v += kBulkThreads) {
                    const int r = v / half_n, j = v - r * half_n;
                    const int col = n0 + 2 * j;
                    double2 cv = make_double2(0.0, 0.0);
                    if (col < ch.ld64)
                        cv = *reinterpret_cast<const double2*>(ch.c64 + static_cast<long long>(aoidx[nkt + r]) * ch.ld64 + col);
                    *reinterpret_cast<double2*>(xs_c + r * N + 2 * j) = cv;
                }
                for (int r = tid; r < nx; r += kBulkThreads) {
                    const int bm = prm.basis.ao_block[aoidx[nkt + r]];
                    xs_shell[r] = bm >> 5;
                    xs_m[r] = bm & 31;
                }
                __syncthreads();
                // Rows in (shell, component) order.
                for (int r = tid; r < nx; r += kBulkThreads) {
                    const int sh = xs_shell[r], mr = xs_m[r];
                    int pos = 0;
                    for (int q = 0; q < nx; ++q) pos += (xs_shell[q] < sh || (xs_shell[q] == sh && xs_m[q] < mr)) ? 1 : 0;
                    grp_rows[pos] = r;
                    grp_m[pos] = xs_m[r];
                }
                __syncthreads();
                if (w == 0) {
                    // Group starts (a new shell in the sorted rows), numbered by a
                    // prefix count over the warp's ballots.
                    int base = 0;
                    for (int j0 = 0; j0 < nx; j0 += 32) {
                        const int j = j0 + lane;
                        const bool first = j < nx && (j == 0 || xs_shell[grp_rows[j]] != xs_shell[grp_rows[j - 1]]);
                        const unsigned b = __ballot_sync(0xffffffffu, first);
                        if (first) grp_first[base + __popc(b & ((1u << lane) - 1u))] = j;
                        base += __popc(b);
                    }
                    if (lane == 0) {
                        grp_first[base] = nx;
                        grp_first[nx + 1] = base;
                    }
                }
                __syncthreads();
                for (int g = tid; g < grp_first[nx + 1]; g += kBulkThreads) {
                    const int j0 = grp_first[g], j1 = grp_first[g + 1];
                    const int sh = xs_shell[grp_rows[j0]];
                    unsigned mask = 0;
                    for (int j = j0; j < j1; ++j) mask |= 1u << grp_m[j];
                    xs_go[g] = prm.basis.origin_r2[sh];
                    xs_gi[g] = prm.basis.info[sh];
                    xs_gmask[g] = mask;
                }
                __syncthreads();
            }
            const int ngrp = nx > 0 ? grp_first[nx + 1] : 0;
            for (int ph0 = 0; ph0 < kBlockPoints; ph0 += ph_points) {
                if (nx > 0) {
                    // FP64 AO values of the exact rows at this phase's points:
                    // each producer thread keeps one point (ph_points divides
                    // the 256 producers) and takes every (256 / ph_points)-th
                    // shell group.
                    if (producer) {
                        const int pp = tid % ph_points;
                        const long long e = start + ph0 + pp;
                        const bool here = ph0 + pp < bcount && point_exists(prm.src, e);
                        double x = 0.0, y = 0.0, z = 0.0;
                        if (here) point_at(prm.src, e, x, y, z);
                        for (int g = tid / ph_points; g < ngrp; g += kThreads / ph_points) {
                            const int j0 = grp_first[g];
                            if (here) {
                                const double4 o = xs_go[g];
                                exact_shell_any<P>(prm.basis, o, xs_gi[g], x - o.x, y - o.y, z - o.z, xs_gmask[g],
                                                   grp_rows + j0, xs_phi, ph_points, pp);
                            } else {
                                for (int j = j0; j < grp_first[g + 1]; ++j)
#pragma unroll
                                    for (int c = 0; c < P; ++c) xs_phi[(grp_rows[j] * P + c) * ph_points + pp] = 0.0;
                            }
                        }
                    }
                    __syncthreads();
                }
                if (point >= ph0 && point < ph0 + ph_points) {
                    const int pq = point - ph0;
                    for (int i0 = i_lo; i0 < i_hi; i0 += MG) {
                        double x[P][MG];
#pragma unroll
                        for (int c = 0; c < P; ++c)
#pragma unroll
                            for (int u = 0; u < MG; ++u) x[c][u] = 0.0;
                        for (int gi = 0; gi < ng; ++gi) {
                            unsigned v[P][MG];
#pragma unroll
                            for (int c = 0; c < P; ++c)
                                tmem_ld<MG>(lane_addr + static_cast<unsigned>(gi) * gcols + static_cast<unsigned>(c * N + i0),
                                            v[c]);
                            tmem_wait_ld();
#pragma unroll
                            for (int c = 0; c < P; ++c) {
                                reg_fence<MG>(v[c]);
#pragma unroll
                                for (int u = 0; u < MG; ++u) x[c][u] += static_cast<double>(__uint_as_float(v[c][u]));
                            }
                        }
                        // The exact rows: FP64 AO values times FP64 coefficients
                        // (two rows per iteration, so that one row's loads overlap
                        // the other's products).
#pragma unroll 2
                        for (int r = 0; r < nx; ++r) {
                            // 64-byte aligned: N and i0 are multiples of 8.
                            const double2* crow = reinterpret_cast<const double2*>(xs_c + r * N + i0);
                            double cv[MG];
#pragma unroll
                            for (int u = 0; u < MG / 2; ++u) {
                                const double2 c2 = crow[u];
                                cv[2 * u] = c2.x;
                                cv[2 * u + 1] = c2.y;
                            }
#pragma unroll
                            for (int c = 0; c < P; ++c) {
                                const double f = xs_phi[(r * P + c) * ph_points + pq];
#pragma unroll
                                for (int u = 0; u < MG; ++u) x[c][u] += f * cv[u];
                            }
                        }
                        fold<P, MG>(x, q, i_hi - i0);
                    }
                }
                // The next phase overwrites the staged AO values.
                if (nx > 0) __syncthreads();
            }
            tc_fence_before();
            __syncthreads();
        }
        if (failed) break;
        if (half == 1)
#pragma unroll
            for (int i = 0; i < Q; ++i) red[i * 128 + point] = q[i];
        __syncthreads();
        if (half == 0) {
#pragma unroll
            for (int i = 0; i < Q; ++i) q[i] += red[i * 128 + point];
            record<P>(q, prm.ao_order, ch.role == 1 ? chan_dd[0] : chan_dd[1]);
        }
        __syncthreads();
    }

    if (failed) {
        if (producer) asm volatile("cp.async.wait_group 0;" ::: "memory");  // no copy in flight at exit
        if (tid == 0) atomicOr(prm.status, 1u);
        // The MMA warp waits for the MMAs it issued and the loader for the rows
        // it requested (bounded), before tensor memory is freed and the CTA exits.
        if ((mma_warp || loader) && lane == 0) {
            const int n = mma_warp ? S : F;
            unsigned long long* b = mma_warp ? a_empty : f_full;
            for (int s = 0; s < n; ++s) {
                const long long lastu = gtile - 1 - ((gtile - 1 - s) % n + n) % n;
                if (lastu >= 0) (void)mbar_wait(&b[lastu % n], static_cast<unsigned>((lastu / n) & 1));
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (w == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, static_cast<unsigned>(prm.tmem_cols));
    }
    if (half != 0 || point >= bcount) return;
    if (failed) {
        const double nan = __longlong_as_double(0x7ff8000000000000ll);
        DevDD d;
        d.value = d.lap = d.tau = nan;
        for (int i = 0; i < 3; ++i) d.grad[i] = d.tau_axes[i] = nan;
        for (int i = 0; i < 6; ++i) d.hess[i] = nan;
        store_point(prm.spec, d, d, false, start + point);
        return;
    }
    // Total and Difference are formed where a property asks for them.
    const DevDD alpha = chan_dd[0];
    const DevDD beta = prm.beta_is_alpha ? chan_dd[0] : chan_dd[1];
    store_point(prm.spec, alpha, beta, false, start + point);
}

// ---------------------------------------------------------------------------
// Fused form: AO rows built in the kernel, K step by K step.
//
// Prologue: the block's bounding box, the AO blocks (shells) whose cutoff
// sphere reaches it in index order, a bound of each one's radial part over
// the box (sum |u_p| exp(-a_p d^2), d the distance from its centre to the
// box), the shells ranked by that bound (ascending, ties by index: the large
// terms are added last, as the row order of the unfused kernel does) and
// packed greedily into K steps of at most 16 rows.  Step t: the two halves of
// the CTA compute alternate shells of the step, thread = point, into an FP32
// staging tile [panel][16 rows][128 points] (padding rows zeroed), which is
// then split into BF16 pieces exactly as the unfused kernel splits the rows it
// loads; the MMAs of step t run while step t+1 is built.
template <int P, int S>
struct FusedSmem {
    static constexpr int Q = NQm<P>::v;
    static constexpr int SB = S + 1;
    static constexpr unsigned a_bytes = 3u * P * kATile;
    static constexpr unsigned stg_bytes = 16u * P * 128u * 4u;
    static constexpr unsigned prologue_bytes = 2u * 4u * kFusedMaxShells;
    static constexpr unsigned red_bytes = 8u * Q * 128u;
    static constexpr unsigned scratch_bytes =
        (stg_bytes > prologue_bytes ? (stg_bytes > red_bytes ? stg_bytes : red_bytes)
                                    : (prologue_bytes > red_bytes ? prologue_bytes : red_bytes));
    __host__ __device__ static unsigned b_bytes(int ncols) { return 3u * 32u * static_cast<unsigned>(ncols); }
    static size_t total(int ncols) {
        return S * static_cast<size_t>(a_bytes) + SB * static_cast<size_t>(b_bytes(ncols)) + scratch_bytes +
               sizeof(int) * (2 * kFusedMaxShells + 2) + sizeof(double) * 8 * 6 + sizeof(int) * 8 + 8 * S + 16;
    }
};

template <int P, int S, int MAXL>
__global__ void __launch_bounds__(kThreads, 1) contract_fused_kernel(const __grid_constant__ ContractFusedParams prm) {
    using L = FusedSmem<P, S>;
    constexpr int Q = L::Q;
    constexpr int SB = L::SB;
    extern __shared__ __align__(1024) unsigned char sm[];
    const int N = prm.ncols;
    const unsigned b_bytes = L::b_bytes(N);
    unsigned char* a_st = sm;
    unsigned char* b_st = sm + S * L::a_bytes;
    unsigned char* scratch = b_st + SB * b_bytes;
    float* stg = reinterpret_cast<float*>(scratch);
    double* red = reinterpret_cast<double*>(scratch);
    int* s_list = reinterpret_cast<int*>(scratch);                        // prologue only
    float* s_key = reinterpret_cast<float*>(s_list + kFusedMaxShells);    // prologue only
    int* s_sorted = reinterpret_cast<int*>(scratch + L::scratch_bytes);
    int* step_first = s_sorted + kFusedMaxShells;
    double* s_box = reinterpret_cast<double*>(step_first + kFusedMaxShells + 2);
    int* s_wcount = reinterpret_cast<int*>(s_box + 8 * 6);
    unsigned long long* bar = reinterpret_cast<unsigned long long*>(s_wcount + 8);
    unsigned* tslot = reinterpret_cast<unsigned*>(bar + S);

    const AoMixedParams& ap = prm.ao;
    const DevBasis& B = ap.basis;
    const int blk = blockIdx.x;
    const long long start = ap.first_point + static_cast<long long>(blk) * ap.block_size;
    long long bcount = prm.count - start;
    if (bcount > ap.block_size) bcount = ap.block_size;
    const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
    const int pj = tid & 127;          // this thread's point in the production
    const int phalf = tid >> 7;        // which alternate shells it builds
    const bool pvalid = pj < bcount && point_exists(ap.src, start + pj);
    double px = 0.0, py = 0.0, pz = 0.0;
    if (pvalid) point_at(ap.src, start + pj, px, py, pz);

    if (tid == 0) {
        for (int q = 0; q < S; ++q) mbar_init(&bar[q], kIssuers<P>);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (w == 0) tmem_alloc(tslot, static_cast<unsigned>(prm.tmem_cols));

    // Bounding box of the block's points (the first 128 threads hold them).
    {
        const double big = 1.0e300;
        const bool mine = pvalid && tid < 128;
        const double pc[3] = {px, py, pz};
        for (int a = 0; a < 3; ++a) {
            const double lo = warp_min_d(mine ? pc[a] : big);
            const double hi = warp_max_d(mine ? pc[a] : -big);
            if (lane == 0) {
                s_box[w * 6 + a] = lo;
                s_box[w * 6 + 3 + a] = hi;
            }
        }
    }
    __syncthreads();
    double lo[3], hi[3];
    for (int a = 0; a < 3; ++a) {
        lo[a] = s_box[a];
        hi[a] = s_box[3 + a];
        for (int q = 1; q < 8; ++q) {
            lo[a] = fmin(lo[a], s_box[q * 6 + a]);
            hi[a] = fmax(hi[a], s_box[q * 6 + 3 + a]);
        }
    }
    // Shells within reach, in index order, with their bounds.
    int nlist = 0;
    for (int c0 = 0; c0 < B.nblocks; c0 += kThreads) {
        const int sh = c0 + tid;
        bool reach = false;
        double d2 = 0.0;
        if (sh < B.nblocks) {
            const double4 o = B.origin_r2[sh];
            const double ox[3] = {o.x, o.y, o.z};
            for (int a = 0; a < 3; ++a) {
                const double d = fmax(0.0, fmax(lo[a] - ox[a], ox[a] - hi[a]));
                d2 += d * d;
            }
            reach = !(d2 > o.w * (1.0 + 1e-10) + 1e-300);
        }
        const unsigned bal = __ballot_sync(0xffffffffu, reach);
        if (lane == 0) s_wcount[w] = __popc(bal);
        __syncthreads();
        int before = nlist, total = nlist;
        for (int q = 0; q < 8; ++q) {
            if (q < w) before += s_wcount[q];
            total += s_wcount[q];
        }
        if (reach) {
            const int pos = before + __popc(bal & ((1u << lane) - 1u));
            const int4 inf = B.info[sh];
            const int nprim = inf.x >> 16;
            float bound = 0.0f;
            for (int q = 0; q < nprim; ++q) {
                const MixPrim pr = ap.prims[inf.y + q];
                bound += fabsf(pr.u) * exp_neg(pr.al2, d2);
            }
            s_list[pos] = sh;
            s_key[pos] = bound;
        }
        nlist = total;
        __syncthreads();
    }
    // Rank by (bound, index) and pack into K steps.
    for (int i = tid; i < nlist; i += kThreads) {
        const float ki = s_key[i];
        int rank = 0;
        for (int q = 0; q < nlist; ++q) {
            const float kq = s_key[q];
            rank += (kq < ki) || (kq == ki && q < i);
        }
        s_sorted[rank] = s_list[i];
    }
    __syncthreads();
    if (tid == 0) {
        int nsteps = 0, rows = 0, total_rows = 0;
        step_first[0] = 0;
        for (int i = 0; i < nlist; ++i) {
            const int4 inf = B.info[s_sorted[i]];
            const int l = inf.x & 0xff;
            const int cnt = ((inf.x >> 8) & 1) ? 2 * l + 1 : (l + 1) * (l + 2) / 2;
            if (rows + cnt > 16) {
                step_first[++nsteps] = i;
                rows = 0;
            }
            rows += cnt;
            total_rows += cnt;
        }
        if (nlist > 0) step_first[++nsteps] = nlist;
        s_wcount[0] = nsteps;
        if (prm.nrows) prm.nrows[blk] = total_rows;
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const unsigned tmem = *tslot;
    const int ntiles = s_wcount[0];
    const int G = prm.groups;
    const unsigned gcols = static_cast<unsigned>(P * N);

    const int k8 = tid & 7, g = (tid >> 3) & 15, kh = tid >> 7;
    const unsigned a_off = static_cast<unsigned>(g * 128 + kh * 2048 + k8 * 16);
    const unsigned idesc = instr_desc(N);
    const unsigned long long a_desc0 = smem_desc(smem_u32(a_st), 2048u, 128u);
    const unsigned long long b_desc0 = smem_desc(smem_u32(b_st), static_cast<unsigned>(N * 16), 128u);
    const unsigned nb8 = static_cast<unsigned>(N / 8);
    const unsigned nb8_mul = (65536u + nb8 - 1u) / nb8;
    const int quarter = w & 3, half = w >> 2;
    const int point = quarter * 32 + lane;

    // AO index of row k of step t (-1 for a padding row).
    auto row_ao = [&](int t, int k) -> int {
        int row = 0;
        for (int f = step_first[t]; f < step_first[t + 1]; ++f) {
            const int4 inf = B.info[s_sorted[f]];
            const int l = inf.x & 0xff;
            const int cnt = ((inf.x >> 8) & 1) ? 2 * l + 1 : (l + 1) * (l + 2) / 2;
            if (k < row + cnt) return inf.w + (k - row);
            row += cnt;
        }
        return -1;
    };
    // FP32 rows of step t into the staging tile.
    auto produce = [&](int t) {
        const size_t pstride = 16 * kBlockPoints;
        int row = 0;
        for (int f = step_first[t]; f < step_first[t + 1]; ++f) {
            const int sh = s_sorted[f];
            const int4 inf = B.info[sh];
            const int l = inf.x & 0xff;
            const bool pure = (inf.x >> 8) & 1;
            const int cnt = pure ? 2 * l + 1 : (l + 1) * (l + 2) / 2;
            if (((f - step_first[t]) & 1) == phalf) {
                const double4 o = B.origin_r2[sh];
                const double dx = px - o.x, dy = py - o.y, dz = pz - o.z;
                const double r2d = dx * dx + dy * dy + dz * dz;
                const bool inside = pvalid && r2d <= o.w;
                float* dst = stg + row * kBlockPoints + pj;
                if (__any_sync(0xffffffffu, inside)) {
                    float R0 = 0.0f, R1 = 0.0f, R2 = 0.0f;
                    if (inside) {
                        const int nprim = inf.x >> 16;
                        for (int q = 0; q < nprim; ++q) {
                            const MixPrim pr = ap.prims[inf.y + q];
                            const float ue = pr.u * exp_neg(pr.al2, r2d);
                            R0 += ue;
                            R1 += ue * pr.alpha;
                            R2 += ue * pr.alpha * pr.alpha;
                        }
                    }
                    const float x = static_cast<float>(dx), y = static_cast<float>(dy), z = static_cast<float>(dz);
                    const float r2 = static_cast<float>(r2d);
                    switch (l | (pure ? 16 : 0)) {
#define KUMO_FUSED(LL, PP)                                                                                          \
    case (LL) | ((PP) ? 16 : 0):                                                                                    \
        if constexpr (LL <= MAXL)                                                                                   \
            mixed_shell<(LL <= MAXL ? LL : 0), PP, P, false>(ap, x, y, z, r2, R0, -2.0f * R1, 4.0f * R2,           \
                                                              (float)(2 * LL + 3) * (-2.0f * R1) + r2 * (4.0f * R2),  \
                                                              dst, pstride, nullptr, lane);                        \
        break;
                        KUMO_FUSED(0, false) KUMO_FUSED(1, false) KUMO_FUSED(2, false) KUMO_FUSED(3, false)
                        KUMO_FUSED(4, false) KUMO_FUSED(2, true) KUMO_FUSED(3, true) KUMO_FUSED(4, true)
#undef KUMO_FUSED
                        default: break;
                    }
                } else {
                    for (int m = 0; m < cnt; ++m)
#pragma unroll
                        for (int c = 0; c < P; ++c) dst[c * pstride + m * kBlockPoints] = 0.0f;
                }
            }
            row += cnt;
        }
        // Padding rows.
        for (int i = tid; i < (16 - row) * P * kBlockPoints; i += kThreads) {
            const int c = i / ((16 - row) * kBlockPoints);
            const int r = row + (i / kBlockPoints) % (16 - row);
            stg[(c * 16 + r) * kBlockPoints + (i % kBlockPoints)] = 0.0f;
        }
    };

    bool failed = false;
    long long gtile = 0;
    DevDD chan_dd[2];
    dd_zero(chan_dd[0]);
    dd_zero(chan_dd[1]);

    for (int ci = 0; ci < prm.nchannels && !failed; ++ci) {
        const MoChannelTC ch = prm.ch[ci];
        double q[Q];
#pragma unroll
        for (int i = 0; i < Q; ++i) q[i] = 0.0;
        for (int n0 = 0; n0 < ch.nocc && !failed; n0 += N) {
            auto load_b = [&](int t, int stage) {
                const unsigned bst = smem_u32(b_st + stage * b_bytes);
                const int nchunk = 3 * 16 * (N / 8);
                for (int v = tid; v < nchunk; v += kThreads) {
                    const int r8 = v & 7;
                    const unsigned rest = static_cast<unsigned>(v) >> 3;
                    const unsigned rest2 = (rest * nb8_mul) >> 16;
                    const int ng = static_cast<int>(rest - rest2 * nb8);
                    const int rh = static_cast<int>(rest2 & 1u), piece = static_cast<int>(rest2 >> 1);
                    const int col = n0 + ng * 8;
                    const int ao = col < ch.ldn ? row_ao(t, rh * 8 + r8) : -1;
                    const bool ok = ao >= 0;
                    const std::uint16_t* src =
                        ch.cs + (ok ? piece * ch.piece_stride + static_cast<long long>(ao) * ch.ldn + col : 0);
                    cp_async16(bst + static_cast<unsigned>(piece * 32 * N + ng * 128 + rh * (N * 16) + r8 * 16), src,
                               ok);
                }
                asm volatile("cp.async.commit_group;" ::: "memory");
            };
            if (ntiles > 0) {
                load_b(0, static_cast<int>(gtile % SB));
                if (ntiles > 1) load_b(1, static_cast<int>((gtile + 1) % SB));
            }
            for (int t = 0; t < ntiles; ++t, ++gtile) {
                const int s = static_cast<int>(gtile % S);
                const int sb = static_cast<int>(gtile % SB);
                produce(t);
                __syncthreads();
                unsigned char* ast = a_st + s * L::a_bytes;
#pragma unroll
                for (int c = 0; c < P; ++c) {
                    const float4* src = reinterpret_cast<const float4*>(stg + (c * 16 + kh * 8 + k8) * kBlockPoints + g * 8);
                    uint4 p0, p1, p2;
                    split8(src[0], src[1], p0, p1, p2);
                    *reinterpret_cast<uint4*>(ast + (0 * P + c) * kATile + a_off) = p0;
                    *reinterpret_cast<uint4*>(ast + (1 * P + c) * kATile + a_off) = p1;
                    *reinterpret_cast<uint4*>(ast + (2 * P + c) * kATile + a_off) = p2;
                }
                if (t + 1 < ntiles)
                    asm volatile("cp.async.wait_group 1;" ::: "memory");
                else
                    asm volatile("cp.async.wait_group 0;" ::: "memory");
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                if (__syncthreads_or(failed)) {
                    failed = true;
                    break;
                }
                if (lane == 0 && w < kIssuers<P>) {
                    tc_fence_after();
                    const unsigned long long as = a_desc0 + ((static_cast<unsigned>(s) * L::a_bytes) >> 4);
                    const unsigned long long bs = b_desc0 + ((static_cast<unsigned>(sb) * b_bytes) >> 4);
                    const unsigned bpiece = (32u * static_cast<unsigned>(N)) >> 4;
                    const unsigned dg = tmem + static_cast<unsigned>(t % G) * gcols;
                    for (int c = w; c < P; c += kIssuers<P>) {
#pragma unroll
                        for (int e = 0; e < 6; ++e) {
                            const unsigned long long ad = as + static_cast<unsigned>(((piece_a(e) * P + c) * kATile) >> 4);
                            const unsigned long long bd = bs + static_cast<unsigned>(piece_b(e)) * bpiece;
                            tc_mma(dg + static_cast<unsigned>(c * N), ad, bd, idesc, (t >= G || e > 0) ? 1u : 0u);
                        }
                    }
                    tc_commit(&bar[s]);
                }
                if (t + 1 < ntiles) {
                    const long long wv = gtile + 1 - S;
                    if (wv >= 0 && !mbar_wait(&bar[wv % S], static_cast<unsigned>((wv / S) & 1), prm.wait_ns)) failed = true;
                    if (t + 2 < ntiles) load_b(t + 2, static_cast<int>((gtile + 2) % SB));
                }
            }
            if (failed || ntiles == 0) continue;
            const long long last = gtile - 1;
            if (!mbar_wait(&bar[last % S], static_cast<unsigned>((last / S) & 1), prm.wait_ns)) failed = true;
            if (__syncthreads_or(failed)) {
                failed = true;
                break;
            }
            tc_fence_after();
            const int nvalid = ch.nocc - n0 < N ? ch.nocc - n0 : N;
            const int i_lo = half * (N / 2), i_hi = min(nvalid, (half + 1) * (N / 2));
            const unsigned lane_addr = tmem + (static_cast<unsigned>(quarter * 32) << 16);
            const int ng = ntiles < G ? ntiles : G;
            constexpr int MG = 4;
            for (int i0 = i_lo; i0 < i_hi; i0 += MG) {
                double x[P][MG];
#pragma unroll
                for (int c = 0; c < P; ++c)
#pragma unroll
                    for (int u = 0; u < MG; ++u) x[c][u] = 0.0;
                for (int gi = 0; gi < ng; ++gi) {
                    unsigned v[P][MG];
#pragma unroll
                    for (int c = 0; c < P; ++c)
                        tmem_ld<MG>(lane_addr + static_cast<unsigned>(gi) * gcols + static_cast<unsigned>(c * N + i0), v[c]);
                    tmem_wait_ld();
#pragma unroll
                    for (int c = 0; c < P; ++c) {
                        reg_fence<MG>(v[c]);
#pragma unroll
                        for (int u = 0; u < MG; ++u) x[c][u] += static_cast<double>(__uint_as_float(v[c][u]));
                    }
                }
                fold<P, MG>(x, q, i_hi - i0);
            }
            tc_fence_before();
            __syncthreads();
        }
        if (failed) break;
        if (half == 1)
#pragma unroll
            for (int i = 0; i < Q; ++i) red[i * 128 + point] = q[i];
        __syncthreads();
        if (half == 0) {
#pragma unroll
            for (int i = 0; i < Q; ++i) q[i] += red[i * 128 + point];
            record<P>(q, prm.ao_order, ch.role == 1 ? chan_dd[0] : chan_dd[1]);
        }
        __syncthreads();
    }

    if (failed) {
        asm volatile("cp.async.wait_group 0;" ::: "memory");
        if (tid == 0) atomicOr(prm.status, 1u);
        for (int q = 0; q < S; ++q) {
            const long long last = gtile - 1 - ((gtile - 1 - q) % S + S) % S;
            if (last >= 0) (void)mbar_wait(&bar[last % S], static_cast<unsigned>((last / S) & 1));
        }
    }
    tc_fence_before();
    __syncthreads();
    if (w == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, static_cast<unsigned>(prm.tmem_cols));
    }
    if (half != 0 || point >= bcount) return;
    DevDD comp[4];
    if (failed) {
        const double nan = __longlong_as_double(0x7ff8000000000000ll);
        DevDD d;
        d.value = d.lap = d.tau = nan;
        for (int i = 0; i < 3; ++i) d.grad[i] = d.tau_axes[i] = nan;
        for (int i = 0; i < 6; ++i) d.hess[i] = nan;
        comp[0] = comp[1] = comp[2] = comp[3] = d;
    } else {
        DevDD alpha = chan_dd[0], beta = chan_dd[1];
        if (prm.beta_is_alpha) beta = alpha;
        comp[1] = alpha;
        comp[2] = beta;
        comp[0] = dd_combine(alpha, beta, 1.0, 1.0, false);
        comp[3] = dd_combine(alpha, beta, -1.0, 1.0, false);
    }
    store_point(prm.spec, comp, start + point);
}

template <int P, int S, int MAXL>
void launch_fused(const ContractFusedParams& p, cudaStream_t stream) {
    constexpr size_t kMaxSmem = 227u * 1024u;
    if (FusedSmem<P, S>::total(p.ncols) > kMaxSmem)
        throw std::invalid_argument("fused tensor-core contraction: stages exceed shared memory");
    KUMO_REGISTER_KERNEL(contract_fused_kernel<P, S, MAXL>);
    ensure_dynamic_smem(reinterpret_cast<const void*>(contract_fused_kernel<P, S, MAXL>), static_cast<int>(kMaxSmem));
    contract_fused_kernel<P, S, MAXL><<<p.ao.nblocks, kThreads, kMaxSmem, stream>>>(p);
}

template <int P>
void fused_maxl(const ContractFusedParams& p, cudaStream_t stream) {
    if (p.ao.basis.max_l <= 2)
        launch_fused<P, 2, 2>(p, stream);
    else if (p.ao.basis.max_l == 3)
        launch_fused<P, 2, 3>(p, stream);
    else
        launch_fused<P, 2, 4>(p, stream);
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (null if
// the driver does not provide it).
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            f = nullptr;
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
    }();
    return fn;
}

// 4-D map of the FP32 panels of a wave, [block][panel][row][point], with a
// box of one row's npanel panel rows.
bool panel_row_map(const ContractMixedParams& p, int npanel, CUtensorMap& map) {
    const PFN_cuTensorMapEncodeTiled_v12000 encode = tensor_map_encoder();
    if (encode == nullptr || reinterpret_cast<std::uintptr_t>(p.scr.panels) % 16 != 0) return false;
    const cuuint64_t row = kBlockPoints * sizeof(float);
    const cuuint64_t dims[4] = {static_cast<cuuint64_t>(kBlockPoints), static_cast<cuuint64_t>(p.scr.row_stride),
                                static_cast<cuuint64_t>(npanel), static_cast<cuuint64_t>(p.nblocks)};
    const cuuint64_t strides[3] = {row, row * p.scr.row_stride, row * p.scr.row_stride * npanel};
    const cuuint32_t box[4] = {static_cast<cuuint32_t>(kBlockPoints), 1u, static_cast<cuuint32_t>(npanel), 1u};
    const cuuint32_t estride[4] = {1u, 1u, 1u, 1u};
    return encode(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, const_cast<float*>(p.scr.panels), dims, strides, box,
                  estride, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int P, int F, int SB>
bool launch_bulk(const ContractMixedParams& p, cudaStream_t stream) {
    constexpr size_t kMaxSmem = 227u * 1024u;
    if (!BulkSmem<P>::rows_fit(p.scr.row_stride) || BulkSmem<P>::total(p.ncols, F, SB, p.scr.row_stride) > kMaxSmem)
        return false;
    CUtensorMap map;
    if (!panel_row_map(p, P, map)) return false;
    KUMO_REGISTER_KERNEL(contract_bulk_kernel<P, F, SB>);
    ensure_dynamic_smem(reinterpret_cast<const void*>(contract_bulk_kernel<P, F, SB>), static_cast<int>(kMaxSmem));
    contract_bulk_kernel<P, F, SB><<<p.nblocks, kBulkThreads, kMaxSmem, stream>>>(p, map);
    return true;
}

// The bulk-copy form where its stages fit (KUMO_MIXED_BULK=0 selects the
// register-staged form, for comparison).
template <int P>
bool try_bulk(const ContractMixedParams& p, cudaStream_t stream) {
    const char* e = std::getenv("KUMO_MIXED_BULK");
    if (e != nullptr && e[0] == '0') return false;
    if constexpr (P == 1) {
        return launch_bulk<1, 4, 3>(p, stream) || launch_bulk<1, 2, 2>(p, stream);
    } else {
        return launch_bulk<P, 2, 3>(p, stream) || launch_bulk<P, 2, 2>(p, stream);
    }
}

template <int P, int S>
void launch(const ContractMixedParams& p, cudaStream_t stream) {
    // The whole 227 KB of shared memory per CTA: one CTA per SM, so each CTA's
    // tensor-memory allocation is granted at once, and every address a matrix
    // descriptor can reach from a stage lies inside the CTA's allocation.
    constexpr size_t kMaxSmem = 227u * 1024u;
    if (Smem<P, S>::total(p.ncols) > kMaxSmem) throw std::invalid_argument("tensor-core contraction: stages exceed shared memory");
    const size_t smem = kMaxSmem;
    KUMO_REGISTER_KERNEL(contract_mixed_kernel<P, S>);
    ensure_dynamic_smem(reinterpret_cast<const void*>(contract_mixed_kernel<P, S>), static_cast<int>(smem));
    contract_mixed_kernel<P, S><<<p.nblocks, kCtaThreads<S>, smem, stream>>>(p);
}

__device__ unsigned g_pipeline_status;

}  // namespace

unsigned* pipeline_status_word() {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_pipeline_status) != cudaSuccess) throw std::runtime_error("cudaGetSymbolAddress (status)");
    return static_cast<unsigned*>(p);
}

unsigned take_pipeline_status() {
    unsigned v = 0;
    if (cudaMemcpyFromSymbol(&v, g_pipeline_status, sizeof v) != cudaSuccess)
        throw std::runtime_error("cudaMemcpyFromSymbol (status)");
    if (v) {
        const unsigned zero = 0;
        cudaMemcpyToSymbol(g_pipeline_status, &zero, sizeof zero);
    }
    return v;
}

void mixed_columns(int npanel, int nocc16, int& ncols, int& groups, int& tmem_cols) {
    const int maxn = std::min(256, (512 / npanel) / 16 * 16);
    const int n = std::max(16, nocc16);
    const int passes = (n + maxn - 1) / maxn;
    ncols = ((n + passes - 1) / passes + 15) / 16 * 16;
    groups = std::max(1, std::min(4, 512 / (npanel * ncols)));
    const int need = groups * npanel * ncols;
    tmem_cols = 32;
    while (tmem_cols < need) tmem_cols *= 2;
}

bool contract_fused_supported(int npanel, int nshells) {
    return (npanel == 1 || npanel == 4 || npanel == 5) && nshells <= kFusedMaxShells;
}

void launch_contract_fused(const ContractFusedParams& p, int npanel, cudaStream_t stream) {
    if (p.ao.nblocks <= 0) return;
    if (p.ncols < 16 || p.ncols % 16 != 0 || p.ncols > 256 || p.groups < 1 ||
        p.groups * npanel * p.ncols > 512 || p.tmem_cols > 512)
        throw std::invalid_argument("tensor-core contraction: unsupported MO column count");
    if (!contract_fused_supported(npanel, p.ao.basis.nblocks))
        throw std::invalid_argument("fused tensor-core contraction: unsupported panel or shell count");
    switch (npanel) {
        case 1: fused_maxl<1>(p, stream); break;
        case 4: fused_maxl<4>(p, stream); break;
        default: fused_maxl<5>(p, stream); break;
    }
}

void upload_exact_tables(const double (&g)[kMaxL + 1][15], const double (&tg)[3][135]) {
    double ig0[kMaxL + 1];
    for (int l = 0; l <= kMaxL; ++l) ig0[l] = 1.0 / g[l][0];
    if (cudaMemcpyToSymbol(c_exact_g, g, sizeof(c_exact_g)) != cudaSuccess ||
        cudaMemcpyToSymbol(c_exact_ig0, ig0, sizeof(c_exact_ig0)) != cudaSuccess ||
        cudaMemcpyToSymbol(c_exact_tg, tg, sizeof(c_exact_tg)) != cudaSuccess)
        throw std::runtime_error("CUDA error in cudaMemcpyToSymbol (exact-row tables)");
}

void launch_contract_mixed(const ContractMixedParams& p, int npanel, cudaStream_t stream) {
    if (p.ncols < 16 || p.ncols % 16 != 0 || p.ncols > 256 || p.groups < 1 ||
        p.groups * npanel * p.ncols > 512 || p.tmem_cols > 512)
        throw std::invalid_argument("tensor-core contraction: unsupported MO column count");
    switch (npanel) {
        case 1: if (!try_bulk<1>(p, stream)) launch<1, 2>(p, stream); break;
        case 4: if (!try_bulk<4>(p, stream)) launch<4, 2>(p, stream); break;
        case 5: if (!try_bulk<5>(p, stream)) launch<5, 2>(p, stream); break;
        case 10: launch<10, 1>(p, stream); break;
        default: throw std::invalid_argument("tensor-core contraction: unsupported panel count");
    }
}

}  // namespace kumo_dev
