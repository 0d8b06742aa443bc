// Mixed-precision AO-P contraction on the tcgen05 tensor cores: the
// reference's density_derivatives_shared (src/density.cpp:150-229) with
// Y = P[kept, kept] Phi[kept, panels 0..3] as tensor-core products.
//
// One CTA (8 warps) per 128-point block.  For each density matrix needed
// (total and/or spin) and each chunk of 128 kept columns k, the CTA computes
// Y_c[point][k] = sum_j Phi_c[j][point] P[j][k] for the value and gradient
// panels c = 0..3 (M = 128 points, N = 128 columns, K = the kept rows j, four
// accumulators of 128 columns = all 512 tensor-memory columns).  Operands are
// split into three BF16 pieces as in the AO-MO contraction (the FP32 panels
// on the fly, P once at upload); the B tile of a K step is gathered from the
// pieces of P through the block's kept AO indices.  The epilogue reads Y from
// tensor memory and folds it, column by column, with the block's FP32 panel
// values of that column into the per-point FP64 partial sums of the FP64
// AO-P kernel (q0 = sum Y0 phi, q[1+a] = sum Y0 d_a phi, q[4+a] = sum Y_a
// d_a phi, then the Laplacian or Hessian terms).  Rows are screened and put
// in ascending order of their block maximum as in the AO-MO contraction.
// Every mbarrier wait is bounded; on expiry the CTA flags *status, stores NaN
// and frees tensor memory after a bounded wait for its MMAs.
#include "func_attr.cuh"
#include <algorithm>
#include <stdexcept>

#include "mixed.cuh"
#include "tc_common.cuh"

namespace kumo_dev {
namespace {

constexpr int kPL = 4;        // left (Y) panels of a matrix with derivatives
constexpr int kCols = 128;    // most columns k per chunk (N of the MMA)
constexpr int kStages = 2;
constexpr int kMaxMats = 2;   // density matrices in one pass

template <int P>
struct NQp {
    static constexpr int v = P == 4 ? 7 : P == 5 ? 8 : 19;
};

template <int P>
__device__ __forceinline__ void record_p(const double* f, int ao_order, DevDD& d) {
    dd_zero(d);
    d.value = f[0];
    if (ao_order == 0) return;
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

template <int P>
struct SmemP {
    static constexpr int Q = NQp<P>::v;
    static constexpr unsigned a_bytes = 3u * kPL * kATile;             // one stage of A pieces
    static constexpr unsigned b_bytes = kMaxMats * 3u * 32u * kCols;   // one stage of B pieces, all matrices of a pass
    // The cross-half sums (Q partials and one value per point) reuse the A
    // stages, which no MMA reads once a pass's last step is done.
    static_assert(sizeof(double) * (Q + 1) * 128 <= kStages * a_bytes, "cross-half sums must fit the A stages");
    static unsigned cap16(int rows) { return (static_cast<unsigned>(rows) + 15u) & ~15u; }
    // rowao (int), perm and colord (u16) and keys (u8) per sortable row.
    static constexpr size_t total(unsigned cap) {
        return kStages * (static_cast<size_t>(a_bytes) + b_bytes) + sizeof(int) * 2 * kCols +
               (sizeof(int) + 2 * sizeof(std::uint16_t) + 1) * static_cast<size_t>(cap) + sizeof(int) * (kBuckets + 4) +
               8 * kStages + 16;
    }
};

template <int P>
__global__ void __launch_bounds__(kThreads, 1) contract_p_mixed_kernel(const __grid_constant__ ContractPMixedParams prm) {
    using L = SmemP<P>;
    constexpr int Q = L::Q;
    constexpr int S = kStages;
    extern __shared__ __align__(1024) unsigned char sm[];
    const int cap = prm.sort_cap;
    unsigned char* a_st = sm;
    unsigned char* b_st = sm + S * L::a_bytes;
    double* red = reinterpret_cast<double*>(sm);
    int* colrow = reinterpret_cast<int*>(b_st + S * L::b_bytes);  // block row of each chunk column (-1: none)
    int* colao = colrow + kCols;                                   // its AO index
    int* rowao = colao + kCols;                                    // AO index of each K row (sorted blocks)
    int* bucket_start = rowao + cap;
    std::uint16_t* perm = reinterpret_cast<std::uint16_t*>(bucket_start + kBuckets + 4);  // K order of the rows
    std::uint16_t* colord = perm + cap;  // the kept rows in AO order: the column order
    unsigned char* keys = reinterpret_cast<unsigned char*>(colord + cap);
    unsigned long long* bar = reinterpret_cast<unsigned long long*>(keys + cap);
    unsigned* tslot = reinterpret_cast<unsigned*>(bar + S);

    const int blk = blockIdx.x;
    const long long start = prm.first_point + static_cast<long long>(blk) * prm.block_size;
    long long bcount = prm.count - start;
    if (bcount > prm.block_size) bcount = prm.block_size;
    const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
    const AoScratch<float>& scr = prm.scr;
    int nk = scr.nkept[blk];
    const size_t pstride = static_cast<size_t>(scr.row_stride) * kBlockPoints;
    const float* pbase = scr.panels + static_cast<size_t>(blk) * P * pstride;
    const int* kept = scr.kept + static_cast<size_t>(blk) * scr.row_stride;
    const long long n = prm.nao;

    if (tid == 0) {
        for (int s = 0; s < S; ++s) mbar_init(&bar[s], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (w == 0) tmem_alloc(tslot, 512u);
    bool sorted = false;
    const int nrows = nk;
    nk = block_row_order(scr.rowmax ? scr.rowmax + static_cast<size_t>(blk) * scr.row_stride * 4 : nullptr, nk,
                         prm.threshold, perm, bucket_start, keys, sorted, cap);
    // The rows kept above the threshold (read back by the profiler).
    if (threadIdx.x == 0) scr.nkept[blk] = nk;
    if (sorted) {
        // Columns k take the kept rows in AO order (runs of consecutive AOs,
        // so that a row of P is read in contiguous pieces); the K rows keep
        // the ascending-maximum order.  Each warp compacts one segment of the
        // rows; the segments' counts give their offsets.
        const int seg = (nrows + 8 * 32 - 1) / (8 * 32) * 32;
        const int lo = w * seg, hi = min(nrows, lo + seg);
        int cnt = 0;
        for (int b = lo; b < hi; b += 32) {
            const int k = b + lane;
            cnt += __popc(__ballot_sync(0xffffffffu, k < hi && keys[k] != 0xffu));
        }
        __syncthreads();  // bucket_start is free again: the counts go there
        if (lane == 0) bucket_start[w] = cnt;
        __syncthreads();
        int pos = 0;
        for (int i = 0; i < w; ++i) pos += bucket_start[i];
        for (int b = lo; b < hi; b += 32) {
            const int k = b + lane;
            const bool keep = k < hi && keys[k] != 0xffu;
            const unsigned bal = __ballot_sync(0xffffffffu, keep);
            if (keep) colord[pos + __popc(bal & ((1u << lane) - 1u))] = static_cast<std::uint16_t>(k);
            pos += __popc(bal);
        }
        for (int k = tid; k < nk; k += kThreads) rowao[k] = kept[perm[k]];
    }
    const int ntiles = (nk + 15) / 16;
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const unsigned tmem = *tslot;

    const int k8 = tid & 7, g = (tid >> 3) & 15, kh = tid >> 7;
    const unsigned a_off = static_cast<unsigned>(g * 128 + kh * 2048 + k8 * 16);
    const unsigned long long a_desc0 = smem_desc(smem_u32(a_st), 2048u, 128u);
    const int quarter = w & 3, half = w >> 2;
    const int point = quarter * 32 + lane;

    bool failed = false;
    long long gtile = 0;
    DevDD tot, spn;
    dd_zero(tot);
    dd_zero(spn);
    // Density matrices: P_total (role 0) and P_spin (role 3), each with the
    // four left panels or (its components needing values only) the value
    // panel.  Two matrices of which at most one has four panels share one
    // pass over the K rows: the A tile serves both (the second uses panel 0)
    // and the chunk width N is what tensor memory holds for all their
    // panels (128 columns, 96 for 4 + 1 panels).  Two four-panel matrices
    // take a pass each.
    const uint2* mp[2];
    int mrole[2], mnpl[2], nm = 0;
    if (prm.total_needed) {
        mp[nm] = reinterpret_cast<const uint2*>(prm.p_total_s);
        mrole[nm] = 0;
        mnpl[nm++] = (prm.value_only & 1) ? 1 : kPL;
    }
    if (prm.spin_needed) {
        mp[nm] = reinterpret_cast<const uint2*>(prm.p_spin_s);
        mrole[nm] = 3;
        mnpl[nm++] = (prm.value_only & 2) ? 1 : kPL;
    }
    if (nm == 2 && mnpl[0] == 1 && mnpl[1] == kPL) {
        const uint2* tp = mp[0];
        mp[0] = mp[1];
        mp[1] = tp;
        const int tr = mrole[0];
        mrole[0] = mrole[1];
        mrole[1] = tr;
        mnpl[0] = kPL;
        mnpl[1] = 1;
    }
    const bool joint = nm == 2 && mnpl[1] == 1;
    const int npass = nm == 0 ? 0 : (joint ? 1 : nm);

    for (int pass = 0; pass < npass && !failed; ++pass) {
        const uint2* P0 = mp[pass];
        const uint2* P1 = joint ? mp[1] : nullptr;
        const int nmp = joint ? 2 : 1;
        const int npl = mnpl[pass];  // A panels (a second matrix uses panel 0)
        const int N = min(kCols, (512 / (npl + nmp - 1)) / 16 * 16);
        const int ngrp = N / 8;
        const unsigned idesc = instr_desc(N);
        const unsigned long long b_desc0 = smem_desc(smem_u32(b_st), static_cast<unsigned>(N * 16), 128u);
        const unsigned bmat = 3u * 32u * static_cast<unsigned>(N);  // one matrix's B tile
        const unsigned col1 = static_cast<unsigned>(npl * N);       // second matrix's accumulator
        double q[Q];
#pragma unroll
        for (int i = 0; i < Q; ++i) q[i] = 0.0;
        double q1 = 0.0;
        for (int c0 = 0; c0 < nk && !failed; c0 += N) {
            for (int c = tid; c < kCols; c += kThreads) {
                const int r = (c < N && c0 + c < nk) ? (sorted ? colord[c0 + c] : c0 + c) : -1;
                colrow[c] = r;
                colao[c] = r >= 0 ? kept[r] : -1;
            }
            __syncthreads();
            float4 ra[kPL][2];
            // Panel rows of step t into registers (read again for every
            // column chunk: default caching).
            auto load_a = [&](int t) {
                const int k = t * 16 + kh * 8 + k8;
                const bool ok = k < nk;
                const int row = ok ? (sorted ? perm[k] : k) : 0;
#pragma unroll
                for (int c = 0; c < kPL; ++c) {
                    if (c >= npl) break;
                    if (ok) {
                        const float4* src =
                            reinterpret_cast<const float4*>(pbase + static_cast<size_t>(c) * pstride +
                                                            static_cast<size_t>(row) * kBlockPoints + g * 8);
                        ra[c][0] = __ldg(src);
                        ra[c][1] = __ldg(src + 1);
                    } else {
                        ra[c][0] = ra[c][1] = make_float4(0.f, 0.f, 0.f, 0.f);
                    }
                }
            };
            // B tiles of step t: the three BF16 pieces of each matrix at (AO
            // of K row j, AO of chunk column c), P stored [row][col] as 8-byte
            // elements (pieces 0..2 and a zero).  Unit v is the 8 columns of
            // group cg of K row jr of matrix mi, gathered with 16-byte loads
            // where they are 8 consecutive AOs, and written as one 16-byte
            // line of each piece.
            auto load_b = [&](int t, int stage) {
                unsigned char* bst = b_st + stage * L::b_bytes;
                const int nunits = nmp * 16 * ngrp;
                for (int v = tid; v < nunits; v += kThreads) {
                    const int cg = v % ngrp, rest = v / ngrp;
                    const int jr = rest & 15, mi = rest >> 4;
                    const uint2* Pm = mi ? P1 : P0;
                    const int j = t * 16 + jr;
                    const int rao = j < nk ? (sorted ? rowao[j] : kept[j]) : -1;
                    uint2 eb[8];
                    const int cao0 = colao[cg * 8];
                    bool run = rao >= 0 && cao0 >= 0;
#pragma unroll
                    for (int u = 1; u < 8; ++u) run = run && colao[cg * 8 + u] == cao0 + u;
                    const long long at = static_cast<long long>(rao) * n + cao0;
                    if (run && (at & 1) == 0) {
                        const uint4* src = reinterpret_cast<const uint4*>(Pm + at);
#pragma unroll
                        for (int h = 0; h < 4; ++h) {
                            const uint4 q4 = __ldg(src + h);
                            eb[2 * h] = make_uint2(q4.x, q4.y);
                            eb[2 * h + 1] = make_uint2(q4.z, q4.w);
                        }
                    } else {
#pragma unroll
                        for (int u = 0; u < 8; ++u) {
                            const int cao = colao[cg * 8 + u];
                            eb[u] = (rao >= 0 && cao >= 0) ? __ldg(Pm + static_cast<long long>(rao) * n + cao)
                                                           : make_uint2(0u, 0u);
                        }
                    }
                    unsigned w0[4], w1[4], w2[4];
#pragma unroll
                    for (int h = 0; h < 4; ++h) {
                        const uint2 a = eb[2 * h], b = eb[2 * h + 1];
                        w0[h] = (a.x & 0xffffu) | (b.x << 16);
                        w1[h] = (a.x >> 16) | (b.x & 0xffff0000u);
                        w2[h] = (a.y & 0xffffu) | (b.y << 16);
                    }
                    unsigned char* dst = bst + mi * bmat + cg * 128 + (jr >> 3) * (N * 16) + (jr & 7) * 16;
                    *reinterpret_cast<uint4*>(dst) = make_uint4(w0[0], w0[1], w0[2], w0[3]);
                    *reinterpret_cast<uint4*>(dst + 32 * N) = make_uint4(w1[0], w1[1], w1[2], w1[3]);
                    *reinterpret_cast<uint4*>(dst + 64 * N) = make_uint4(w2[0], w2[1], w2[2], w2[3]);
                }
            };
            if (ntiles > 0) {
                load_a(0);
                load_b(0, static_cast<int>(gtile % S));
            }
            for (int t = 0; t < ntiles; ++t, ++gtile) {
                const int s = static_cast<int>(gtile % S);
                unsigned char* ast = a_st + s * L::a_bytes;
#pragma unroll
                for (int c = 0; c < kPL; ++c) {
                    if (c >= npl) break;
                    uint4 p0, p1, p2;
                    split8(ra[c][0], ra[c][1], p0, p1, p2);
                    *reinterpret_cast<uint4*>(ast + (0 * kPL + c) * kATile + a_off) = p0;
                    *reinterpret_cast<uint4*>(ast + (1 * kPL + c) * kATile + a_off) = p1;
                    *reinterpret_cast<uint4*>(ast + (2 * kPL + c) * kATile + a_off) = p2;
                }
                if (t + 1 < ntiles) load_a(t + 1);
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                if (__syncthreads_or(failed)) {
                    failed = true;
                    break;
                }
                if (tid == 0) {
                    tc_fence_after();
                    const unsigned long long as = a_desc0 + ((static_cast<unsigned>(s) * L::a_bytes) >> 4);
                    const unsigned long long bs = b_desc0 + ((static_cast<unsigned>(s) * L::b_bytes) >> 4);
                    const unsigned bpiece = (32u * static_cast<unsigned>(N)) >> 4;
#pragma unroll
                    for (int c = 0; c < kPL; ++c) {
                        if (c >= npl) break;
#pragma unroll
                        for (int e = 0; e < 6; ++e) {
                            const unsigned long long ad = as + static_cast<unsigned>(((piece_a(e) * kPL + c) * kATile) >> 4);
                            const unsigned long long bd = bs + static_cast<unsigned>(piece_b(e)) * bpiece;
                            tc_mma(tmem + static_cast<unsigned>(c * N), ad, bd, idesc, (t > 0 || e > 0) ? 1u : 0u);
                        }
                    }
                    if (joint) {
#pragma unroll
                        for (int e = 0; e < 6; ++e) {
                            const unsigned long long ad = as + static_cast<unsigned>((piece_a(e) * kPL * kATile) >> 4);
                            const unsigned long long bd = bs + (bmat >> 4) + static_cast<unsigned>(piece_b(e)) * bpiece;
                            tc_mma(tmem + col1, ad, bd, idesc, (t > 0 || e > 0) ? 1u : 0u);
                        }
                    }
                    tc_commit(&bar[s]);
                }
                if (t + 1 < ntiles) {
                    // Stage (t + 1) % S was last read by the MMAs of step t - 1.
                    const long long wt = gtile + 1 - S;
                    if (wt >= 0 && !mbar_wait(&bar[wt % S], static_cast<unsigned>((wt / S) & 1), prm.wait_ns)) failed = true;
                    load_b(t + 1, static_cast<int>((gtile + 1) % S));
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
            // Fold: columns [half*N/2, half*N/2 + N/2) of the chunk.  The
            // panel values of a group's columns are loaded one group ahead,
            // so that their latency overlaps the previous group's products.
            const unsigned lane_addr = tmem + (static_cast<unsigned>(quarter * 32) << 16);
            const int i_lo = half * (N / 2);
            const int c_hi = min(nk - c0, i_lo + N / 2);
            if (npl == 1) {
                float rv[2][8];
                auto rows8 = [&](float (&r)[8], int i0) {
#pragma unroll
                    for (int u = 0; u < 8; ++u)
                        r[u] = i0 + u < c_hi ? pbase[static_cast<size_t>(colrow[i0 + u]) * kBlockPoints + point] : 0.0f;
                };
                auto fold8 = [&](const float (&r)[8], int i0) {
                    unsigned v[8], v1[8];
                    tmem_ld<8>(lane_addr + static_cast<unsigned>(i0), v);
                    if (joint) tmem_ld<8>(lane_addr + col1 + static_cast<unsigned>(i0), v1);
                    tmem_wait_ld();
                    reg_fence<8>(v);
                    if (joint) reg_fence<8>(v1);
#pragma unroll
                    for (int u = 0; u < 8; ++u) {
                        if (i0 + u >= c_hi) break;
                        const double f = static_cast<double>(r[u]);
                        q[0] += f * static_cast<double>(__uint_as_float(v[u]));
                        if (joint) q1 += f * static_cast<double>(__uint_as_float(v1[u]));
                    }
                };
                if (i_lo < c_hi) rows8(rv[0], i_lo);
                for (int i0 = i_lo; i0 < c_hi; i0 += 16) {
                    if (i0 + 8 < c_hi) rows8(rv[1], i0 + 8);
                    fold8(rv[0], i0);
                    if (i0 + 8 < c_hi) {
                        if (i0 + 16 < c_hi) rows8(rv[0], i0 + 16);
                        fold8(rv[1], i0 + 8);
                    }
                }
            } else {
                // Panel values of CG columns, r[u][c] of panel c (all P
                // panels); two columns at a time with the Hessian panels.
                constexpr int CG = P == 10 ? 2 : 4;
                float rv[2][CG][P];
                auto rows4 = [&](float (&r)[CG][P], int i0) {
#pragma unroll
                    for (int u = 0; u < CG; ++u) {
                        const bool ok = i0 + u < c_hi;
                        const float* row = pbase + static_cast<size_t>(ok ? colrow[i0 + u] : 0) * kBlockPoints + point;
#pragma unroll
                        for (int c = 0; c < P; ++c) r[u][c] = ok ? row[c * pstride] : 0.0f;
                    }
                };
                auto fold4 = [&](const float (&r)[CG][P], int i0) {
                    unsigned v[kPL][CG], v1[CG];
#pragma unroll
                    for (int c = 0; c < kPL; ++c) tmem_ld<CG>(lane_addr + static_cast<unsigned>(c * N + i0), v[c]);
                    if (joint) tmem_ld<CG>(lane_addr + col1 + static_cast<unsigned>(i0), v1);
                    tmem_wait_ld();
#pragma unroll
                    for (int c = 0; c < kPL; ++c) reg_fence<CG>(v[c]);
                    if (joint) reg_fence<CG>(v1);
#pragma unroll
                    for (int u = 0; u < CG; ++u) {
                        if (i0 + u >= c_hi) break;
                        double y[kPL];
#pragma unroll
                        for (int c = 0; c < kPL; ++c) y[c] = static_cast<double>(__uint_as_float(v[c][u]));
                        q[0] += static_cast<double>(r[u][0]) * y[0];
                        if (joint) q1 += static_cast<double>(r[u][0]) * static_cast<double>(__uint_as_float(v1[u]));
                        double fa[3];
#pragma unroll
                        for (int a = 0; a < 3; ++a) {
                            fa[a] = r[u][1 + a];
                            q[1 + a] += fa[a] * y[0];
                            q[4 + a] += fa[a] * y[1 + a];
                        }
                        if constexpr (P == 5) q[7] += static_cast<double>(r[u][4]) * y[0];
                        if constexpr (P == 10) {
                            constexpr int pa[6] = {0, 0, 0, 1, 1, 2}, pc[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
                            for (int h = 0; h < 6; ++h) {
                                q[7 + h] += static_cast<double>(r[u][4 + h]) * y[0];
                                q[13 + h] += fa[pa[h]] * y[1 + pc[h]];
                            }
                        }
                    }
                };
                if (i_lo < c_hi) rows4(rv[0], i_lo);
                for (int i0 = i_lo; i0 < c_hi; i0 += 2 * CG) {
                    if (i0 + CG < c_hi) rows4(rv[1], i0 + CG);
                    fold4(rv[0], i0);
                    if (i0 + CG < c_hi) {
                        if (i0 + 2 * CG < c_hi) rows4(rv[0], i0 + 2 * CG);
                        fold4(rv[1], i0 + CG);
                    }
                }
            }
            tc_fence_before();
            __syncthreads();
        }
        if (failed) break;
        // Cross-half sums in the A stages (no MMA reads them now).
        if (half == 1) {
#pragma unroll
            for (int i = 0; i < Q; ++i) red[i * 128 + point] = q[i];
            red[Q * 128 + point] = q1;
        }
        __syncthreads();
        if (half == 0) {
#pragma unroll
            for (int i = 0; i < Q; ++i) q[i] += red[i * 128 + point];
            record_p<P>(q, npl == 1 ? 0 : prm.ao_order, mrole[pass] == 0 ? tot : spn);
            if (joint) {
                DevDD& d1 = mrole[1] == 0 ? tot : spn;
                dd_zero(d1);
                d1.value = q1 + red[Q * 128 + point];
            }
        }
        __syncthreads();
    }

    if (failed) {
        if (tid == 0) atomicOr(prm.status, 1u);
        for (int s = 0; s < S; ++s) {
            const long long last = gtile - 1 - ((gtile - 1 - s) % S + S) % S;
            if (last >= 0) (void)mbar_wait(&bar[last % S], static_cast<unsigned>((last / S) & 1));
        }
    }
    tc_fence_before();
    __syncthreads();
    if (w == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, 512u);
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
        const bool full = P == 10 && prm.ao_order == 2;
        comp[0] = tot;
        comp[3] = spn;
        comp[1] = dd_combine(tot, spn, 1.0, 0.5, full);
        comp[2] = dd_combine(tot, spn, -1.0, 0.5, full);
    }
    store_point(prm.spec, comp, start + point);
}

template <int P>
void launch(const ContractPMixedParams& p, cudaStream_t stream) {
    constexpr size_t kMaxSmem = 227u * 1024u;
    static_assert(SmemP<P>::total(kSortCap) <= kMaxSmem, "AO-P stages exceed shared memory");
    // The row-order arrays hold the block's rows (blocks with more rows than
    // kSortCap keep AO order).
    ContractPMixedParams q = p;
    q.sort_cap = static_cast<int>(std::min<unsigned>(SmemP<P>::cap16(p.scr.row_stride), kSortCap));
    const size_t smem = SmemP<P>::total(static_cast<unsigned>(q.sort_cap));
    KUMO_REGISTER_KERNEL(contract_p_mixed_kernel<P>);
    ensure_dynamic_smem(reinterpret_cast<const void*>(contract_p_mixed_kernel<P>), static_cast<int>(kMaxSmem));
    contract_p_mixed_kernel<P><<<p.nblocks, kThreads, smem, stream>>>(q);
}

}  // namespace

void launch_contract_p_mixed(const ContractPMixedParams& p, int npanel, cudaStream_t stream) {
    switch (npanel) {
        case 4: launch<4>(p, stream); break;
        case 5: launch<5>(p, stream); break;
        case 10: launch<10>(p, stream); break;
        default: throw std::invalid_argument("tensor-core AO-P contraction: unsupported panel count");
    }
}

}  // namespace kumo_dev
