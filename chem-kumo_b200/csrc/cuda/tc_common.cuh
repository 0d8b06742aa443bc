// Device helpers shared by the tcgen05 contractions (inline PTX for
// mbarriers, tensor memory, tcgen05.mma/ld and cp.async; the BF16 three-piece
// split; the screening and K order of a block's rows).
#pragma once

#include <cuda_bf16.h>

namespace kumo_dev {
namespace {

constexpr int kThreads = 256;

// The six BF16 products a_i b_j (i + j <= 2) of one FP32 product, in the
// order they are accumulated: the terms of order 2^-16, then 2^-8, then
// a_0 b_0, so that the small terms meet a small partial sum.
// Pieces (a_i, b_j) of product e: (1,1) (0,2) (2,0) (0,1) (1,0) (0,0).
__host__ __device__ constexpr int piece_a(int e) { return e == 0 || e == 4 ? 1 : (e == 2 ? 2 : 0); }
__host__ __device__ constexpr int piece_b(int e) { return e == 1 ? 2 : (e == 0 || e == 3 ? 1 : 0); }
constexpr unsigned kATile = 4096;            // 128 points x 16 rows x 2 B
constexpr unsigned long long kWaitNs = 1000000000ull;  // 1 s per wait

__device__ __forceinline__ unsigned smem_u32(const void* p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// As mbar_try_wait, but the thread may be suspended until the phase
// completes or about `hint_ns` nanoseconds pass, instead of returning at once
// (a waiting warp then does not poll the barrier through the shared-memory
// port).
__device__ __forceinline__ bool mbar_try_wait_suspend(unsigned long long* bar, unsigned parity, unsigned hint_ns) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity), "r"(hint_ns)
        : "memory");
    return ok != 0;
}

// One arrival (release semantics) on an mbarrier, without waiting.
__device__ __forceinline__ void mbar_arrive(unsigned long long* bar) {
    asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Whether the phase has completed, without waiting.
__device__ __forceinline__ bool mbar_test_wait(unsigned long long* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits until the phase with the given parity has completed; false if that
// did not happen within limit_ns (0: kWaitNs).  The pipeline waits take the
// evaluation's limit (kernel parameter wait_ns); the waits that drain a
// failed CTA's MMAs and copies before it frees tensor memory always take
// kWaitNs.
constexpr unsigned kSuspendNs = 20000;
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity, unsigned long long limit_ns = 0) {
    const unsigned long long limit = limit_ns ? limit_ns : kWaitNs;
    // A limit below the suspend hint (finer than the global timer resolves)
    // allows no waiting at all: try_wait may itself block for a
    // system-dependent time, test_wait never does.
    if (limit < kSuspendNs) return mbar_test_wait(bar, parity);
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    while (!mbar_try_wait_suspend(bar, parity, kSuspendNs))
        if (global_ns() - t0 > limit) return false;
    return true;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_alloc(unsigned* slot, unsigned ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)), "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(unsigned taddr, unsigned ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void tc_commit(unsigned long long* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// D[tmem] (+)= A[smem] * B[smem], BF16 inputs, FP32 accumulators.
__device__ __forceinline__ void tc_mma(unsigned d_tmem, unsigned long long adesc, unsigned long long bdesc,
                                       unsigned idesc, unsigned accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}\n" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u)
        : "memory");
}

// Shared-memory matrix descriptor, no swizzle: start address, leading byte
// offset (between core matrices along K), stride byte offset (between core
// matrices along M or N), descriptor version 1.
__device__ __forceinline__ unsigned long long smem_desc(unsigned saddr, unsigned lbo, unsigned sbo) {
    return static_cast<unsigned long long>((saddr >> 4) & 0x3FFFu) |
           (static_cast<unsigned long long>((lbo >> 4) & 0x3FFFu) << 16) |
           (static_cast<unsigned long long>((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both
// MN-major, M = 128, N = n.
__device__ __forceinline__ unsigned instr_desc(int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | (1u << 15) | (1u << 16) | (static_cast<unsigned>(n >> 3) << 17) |
           (static_cast<unsigned>(128 >> 4) << 24);
}

// MG (8, 4 or 2) consecutive FP32 columns of the warp's 32 lanes.
template <int MG>
__device__ __forceinline__ void tmem_ld(unsigned taddr, unsigned (&r)[MG]) {
    if constexpr (MG == 2) {
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0,%1}, [%2];" : "=r"(r[0]), "=r"(r[1]) : "r"(taddr));
    } else if constexpr (MG == 8) {
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                     : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                     : "r"(taddr));
    } else {
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0,%1,%2,%3}, [%4];"
                     : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                     : "r"(taddr));
    }
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
// Orders later uses of r after the preceding wait::ld.
template <int MG>
__device__ __forceinline__ void reg_fence(unsigned (&r)[MG]) {
    if constexpr (MG == 2)
        asm volatile("" : "+r"(r[0]), "+r"(r[1]));
    else if constexpr (MG == 8)
        asm volatile("" : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]));
    else
        asm volatile("" : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]));
}

// One arrival that also expects `bytes` of asynchronous copies on the phase.
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// Tiled tensor copy global -> shared of the box at (x, y, z, w) of a 4-D
// tensor map (a __grid_constant__ parameter); x * element size must be a
// multiple of 16 bytes and the shared address 128-byte aligned.
__device__ __forceinline__ void tma_load_4d(unsigned saddr, const void* map, int x, int y, int z, int w,
                                            unsigned long long* bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
        "[%6];" ::"r"(saddr),
        "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(z), "r"(w), "r"(smem_u32(bar))
        : "memory");
}

// 16-byte shared-memory load at a fixed address (the compiler may not fold a
// later select of the result into the address, which would change the banks
// the warp's lanes touch).
__device__ __forceinline__ float4 lds128(unsigned saddr) {
    float4 v;
    asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "r"(saddr) : "memory");
    return v;
}

__device__ __forceinline__ void cp_async16(unsigned saddr, const void* gmem, bool valid) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(saddr), "l"(gmem), "r"(valid ? 16 : 0)
                 : "memory");
}

__device__ __forceinline__ unsigned bf2_bits(__nv_bfloat162 h) { return *reinterpret_cast<unsigned*>(&h); }

// Three BF16 pieces of 8 FP32 values (x = p0 + p1 + p2 exactly).
__device__ __forceinline__ void split8(const float4& lo, const float4& hi, uint4& p0, uint4& p1, uint4& p2) {
    const float x[8] = {lo.x, lo.y, lo.z, lo.w, hi.x, hi.y, hi.z, hi.w};
    unsigned a[4], b[4], c[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const float u = x[2 * i], v = x[2 * i + 1];
        const __nv_bfloat162 h0 = __floats2bfloat162_rn(u, v);
        const float2 f0 = __bfloat1622float2(h0);
        const float ru = __fsub_rn(u, f0.x), rv = __fsub_rn(v, f0.y);
        const __nv_bfloat162 h1 = __floats2bfloat162_rn(ru, rv);
        const float2 f1 = __bfloat1622float2(h1);
        const __nv_bfloat162 h2 = __floats2bfloat162_rn(__fsub_rn(ru, f1.x), __fsub_rn(rv, f1.y));
        a[i] = bf2_bits(h0);
        b[i] = bf2_bits(h1);
        c[i] = bf2_bits(h2);
    }
    p0 = make_uint4(a[0], a[1], a[2], a[3]);
    p1 = make_uint4(b[0], b[1], b[2], b[3]);
    p2 = make_uint4(c[0], c[1], c[2], c[3]);
}

// Rows of a block put in ascending order of their block maximum (at most
// kSortCap rows; larger blocks keep AO order).
constexpr int kSortCap = 8192;
constexpr int kBuckets = 128;

// Screening and K order of a block's rows, run by all kThreads threads.
// rowmax4 holds the four per-warp maxima of each row (null: keep all rows in
// AO order).  On return perm[0..nk) lists the kept rows (block maximum above
// the threshold; threshold 0 keeps every row) and `sorted` says whether perm
// is in use (blocks of at most `cap` rows); keys and bucket_start are shared
// scratch of cap bytes and kBuckets + 4 ints.
template <typename PermT>
__device__ __forceinline__ int block_row_order(const float* rowmax4, int nk, float threshold, PermT* perm,
                                               int* bucket_start, unsigned char* keys, bool& sorted,
                                               int cap = kSortCap) {
    const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
    // K order: rows in ascending order of their block maximum (a stable
    // counting sort on the FP32 exponent), so that the accumulators are small
    // while most rows are added and the largest terms come last.  The
    // tensor-core accumulation truncates, and its error grows with the
    // magnitude of the accumulator at each step.
    // Rows whose block maximum is not above the screening threshold are left
    // out here (src/ao_screening.hpp:35-50 on the FP32 panels; threshold 0
    // keeps every row).
    sorted = rowmax4 != nullptr && nk <= cap;
    if (sorted) {
        const float4* rmax = reinterpret_cast<const float4*>(rowmax4);
        // Threads beyond kThreads (a CTA's MMA warp) only meet the barriers.
        for (int k = tid; tid < kThreads && k < nk; k += kThreads) {
            const float4 v = rmax[k];
            const float mx = fmaxf(fmaxf(v.x, v.y), fmaxf(v.z, v.w));
            const int e = static_cast<int>((__float_as_uint(mx) >> 23) & 0xffu) - 127 + kBuckets / 2;
            const bool keep = threshold == 0.0f || mx > threshold;
            keys[k] = keep ? static_cast<unsigned char>(e < 0 ? 0 : (e >= kBuckets ? kBuckets - 1 : e)) : 0xffu;
        }
        for (int b = tid; tid < kThreads && b <= kBuckets; b += kThreads) bucket_start[b] = 0;
        __syncthreads();
        for (int k = tid; tid < kThreads && k < nk; k += kThreads)
            if (keys[k] != 0xffu) atomicAdd(&bucket_start[keys[k]], 1);
        __syncthreads();
        if (w == 0) {
            // Exclusive scan of the 128 bucket counts, 4 buckets per lane.
            int c[4], local = 0;
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                c[i] = bucket_start[4 * lane + i];
                local += c[i];
            }
            int incl = local;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += y;
            }
            int run = incl - local;
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                bucket_start[4 * lane + i] = run;
                run += c[i];
            }
            if (lane == 31) bucket_start[kBuckets] = incl;
            __syncwarp();
            // Stable scatter in row order, 32 rows at a time.
            for (int base = 0; base < nk; base += 32) {
                const int k = base + lane;
                const unsigned key = k < nk ? keys[k] : 0xffu;
                const unsigned same = __match_any_sync(0xffffffffu, key);
                const int rank = __popc(same & ((1u << lane) - 1u));
                const int start = key != 0xffu ? bucket_start[key] : 0;
                __syncwarp();
                if (key != 0xffu) {
                    perm[start + rank] = static_cast<PermT>(k);
                    if (rank == __popc(same) - 1) bucket_start[key] = start + rank + 1;
                }
                __syncwarp();
            }
        }
        __syncthreads();
        nk = bucket_start[kBuckets];
    }
    return nk;
}

}  // namespace
}  // namespace kumo_dev
