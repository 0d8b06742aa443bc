// FP64 contraction kernels; see contract.cuh.
//
// AO-MO kernel layout: one CTA per 32 points of a screening block, 8 warps.
// Lane l of every warp owns point l of the 32; warp w owns MOs
// [w*MPT, (w+1)*MPT) of the current chunk of 8*MPT occupied MOs.  The K loop
// walks the block's kept AO rows in tiles of KT, double-buffered in shared
// memory with cp.async: the compacted panels Phi[k][a][32 points] and the
// gathered MO rows C[kept[k]][chunk].  Each thread accumulates
// V_a[mo][point] for its MPT MOs and P panels in registers (DFMA), then folds
// them into per-point partial sums (rho, grad, tau axes, Hessian terms); the
// partials of the 8 warps are summed in a fixed order, so results do not
// depend on scheduling.
#include "func_attr.cuh"
#include <cstdio>
#include <initializer_list>

#include "contract.cuh"

namespace kumo_dev {

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool valid) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    const int n = valid ? 16 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(n));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

template <int P>
struct NQ;
template <>
struct NQ<1> {
    static constexpr int v = 1;
};
template <>
struct NQ<4> {
    static constexpr int v = 7;
};
template <>
struct NQ<5> {
    static constexpr int v = 8;
};
template <>
struct NQ<10> {
    static constexpr int v = 19;
};

// Partial layout: 0 value; 1..3 v0.va; 4..6 va.va; P=5: 7 v0.vlap;
// P=10: 7..12 v0.v_h (xx xy xz yy yz zz), 13..18 va.vc (same pairs).
template <int P, int MPT>
__device__ __forceinline__ void fold_partials(const double (&acc)[P][MPT], double (&q)[NQ<P>::v]) {
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
__device__ __forceinline__ void record_from_partials(const double* f, int ao_order, DevDD& d) {
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
__global__ void __launch_bounds__(256, 1) contract_mo_f64_kernel(const __grid_constant__ ContractMoParams prm) {
    constexpr int MOC = 8 * MPT;
    constexpr int Q = NQ<P>::v;
    extern __shared__ __align__(16) double sm[];
    double* phs = sm;                        // [2][KT][P][32]
    double* cs = phs + 2 * KT * P * 32;      // [2][KT][MOC]
    double* fin = cs + 2 * KT * MOC;         // [2][Q][32]

    const int blk = blockIdx.x >> 2;
    const int j0 = (blockIdx.x & 3) * 32;
    long long start, b;
    int sblock_unused;
    cta_points(prm.first_point, prm.block_size, prm.screen_block, prm.count, blk, start, b, sblock_unused);
    if (j0 >= b) return;
    const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
    const AoScratch<double>& scr = prm.scr;
    const int nk = scr.nkept[blk];
    const double* pbase = scr.panels + (size_t)blk * P * scr.row_stride * kBlockPoints + j0;
    const int* kept = scr.kept + (size_t)blk * scr.row_stride;

    for (int ci = 0; ci < prm.nchannels; ++ci) {
        const MoChannel ch = prm.ch[ci];
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
                double* ph = phs + buf * KT * P * 32;
                for (int c = tid; c < KT * P * 16; c += 256) {
                    const int kk = c / (P * 16), rem = c % (P * 16), cc = rem / 16, jj = (rem % 16) * 2;
                    const bool ok = k0 + kk < nk;
                    const double* src = pbase + ((size_t)cc * scr.row_stride + (ok ? k0 + kk : 0)) * kBlockPoints + jj;
                    cp_async16(ph + (kk * P + cc) * 32 + jj, src, ok);
                }
                double* cb = cs + buf * KT * MOC;
                for (int c = tid; c < KT * MOC / 2; c += 256) {
                    const int kk = c / (MOC / 2), col = (c % (MOC / 2)) * 2;
                    const bool ok = (k0 + kk < nk) && (mo0 + col < ch.ldc);
                    const double* src = ch.ct + (size_t)(ok ? kept[k0 + kk] : 0) * ch.ldc + (ok ? mo0 + col : 0);
                    cp_async16(cb + kk * MOC + col, src, ok);
                }
                cp_async_commit();
            };
            if (ntiles > 0) load_tile(0, 0);
            for (int t = 0; t < ntiles; ++t) {
                if (t + 1 < ntiles) {
                    load_tile(t + 1, (t + 1) & 1);
                    cp_async_wait<1>();
                } else {
                    cp_async_wait<0>();
                }
                __syncthreads();
                const double* ph = phs + (t & 1) * KT * P * 32;
                const double* cb = cs + (t & 1) * KT * MOC + w * MPT;
#pragma unroll 4
                for (int kk = 0; kk < KT; ++kk) {
                    double phi[P];
#pragma unroll
                    for (int c = 0; c < P; ++c) phi[c] = ph[(kk * P + c) * 32 + lane];
                    double cv[MPT];
#pragma unroll
                    for (int t2 = 0; t2 < MPT / 2; ++t2) {
                        const double2 v = reinterpret_cast<const double2*>(cb + kk * MOC)[t2];
                        cv[2 * t2] = v.x;
                        cv[2 * t2 + 1] = v.y;
                    }
#pragma unroll
                    for (int c = 0; c < P; ++c)
#pragma unroll
                        for (int tt = 0; tt < MPT; ++tt) acc[c][tt] = fma(phi[c], cv[tt], acc[c][tt]);
                }
                __syncthreads();
            }
            fold_partials<P, MPT>(acc, q);
        }
        // Sum the partials of the 8 warps (fixed order) into fin[ci].
        double* red = phs;  // [8][Q][32], the tile buffers are idle here
#pragma unroll
        for (int i = 0; i < Q; ++i) red[(w * Q + i) * 32 + lane] = q[i];
        __syncthreads();
        for (int i = tid; i < Q * 32; i += 256) {
            const int qi = i / 32, l = i % 32;
            double s = red[(0 * Q + qi) * 32 + l];
#pragma unroll
            for (int ww = 1; ww < 8; ++ww) s += red[(ww * Q + qi) * 32 + l];
            fin[(ci * Q + qi) * 32 + l] = s;
        }
        __syncthreads();
    }

    if (w != 0 || j0 + lane >= b) return;
    double f[Q];
    DevDD alpha, beta;
    dd_zero(alpha);
    dd_zero(beta);
    for (int ci = 0; ci < prm.nchannels; ++ci) {
        for (int i = 0; i < Q; ++i) f[i] = fin[(ci * Q + i) * 32 + lane];
        if (prm.ch[ci].role == 1)
            record_from_partials<P>(f, prm.ao_order, alpha);
        else
            record_from_partials<P>(f, prm.ao_order, beta);
    }
    if (prm.beta_is_alpha) beta = alpha;
    store_point(prm.spec, alpha, beta, P == 10 && prm.ao_order == 2, start + j0 + lane);
}

template <int P, int MPT, int KT>
static void launch_mo(const ContractMoParams& p, cudaStream_t stream) {
    constexpr int MOC = 8 * MPT;
    constexpr int Q = NQ<P>::v;
    const size_t smem = sizeof(double) * (size_t)(2 * KT * P * 32 + 2 * KT * MOC + 2 * Q * 32);
    KUMO_REGISTER_KERNEL(contract_mo_f64_kernel<P, MPT, KT>);
    ensure_dynamic_smem(reinterpret_cast<const void*>(contract_mo_f64_kernel<P, MPT, KT>), (int)smem);
    contract_mo_f64_kernel<P, MPT, KT><<<p.nblocks * 4, 256, smem, stream>>>(p);
}

// MOs per warp and pass: the fewest passes the largest width allows, then the
// narrowest listed width that covers the channel's occupied MOs in that many
// passes (MO columns past the last occupied one are zero and cost as much as
// real ones: 76 MOs in one pass of 8 x 16 columns would be 40% padding).
static int mo_width(int nocc, std::initializer_list<int> widths) {
    const int widest = *(widths.end() - 1);
    const int passes = nocc > 0 ? (nocc + 8 * widest - 1) / (8 * widest) : 1;
    const int need = (nocc + 8 * passes - 1) / (8 * passes);
    for (int w : widths)
        if (w >= need) return w;
    return widest;
}

template <int P>
static void launch_mo_width(const ContractMoParams& p, int width, cudaStream_t stream) {
    switch (width) {
        case 4: launch_mo<P, 4, 16>(p, stream); break;
        case 8: launch_mo<P, 8, 16>(p, stream); break;
        case 10: launch_mo<P, 10, 16>(p, stream); break;
        case 12: launch_mo<P, 12, 16>(p, stream); break;
        default: launch_mo<P, 16, 16>(p, stream); break;
    }
}

void launch_contract_mo_f64(const ContractMoParams& p, int npanel, cudaStream_t stream) {
    int nocc = 0;
    for (int i = 0; i < p.nchannels; ++i) nocc = p.ch[i].nocc > nocc ? p.ch[i].nocc : nocc;
    switch (npanel) {
        case 1: launch_mo_width<1>(p, mo_width(nocc, {4, 8, 10, 12, 16}), stream); break;
        case 4: launch_mo_width<4>(p, mo_width(nocc, {4, 8, 10, 12, 16}), stream); break;
        case 5: launch_mo_width<5>(p, mo_width(nocc, {4, 8, 10, 12, 16}), stream); break;
        case 10:
            switch (mo_width(nocc, {4, 6, 8})) {
                case 4: launch_mo<10, 4, 8>(p, stream); break;
                case 6: launch_mo<10, 6, 8>(p, stream); break;
                default: launch_mo<10, 8, 8>(p, stream); break;
            }
            break;
        default: break;
    }
}

// Orbital-energy sums: one CTA per 32 points of a block, 8 warps x 16
// columns of each 128-column chunk, cp.async double-buffered tiles of the AO
// values and of the column rows; per point the ten set sums are reduced
// across the warps in a fixed order and the fields are stored.
template <int KT>
__global__ void __launch_bounds__(256, 1) orbital_energy_f64_kernel(const __grid_constant__ OrbitalEnergyParams prm) {
    constexpr int MPT = 16;
    constexpr int MOC = 8 * MPT;
    constexpr int NS = kOrbitalEnergySets;
    extern __shared__ __align__(16) double sm[];
    double* phs = sm;                  // [2][KT][32]
    double* cs = phs + 2 * KT * 32;    // [2][KT][MOC]
    double* red = cs + 2 * KT * MOC;   // [8][2 NS][32]

    const int blk = blockIdx.x >> 2;
    const int j0 = (blockIdx.x & 3) * 32;
    long long start, b;
    int sblock_unused;
    cta_points(prm.first_point, prm.block_size, prm.screen_block, prm.count, blk, start, b, sblock_unused);
    if (j0 >= b) return;
    const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
    const AoScratch<double>& scr = prm.scr;
    const int nk = scr.nkept[blk];
    const double* pbase = scr.panels + (size_t)blk * scr.row_stride * kBlockPoints + j0;
    const int* kept = scr.kept + (size_t)blk * scr.row_stride;

    double D[NS], E[NS];
#pragma unroll
    for (int s = 0; s < NS; ++s) D[s] = E[s] = 0.0;
    const int ntiles = (nk + KT - 1) / KT;
    for (int chunk = 0; chunk < prm.nchunks; ++chunk) {
        const int mo0 = chunk * MOC;
        double acc[MPT];
#pragma unroll
        for (int t = 0; t < MPT; ++t) acc[t] = 0.0;
        auto load_tile = [&](int tile, int buf) {
            const int k0 = tile * KT;
            double* ph = phs + buf * KT * 32;
            for (int c = tid; c < KT * 16; c += 256) {
                const int kk = c / 16, jj = (c % 16) * 2;
                const bool ok = k0 + kk < nk;
                cp_async16(ph + kk * 32 + jj, pbase + (size_t)(ok ? k0 + kk : 0) * kBlockPoints + jj, ok);
            }
            double* cb = cs + buf * KT * MOC;
            for (int c = tid; c < KT * MOC / 2; c += 256) {
                const int kk = c / (MOC / 2), col = (c % (MOC / 2)) * 2;
                const bool ok = k0 + kk < nk;
                const double* src = prm.w + (size_t)(ok ? kept[k0 + kk] : 0) * prm.ldw + mo0 + col;
                cp_async16(cb + kk * MOC + col, src, ok);
            }
            cp_async_commit();
        };
        if (ntiles > 0) load_tile(0, 0);
        for (int t = 0; t < ntiles; ++t) {
            if (t + 1 < ntiles) {
                load_tile(t + 1, (t + 1) & 1);
                cp_async_wait<1>();
            } else {
                cp_async_wait<0>();
            }
            __syncthreads();
            const double* ph = phs + (t & 1) * KT * 32;
            const double* cb = cs + (t & 1) * KT * MOC + w * MPT;
#pragma unroll 4
            for (int kk = 0; kk < KT; ++kk) {
                const double phi = ph[kk * 32 + lane];
#pragma unroll
                for (int t2 = 0; t2 < MPT / 2; ++t2) {
                    const double2 v = reinterpret_cast<const double2*>(cb + kk * MOC)[t2];
                    acc[2 * t2] = fma(phi, v.x, acc[2 * t2]);
                    acc[2 * t2 + 1] = fma(phi, v.y, acc[2 * t2 + 1]);
                }
            }
            __syncthreads();
        }
        const int set = prm.chunk_set[chunk];
        const double* e = prm.col_energy + mo0 + w * MPT;
        double d = 0.0, en = 0.0;
#pragma unroll
        for (int t = 0; t < MPT; ++t) {
            const double x2 = acc[t] * acc[t];
            d += x2;
            en += e[t] * x2;
        }
#pragma unroll
        for (int s = 0; s < NS; ++s)
            if (s == set) {
                D[s] += d;
                E[s] += en;
            }
    }
#pragma unroll
    for (int s = 0; s < NS; ++s) {
        red[(w * 2 * NS + s) * 32 + lane] = D[s];
        red[(w * 2 * NS + NS + s) * 32 + lane] = E[s];
    }
    __syncthreads();
    if (w != 0 || j0 + lane >= b) return;
    double tot[2 * NS];
#pragma unroll
    for (int i = 0; i < 2 * NS; ++i) {
        double v = red[i * 32 + lane];
#pragma unroll
        for (int ww = 1; ww < 8; ++ww) v += red[(ww * 2 * NS + i) * 32 + lane];
        tot[i] = v;
    }
    // store_orbital_energy_block (src/evaluator.cpp:485-516).
    const double rho = tot[0];
    const double alie = rho > 0.0 ? tot[NS + 0] / rho : 0.0;
    double lea = 0.0, attachment = 0.0;
    if (prm.have_virtuals) {
        const double vir = tot[1];
        lea = vir > 0.0 ? -tot[NS + 1] / vir : 0.0;
        attachment = rho > 0.0 ? tot[NS + 2] / rho : 0.0;
    }
    double plus = 0.0, minus = 0.0;
    if (prm.have_fukui) {
        plus = tot[3];
        minus = tot[4];
    }
    const long long q = start + j0 + lane - prm.out_base;
    for (int o = 0; o < prm.nout; ++o) {
        double v;
        switch (prm.kinds[o]) {
            case 19: v = alie; break;                  // AverageLocalIonizationEnergy
            case 20: v = lea; break;                   // LocalElectronAffinity
            case 21: v = attachment; break;            // LocalElectronAttachmentEnergy
            case 22: v = 0.5 * (alie + lea); break;    // LocalElectronegativity
            case 23: v = 0.5 * (alie - lea); break;    // LocalHardness
            case 26: v = plus; break;                  // OrbitalWeightedFukuiPlus
            case 27: v = minus; break;                 // OrbitalWeightedFukuiMinus
            case 28: v = 0.5 * (plus + minus); break;  // OrbitalWeightedFukuiZero
            default: v = plus - minus; break;          // OrbitalWeightedDualDescriptor
        }
        prm.outs[o][q] = v;
    }
}

void launch_orbital_energy_f64(const OrbitalEnergyParams& p, cudaStream_t stream) {
    constexpr int KT = 16;
    const size_t smem = sizeof(double) * (size_t)(2 * KT * 32 + 2 * KT * 128 + 8 * 2 * kOrbitalEnergySets * 32);
    KUMO_REGISTER_KERNEL(orbital_energy_f64_kernel<KT>);
    ensure_dynamic_smem(reinterpret_cast<const void*>(orbital_energy_f64_kernel<KT>), (int)smem);
    orbital_energy_f64_kernel<KT><<<p.nblocks * 4, 256, smem, stream>>>(p);
}

// MO amplitudes (and derivatives) of up to 8 selected MOs: thread per point,
// summing over every AO in order, as selected^T * phi.
__global__ void __launch_bounds__(128) orbitals_f64_kernel(const __grid_constant__ OrbitalParams prm) {
    const int blk = blockIdx.x;
    const int j = threadIdx.x;
    const long long start = prm.first_point + (long long)blk * prm.block_size;
    long long b = prm.count - start;
    if (b > prm.block_size) b = prm.block_size;
    if (j >= b) return;
    const AoScratch<double>& scr = prm.scr;
    const double* base = scr.panels + (size_t)blk * prm.npanel * scr.row_stride * kBlockPoints + j;
    const int* kept = scr.kept + (size_t)blk * scr.row_stride;
    const int nk = scr.nkept[blk];
    const long long q = start + j;
    for (int s = 0; s < prm.nsel; ++s) {
        const double* c = prm.coef[s];
        for (int ch = 0; ch < prm.nchan[s]; ++ch) {
            const int panel = prm.first_channel[s] + ch;
            const double* ph = base + (size_t)panel * scr.row_stride * kBlockPoints;
            // Kept rows in AO order: the AOs left out are cutoff zeros here.
            double acc = 0.0;
            for (int k = 0; k < nk; ++k) acc += c[kept[k]] * ph[(size_t)k * kBlockPoints];
            prm.out[s][ch * prm.stride + (q - prm.out_base)] = acc;
        }
    }
}

void launch_orbitals_f64(const OrbitalParams& p, cudaStream_t stream) {
    KUMO_REGISTER_KERNEL(orbitals_f64_kernel);
    orbitals_f64_kernel<<<p.nblocks, 128, 0, stream>>>(p);
}

}  // namespace kumo_dev

namespace kumo_dev {

// AO-P kernel: one CTA per 32 points of a block, 8 warps; warp w owns RPT
// rows r of the current row chunk and accumulates Y[q][r] (q < NY panels of
// P*Phi) for its lane's point over the K loop of kept AOs; the tiles of
// Phi[k][q][32 points] and P[kept[k]][kept[r]] are double-buffered with
// cp.async.  After the K loop each thread folds its rows into the per-point
// partial sums with the row's own panels.
template <int P, bool VALUES, int RPT, int KT>
__global__ void __launch_bounds__(256, 1) contract_p_f64_kernel(const __grid_constant__ ContractPParams prm) {
    constexpr int NY = VALUES ? 1 : 4;
    constexpr int RC = 8 * RPT;
    constexpr int Q = NQ<P>::v;
    extern __shared__ __align__(16) double sm[];
    double* phs = sm;                    // [2][KT][NY][32]
    double* ps = phs + 2 * KT * NY * 32; // [2][KT][RC]
    double* fin = ps + 2 * KT * RC;      // [2][Q][32]
    int* s_rows = reinterpret_cast<int*>(fin + 2 * Q * 32);  // [RC] kept AO index of each chunk row

    const int blk = blockIdx.x >> 2;
    const int j0 = (blockIdx.x & 3) * 32;
    long long start, b;
    int sblock_unused;
    cta_points(prm.first_point, prm.block_size, prm.screen_block, prm.count, blk, start, b, sblock_unused);
    if (j0 >= b) return;
    const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
    const AoScratch<double>& scr = prm.scr;
    const int nk = scr.nkept[blk];
    const double* pbase = scr.panels + (size_t)blk * P * scr.row_stride * kBlockPoints + j0;
    const int* kept = scr.kept + (size_t)blk * scr.row_stride;
    const int n = prm.nao;

    // Matrices: VALUES -> one (the component's); otherwise total and/or spin.
    int nmat = 0;
    const double* mats[2];
    int roles[2];
    if (VALUES) {
        mats[0] = prm.density_component == 3 ? prm.p_spin : prm.p_total;
        roles[0] = prm.density_component;
        nmat = 1;
    } else {
        if (prm.total_needed) {
            mats[nmat] = prm.p_total;
            roles[nmat++] = 0;
        }
        if (prm.spin_needed) {
            mats[nmat] = prm.p_spin;
            roles[nmat++] = 3;
        }
    }
    for (int mi = 0; mi < nmat; ++mi) {
        const double* Pm = mats[mi];
        // Alpha / beta grid densities use 0.5 * (P_total +/- P_spin).
        const int comp = roles[mi];
        const bool half = VALUES && (comp == 1 || comp == 2);
        const double sign = comp == 2 ? -1.0 : 1.0;
        double q[Q];
#pragma unroll
        for (int i = 0; i < Q; ++i) q[i] = 0.0;
        for (int r0 = 0; r0 < nk; r0 += RC) {
            for (int i = tid; i < RC; i += 256) s_rows[i] = r0 + i < nk ? kept[r0 + i] : -1;
            __syncthreads();
            double acc[NY][RPT];
#pragma unroll
            for (int c = 0; c < NY; ++c)
#pragma unroll
                for (int t = 0; t < RPT; ++t) acc[c][t] = 0.0;
            const int ntiles = (nk + KT - 1) / KT;
            auto load_tile = [&](int tile, int buf) {
                const int k0 = tile * KT;
                double* ph = phs + buf * KT * NY * 32;
                for (int c = tid; c < KT * NY * 16; c += 256) {
                    const int kk = c / (NY * 16), rem = c % (NY * 16), cc = rem / 16, jj = (rem % 16) * 2;
                    const bool ok = k0 + kk < nk;
                    const double* src = pbase + ((size_t)cc * scr.row_stride + (ok ? k0 + kk : 0)) * kBlockPoints + jj;
                    cp_async16(ph + (kk * NY + cc) * 32 + jj, src, ok);
                }
                cp_async_commit();
                double* pb = ps + buf * KT * RC;
                for (int c = tid; c < KT * RC; c += 256) {
                    const int kk = c / RC, rr = c % RC;
                    const int col = k0 + kk < nk ? kept[k0 + kk] : -1;
                    const int row = s_rows[rr];
                    double v = 0.0;
                    if (col >= 0 && row >= 0) {
                        v = Pm[(size_t)col * n + row];
                        if (half) v = 0.5 * (prm.p_total[(size_t)col * n + row] + sign * prm.p_spin[(size_t)col * n + row]);
                    }
                    pb[kk * RC + rr] = v;
                }
            };
            if (ntiles > 0) load_tile(0, 0);
            for (int t = 0; t < ntiles; ++t) {
                if (t + 1 < ntiles) {
                    load_tile(t + 1, (t + 1) & 1);
                    cp_async_wait<1>();
                } else {
                    cp_async_wait<0>();
                }
                __syncthreads();
                const double* ph = phs + (t & 1) * KT * NY * 32;
                const double* pb = ps + (t & 1) * KT * RC + w * RPT;
#pragma unroll 4
                for (int kk = 0; kk < KT; ++kk) {
                    double phi[NY];
#pragma unroll
                    for (int c = 0; c < NY; ++c) phi[c] = ph[(kk * NY + c) * 32 + lane];
                    double pv[RPT];
#pragma unroll
                    for (int t2 = 0; t2 < RPT / 2; ++t2) {
                        const double2 v = reinterpret_cast<const double2*>(pb + kk * RC)[t2];
                        pv[2 * t2] = v.x;
                        pv[2 * t2 + 1] = v.y;
                    }
#pragma unroll
                    for (int c = 0; c < NY; ++c)
#pragma unroll
                        for (int tt = 0; tt < RPT; ++tt) acc[c][tt] = fma(pv[tt], phi[c], acc[c][tt]);
                }
                __syncthreads();
            }
            // Fold rows r = r0 + w*RPT + t into the partials.
#pragma unroll
            for (int t = 0; t < RPT; ++t) {
                const int r = r0 + w * RPT + t;
                if (r >= nk) break;
                const double* row = pbase + (size_t)r * kBlockPoints + lane;
                const size_t ps_ = (size_t)scr.row_stride * kBlockPoints;
                const double f0 = row[0];
                q[0] += f0 * acc[0][t];
                if constexpr (!VALUES) {
                    double fa[3];
#pragma unroll
                    for (int a = 0; a < 3; ++a) {
                        fa[a] = row[(1 + a) * ps_];
                        q[1 + a] += fa[a] * acc[0][t];
                        q[4 + a] += fa[a] * acc[1 + a][t];
                    }
                    if constexpr (P == 5) q[7] += row[4 * ps_] * acc[0][t];
                    if constexpr (P == 10) {
                        constexpr int pa[6] = {0, 0, 0, 1, 1, 2}, pc[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
                        for (int h = 0; h < 6; ++h) {
                            q[7 + h] += row[(4 + h) * ps_] * acc[0][t];
                            q[13 + h] += fa[pa[h]] * acc[1 + pc[h]][t];
                        }
                    }
                }
            }
            __syncthreads();
        }
        double* red = phs;
#pragma unroll
        for (int i = 0; i < Q; ++i) red[(w * Q + i) * 32 + lane] = q[i];
        __syncthreads();
        for (int i = tid; i < Q * 32; i += 256) {
            const int qi = i / 32, l = i % 32;
            double s = red[(0 * Q + qi) * 32 + l];
#pragma unroll
            for (int ww = 1; ww < 8; ++ww) s += red[(ww * Q + qi) * 32 + l];
            fin[(mi * Q + qi) * 32 + l] = s;
        }
        __syncthreads();
    }

    if (w != 0 || j0 + lane >= b) return;
    const long long qpt = start + j0 + lane;
    if (VALUES) {
        prm.spec.props[0].out[qpt - prm.spec.out_base] = fin[lane];
        return;
    }
    double f[Q];
    DevDD t, s;
    dd_zero(t);
    dd_zero(s);
    for (int mi = 0; mi < nmat; ++mi) {
        for (int i = 0; i < Q; ++i) f[i] = fin[(mi * Q + i) * 32 + lane];
        record_from_partials<P>(f, prm.ao_order, roles[mi] == 0 ? t : s);
    }
    const bool full = P == 10 && prm.ao_order == 2;
    DevDD comp[4];
    comp[0] = t;
    comp[3] = s;
    comp[1] = dd_combine(t, s, 1.0, 0.5, full);
    comp[2] = dd_combine(t, s, -1.0, 0.5, full);
    store_point(prm.spec, comp, qpt);
}

template <int P, bool VALUES, int RPT, int KT>
static void launch_p(const ContractPParams& p, cudaStream_t stream) {
    constexpr int NY = VALUES ? 1 : 4;
    constexpr int RC = 8 * RPT;
    constexpr int Q = NQ<P>::v;
    const size_t smem = sizeof(double) * (size_t)(2 * KT * NY * 32 + 2 * KT * RC + 2 * Q * 32) + sizeof(int) * RC;
    static_assert(8 * Q * 32 <= 2 * KT * NY * 32 || VALUES, "reduction buffer must fit the tile buffers");
    KUMO_REGISTER_KERNEL(contract_p_f64_kernel<P, VALUES, RPT, KT>);
    ensure_dynamic_smem(reinterpret_cast<const void*>(contract_p_f64_kernel<P, VALUES, RPT, KT>), (int)smem);
    contract_p_f64_kernel<P, VALUES, RPT, KT><<<p.nblocks * 4, 256, smem, stream>>>(p);
}

void launch_contract_p_f64(const ContractPParams& p, int npanel, cudaStream_t stream) {
    switch (npanel) {
        case 4: launch_p<4, false, 16, 16>(p, stream); break;
        case 5: launch_p<5, false, 16, 16>(p, stream); break;
        case 10: launch_p<10, false, 16, 32>(p, stream); break;
        default: break;
    }
}

void launch_density_values_f64(const ContractPParams& p, cudaStream_t stream) {
    launch_p<1, true, 32, 32>(p, stream);
}

}  // namespace kumo_dev
