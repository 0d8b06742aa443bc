// Mixed-precision contraction of the AO-MO path on the fifth-generation
// tensor cores: FP32 AO panels and FP64 MO coefficients are each split into
// three BF16 pieces, the six products whose pieces sum to order <= 2 are
// accumulated by tcgen05.mma in FP32 in tensor memory, and the per-point
// reductions (rho, grad, tau, Laplacian/Hessian) and fields are done in FP64.
#pragma once

#include <cstdint>

#include "ao_mixed.cuh"
#include "fields.cuh"
#include "kumo_device.cuh"

namespace kumo_dev {

struct MoChannelTC {
    const std::uint16_t* cs = nullptr;  // [3][nao][ldn] BF16 pieces, MO contiguous
    long long piece_stride = 0;         // nao * ldn
    int ldn = 0;                        // multiple of 16, >= nocc
    int nocc = 0;
    int role = 0;  // 1 alpha, 2 beta
    const double* c64 = nullptr;  // FP64 coefficients [nao][ld64] (rows padded to a multiple of 4 MOs)
    int ld64 = 0;
};

struct ContractMixedParams {
    // AO rows of the wave's blocks (ao_mixed layout, rowmax with 4 entries per row).
    AoScratch<float> scr;
    long long first_point = 0;
    long long block_size = 128;
    long long count = 0;
    int nblocks = 0;
    int nchannels = 0;
    MoChannelTC ch[2];
    int beta_is_alpha = 0;
    int ao_order = 2;
    int ncols = 16;       // MO columns per pass (multiple of 16, npanel * ncols <= 512)
    int groups = 1;       // accumulator groups (K steps round-robin), groups * npanel * ncols <= 512
    int tmem_cols = 32;   // power of two >= groups * npanel * ncols
    float threshold = 0.0f;      // screening threshold on the rows' block maxima
    FieldSpec spec;
    unsigned* status = nullptr;  // set nonzero if a pipeline wait ran out
    // Rows at the end of each block's K order (largest block maxima) that the
    // bulk-copy kernel adds in FP64 with ch[].c64 instead of on the tensor
    // cores (0: all rows on the tensor cores), with their AO values computed
    // in FP64 from the basis at the block's points.
    int exact_rows = 0;
    // Only rows whose block maximum reaches exact_min are taken exact (0: any
    // row), so blocks whose rows are all small skip the FP64 epilogue.
    float exact_min = 0.0f;
    PointSource src;        // the evaluation's points (for the exact rows)
    DevBasis basis;         // FP64 exponents and weights (for the exact rows)
    // Limit of each tensor-core pipeline wait in ns (0: one second); a wait
    // that runs out sets *status and the CTA stores NaN for its points.
    unsigned long long wait_ns = 0;
};

// AO-P form (density_derivatives_shared): Y = P[kept, kept] Phi[kept, 0..3]
// on the tensor cores, folded with the FP32 panels (4, 5 or 10 of them).
struct ContractPMixedParams {
    AoScratch<float> scr;  // ao_mixed layout
    long long first_point = 0;
    long long block_size = 128;
    long long count = 0;
    int nblocks = 0;
    int nao = 0;
    const std::uint16_t* p_total_s = nullptr;  // [nao][nao][4]: BF16 pieces 0..2 of P_total and a zero
    const std::uint16_t* p_spin_s = nullptr;   // same for P_spin
    int total_needed = 0;
    int spin_needed = 0;
    int ao_order = 2;
    // Bit 0 (P_total) and bit 1 (P_spin): that matrix's components need
    // values only, so only Y_0 = Phi_0 P is formed and folded.
    int value_only = 0;
    float threshold = 0.0f;
    int sort_cap = 0;  // rows the row-order arrays hold (set at launch)
    FieldSpec spec;
    unsigned* status = nullptr;
    // Limit of each tensor-core pipeline wait in ns (0: one second); a wait
    // that runs out sets *status and the CTA stores NaN for its points.
    unsigned long long wait_ns = 0;
};

void launch_contract_p_mixed(const ContractPMixedParams& p, int npanel, cudaStream_t stream);

// MO columns per pass, accumulator groups and tensor-memory columns for
// npanel panels and at most nocc16 (a multiple of 16) occupied MOs per channel.
void mixed_columns(int npanel, int nocc16, int& ncols, int& groups, int& tmem_cols);

// Device word the contraction sets when a pipeline wait runs out (per device),
// and a synchronous read-and-clear of it.
unsigned* pipeline_status_word();
unsigned take_pipeline_status();

void launch_contract_mixed(const ContractMixedParams& p, int npanel, cudaStream_t stream);

// Copies the FP64 normalisation tables of the exact rows to the current
// device: g[l][k] (Cartesian component k of order l, Gaussian order) and
// tg[l - 2][m * nc + k] = T[m][k] g[l][k] of the Cartesian-to-pure
// transforms.  Synchronous; call outside stream capture, before the first
// mixed contraction on the device.
void upload_exact_tables(const double (&g)[kMaxL + 1][15], const double (&tg)[3][135]);

// Fused form of the mixed AO-MO path: the FP32 AO rows of each K step are
// computed in the contraction kernel itself (no panels in global memory).
// Rows are those of the AO blocks whose cutoff sphere reaches the point
// block, in ascending order of a bound of their radial part over the block;
// the K steps hold whole AO blocks (zero rows pad a step).
constexpr int kFusedMaxShells = 2048;

struct ContractFusedParams {
    AoMixedParams ao;  // basis, primitives, points, first_point, block_size, nblocks, tpure, gcart
    long long count = 0;
    int nchannels = 0;
    MoChannelTC ch[2];
    int beta_is_alpha = 0;
    int ao_order = 2;
    int ncols = 16;
    int groups = 1;
    int tmem_cols = 32;
    FieldSpec spec;
    unsigned* status = nullptr;
    int* nrows = nullptr;  // optional: AO rows contracted per block (for the profiler)
    // Limit of each tensor-core pipeline wait in ns (0: one second); a wait
    // that runs out sets *status and the CTA stores NaN for its points.
    unsigned long long wait_ns = 0;
};

bool contract_fused_supported(int npanel, int nshells);
void launch_contract_fused(const ContractFusedParams& p, int npanel, cudaStream_t stream);

}  // namespace kumo_dev
