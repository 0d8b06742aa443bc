// Mixed-precision contraction of the AO-MO path: FP32 AO panels and FP32 MO
// coefficients, products accumulated in FP32 per K tile, and the per-point
// reductions (rho, grad, tau, Laplacian/Hessian) and fields in FP64.
#pragma once

#include "fields.cuh"
#include "kumo_device.cuh"

namespace kumo_dev {

struct MoChannelF {
    const float* ct = nullptr;  // [nao][ldc], MO contiguous
    int ldc = 0;
    int nocc = 0;
    int role = 0;  // 1 alpha, 2 beta
};

struct ContractMixedParams {
    AoScratch<float> scr;
    long long first_point = 0;
    long long block_size = 128;
    long long count = 0;
    int nblocks = 0;
    int nchannels = 0;
    MoChannelF ch[2];
    int beta_is_alpha = 0;
    int ao_order = 2;
    FieldSpec spec;
};

void launch_contract_mixed(const ContractMixedParams& p, int npanel, cudaStream_t stream);

}  // namespace kumo_dev
