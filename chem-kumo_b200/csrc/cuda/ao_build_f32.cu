// FP32 AO build of the mixed-precision form (fused multiply-add allowed); the
// cutoff test and the point displacements stay FP64.
#include "ao_build.cuh"

namespace kumo_dev {

template <int ORDER, int P>
static void launch(const AoBuildParams<float>& p, cudaStream_t stream) {
    const size_t smem = sizeof(float) * ((size_t)p.basis.max_count * P * kBlockPoints + (size_t)kMaxPrim * kBlockPoints);
    cudaFuncSetAttribute(ao_build_kernel<float, ORDER, P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    ao_build_kernel<float, ORDER, P><<<p.nblocks, kBlockPoints, smem, stream>>>(p);
}

template <>
void launch_ao_build<float>(const AoBuildParams<float>& p, int order, int npanel, cudaStream_t stream) {
    if (order == 0) launch<0, 1>(p, stream);
    else if (order == 1) launch<1, 4>(p, stream);
    else if (npanel == 5) launch<2, 5>(p, stream);
    else launch<2, 10>(p, stream);
}

}  // namespace kumo_dev
