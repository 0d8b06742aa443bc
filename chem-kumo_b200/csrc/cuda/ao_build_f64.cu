// FP64 AO build.  Compiled with -fmad=false: every product and sum of the AO
// arithmetic is rounded as written, in the reference's order.
#include "ao_build.cuh"

namespace kumo_dev {

template <int ORDER, int P>
static void launch(const AoBuildParams<double>& p, cudaStream_t stream) {
    const size_t smem = sizeof(double) * ((size_t)p.basis.max_count * P * kBlockPoints + (size_t)kMaxPrim * kBlockPoints);
    cudaFuncSetAttribute(ao_build_kernel<double, ORDER, P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    ao_build_kernel<double, ORDER, P><<<p.nblocks, kBlockPoints, smem, stream>>>(p);
}

template <>
void launch_ao_build<double>(const AoBuildParams<double>& p, int order, int npanel, cudaStream_t stream) {
    if (order == 0) launch<0, 1>(p, stream);
    else if (order == 1) launch<1, 4>(p, stream);
    else if (npanel == 5) launch<2, 5>(p, stream);
    else launch<2, 10>(p, stream);
}

}  // namespace kumo_dev
