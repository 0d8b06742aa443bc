// FP64 AO build.  Compiled with -fmad=false: every product and sum of the AO
// arithmetic is rounded as written, in the reference's order.
#include "func_attr.cuh"
#include "ao_build.cuh"

namespace kumo_dev {

template <int ORDER, int P, int MAXL>
static void launch(const AoBuildParams<double>& p, cudaStream_t stream) {
    const size_t smem = sizeof(double) * ((size_t)p.basis.max_count * P * kBlockPoints + (size_t)kMaxPrim * kBlockPoints) +
                        sizeof(int) * (size_t)p.basis.nblocks;
    KUMO_REGISTER_KERNEL(ao_build_kernel<double, ORDER, P, MAXL>);
    ensure_dynamic_smem(reinterpret_cast<const void*>(ao_build_kernel<double, ORDER, P, MAXL>), (int)smem);
    ao_build_kernel<double, ORDER, P, MAXL><<<p.nblocks, kBlockPoints, smem, stream>>>(p);
}

template <int MAXL>
static void dispatch(const AoBuildParams<double>& p, int order, int npanel, cudaStream_t stream) {
    if (order == 0) launch<0, 1, MAXL>(p, stream);
    else if (order == 1) launch<1, 4, MAXL>(p, stream);
    else if (npanel == 5) launch<2, 5, MAXL>(p, stream);
    else launch<2, 10, MAXL>(p, stream);
}

template <>
void launch_ao_build<double>(const AoBuildParams<double>& p, int order, int npanel, cudaStream_t stream) {
    if (p.basis.max_l <= 2) dispatch<2>(p, order, npanel, stream);
    else if (p.basis.max_l == 3) dispatch<3>(p, order, npanel, stream);
    else dispatch<4>(p, order, npanel, stream);
}

}  // namespace kumo_dev
