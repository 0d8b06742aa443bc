// Allocation-free evaluation at device points (kumo_evaluate_points_noalloc).
//
// Who needs it: some hosts cannot let a library call cudaMalloc.  A serving
// process that budgets every byte of HBM for its own admission control, or
// an application whose memory manager owns the device and forbids foreign
// allocations, must run the evaluator inside memory it already controls;
// cudaMalloc can also block until the device is idle, which stalls the
// host's other streams.  For such callers this entry point runs the FP64
// AO-MO point path (AO build with screening, then the contraction with its
// field epilogue) with its AO scratch in a fixed array that this library
// reserves once, in every GPU that loads it, until the process exits.
//
// The caller passes everything else: a molecule whose device copy already
// exists (made by any earlier evaluation of that molecule on this device),
// the points and the outputs, all in device memory.
//
// Use rules:
//  - the first call on each device looks up the scratch array's device
//    address (cudaGetSymbolAddress); make that first call before any stream
//    capture;
//  - every call shares the one array: calls whose work overlaps on the GPU
//    (different streams, or different host threads) race and corrupt each
//    other's results, so serialize them;
//  - the array keeps whatever the last call left in it; nothing in it has to
//    start at zero (each wave writes every entry it later reads);
//  - a molecule that needs more than the whole array for one 128-point block
//    is rejected with KUMO_INVALID_ARGUMENT.
#include <cstring>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "../cuda/contract.cuh"
#include "chem/kumo/evaluator.hpp"
#include "device_state.hpp"
#include "kumo_b200.h"
#include "plan.hpp"

struct kumo_molecule {
    chem::kumo::Molecule mol;
};

namespace {

using namespace chem::kumo;

// Size of the fixed AO scratch of the allocation-free entry point.
constexpr std::size_t kNoAllocScratchBytes = std::size_t(64) << 20;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
void* g_scratch_address[kMaxDevices] = {};

// Device address of the scratch array on the current device (looked up once
// per device, with that device current).
void* scratch_address() {
    int dev = 0;
    detail::check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices) throw std::runtime_error("device index out of range for the scratch table");
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_address[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) detail::throw_cuda(e, "cudaGetSymbolAddress (no-allocation scratch)");
        g_scratch_address[dev] = p;
    }
    return g_scratch_address[dev];
}

void put(char* err, size_t errlen, const std::string& msg) {
    if (err && errlen) {
        const size_t n = std::min(errlen - 1, msg.size());
        std::memcpy(err, msg.data(), n);
        err[n] = '\0';
    }
}

bool point_path_kind(PropertyKind k) {
    return !detail::is_orbital_kind(k) && !detail::is_orbital_energy_kind(k) && k != PropertyKind::ElectrostaticPotential;
}

bool needs_hessian(PropertyKind k) {
    return k == PropertyKind::Hessian || k == PropertyKind::SignLambda2Density ||
           k == PropertyKind::DensityOverlapRegionsIndicator || k == PropertyKind::HamiltonianKineticEnergyComponents;
}

void run(const kumo_molecule* m, const kumo_options* opt, const double* device_points, long long npoints,
         const kumo_property* props, int nprops, double* const* outputs, void* stream) {
    if (!m) throw std::invalid_argument("null molecule");
    if (npoints < 0 || (npoints > 0 && !device_points)) throw std::invalid_argument("invalid points");
    if (nprops <= 0 || !props || !outputs) throw std::invalid_argument("invalid property list");
    const std::size_t bs = opt ? static_cast<std::size_t>(opt->block_size) : 128;
    const double thr = opt ? opt->screening_threshold : default_screening_threshold;
    if (bs == 0 || bs > static_cast<std::size_t>(kumo_dev::kBlockPoints))
        throw std::invalid_argument("the no-allocation entry point supports block_size 1 to 128");
    if (!std::isfinite(thr) || thr < 0.0) throw std::invalid_argument("screening threshold must be finite and nonnegative");
    if (opt && opt->precision != 0) throw std::invalid_argument("the no-allocation entry point is FP64 only");
    if (opt && opt->backend != 0 && opt->backend != 2)
        throw std::invalid_argument("the no-allocation entry point takes backend AUTO or AO_MO");
    Request req;
    for (int i = 0; i < nprops; ++i) {
        if (props[i].kind < 0 || props[i].kind > static_cast<int>(PropertyKind::LolTsirelsonStash) || props[i].component < 0 ||
            props[i].component > 3)
            throw std::invalid_argument("unknown property");
        if (!outputs[i]) throw std::invalid_argument("null output array for property " + std::to_string(i));
        const PropertyKind k = static_cast<PropertyKind>(props[i].kind);
        if (!point_path_kind(k))
            throw std::invalid_argument("the no-allocation entry point evaluates density properties only");
        req.add({k, static_cast<DensityComponent>(props[i].component)});
    }
    const detail::Plan plan = detail::Plan::from(req);
    if (!m->mol.electronic_structure_info().ao_mo_eligible())
        throw std::invalid_argument("AO_MO backend requested but orbital representation is not eligible");
    const detail::DeviceMolecule* dev = m->mol.device_if_resident();
    if (!dev)
        throw std::invalid_argument(
            "the molecule has no device copy on this device: run one evaluation of it before this call");
    if (npoints == 0) return;
    // Point path of an evaluation at arbitrary points (src/evaluator.cpp:638-657).
    const int ao_order = std::max(1, plan.max_order);
    bool full = false;
    for (const auto& p : req.properties()) full |= needs_hessian(p.kind);
    const int npanel = ao_order == 1 ? kumo_dev::kPanelsGradient : (full ? kumo_dev::kPanelsFull : kumo_dev::kPanelsLaplacian);
    const int nao = dev->basis.nao;
    const std::size_t panel_bytes = sizeof(double) * npanel * static_cast<std::size_t>(nao) * kumo_dev::kBlockPoints;
    const std::size_t kept_bytes = (sizeof(int) * static_cast<std::size_t>(nao) + 255) / 256 * 256;
    const std::size_t per_block = panel_bytes + kept_bytes + 256;
    const std::size_t max_blocks = kNoAllocScratchBytes / per_block;
    if (max_blocks == 0)
        throw std::invalid_argument("one 128-point block of this molecule needs " + std::to_string(per_block) +
                                    " bytes of AO scratch; the no-allocation entry point has " +
                                    std::to_string(kNoAllocScratchBytes));
    const std::size_t n = static_cast<std::size_t>(npoints);
    const std::size_t nblocks = (n + bs - 1) / bs;
    const int W = static_cast<int>(std::min(max_blocks, nblocks));
    unsigned char* base = static_cast<unsigned char*>(scratch_address());
    double* panels = reinterpret_cast<double*>(base);
    int* kept = reinterpret_cast<int*>(base + panel_bytes * W);
    int* nkept = reinterpret_cast<int*>(base + (panel_bytes + kept_bytes) * W);

    kumo_dev::PointSource src{};
    src.points = device_points;
    src.count = npoints;
    kumo_dev::AoBuildParams<double> bp{};
    bp.basis = dev->basis;
    bp.src = src;
    bp.block_size = static_cast<long long>(bs);
    bp.threshold = thr;
    bp.out = {panels, kept, nkept, nao, npanel};
    for (int l = 0; l < 3; ++l)
        for (int i = 0; i < 135; ++i) bp.pure[l][i] = dev->pure_d[l][i];
    kumo_dev::ContractMoParams cp{};
    cp.scr = bp.out;
    cp.block_size = bp.block_size;
    cp.count = npoints;
    cp.ao_order = ao_order;
    cp.spec.stride = npoints;
    for (int i = 0; i < nprops; ++i) {
        if (cp.spec.nprops == kumo_dev::kMaxProps) throw std::invalid_argument("too many properties in one request");
        cp.spec.props[cp.spec.nprops++] = {props[i].kind, props[i].component, outputs[i]};
    }
    // Occupied-MO channels (src/density.cpp:257-273).
    std::array<bool, 4> needed{};
    for (int c = 0; c < 4; ++c) needed[static_cast<std::size_t>(c)] = plan.c[static_cast<std::size_t>(c)].derivatives() ||
                                                                      plan.c[static_cast<std::size_t>(c)].density;
    const bool need_a = needed[1] || needed[0] || needed[3];
    const bool need_b = needed[2] || needed[0] || needed[3];
    const int na = static_cast<int>(m->mol.occupied_count(SpinChannel::Alpha));
    const int nb = static_cast<int>(m->mol.occupied_count(SpinChannel::Beta));
    const bool bia = need_a && need_b && !m->mol.unrestricted() && na == nb;
    if (need_a && na > 0) cp.ch[cp.nchannels++] = {dev->ct_alpha, dev->ldc_alpha, na, 1};
    if (need_b && !bia && nb > 0) cp.ch[cp.nchannels++] = {dev->ct_beta, dev->ldc_beta, nb, 2};
    cp.beta_is_alpha = bia;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    for (std::size_t b0 = 0; b0 < nblocks; b0 += static_cast<std::size_t>(W)) {
        const int nbw = static_cast<int>(std::min<std::size_t>(W, nblocks - b0));
        bp.first_point = static_cast<long long>(b0 * bs);
        bp.nblocks = nbw;
        kumo_dev::launch_ao_build<double>(bp, ao_order, npanel, s);
        cp.first_point = bp.first_point;
        cp.nblocks = nbw;
        kumo_dev::launch_contract_mo_f64(cp, npanel, s);
    }
    detail::check_cuda(cudaGetLastError(), "kernel launch (no-allocation entry point)");
}

}  // namespace

extern "C" int kumo_evaluate_points_noalloc(const kumo_molecule* m, const kumo_options* opt, const double* device_points,
                                            long long npoints, const kumo_property* props, int nprops,
                                            double* const* outputs, void* stream, char* err, size_t errlen) {
    try {
        run(m, opt, device_points, npoints, props, nprops, outputs, stream);
        put(err, errlen, "");
        return KUMO_OK;
    } catch (const std::out_of_range& e) {
        put(err, errlen, e.what());
        return KUMO_OUT_OF_RANGE;
    } catch (const std::invalid_argument& e) {
        put(err, errlen, e.what());
        return KUMO_INVALID_ARGUMENT;
    } catch (const std::exception& e) {
        const std::string w = e.what();
        put(err, errlen, w);
        return w.rfind("CUDA error", 0) == 0 ? KUMO_CUDA_ERROR : KUMO_RUNTIME_ERROR;
    }
}
