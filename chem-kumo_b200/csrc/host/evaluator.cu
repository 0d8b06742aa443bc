// Evaluator: one evaluation runs the passes of chem-kumo's Evaluator::Run
// (src/evaluator.cpp:545-615) on the GPU:
//  - point path: AO panels + screening (ao_build) and the AO-MO or AO-P
//    contraction with the fused field epilogue, in waves of point blocks;
//  - electrostatic potential;
//  - orbital pass / grid-path orbital amplitudes;
//  - grid-path AO-P densities.
// The field each property comes from follows src/evaluator.cpp:79-111.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "../cuda/contract.cuh"
#include "../cuda/esp.cuh"
#include "../cuda/func_attr.cuh"
#include "../cuda/mixed.cuh"
#include "chem/kumo/evaluator.hpp"
#include "device_state.hpp"
#include "grid_geometry.hpp"
#include "plan.hpp"
#include "profile.hpp"

namespace chem::kumo {

std::size_t property_channels(PropertyKind k) {
    switch (k) {
        case PropertyKind::Gradient:
        case PropertyKind::OrbitalGradient:
        case PropertyKind::TauComponents:
        case PropertyKind::HamiltonianKineticEnergyComponents: return 3;
        case PropertyKind::Hessian:
        case PropertyKind::OrbitalHessian: return 6;
        default: return 1;
    }
}

namespace {

using detail::check_cuda;

// Rows per block that the mixed AO-MO contraction adds in FP64 (AO values
// and products) rather than on the tensor cores (KUMO_MIXED_EXACT_ROWS, read
// at each evaluation; default 38, 0 turns it off): the largest rows of each
// block, whose FP32 rounding and truncated tensor-core sums would otherwise
// set the error of the densities at the block's points.
int mixed_exact_rows() {
    const char* e = std::getenv("KUMO_MIXED_EXACT_ROWS");
    return e ? std::max(0, std::atoi(e)) : 38;
}

// Smallest block maximum of an exact row (KUMO_MIXED_EXACT_MIN, read at each
// evaluation; 0: the largest rows of every block are exact).  Default 1e-3:
// on the 740-AO workload's 128^3 grid the blocks whose rows all stay below it
// (far from the nuclei) then skip the FP64 epilogue, 13.2 -> 10.9 ms per
// step, with every field's error against FP64 unchanged in all three metrics
// (1e-2 kept the scaled errors but raised the relative error of rho where
// rho > 1e-6 from 6.2e-7 to 9.8e-7; 1e-1 took ELF past 1e-7).
float mixed_exact_min() {
    const char* e = std::getenv("KUMO_MIXED_EXACT_MIN");
    const double v = e ? std::atof(e) : 1e-3;
    return v > 0.0 && std::isfinite(v) ? static_cast<float>(v) : 0.0f;
}

// The mixed form of the potential (FP32 Hermite sums) is opt-in
// (KUMO_ESP_MIXED=1, read at each evaluation): on a 1260-AO molecule it was
// 1.07x faster than FP64 with 9e-4 scaled error on its density isosurface, so
// by default Precision::Mixed evaluates the potential in FP64.
// Limit of the tensor-core pipeline waits (KUMO_PIPELINE_WAIT_NS, read at
// each evaluation; 0 or unset: one second).  Tests shorten it to make the
// waits run out and check that the failure is reported.
unsigned long long pipeline_wait_ns() {
    const char* e = std::getenv("KUMO_PIPELINE_WAIT_NS");
    return e ? std::strtoull(e, nullptr, 10) : 0ull;
}

bool esp_mixed_opt_in() {
    const char* e = std::getenv("KUMO_ESP_MIXED");
    return e != nullptr && e[0] == '1';
}

// Which pass computes each requested property.  Grid-path orbital amplitudes
// follow src/orbitals.cpp:66-102.  AO-P densities on a grid take the
// reference's blocked grid path (src/density.cpp:366-444) in the FP64 form;
// the mixed form computes them in its tensor-core point pass, where one
// contraction per density matrix serves every component.
struct Route {
    Backend backend = Backend::AO_P;
    bool grid = false;
    bool mixed = false;
    bool grid_densities() const { return grid && backend == Backend::AO_P && !mixed; }
};

bool uses_point_path(const detail::ComponentNeeds& c, const Route& r) {
    return c.derivatives() || (!r.grid_densities() && c.density);
}

bool on_grid_path(const Property& p, const Route& r) {
    return r.grid && (p.kind == PropertyKind::Orbital || (p.kind == PropertyKind::Density && r.grid_densities()));
}

bool from_point_path(const Property& p, const Route& r) {
    return !on_grid_path(p, r) && !detail::is_orbital_kind(p.kind) &&
           p.kind != PropertyKind::ElectrostaticPotential && !detail::is_orbital_energy_kind(p.kind);
}

bool needs_full_hessian(PropertyKind k) {
    return k == PropertyKind::Hessian || k == PropertyKind::SignLambda2Density ||
           k == PropertyKind::DensityOverlapRegionsIndicator ||
           k == PropertyKind::HamiltonianKineticEnergyComponents;
}

// Stream-ordered device allocation, freed when the owner goes out of scope.
class DeviceAlloc {
public:
    DeviceAlloc() = default;
    DeviceAlloc(std::size_t bytes, cudaStream_t s) : stream_(s) {
        if (bytes) check_cuda(cudaMallocAsync(&ptr_, bytes, s), "cudaMallocAsync (evaluation scratch)");
    }
    DeviceAlloc(const DeviceAlloc&) = delete;
    DeviceAlloc& operator=(const DeviceAlloc&) = delete;
    DeviceAlloc(DeviceAlloc&& o) noexcept : ptr_(o.ptr_), stream_(o.stream_) { o.ptr_ = nullptr; }
    DeviceAlloc& operator=(DeviceAlloc&& o) noexcept {
        std::swap(ptr_, o.ptr_);
        std::swap(stream_, o.stream_);
        return *this;
    }
    ~DeviceAlloc() {
        if (ptr_) cudaFreeAsync(ptr_, stream_);
    }
    template <typename T>
    T* as() const {
        return static_cast<T*>(ptr_);
    }

private:
    void* ptr_ = nullptr;
    cudaStream_t stream_ = nullptr;
};

// The wave scratch comes from the device's default stream-ordered pool.  With
// the pool's default release threshold (0) every synchronization hands the
// memory back to the driver and the next evaluation maps it again, which
// blocks the host for tens to hundreds of milliseconds per call; keep it
// cached instead (once per device).
//
// The pool may also hand an allocation on one stream memory whose free is
// still queued on another stream, making the first stream wait for all the
// work queued before that free.  Evaluations issued concurrently on separate
// streams (the serving loop's slots) would then wait for one another: a small
// request for a large one that happened to free a block first.  That reuse is
// turned off; memory freed by work that has completed is still reused.
void keep_pool_memory() {
    static std::once_flag flags[64];
    int dev = 0;
    check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev < 0 || dev >= 64) return;
    std::call_once(flags[dev], [dev] {
        cudaMemPool_t pool;
        check_cuda(cudaDeviceGetDefaultMemPool(&pool, dev), "cudaDeviceGetDefaultMemPool");
        unsigned long long keep = ~0ull;
        check_cuda(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep),
                   "cudaMemPoolSetAttribute");
        int no_wait = 0;
        check_cuda(cudaMemPoolSetAttribute(pool, cudaMemPoolReuseAllowInternalDependencies, &no_wait),
                   "cudaMemPoolSetAttribute");
    });
}

// ---------------------------------------------------------------------------
// Tile-shape autotuner of the mixed form.  For grids of more than
// kTuneMinPoints points (KUMO_TILE_AUTOTUNE=0 turns it off) the tile shape is
// chosen by measurement: per molecule, backend, stored panels, exact-row count
// and grid step lengths, each compact candidate shape (see tile_candidates) is
// timed on a probe: the request's point-path properties on a sub-grid of at
// most 32 points per axis around the grid's centre, once untimed and twice
// timed with CUDA events, the faster time kept.  The ranking is cached; a
// later grid takes the best-ranked candidate among the shapes with its own
// fewest padding points.  Smaller grids (among them every grid the serving
// loop replays from a graph) keep the default shape.
constexpr std::size_t kTuneMinPoints = std::size_t(1) << 17;

struct TileRank {
    int sa, sb, sc;
    double ms;  // probe time
};

struct TileTuner {
    std::mutex mu;
    std::map<std::string, std::vector<TileRank>> ranked;
};

TileTuner& tile_tuner() {
    static TileTuner t;
    return t;
}

// Shape forced on the probe evaluations of this thread (sa, sb, sc), or null.
thread_local const int* t_forced_shape = nullptr;
// Whether evaluations on this thread may run probes (the serving loop's
// scheduler thread may not: it only takes rankings already measured).
thread_local bool t_probe_tiles = true;

bool tile_autotune_enabled() {
    const char* e = std::getenv("KUMO_TILE_AUTOTUNE");
    return !(e && e[0] == '0');
}

detail::TileShape shape_on(const Grid& g, int sa, int sb, int sc) {
    return {sa, sb, sc, (g.counts[0] + (1ll << sa) - 1) >> sa, (g.counts[1] + (1ll << sb) - 1) >> sb,
            (g.counts[2] + (1ll << sc) - 1) >> sc};
}

// Candidate shapes for a grid: padding within 5% of the fewest and a
// diagonal within 1.25 times the most compact's (the compact shapes, whose
// accuracy is the same), the most compact first, at most 8.
std::vector<detail::TileShape> tile_candidates(const Grid& g) {
    double len[3];
    for (int a = 0; a < 3; ++a)
        len[a] = std::sqrt(g.steps(0, a) * g.steps(0, a) + g.steps(1, a) * g.steps(1, a) + g.steps(2, a) * g.steps(2, a));
    const detail::TileShape best = detail::choose_tiles(g);
    auto diag = [&](const detail::TileShape& t) {
        const double da = len[0] * double(1 << t.sa), db = len[1] * double(1 << t.sb), dc = len[2] * double(1 << t.sc);
        return da * da + db * db + dc * dc;
    };
    std::vector<std::pair<double, detail::TileShape>> c;
    for (int sa = 0; sa <= 7; ++sa)
        for (int sb = 0; sa + sb <= 7; ++sb) {
            const detail::TileShape t = shape_on(g, sa, sb, 7 - sa - sb);
            if (t.padded() <= best.padded() * 1.05 && diag(t) <= 1.25 * diag(best)) c.emplace_back(diag(t), t);
        }
    std::stable_sort(c.begin(), c.end(), [](const auto& x, const auto& y) { return x.first < y.first; });
    std::vector<detail::TileShape> out;
    for (std::size_t i = 0; i < c.size() && i < 8; ++i) out.push_back(c[i].second);
    return out;
}

// AO scratch of one wave (KUMO_SCRATCH_MB): by default a quarter of the
// device memory free at the evaluation, between 4 and 32 GiB.  Molecules of
// thousands of AOs need tens of MB per block (every AO row is reserved), so
// a fixed 4 GiB left their waves at one or two hundred blocks, fewer than two
// per SM.
std::size_t scratch_budget() {
    if (const char* e = std::getenv("KUMO_SCRATCH_MB")) {
        const long long mb = std::atoll(e);
        if (mb > 0) return static_cast<std::size_t>(mb) << 20;
    }
    std::size_t free_b = 0, total_b = 0;
    const std::size_t lo = std::size_t(4) << 30, hi = std::size_t(32) << 30;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
        cudaGetLastError();
        return lo;
    }
    return std::clamp(free_b / 4, lo, hi);
}

// SMs of the current device (cached per device).
int sm_count() {
    static int counts[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    if (!counts[dev]) {
        int n = 0;
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
        counts[dev] = n;
    }
    return counts[dev];
}

}  // namespace

}  // namespace chem::kumo

namespace kumo_dev {

std::vector<const void*>& kernel_registry() {
    static std::vector<const void*> kernels;
    return kernels;
}

// Loads every listed kernel on the current device, once per device: asking
// for a kernel's attributes makes CUDA load it.
void preload_kernels() {
    static std::once_flag flags[64];
    int dev = 0;
    chem::kumo::detail::check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev < 0 || dev >= 64) return;
    std::call_once(flags[dev], [] {
        for (const void* f : kernel_registry()) {
            cudaFuncAttributes a;
            chem::kumo::detail::check_cuda(cudaFuncGetAttributes(&a, f), "cudaFuncGetAttributes (kernel preload)");
        }
    });
}

}  // namespace kumo_dev

namespace chem::kumo {

namespace detail {
// Once-per-device set-up that must not run inside a CUDA stream capture: the
// pool's settings, the tensor-core status word's address and every kernel of
// the library loaded (a serving loop's threads would otherwise wait while
// CUDA loads each kernel at its first launch).
void prepare_device_for_capture() {
    keep_pool_memory();
    (void)kumo_dev::pipeline_status_word();
    kumo_dev::preload_kernels();
}
}  // namespace detail

Evaluator::Evaluator(const Molecule& molecule, EvaluationOptions options) : molecule_(&molecule), options_(std::move(options)) {
    if (options_.block_size == 0 || options_.block_size > max_block_size)
        throw std::invalid_argument("evaluation block_size must be in [1, " + std::to_string(max_block_size) + "]");
    if (options_.threads < 0) throw std::invalid_argument("invalid evaluation options");
    if (!std::isfinite(options_.screening_threshold) || options_.screening_threshold < 0.0)
        throw std::invalid_argument("screening threshold must be finite and nonnegative");
    if (!std::isfinite(options_.potential_tolerance) || options_.potential_tolerance < 0.0)
        throw std::invalid_argument("potential tolerance must be finite and nonnegative");
    if (!std::isfinite(options_.fukui_delta) || options_.fukui_delta <= 0.0)
        throw std::invalid_argument("fukui_delta must be finite and positive");
    if (options_.backend != Backend::AUTO && options_.backend != Backend::AO_P && options_.backend != Backend::AO_MO)
        throw std::invalid_argument("unknown evaluation backend");
    if (options_.backend == Backend::AO_MO && !molecule.electronic_structure_info().ao_mo_eligible())
        throw std::invalid_argument("AO_MO backend requested but orbital representation is not eligible");
    if (options_.threads > 1)
        throw std::invalid_argument("explicit multi-thread control is not implemented in the API adapter");
}

// One evaluation on the device.  `outs` pairs each requested property with
// its device output (channels x n doubles).
class Evaluator::Run {
public:
    Run(const Evaluator& ev, const Grid* grid, const double* device_points, std::size_t n, const Request& request,
        cudaStream_t stream)
        : mol_(*ev.molecule_), opt_(ev.options_), grid_(grid), points_(device_points), n_(n), stream_(stream),
          plan_(detail::Plan::from(request)) {
        backend_ = detail::choose_backend(opt_.backend, mol_.electronic_structure_info().ao_mo_eligible(), plan_);
        // The orbital-energy checks come first, naming the most restrictive
        // group (src/evaluator.cpp:579-597).
        if (plan_.orbital_energies) {
            oe_needs_.virtuals = plan_.virtual_orbitals;
            oe_needs_.fukui = plan_.orbital_weighted_fukui;
            oe_needs_.fukui_delta = opt_.fukui_delta;
            oe_what_ = plan_.orbital_weighted_fukui ? "the orbital-weighted Fukui function or dual descriptor"
                       : plan_.virtual_orbitals    ? "the local electron affinity and related fields"
                                                   : "the average local ionization energy";
            detail::check_orbital_energy_fields(mol_, oe_needs_, oe_what_);
        }
        for (const auto& p : request.properties()) {
            // Orbital requests are checked before any pass (src/evaluator.cpp:623-636).
            if (detail::is_orbital_kind(p.kind)) {
                const auto& c = mol_.mo_coefficients(p.channel);
                if (c.cols() == 0) throw std::runtime_error("FCHK has no MO coefficients");
                if (p.orbital_index > c.cols()) throw std::out_of_range("MO index outside available coefficient range");
            }
        }
    }

    Backend backend() const { return backend_; }

    void execute(const std::vector<std::pair<Property, double*>>& outs, const ReadyCallback& ready = {}) {
        outs_ = outs;
        ready_ = &ready;
        if (n_ == 0) return;
        keep_pool_memory();
        dev_ = &mol_.device();
        src_ = kumo_dev::PointSource{};
        src_.count = static_cast<long long>(n_);
        if (grid_) {
            for (int k = 0; k < 3; ++k) src_.origin[k] = grid_->origin[k];
            for (int i = 0; i < 9; ++i) src_.steps[i] = grid_->steps.m[static_cast<std::size_t>(i)];
            src_.ny = grid_->counts[1];
            src_.nz = grid_->counts[2];
        } else {
            src_.points = points_;
        }
        const Route rt = route();
        bool point_path = false;
        for (const auto& c : plan_.c) point_path |= uses_point_path(c, rt);
        // Progress over all passes, src/evaluator.cpp:599-607.
        passes_ = (point_path ? 1 : 0) + (plan_.needs_esp() ? 1 : 0) + (plan_.orbital_energies ? 1 : 0);
        bool orbital_pass = false;
        bool grid_orbitals[2] = {false, false};
        std::size_t grid_densities = 0;
        for (const auto& [key, ptr] : outs_) {
            if (detail::is_orbital_kind(key.kind)) {
                if (on_grid_path(key, rt))
                    grid_orbitals[key.channel == SpinChannel::Beta ? 1 : 0] = true;
                else
                    orbital_pass = true;
            } else if (on_grid_path(key, rt)) {
                ++grid_densities;
            }
        }
        passes_ += (orbital_pass ? 1 : 0) + grid_densities + (grid_orbitals[0] ? 1 : 0) + (grid_orbitals[1] ? 1 : 0);

        if (point_path) point_pass();
        if (plan_.needs_esp()) potential_pass();
        if (plan_.orbital_energies) orbital_energy_pass();
        if (orbital_pass) orbital_pass_run(false);
        for (const auto& [key, ptr] : outs_)
            if (on_grid_path(key, rt) && key.kind == PropertyKind::Density) grid_density_pass(key, ptr);
        for (int ch = 0; ch < 2; ++ch)
            if (grid_orbitals[ch]) orbital_pass_run(true, ch);
        check_cuda(cudaGetLastError(), "kernel launch");
    }

private:
    void report(std::size_t done_in_pass) {
        // With one pass, every output of points [0, done) is final once the
        // launches enqueued so far have run.
        if (ready_ && *ready_ && passes_ == 1) (*ready_)(std::min(n_, completed_ + done_in_pass));
        if (!opt_.progress) return;
        check_cuda(cudaStreamSynchronize(stream_), "cudaStreamSynchronize (progress)");
        opt_.progress(completed_ + done_in_pass, passes_ * n_);
    }

    // Screening block of the FP64 passes (1 .. 65536 points, as the reference).
    std::size_t block_size() const { return opt_.block_size; }
    // Points per CTA of passes whose results do not depend on the block (no
    // screening, or the mixed form): the screening block, at most 128.
    std::size_t cta_block() const { return std::min<std::size_t>(opt_.block_size, kumo_dev::kBlockPoints); }

    // FP64 screening passes: CTAs take chunks of at most 128 points of a
    // screening block (kumo_dev::cta_points).
    struct F64Blocks {
        std::size_t screen = 128;  // points per screening block
        std::size_t chunk = 128;   // points per CTA
        std::size_t per = 1;       // CTAs per screening block
        std::size_t nscreen = 0;   // screening blocks
    };
    F64Blocks f64_blocks() const {
        F64Blocks b;
        b.screen = block_size();
        b.chunk = cta_block();
        b.per = (b.screen + b.chunk - 1) / b.chunk;
        b.nscreen = (n_ + b.screen - 1) / b.screen;
        return b;
    }

    // CTAs of one wave for `per_cta` bytes of AO scratch each: whole
    // screening blocks, at least one.
    int f64_wave_ctas(const F64Blocks& fb, std::size_t per_cta) const {
        const std::size_t w = static_cast<std::size_t>(wave_blocks(fb.nscreen * fb.per, per_cta));
        return static_cast<int>(std::max<std::size_t>(w / fb.per, 1) * fb.per);
    }

    // Runs the waves of an FP64 screening pass: per wave the AO build (for
    // screening blocks above 128 points first a launch that records each
    // AO's maximum over the whole block, src/ao_screening.hpp:35-50, then the
    // build that keeps rows by it) and `contract(first_point, ctas)`.
    template <class Contract>
    void f64_waves(const F64Blocks& fb, int W, kumo_dev::AoBuildParams<double>& bp, int ao_order, int npanel,
                   Contract&& contract) {
        const std::size_t ws = static_cast<std::size_t>(W) / fb.per;
        const bool mask = fb.per > 1 && bp.threshold > 0.0;
        const std::size_t nao = static_cast<std::size_t>(dev_->basis.nao);
        DeviceAlloc bmax(mask ? sizeof(double) * ws * nao : 0, stream_);
        bp.block_size = static_cast<long long>(fb.chunk);
        bp.screen_block = static_cast<long long>(fb.screen);
        for (std::size_t s0 = 0; s0 < fb.nscreen; s0 += ws) {
            const std::size_t ns = std::min(ws, fb.nscreen - s0);
            const int ctas = static_cast<int>(ns * fb.per);
            bp.first_point = static_cast<long long>(s0 * fb.screen);
            bp.nblocks = ctas;
            if (mask) {
                check_cuda(cudaMemsetAsync(bmax.as<double>(), 0, sizeof(double) * ns * nao, stream_),
                           "cudaMemsetAsync (block maxima)");
                bp.mask_pass = 1;
                bp.block_max = bmax.as<double>();
                kumo_dev::launch_ao_build<double>(bp, ao_order, npanel, stream_);
                bp.mask_pass = 2;
            }
            const int tok = detail::profile_begin(detail::kProfAoBuild, stream_);
            kumo_dev::launch_ao_build<double>(bp, ao_order, npanel, stream_);
            detail::profile_end(tok, stream_);
            count_ao_rows(bp.out.nkept, ctas);
            contract(bp.first_point, ctas);
            report(std::min(n_, (s0 + ns) * fb.screen));
        }
        bp.mask_pass = 0;
        bp.block_max = nullptr;
    }

    // Blocks per wave for a scratch of `per_block` bytes per block: as many as
    // the scratch holds, but with the default scratch no more than an eighth
    // of the blocks (down to 8 per SM), so that a large grid still has waves
    // whose results the host-output calls copy while later waves compute.
    int wave_blocks(std::size_t total_blocks, std::size_t per_block) const {
        const std::size_t budget = opt_.scratch_bytes ? opt_.scratch_bytes : scratch_budget();
        std::size_t w = budget / std::max<std::size_t>(per_block, 1);
        if (!opt_.scratch_bytes)
            w = std::min(w, std::max<std::size_t>((total_blocks + 7) / 8, static_cast<std::size_t>(8 * sm_count())));
        w = std::max<std::size_t>(1, std::min(w, total_blocks));
        w = std::min<std::size_t>(w, kumo_dev::kMaxBlocksPerWave);
        return static_cast<int>(w);
    }

    template <typename T>
    kumo_dev::AoBuildParams<T> build_params(double threshold) const {
        kumo_dev::AoBuildParams<T> p{};
        p.basis = dev_->basis;
        p.src = src_;
        p.threshold = threshold;
        for (int l = 0; l < 3; ++l)
            for (int i = 0; i < 135; ++i)
                p.pure[l][i] = sizeof(T) == 8 ? static_cast<T>(dev_->pure_d[l][i]) : static_cast<T>(dev_->pure_f[l][i]);
        return p;
    }

    Route route() const { return {backend_, grid_ != nullptr, opt_.precision == Precision::Mixed}; }

    kumo_dev::FieldSpec field_spec(bool (*select)(const Property&, const Route&)) const {
        kumo_dev::FieldSpec spec{};
        spec.stride = static_cast<long long>(n_);
        spec.out_base = 0;
        for (const auto& [key, ptr] : outs_) {
            if (!select(key, route())) continue;
            if (spec.nprops == kumo_dev::kMaxProps) throw std::invalid_argument("too many properties in one request");
            spec.props[spec.nprops++] = {static_cast<int>(key.kind), static_cast<int>(key.component), ptr};
        }
        return spec;
    }

    void point_pass() {
        const bool grid = grid_ != nullptr;
        std::array<bool, 4> needed{};
        const Route rt = route();
        for (int c = 0; c < 4; ++c) needed[c] = uses_point_path(plan_.c[c], rt);
        const int ao_order = grid ? plan_.max_order : std::max(1, plan_.max_order);
        bool full = false;
        for (const auto& [key, ptr] : outs_)
            if (from_point_path(key, rt) && needs_full_hessian(key.kind)) full = true;
        int npanel;
        if (ao_order <= 0)
            npanel = kumo_dev::kPanelsValue;
        else if (ao_order == 1)
            npanel = kumo_dev::kPanelsGradient;
        else
            npanel = full ? kumo_dev::kPanelsFull : kumo_dev::kPanelsLaplacian;
        const kumo_dev::FieldSpec spec = field_spec(&from_point_path);
        if (backend_ == Backend::AO_MO) {
            if (opt_.precision == Precision::Mixed)
                mo_pass_mixed(std::max(0, ao_order), npanel, needed, spec);
            else
                mo_pass_f64(std::max(0, ao_order), npanel, needed, spec);
        } else {
            const int np = npanel == kumo_dev::kPanelsValue ? kumo_dev::kPanelsGradient : npanel;
            if (opt_.precision == Precision::Mixed)
                p_pass_mixed(std::max(1, ao_order), np, needed, spec);
            else
                p_pass_f64(std::max(1, ao_order), np, needed, spec);
        }
        completed_ += n_;
    }

    // Rows written by one AO-build wave (counted right after its launch: the
    // mixed contractions then overwrite nkept with the rows they keep).
    void count_ao_rows(const int* nkept, int nb) const {
        if (!detail::profiling_enabled()) return;
        detail::profile_count(detail::kProfAoBuild, nkept, nb, 0.0, nb, 0.0, 0.0, stream_);
    }

    // Algorithmic counters of one contraction wave: per kept AO row of a
    // block (above the screening threshold), 2 * 128 points * panels *
    // occupied MOs FLOPs (the dense product C_kept^T Phi_kept of every stored
    // panel).
    void count_contraction(detail::ProfileKernel k, const int* nkept, int nb, int npanel, int nch, int nocc0,
                           int nocc1) const {
        if (!detail::profiling_enabled()) return;
        const double mos = static_cast<double>(nocc0) + (nch > 1 ? nocc1 : 0);
        const double per_row = 2.0 * kumo_dev::kBlockPoints * npanel * mos;
        detail::profile_count(k, nkept, nb, per_row, nb, 0.0, 0.0, stream_);
    }

    // AO-P contraction of a wave: per block and density matrix, the product
    // P[kept, kept] Phi[kept, 4 panels], 2 * m^2 * 4 * 128 FLOPs.
    // npanels: left panels summed over the density matrices contracted (4 per
    // matrix, 1 for a matrix whose components need values only).
    void count_ao_p(const int* nkept, int nb, int npanels) const {
        if (!detail::profiling_enabled()) return;
        detail::profile_count_sq(detail::kProfContractP, nkept, nb, 2.0 * kumo_dev::kBlockPoints * npanels, stream_);
    }

    // Occupied-MO channels needed by the AO-MO contraction
    // (src/density.cpp:257-273).
    int mo_channels(const std::array<bool, 4>& needed, kumo_dev::MoChannel* ch, bool& beta_is_alpha, bool mixed) const {
        const bool need_a = needed[1] || needed[0] || needed[3];
        const bool need_b = needed[2] || needed[0] || needed[3];
        const int na = static_cast<int>(mol_.occupied_count(SpinChannel::Alpha));
        const int nb = static_cast<int>(mol_.occupied_count(SpinChannel::Beta));
        beta_is_alpha = need_a && need_b && !mol_.unrestricted() && na == nb;
        int nch = 0;
        (void)mixed;
        auto ct = [&](bool beta) -> const double* { return beta ? dev_->ct_beta : dev_->ct_alpha; };
        if (need_a && na > 0) ch[nch++] = {ct(false), dev_->ldc_alpha, na, 1};
        if (need_b && !beta_is_alpha && nb > 0) ch[nch++] = {ct(true), dev_->ldc_beta, nb, 2};
        return nch;
    }

    // Evaluation layout of a mixed-form pass (blocks of at most 128 points:
    // a larger screening block only widens the FP64 form's kept sets, by
    // rows below the threshold).  On a grid with 128-point (or larger)
    // blocks the mixed form evaluates compact tiles (GridTiles) instead of
    // runs of 128 points along k: the tile shape (powers of two, 128 points)
    // leaves the fewest padding points, and among those spans the shortest
    // diagonal.  The FP64 form keeps the reference's blocks, whose screening
    // it reproduces bit for bit; the mixed form only has to agree with it to
    // its tolerance, and a compact block lets its FP64 exact rows (the
    // block's largest rows) cover the dominant terms of every point.
    // KUMO_MIXED_TILES=0 keeps the linear blocks.
    struct MixedLayout {
        kumo_dev::PointSource src;
        kumo_dev::GridTiles tiles;
        std::size_t nblocks = 0;
        long long count = 0;  // evaluation indices
    };

    // The tile shape of this run's grid: measured (see TileTuner) or, for
    // small grids, under stream capture or with the tuner off, the default.
    detail::TileShape tuned_shape(int npanel) const {
        const detail::TileShape def = detail::choose_tiles(*grid_);
        cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
        if (n_ <= kTuneMinPoints || !tile_autotune_enabled() ||
            cudaStreamIsCapturing(stream_, &cap) != cudaSuccess || cap != cudaStreamCaptureStatusNone)
            return def;
        char key[256];
        double len[3];
        for (int a = 0; a < 3; ++a)
            len[a] = std::sqrt(grid_->steps(0, a) * grid_->steps(0, a) + grid_->steps(1, a) * grid_->steps(1, a) +
                               grid_->steps(2, a) * grid_->steps(2, a));
        std::snprintf(key, sizeof key, "%p|%d|%d|%d|%.6g,%.6g,%.6g", static_cast<const void*>(&mol_),
                      static_cast<int>(backend_), npanel, mixed_exact_rows(), len[0], len[1], len[2]);
        TileTuner& tt = tile_tuner();
        std::vector<TileRank> rank;
        {
            std::lock_guard<std::mutex> lock(tt.mu);
            auto it = tt.ranked.find(key);
            if (it != tt.ranked.end()) rank = it->second;
        }
        const auto cands = tile_candidates(*grid_);
        if (rank.empty() && !t_probe_tiles) return def;
        if (rank.empty()) {
            rank = probe_shapes(cands);
            std::lock_guard<std::mutex> lock(tt.mu);
            tt.ranked[key] = rank;
        }
        for (const auto& r : rank)
            for (const auto& c : cands)
                if (c.sa == r.sa && c.sb == r.sb && c.sc == r.sc && c.padded() == def.padded()) return c;
        return def;
    }

    // Times each candidate on the probe sub-grid; fastest first.
    std::vector<TileRank> probe_shapes(const std::vector<detail::TileShape>& cands) const {
        Grid sub = *grid_;
        long long lo[3];
        for (int a = 0; a < 3; ++a) {
            const int n = std::min(grid_->counts[a], 32);
            lo[a] = (grid_->counts[a] - n) / 2;
            sub.counts[a] = n;
        }
        for (int r = 0; r < 3; ++r)
            sub.origin[r] = grid_->origin[r] + ((grid_->steps(r, 0) * double(lo[0]) + grid_->steps(r, 1) * double(lo[1])) +
                                                grid_->steps(r, 2) * double(lo[2]));
        Request probe;
        std::size_t chans = 0;
        for (const auto& [key, ptr] : outs_)
            if (from_point_path(key, route())) {
                probe.add(key);
                chans += property_channels(key.kind);
            }
        const std::size_t np = detail::validated_point_count(sub);
        DeviceAlloc buf(sizeof(double) * std::max<std::size_t>(chans * np, 1), stream_);
        std::vector<double*> outs;
        std::size_t off = 0;
        for (const auto& q : probe.properties()) {
            outs.push_back(buf.as<double>() + off * np);
            off += property_channels(q.kind);
        }
        EvaluationOptions o = opt_;
        o.progress = {};
        o.backend = backend_;
        const Evaluator ev(mol_, o);
        cudaEvent_t e0, e1;
        check_cuda(cudaEventCreate(&e0), "cudaEventCreate");
        check_cuda(cudaEventCreate(&e1), "cudaEventCreate");
        std::vector<TileRank> rank;
        for (const auto& c : cands) {
            const int shape[3] = {c.sa, c.sb, c.sc};
            t_forced_shape = shape;
            double best = 1e300;
            try {
                for (int rep = 0; rep < 3; ++rep) {
                    check_cuda(cudaEventRecord(e0, stream_), "cudaEventRecord");
                    ev.evaluate_device(sub, probe, outs.data(), stream_);
                    check_cuda(cudaEventRecord(e1, stream_), "cudaEventRecord");
                    check_cuda(cudaEventSynchronize(e1), "cudaEventSynchronize (tile tuning)");
                    float ms = 0.f;
                    check_cuda(cudaEventElapsedTime(&ms, e0, e1), "cudaEventElapsedTime");
                    if (rep > 0) best = std::min(best, static_cast<double>(ms));
                }
            } catch (...) {
                t_forced_shape = nullptr;
                cudaEventDestroy(e0);
                cudaEventDestroy(e1);
                throw;
            }
            t_forced_shape = nullptr;
            rank.push_back({c.sa, c.sb, c.sc, best});
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        std::stable_sort(rank.begin(), rank.end(), [](const TileRank& x, const TileRank& y) { return x.ms < y.ms; });
        return rank;
    }

    MixedLayout mixed_layout(int npanel) const {
        MixedLayout L;
        L.src = src_;
        const std::size_t bs = cta_block();
        const bool tiled = grid_ && detail::mixed_grid_tiles(opt_.block_size);
        if (!tiled) {
            L.nblocks = (n_ + bs - 1) / bs;
            L.count = static_cast<long long>(n_);
            return L;
        }
        const detail::TileShape ts = t_forced_shape ? shape_on(*grid_, t_forced_shape[0], t_forced_shape[1], t_forced_shape[2])
                                                    : tuned_shape(npanel);
        const kumo_dev::GridTiles t{1,           ts.sa,       ts.sb,   ts.sc, grid_->counts[0], grid_->counts[1],
                                    grid_->counts[2], ts.tny, ts.tnz};
        const long long best_pad = ts.padded();
        L.tiles = t;
        L.src.tiles = t;
        L.count = best_pad;
        L.src.count = best_pad;
        L.nblocks = static_cast<std::size_t>(best_pad / 128);
        return L;
    }

    // Points of the grid whose results are final once the first `blocks`
    // blocks of a pass have run (tiles run with i slowest, so finished tiles
    // complete whole planes of the grid).
    std::size_t done_points(const MixedLayout& L, std::size_t blocks) const {
        const std::size_t bs = cta_block();
        if (!L.tiles.on) return std::min(n_, blocks * bs);
        const std::size_t per_slab = static_cast<std::size_t>(L.tiles.tny * L.tiles.tnz);
        const std::size_t planes = (blocks / per_slab) << L.tiles.sa;
        return std::min(n_, planes * static_cast<std::size_t>(L.tiles.ny * L.tiles.nz));
    }

    void mo_pass_f64(int ao_order, int npanel, const std::array<bool, 4>& needed, const kumo_dev::FieldSpec& spec) {
        const F64Blocks fb = f64_blocks();
        const int nao = dev_->basis.nao;
        const int stride = nao;
        const std::size_t per_cta = sizeof(double) * npanel * (std::size_t)stride * kumo_dev::kBlockPoints +
                                    sizeof(int) * ((std::size_t)stride + 1);
        const int W = f64_wave_ctas(fb, per_cta);
        DeviceAlloc panels(sizeof(double) * npanel * (std::size_t)stride * kumo_dev::kBlockPoints * W, stream_);
        DeviceAlloc kept(sizeof(int) * (std::size_t)stride * W, stream_);
        DeviceAlloc nkept(sizeof(int) * (std::size_t)W, stream_);
        kumo_dev::AoBuildParams<double> bp = build_params<double>(opt_.screening_threshold);
        bp.out = {panels.as<double>(), kept.as<int>(), nkept.as<int>(), stride, npanel};
        kumo_dev::ContractMoParams cp{};
        cp.scr = bp.out;
        cp.block_size = static_cast<long long>(fb.chunk);
        cp.screen_block = static_cast<long long>(fb.screen);
        cp.count = static_cast<long long>(n_);
        bool bia = false;
        cp.nchannels = mo_channels(needed, cp.ch, bia, false);
        cp.beta_is_alpha = bia;
        cp.ao_order = ao_order;
        cp.spec = spec;
        f64_waves(fb, W, bp, ao_order, npanel, [&](long long first, int ctas) {
            cp.first_point = first;
            cp.nblocks = ctas;
            const int tok = detail::profile_begin(detail::kProfContractMo, stream_);
            kumo_dev::launch_contract_mo_f64(cp, npanel, stream_);
            detail::profile_end(tok, stream_);
            count_contraction(detail::kProfContractMo, bp.out.nkept, ctas, npanel, cp.nchannels, cp.ch[0].nocc,
                              cp.nchannels > 1 ? cp.ch[1].nocc : 0);
        });
    }

    // Fused mixed AO-MO pass: the AO rows are built inside the tensor-core
    // kernel, so no AO panels (and no AO scratch) go through device memory.
    // Opt-in with KUMO_MIXED_FUSED=1, where the AO rows are built at most
    // twice per block (MO passes x spin channels <= 2): on organic_740 it
    // takes 26.4 ms per 128^3 step against 13.3 ms for the two-kernel form,
    // whose AO build runs at twice the warps per SM and without the
    // per-step barriers.
    bool mo_pass_fused(int ao_order, int npanel, const std::array<bool, 4>& needed, const kumo_dev::FieldSpec& spec) {
        const char* e = std::getenv("KUMO_MIXED_FUSED");
        if (!e || std::string(e) != "1") return false;
        if (!kumo_dev::contract_fused_supported(npanel, dev_->basis.nblocks)) return false;
        const std::size_t bs = cta_block();
        const MixedLayout lay = mixed_layout(npanel);
        const std::size_t nblocks = lay.nblocks;
        const int nao = dev_->basis.nao;
        kumo_dev::ContractFusedParams cp{};
        bool bia = false;
        kumo_dev::MoChannel ch[2];
        cp.nchannels = mo_channels(needed, ch, bia, true);
        int nocc16 = 16;
        for (int i = 0; i < cp.nchannels; ++i) {
            const bool beta = ch[i].role == 2;
            const int ldn = beta ? dev_->ldn_beta : dev_->ldn_alpha;
            cp.ch[i] = {beta ? dev_->cs_beta : dev_->cs_alpha, static_cast<long long>(nao) * ldn, ldn, ch[i].nocc,
                        ch[i].role};
            nocc16 = std::max(nocc16, (ch[i].nocc + 15) / 16 * 16);
        }
        kumo_dev::mixed_columns(npanel, nocc16, cp.ncols, cp.groups, cp.tmem_cols);
        int builds = 0;
        for (int i = 0; i < cp.nchannels; ++i) builds += (cp.ch[i].nocc + cp.ncols - 1) / cp.ncols;
        if (builds > 2) return false;
        cp.ao.basis = dev_->basis;
        cp.ao.prims = dev_->mix_prims;
        cp.ao.src = lay.src;
        cp.ao.block_size = static_cast<long long>(bs);
        std::memcpy(cp.ao.tpure, dev_->tpure_g, sizeof cp.ao.tpure);
        std::memcpy(cp.ao.gcart, dev_->gcart, sizeof cp.ao.gcart);
        cp.count = lay.count;
        cp.status = kumo_dev::pipeline_status_word();
        cp.wait_ns = pipeline_wait_ns();
        cp.beta_is_alpha = bia;
        cp.ao_order = ao_order;
        cp.spec = spec;
        cp.spec.tiles = lay.tiles;
        const int W = static_cast<int>(std::min<std::size_t>(nblocks, 1u << 16));
        DeviceAlloc nrows(sizeof(int) * static_cast<std::size_t>(W), stream_);
        cp.nrows = detail::profiling_enabled() ? nrows.as<int>() : nullptr;
        for (std::size_t b0 = 0; b0 < nblocks; b0 += static_cast<std::size_t>(W)) {
            const int nb = static_cast<int>(std::min<std::size_t>(W, nblocks - b0));
            cp.ao.first_point = static_cast<long long>(b0 * bs);
            cp.ao.nblocks = nb;
            const int tok = detail::profile_begin(detail::kProfContractMixed, stream_);
            kumo_dev::launch_contract_fused(cp, npanel, stream_);
            detail::profile_end(tok, stream_);
            if (cp.nrows)
                count_contraction(detail::kProfContractMixed, cp.nrows, nb, npanel, cp.nchannels, cp.ch[0].nocc,
                                  cp.nchannels > 1 ? cp.ch[1].nocc : 0);
            report(done_points(lay, b0 + nb));
        }
        return true;
    }

    void mo_pass_mixed(int ao_order, int npanel, const std::array<bool, 4>& needed, const kumo_dev::FieldSpec& spec) {
        if (mo_pass_fused(ao_order, npanel, needed, spec)) return;
        const std::size_t bs = cta_block();
        const MixedLayout lay = mixed_layout(npanel);
        const std::size_t nblocks = lay.nblocks;
        const int nao = dev_->basis.nao;
        const int stride = (nao + 7) / 8 * 8;
        const std::size_t per_block = sizeof(float) * npanel * (std::size_t)stride * kumo_dev::kBlockPoints +
                                      sizeof(int) * ((std::size_t)stride + 1) + sizeof(float) * 4 * (std::size_t)stride;
        const int W = wave_blocks(nblocks, per_block);
        DeviceAlloc panels(sizeof(float) * npanel * (std::size_t)stride * kumo_dev::kBlockPoints * W, stream_);
        DeviceAlloc kept(sizeof(int) * (std::size_t)stride * W, stream_);
        DeviceAlloc nkept(sizeof(int) * (std::size_t)W, stream_);
        DeviceAlloc rowmax(sizeof(float) * 4 * (std::size_t)stride * W, stream_);
        kumo_dev::AoMixedParams bp{};
        bp.basis = dev_->basis;
        bp.prims = dev_->mix_prims;
        bp.src = lay.src;
        bp.block_size = static_cast<long long>(bs);
        std::memcpy(bp.tpure, dev_->tpure_g, sizeof bp.tpure);
        std::memcpy(bp.gcart, dev_->gcart, sizeof bp.gcart);
        bp.out = {panels.as<float>(), kept.as<int>(), nkept.as<int>(), stride, npanel, rowmax.as<float>()};
        kumo_dev::ContractMixedParams cp{};
        cp.scr = bp.out;
        cp.block_size = static_cast<long long>(bs);
        cp.count = lay.count;
        bool bia = false;
        kumo_dev::MoChannel ch[2];
        cp.nchannels = mo_channels(needed, ch, bia, true);
        int nocc16 = 16;
        for (int i = 0; i < cp.nchannels; ++i) {
            const bool beta = ch[i].role == 2;
            const int ldn = beta ? dev_->ldn_beta : dev_->ldn_alpha;
            cp.ch[i] = {beta ? dev_->cs_beta : dev_->cs_alpha, static_cast<long long>(nao) * ldn, ldn, ch[i].nocc,
                        ch[i].role, beta ? dev_->ct_beta : dev_->ct_alpha, beta ? dev_->ldc_beta : dev_->ldc_alpha};
            nocc16 = std::max(nocc16, (ch[i].nocc + 15) / 16 * 16);
        }
        kumo_dev::mixed_columns(npanel, nocc16, cp.ncols, cp.groups, cp.tmem_cols);
        cp.status = kumo_dev::pipeline_status_word();
        cp.wait_ns = pipeline_wait_ns();
        cp.threshold = static_cast<float>(opt_.screening_threshold);
        cp.beta_is_alpha = bia;
        cp.ao_order = ao_order;
        cp.spec = spec;
        cp.spec.tiles = lay.tiles;
        cp.exact_rows = mixed_exact_rows();
        cp.exact_min = mixed_exact_min();
        cp.src = lay.src;
        cp.basis = dev_->basis;
        for (std::size_t b0 = 0; b0 < nblocks; b0 += static_cast<std::size_t>(W)) {
            const int nb = static_cast<int>(std::min<std::size_t>(W, nblocks - b0));
            bp.first_point = static_cast<long long>(b0 * bs);
            bp.nblocks = nb;
            int tok = detail::profile_begin(detail::kProfAoBuild, stream_);
            kumo_dev::launch_ao_mixed(bp, npanel, stream_);
            detail::profile_end(tok, stream_);
            count_ao_rows(bp.out.nkept, nb);
            cp.first_point = bp.first_point;
            cp.nblocks = nb;
            tok = detail::profile_begin(detail::kProfContractMixed, stream_);
            kumo_dev::launch_contract_mixed(cp, npanel, stream_);
            detail::profile_end(tok, stream_);
            count_contraction(detail::kProfContractMixed, bp.out.nkept, nb, npanel, cp.nchannels, cp.ch[0].nocc,
                              cp.nchannels > 1 ? cp.ch[1].nocc : 0);
            report(done_points(lay, b0 + nb));
        }
    }

    // Mixed AO-P form: FP32 AO rows (ao_mixed) and the tensor-core
    // Y = P[kept, kept] Phi contraction (density_derivatives_shared).
    void p_pass_mixed(int ao_order, int npanel, const std::array<bool, 4>& needed, const kumo_dev::FieldSpec& spec) {
        const std::size_t bs = cta_block();
        const MixedLayout lay = mixed_layout(npanel);
        const std::size_t nblocks = lay.nblocks;
        const int nao = dev_->basis.nao;
        const int stride = (nao + 7) / 8 * 8;
        const std::size_t per_block = sizeof(float) * npanel * (std::size_t)stride * kumo_dev::kBlockPoints +
                                      sizeof(int) * ((std::size_t)stride + 1) + sizeof(float) * 4 * (std::size_t)stride;
        const int W = wave_blocks(nblocks, per_block);
        DeviceAlloc panels(sizeof(float) * npanel * (std::size_t)stride * kumo_dev::kBlockPoints * W, stream_);
        DeviceAlloc kept(sizeof(int) * (std::size_t)stride * W, stream_);
        DeviceAlloc nkept(sizeof(int) * (std::size_t)W, stream_);
        DeviceAlloc rowmax(sizeof(float) * 4 * (std::size_t)stride * W, stream_);
        kumo_dev::AoMixedParams bp{};
        bp.basis = dev_->basis;
        bp.prims = dev_->mix_prims;
        bp.src = lay.src;
        bp.block_size = static_cast<long long>(bs);
        std::memcpy(bp.tpure, dev_->tpure_g, sizeof bp.tpure);
        std::memcpy(bp.gcart, dev_->gcart, sizeof bp.gcart);
        bp.out = {panels.as<float>(), kept.as<int>(), nkept.as<int>(), stride, npanel, rowmax.as<float>()};
        kumo_dev::ContractPMixedParams cp{};
        cp.scr = bp.out;
        cp.block_size = static_cast<long long>(bs);
        cp.count = lay.count;
        cp.nao = nao;
        dev_->ensure_p_pieces(mol_);
        cp.p_total_s = dev_->p_total_s;
        cp.p_spin_s = dev_->p_spin_s;
        cp.total_needed = needed[0] || needed[1] || needed[2];
        cp.spin_needed = needed[3] || needed[1] || needed[2];
        cp.ao_order = ao_order;
        // A density matrix whose components need values only (the alpha, beta
        // and spin densities beside a Total-only RDG, say) is contracted with
        // the value panel alone.
        int order_total = -1, order_spin = -1;
        for (int c = 0; c < 4; ++c) {
            if (!needed[c]) continue;
            const int o = std::max(0, plan_.c[c].ao_order());
            if (c != 3) order_total = std::max(order_total, o);
            if (c != 0) order_spin = std::max(order_spin, o);
        }
        cp.value_only = (order_total == 0 ? 1 : 0) | (order_spin == 0 ? 2 : 0);
        cp.threshold = static_cast<float>(opt_.screening_threshold);
        cp.spec = spec;
        cp.spec.tiles = lay.tiles;
        cp.status = kumo_dev::pipeline_status_word();
        cp.wait_ns = pipeline_wait_ns();
        for (std::size_t b0 = 0; b0 < nblocks; b0 += static_cast<std::size_t>(W)) {
            const int nb = static_cast<int>(std::min<std::size_t>(W, nblocks - b0));
            bp.first_point = static_cast<long long>(b0 * bs);
            bp.nblocks = nb;
            int tok = detail::profile_begin(detail::kProfAoBuild, stream_);
            kumo_dev::launch_ao_mixed(bp, npanel, stream_);
            detail::profile_end(tok, stream_);
            count_ao_rows(bp.out.nkept, nb);
            cp.first_point = bp.first_point;
            cp.nblocks = nb;
            tok = detail::profile_begin(detail::kProfContractP, stream_);
            kumo_dev::launch_contract_p_mixed(cp, npanel, stream_);
            detail::profile_end(tok, stream_);
            count_ao_p(bp.out.nkept, nb,
                       (cp.total_needed ? (cp.value_only & 1 ? 1 : 4) : 0) + (cp.spin_needed ? (cp.value_only & 2 ? 1 : 4) : 0));
            report(done_points(lay, b0 + nb));
        }
    }

    void p_pass_f64(int ao_order, int npanel, const std::array<bool, 4>& needed, const kumo_dev::FieldSpec& spec) {
        const F64Blocks fb = f64_blocks();
        const int nao = dev_->basis.nao;
        const int stride = nao;
        const std::size_t per_cta = sizeof(double) * npanel * (std::size_t)stride * kumo_dev::kBlockPoints +
                                    sizeof(int) * ((std::size_t)stride + 1);
        const int W = f64_wave_ctas(fb, per_cta);
        DeviceAlloc panels(sizeof(double) * npanel * (std::size_t)stride * kumo_dev::kBlockPoints * W, stream_);
        DeviceAlloc kept(sizeof(int) * (std::size_t)stride * W, stream_);
        DeviceAlloc nkept(sizeof(int) * (std::size_t)W, stream_);
        kumo_dev::AoBuildParams<double> bp = build_params<double>(opt_.screening_threshold);
        bp.out = {panels.as<double>(), kept.as<int>(), nkept.as<int>(), stride, npanel};
        kumo_dev::ContractPParams cp{};
        cp.scr = bp.out;
        cp.block_size = static_cast<long long>(fb.chunk);
        cp.screen_block = static_cast<long long>(fb.screen);
        cp.count = static_cast<long long>(n_);
        cp.nao = nao;
        cp.total_needed = needed[0] || needed[1] || needed[2];
        cp.spin_needed = needed[3] || needed[1] || needed[2];
        cp.p_total = dev_->p_total;
        cp.p_spin = dev_->p_spin;
        cp.ao_order = ao_order;
        cp.spec = spec;
        f64_waves(fb, W, bp, ao_order, npanel, [&](long long first, int ctas) {
            cp.first_point = first;
            cp.nblocks = ctas;
            const int tok = detail::profile_begin(detail::kProfContractP, stream_);
            kumo_dev::launch_contract_p_f64(cp, npanel, stream_);
            detail::profile_end(tok, stream_);
            count_ao_p(bp.out.nkept, ctas, 4 * ((cp.total_needed ? 1 : 0) + (cp.spin_needed ? 1 : 0)));
        });
    }

    // Molecule::densities_blocked for one component (src/density.cpp:366-444).
    void grid_density_pass(const Property& key, double* out) {
        const F64Blocks fb = f64_blocks();
        const int nao = dev_->basis.nao;
        const std::size_t per_cta =
            sizeof(double) * (std::size_t)nao * kumo_dev::kBlockPoints + sizeof(int) * ((std::size_t)nao + 1);
        const int W = f64_wave_ctas(fb, per_cta);
        DeviceAlloc panels(sizeof(double) * (std::size_t)nao * kumo_dev::kBlockPoints * W, stream_);
        DeviceAlloc kept(sizeof(int) * (std::size_t)nao * W, stream_);
        DeviceAlloc nkept(sizeof(int) * (std::size_t)W, stream_);
        kumo_dev::AoBuildParams<double> bp = build_params<double>(opt_.screening_threshold);
        bp.out = {panels.as<double>(), kept.as<int>(), nkept.as<int>(), nao, 1};
        kumo_dev::ContractPParams cp{};
        cp.scr = bp.out;
        cp.block_size = static_cast<long long>(fb.chunk);
        cp.screen_block = static_cast<long long>(fb.screen);
        cp.count = static_cast<long long>(n_);
        cp.nao = nao;
        cp.density_component = static_cast<int>(key.component);
        cp.p_total = dev_->p_total;
        cp.p_spin = dev_->p_spin;
        cp.ao_order = 0;
        cp.spec.stride = static_cast<long long>(n_);
        cp.spec.nprops = 1;
        cp.spec.props[0] = {static_cast<int>(key.kind), static_cast<int>(key.component), out};
        f64_waves(fb, W, bp, 0, 1, [&](long long first, int ctas) {
            cp.first_point = first;
            cp.nblocks = ctas;
            const int tok = detail::profile_begin(detail::kProfContractP, stream_);
            kumo_dev::launch_density_values_f64(cp, stream_);
            detail::profile_end(tok, stream_);
            // 2 m^2 FLOPs per point (one panel, one density matrix).
            if (detail::profiling_enabled())
                detail::profile_count_sq(detail::kProfContractP, bp.out.nkept, ctas, 2.0 * kumo_dev::kBlockPoints,
                                         stream_);
        });
        completed_ += n_;
    }

    // Orbital amplitudes and derivatives (src/evaluator.cpp:688-730) or the
    // grid-path amplitudes of one channel (src/orbitals.cpp:66-102): every AO
    // kept (no screening), values from evaluate_batch and derivatives from
    // evaluate_derivatives_batch.
    void orbital_pass_run(bool grid_path, int channel = 0) {
        const bool grid = grid_ != nullptr;
        std::vector<std::pair<Property, double*>> sel;
        int order = 0;
        for (const auto& [key, ptr] : outs_) {
            if (!detail::is_orbital_kind(key.kind)) continue;
            const bool gp = on_grid_path(key, route());
            if (gp != grid_path) continue;
            if (grid_path && static_cast<int>(key.channel) != channel) continue;
            sel.emplace_back(key, ptr);
            if (key.kind == PropertyKind::OrbitalGradient) order = std::max(order, 1);
            if (key.kind == PropertyKind::OrbitalHessian) order = 2;
        }
        if (sel.empty()) return;
        const std::size_t bs = grid_path ? 128 : cta_block();  // no screening: any chunking gives the same values
        const std::size_t nblocks = (n_ + bs - 1) / bs;
        const int nao = dev_->basis.nao;
        // Values come from the value path (npanel 1); derivatives from the
        // derivative path with 4 or 10 panels.
        for (int pass = 0; pass < (order > 0 ? 2 : 1); ++pass) {
            const int npanel = pass == 0 ? 1 : (order == 1 ? 4 : 10);
            const int aord = pass == 0 ? 0 : order;
            const std::size_t per_block = sizeof(double) * npanel * (std::size_t)nao * kumo_dev::kBlockPoints +
                                          sizeof(int) * ((std::size_t)nao + 1);
            const int W = wave_blocks(nblocks, per_block);
            DeviceAlloc panels(sizeof(double) * npanel * (std::size_t)nao * kumo_dev::kBlockPoints * W, stream_);
            DeviceAlloc kept(sizeof(int) * (std::size_t)nao * W, stream_);
            DeviceAlloc nkept(sizeof(int) * (std::size_t)W, stream_);
            kumo_dev::AoBuildParams<double> bp = build_params<double>(0.0);
            bp.keep_reaching = 1;
            bp.block_size = static_cast<long long>(bs);
            bp.out = {panels.as<double>(), kept.as<int>(), nkept.as<int>(), nao, npanel};
            kumo_dev::OrbitalParams op{};
            op.scr = bp.out;
            op.block_size = static_cast<long long>(bs);
            op.count = static_cast<long long>(n_);
            op.nao = nao;
            op.npanel = npanel;
            op.stride = static_cast<long long>(n_);
            for (const auto& [key, ptr] : sel) {
                const bool value = key.kind == PropertyKind::Orbital;
                if ((pass == 0) != value) continue;
                if (op.nsel == 8) {
                    run_orbital_waves(bp, op, nblocks, W, bs, aord, npanel);
                    op.nsel = 0;
                }
                const bool beta = key.channel == SpinChannel::Beta;
                const double* c = beta ? dev_->c_beta : dev_->c_alpha;
                op.coef[op.nsel] = c + (key.orbital_index - 1) * static_cast<std::size_t>(nao);
                op.out[op.nsel] = ptr;
                op.first_channel[op.nsel] = value ? 0 : (key.kind == PropertyKind::OrbitalGradient ? 1 : 4);
                op.nchan[op.nsel] = static_cast<int>(property_channels(key.kind));
                ++op.nsel;
            }
            if (op.nsel) run_orbital_waves(bp, op, nblocks, W, bs, aord, npanel);
        }
        completed_ += n_;
    }

    // Orbital-energy fields (src/evaluator.cpp:676-682): per block the AO
    // values with every AO kept (evaluate_batch: shell cutoff only), then the
    // set sums over the scaled MO columns and the fields from them.
    void orbital_energy_pass() {
        const auto& st = dev_->orbital_energy_state(mol_, oe_needs_, oe_what_);
        const std::size_t bs = cta_block();  // no screening: any chunking gives the same values
        const std::size_t nblocks = (n_ + bs - 1) / bs;
        const int nao = dev_->basis.nao;
        const std::size_t per_block =
            sizeof(double) * (std::size_t)nao * kumo_dev::kBlockPoints + sizeof(int) * ((std::size_t)nao + 1);
        const int W = wave_blocks(nblocks, per_block);
        DeviceAlloc panels(sizeof(double) * (std::size_t)nao * kumo_dev::kBlockPoints * W, stream_);
        DeviceAlloc kept(sizeof(int) * (std::size_t)nao * W, stream_);
        DeviceAlloc nkept(sizeof(int) * (std::size_t)W, stream_);
        kumo_dev::AoBuildParams<double> bp = build_params<double>(0.0);
        bp.keep_reaching = 1;
        bp.block_size = static_cast<long long>(bs);
        bp.out = {panels.as<double>(), kept.as<int>(), nkept.as<int>(), nao, 1};
        kumo_dev::OrbitalEnergyParams op{};
        op.scr = bp.out;
        op.block_size = static_cast<long long>(bs);
        op.count = static_cast<long long>(n_);
        op.w = st.w;
        op.ldw = st.ldw;
        op.nchunks = st.nchunks;
        op.chunk_set = st.chunk_set;
        op.col_energy = st.energy;
        op.have_virtuals = oe_needs_.virtuals ? 1 : 0;
        op.have_fukui = oe_needs_.fukui ? 1 : 0;
        for (const auto& [key, ptr] : outs_) {
            if (!detail::is_orbital_energy_kind(key.kind)) continue;
            op.kinds[op.nout] = static_cast<int>(key.kind);
            op.outs[op.nout++] = ptr;
        }
        for (std::size_t b0 = 0; b0 < nblocks; b0 += static_cast<std::size_t>(W)) {
            const int nb = static_cast<int>(std::min<std::size_t>(W, nblocks - b0));
            bp.first_point = static_cast<long long>(b0 * bs);
            bp.nblocks = nb;
            kumo_dev::launch_ao_build<double>(bp, 0, 1, stream_);
            op.first_point = bp.first_point;
            op.nblocks = nb;
            kumo_dev::launch_orbital_energy_f64(op, stream_);
        }
        completed_ += n_;
    }

    void run_orbital_waves(kumo_dev::AoBuildParams<double>& bp, kumo_dev::OrbitalParams& op, std::size_t nblocks, int W,
                           std::size_t bs, int order, int npanel) {
        for (std::size_t b0 = 0; b0 < nblocks; b0 += static_cast<std::size_t>(W)) {
            const int nb = static_cast<int>(std::min<std::size_t>(W, nblocks - b0));
            bp.first_point = static_cast<long long>(b0 * bs);
            bp.nblocks = nb;
            kumo_dev::launch_ao_build<double>(bp, order, npanel, stream_);
            op.first_point = bp.first_point;
            op.nblocks = nb;
            kumo_dev::launch_orbitals_f64(op, stream_);
        }
    }

    void potential_pass() {
        double* out = nullptr;
        for (const auto& [key, ptr] : outs_)
            if (key.kind == PropertyKind::ElectrostaticPotential) out = ptr;
        // potential_tolerance as the reference's (src/electrostatic_potential.cpp:501-521:
        // every value within the tolerance of the exact potential): the pairs
        // whose bounds (valid at every point) sum to at most half of it are
        // left out, the others are evaluated exactly.  The opt-in mixed
        // form adds its FP32 rounding.
        kumo_dev::EspDevice& esp = esp_state();
        kumo_dev::EspParams ep{};
        ep.esp = esp.view_for(opt_.potential_tolerance, stream_);
        ep.src = src_;
        ep.out = out;
        ep.mixed = opt_.precision == Precision::Mixed && esp_mixed_opt_in();
        const int tok = detail::profile_begin(detail::kProfEsp, stream_);
        kumo_dev::launch_esp(ep, stream_);
        detail::profile_end(tok, stream_);
        detail::profile_count(detail::kProfEsp, nullptr, 0, 0.0, static_cast<double>(n_) * ep.esp.npairs, 0.0, 0.0,
                              stream_);
        completed_ += n_;
        report(0);
    }

    kumo_dev::EspDevice& esp_state();

    const Molecule& mol_;
    const EvaluationOptions& opt_;
    const Grid* grid_;
    const double* points_;
    std::size_t n_;
    cudaStream_t stream_;
    detail::Plan plan_;
    Backend backend_ = Backend::AO_P;
    detail::DeviceMolecule* dev_ = nullptr;
    kumo_dev::PointSource src_{};
    std::vector<std::pair<Property, double*>> outs_;
    std::size_t passes_ = 0, completed_ = 0;
    const ReadyCallback* ready_ = nullptr;
    detail::OrbitalEnergyNeeds oe_needs_;
    std::string oe_what_;
};

kumo_dev::EspDevice& Evaluator::Run::esp_state() { return dev_->esp_state(mol_, stream_); }

namespace {

std::vector<Property> unique_keys(const Request& request) {
    std::vector<Property> keys;
    for (const auto& p : request.properties())
        if (std::find(keys.begin(), keys.end(), p) == keys.end()) keys.push_back(p);
    return keys;
}

// A tensor-core pipeline wait that ran out leaves NaN in its block's outputs
// and a flag on the device; host-returning calls turn the flag into an error.
void check_pipeline_status(Precision precision) {
    if (precision == Precision::Mixed && kumo_dev::take_pipeline_status() != 0)
        throw std::runtime_error("mixed-precision contraction: a tensor-core pipeline wait timed out");
}

}  // namespace

Results Evaluator::evaluate(const Grid& grid, const Request& request) const {
    const std::size_t n = detail::validated_point_count(grid);
    Run run(*this, &grid, nullptr, n, request, nullptr);
    const auto keys = unique_keys(request);
    std::size_t total = 0;
    for (const auto& k : keys) total += property_channels(k.kind) * n;
    DeviceAlloc out(sizeof(double) * std::max<std::size_t>(total, 1), nullptr);
    std::vector<std::pair<Property, double*>> outs;
    std::size_t off = 0;
    for (const auto& k : keys) {
        outs.emplace_back(k, out.as<double>() + off);
        off += property_channels(k.kind) * n;
    }
    if (total) check_cuda(cudaMemsetAsync(out.as<double>(), 0, sizeof(double) * total, nullptr), "cudaMemsetAsync");
    run.execute(outs);
    Results res;
    res.backend_used_ = run.backend();
    std::vector<double> host(total);
    if (total) check_cuda(cudaMemcpy(host.data(), out.as<double>(), sizeof(double) * total, cudaMemcpyDeviceToHost),
                          "cudaMemcpy (results)");
    check_pipeline_status(options_.precision);
    off = 0;
    for (const auto& k : keys) {
        PropertyField f;
        f.points = n;
        const std::size_t ch = property_channels(k.kind);
        f.components.resize(ch);
        for (std::size_t c = 0; c < ch; ++c) {
            f.components[c].assign(host.begin() + static_cast<std::ptrdiff_t>(off), host.begin() + static_cast<std::ptrdiff_t>(off + n));
            off += n;
        }
        res.fields_.emplace(k, std::move(f));
    }
    return res;
}

Results Evaluator::evaluate(Points points, const Request& request) const {
    for (std::size_t i = 0; i < 3 * points.count; ++i)
        if (!std::isfinite(points.data[i])) throw std::invalid_argument("evaluation points must be finite");
    const std::size_t n = points.count;
    DeviceAlloc dpts(sizeof(double) * 3 * std::max<std::size_t>(n, 1), nullptr);
    if (n) check_cuda(cudaMemcpy(dpts.as<double>(), points.data, sizeof(double) * 3 * n, cudaMemcpyHostToDevice),
                      "cudaMemcpy (points)");
    Run run(*this, nullptr, dpts.as<double>(), n, request, nullptr);
    const auto keys = unique_keys(request);
    std::size_t total = 0;
    for (const auto& k : keys) total += property_channels(k.kind) * n;
    DeviceAlloc out(sizeof(double) * std::max<std::size_t>(total, 1), nullptr);
    std::vector<std::pair<Property, double*>> outs;
    std::size_t off = 0;
    for (const auto& k : keys) {
        outs.emplace_back(k, out.as<double>() + off);
        off += property_channels(k.kind) * n;
    }
    if (total) check_cuda(cudaMemsetAsync(out.as<double>(), 0, sizeof(double) * total, nullptr), "cudaMemsetAsync");
    run.execute(outs);
    Results res;
    res.backend_used_ = run.backend();
    std::vector<double> host(total);
    if (total) check_cuda(cudaMemcpy(host.data(), out.as<double>(), sizeof(double) * total, cudaMemcpyDeviceToHost),
                          "cudaMemcpy (results)");
    check_pipeline_status(options_.precision);
    off = 0;
    for (const auto& k : keys) {
        PropertyField f;
        f.points = n;
        const std::size_t ch = property_channels(k.kind);
        f.components.resize(ch);
        for (std::size_t c = 0; c < ch; ++c) {
            f.components[c].assign(host.begin() + static_cast<std::ptrdiff_t>(off), host.begin() + static_cast<std::ptrdiff_t>(off + n));
            off += n;
        }
        res.fields_.emplace(k, std::move(f));
    }
    return res;
}

namespace detail {
void set_tile_probing(bool on) { t_probe_tiles = on; }

std::string tile_tuning_report() {
    TileTuner& tt = tile_tuner();
    std::lock_guard<std::mutex> lock(tt.mu);
    std::string out;
    for (const auto& [key, rank] : tt.ranked) {
        out += key;
        for (const auto& r : rank) {
            char b[64];
            std::snprintf(b, sizeof b, " %dx%dx%d:%.4fms", 1 << r.sa, 1 << r.sb, 1 << r.sc, r.ms);
            out += b;
        }
        out += '\n';
    }
    return out;
}
}  // namespace detail

void Evaluator::validate(const Request& request) const { Run run(*this, nullptr, nullptr, 0, request, nullptr); }

Backend Evaluator::evaluate_device(const Grid& grid, const Request& request, double* const* outputs, void* stream,
                                   const ReadyCallback& ready) const {
    const std::size_t n = detail::validated_point_count(grid);
    Run run(*this, &grid, nullptr, n, request, static_cast<cudaStream_t>(stream));
    std::vector<std::pair<Property, double*>> outs;
    for (std::size_t i = 0; i < request.properties().size(); ++i) outs.emplace_back(request.properties()[i], outputs[i]);
    run.execute(outs, ready);
    return run.backend();
}

Backend Evaluator::evaluate_device(Points device_points, const Request& request, double* const* outputs, void* stream,
                                   const ReadyCallback& ready) const {
    Run run(*this, nullptr, device_points.data, device_points.count, request, static_cast<cudaStream_t>(stream));
    std::vector<std::pair<Property, double*>> outs;
    for (std::size_t i = 0; i < request.properties().size(); ++i) outs.emplace_back(request.properties()[i], outputs[i]);
    run.execute(outs, ready);
    return run.backend();
}

Field Evaluator::field(const Grid& grid, Property property) const {
    if (property_channels(property.kind) != 1)
        throw std::invalid_argument(
            "Evaluator::field needs a one-component property (not a gradient, a Hessian or the Cartesian terms of G "
            "or K)");
    const auto results = evaluate(grid, Request().add(property));
    const auto v = results.get(property).component();
    return Field(grid, molecule_->atoms(), std::vector<double>(v.begin(), v.end()));
}

}  // namespace chem::kumo
