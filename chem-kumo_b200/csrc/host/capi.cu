// extern "C" boundary of the B200 grid evaluator (include/kumo_b200.h).
#include "kumo_b200.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <new>
#include <stdexcept>
#include <string>
#include <array>
#include <mutex>
#include <vector>

#include "../cuda/esp.cuh"
#include "../cuda/func_attr.cuh"
#include "../cuda/mixed.cuh"
#include "grid_geometry.hpp"
#include "chem/kumo/cube.hpp"
#include "chem/kumo/evaluator.hpp"
#include "chem/kumo/server.hpp"
#include "chem/kumo/surface.hpp"
#include "device_state.hpp"
#include "profile.hpp"

namespace chem::kumo::detail {
std::string tile_tuning_report();  // evaluator.cu
}

struct kumo_molecule {
    chem::kumo::Molecule mol;
};

struct kumo_surface {
    chem::kumo::TriangleMesh mesh;
    std::vector<chem::kumo::IVec3> cells;
    std::vector<std::vector<double>> values;
    std::vector<chem::kumo::SurfaceStatistics> stats;
};

namespace {

using namespace chem::kumo;

void put(char* err, size_t errlen, const std::string& msg) {
    if (err && errlen) {
        const size_t n = std::min(errlen - 1, msg.size());
        std::memcpy(err, msg.data(), n);
        err[n] = '\0';
    }
}

template <typename F>
int guarded(char* err, size_t errlen, F&& f) {
    try {
        f();
        put(err, errlen, "");
        return KUMO_OK;
    } catch (const std::bad_alloc& e) {
        put(err, errlen, "out of memory");
        return KUMO_OUT_OF_MEMORY;
    } catch (const std::out_of_range& e) {
        put(err, errlen, e.what());
        return KUMO_OUT_OF_RANGE;
    } catch (const std::invalid_argument& e) {
        put(err, errlen, e.what());
        return KUMO_INVALID_ARGUMENT;
    } catch (const std::runtime_error& e) {
        const std::string w = e.what();
        put(err, errlen, w);
        return w.rfind("CUDA error", 0) == 0 ? KUMO_CUDA_ERROR : KUMO_RUNTIME_ERROR;
    } catch (const std::exception& e) {
        put(err, errlen, e.what());
        return KUMO_RUNTIME_ERROR;
    } catch (...) {
        put(err, errlen, "unknown error");
        return KUMO_RUNTIME_ERROR;
    }
}

EvaluationOptions to_options(const kumo_options* o) {
    EvaluationOptions e;
    if (!o) return e;
    if (o->block_size < 0) throw std::invalid_argument("evaluation block_size must be in [1, 65536]");
    e.block_size = static_cast<std::size_t>(o->block_size);
    if (o->backend < 0 || o->backend > 2) throw std::invalid_argument("unknown evaluation backend");
    e.backend = static_cast<Backend>(o->backend);
    e.screening_threshold = o->screening_threshold;
    e.potential_tolerance = o->potential_tolerance;
    if (o->precision != 0 && o->precision != 1) throw std::invalid_argument("unknown precision");
    e.precision = o->precision ? Precision::Mixed : Precision::FP64;
    e.fukui_delta = o->fukui_delta;
    return e;
}

void fill_stats(const SurfaceStatistics& s, kumo_surface_stats* o, long long* minima, long long cap_min,
                long long* maxima, long long cap_max) {
    if (o) {
        o->area = s.area;
        o->positive_area = s.positive_area;
        o->negative_area = s.negative_area;
        o->nonpolar_area = s.nonpolar_area;
        o->minimum = s.minimum;
        o->maximum = s.maximum;
        o->minimum_vertex = static_cast<long long>(s.minimum_vertex);
        o->maximum_vertex = static_cast<long long>(s.maximum_vertex);
        o->average = s.average;
        o->positive_average = s.positive_average;
        o->negative_average = s.negative_average;
        o->positive_variance = s.positive_variance;
        o->negative_variance = s.negative_variance;
        o->total_variance = s.total_variance;
        o->balance = s.balance;
        o->charge_separation = s.charge_separation;
        o->polarity_index = s.polarity_index;
        o->n_local_minima = static_cast<long long>(s.local_minima.size());
        o->n_local_maxima = static_cast<long long>(s.local_maxima.size());
    }
    for (long long i = 0; minima && i < cap_min && i < static_cast<long long>(s.local_minima.size()); ++i)
        minima[i] = static_cast<long long>(s.local_minima[static_cast<std::size_t>(i)]);
    for (long long i = 0; maxima && i < cap_max && i < static_cast<long long>(s.local_maxima.size()); ++i)
        maxima[i] = static_cast<long long>(s.local_maxima[static_cast<std::size_t>(i)]);
}

TriangleMesh to_mesh(const double* vertices, long long nv, const long long* triangles, long long nt) {
    if (nv < 0 || nt < 0 || (nv > 0 && !vertices) || (nt > 0 && !triangles))
        throw std::invalid_argument("invalid mesh arrays");
    TriangleMesh mesh;
    mesh.vertices.resize(static_cast<std::size_t>(nv));
    for (long long v = 0; v < nv; ++v)
        for (int r = 0; r < 3; ++r) mesh.vertices[static_cast<std::size_t>(v)][static_cast<std::size_t>(r)] = vertices[3 * v + r];
    mesh.triangles.resize(static_cast<std::size_t>(nt));
    for (long long t = 0; t < nt; ++t)
        for (int r = 0; r < 3; ++r) {
            if (triangles[3 * t + r] < 0) throw std::invalid_argument("surface triangle refers to a missing vertex");
            mesh.triangles[static_cast<std::size_t>(t)][static_cast<std::size_t>(r)] =
                static_cast<std::size_t>(triangles[3 * t + r]);
        }
    return mesh;
}

Grid to_grid(const kumo_grid* g) {
    if (!g) throw std::invalid_argument("null grid");
    Grid r;
    for (int k = 0; k < 3; ++k) r.origin[k] = g->origin[k];
    for (int i = 0; i < 9; ++i) r.steps.m[static_cast<std::size_t>(i)] = g->steps[i];
    for (int k = 0; k < 3; ++k) r.counts[k] = g->counts[k];
    return r;
}

Request to_request(const kumo_property* props, int n) {
    if (n < 0 || (n > 0 && !props)) throw std::invalid_argument("invalid property list");
    Request r;
    for (int i = 0; i < n; ++i) {
        if (props[i].kind < 0 || props[i].kind > static_cast<int>(PropertyKind::LolTsirelsonStash))
            throw std::invalid_argument("unknown property kind");
        if (props[i].component < 0 || props[i].component > 3) throw std::invalid_argument("invalid density spin component");
        if (props[i].channel < 0 || props[i].channel > 1) throw std::invalid_argument("MO spin channel must be alpha or beta");
        if (props[i].orbital_index < 0) throw std::invalid_argument("orbital indices are one-based");
        r.add({static_cast<PropertyKind>(props[i].kind), static_cast<DensityComponent>(props[i].component),
               static_cast<SpinChannel>(props[i].channel), static_cast<std::size_t>(props[i].orbital_index)});
    }
    return r;
}

// A non-blocking stream per device for result copies that overlap the
// evaluation (it waits only on events of the evaluation's stream).
cudaStream_t copy_stream() {
    static std::mutex mu;
    static std::array<cudaStream_t, 64> streams{};
    int dev = 0;
    detail::check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev < 0 || dev >= static_cast<int>(streams.size())) throw std::runtime_error("device index out of range");
    std::lock_guard<std::mutex> lock(mu);
    if (!streams[static_cast<std::size_t>(dev)])
        detail::check_cuda(cudaStreamCreateWithFlags(&streams[static_cast<std::size_t>(dev)], cudaStreamNonBlocking),
                           "cudaStreamCreateWithFlags (copies)");
    return streams[static_cast<std::size_t>(dev)];
}

bool page_locked(const void* p) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        (void)cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

// Evaluation into the caller's host arrays: device outputs from the
// stream-ordered pool, the device evaluation, and device-to-host copies
// straight into the caller's arrays (no intermediate host copies).  When
// every output is page-locked, each finished range of points (the
// evaluator's ready callback, after each wave of blocks) is copied on a
// separate stream while the next wave runs; otherwise all results are copied
// at the end.
template <typename Launch>
Backend evaluate_to_host(const Request& req, std::size_t n, double* const* outputs, Precision precision,
                         Launch&& launch) {
    const auto& props = req.properties();
    std::vector<std::size_t> chans(props.size());
    std::size_t total = 0;
    bool locked = true;
    for (std::size_t i = 0; i < props.size(); ++i) {
        chans[i] = property_channels(props[i].kind);
        total += chans[i] * n;
        locked = locked && (n == 0 || page_locked(outputs[i]));
    }
    void* dev = nullptr;
    if (total) detail::check_cuda(cudaMallocAsync(&dev, sizeof(double) * total, nullptr), "cudaMallocAsync (outputs)");
    cudaStream_t cs = locked && total ? copy_stream() : nullptr;
    cudaEvent_t ev = nullptr;
    if (cs) detail::check_cuda(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "cudaEventCreateWithFlags");
    // Declared after `dev`: on every exit the copies end before the buffer is freed.
    struct Release {
        void* dev;
        cudaStream_t cs;
        cudaEvent_t ev;
        ~Release() {
            if (cs) cudaStreamSynchronize(cs);
            if (ev) cudaEventDestroy(ev);
            if (dev) cudaFreeAsync(dev, nullptr);
        }
    } guard{dev, cs, ev};
    std::vector<double*> dptr(props.size());
    std::size_t off = 0;
    for (std::size_t i = 0; i < props.size(); ++i) {
        dptr[i] = static_cast<double*>(dev) + off;
        off += chans[i] * n;
    }
    if (total)
        detail::check_cuda(cudaMemsetAsync(dev, 0, sizeof(double) * total, nullptr), "cudaMemsetAsync (outputs)");
    std::size_t copied = 0;
    // Points [copied, done) of every channel, on the copy stream once the
    // evaluation's launches enqueued so far have run.
    auto copy_range = [&](std::size_t done) {
        if (!cs || done <= copied) return;
        detail::check_cuda(cudaEventRecord(ev, nullptr), "cudaEventRecord");
        detail::check_cuda(cudaStreamWaitEvent(cs, ev, 0), "cudaStreamWaitEvent");
        for (std::size_t i = 0; i < props.size(); ++i)
            for (std::size_t c = 0; c < chans[i]; ++c)
                detail::check_cuda(cudaMemcpyAsync(outputs[i] + c * n + copied, dptr[i] + c * n + copied,
                                                   sizeof(double) * (done - copied), cudaMemcpyDeviceToHost, cs),
                                   "cudaMemcpyAsync (results)");
        copied = done;
    };
    const Evaluator::ReadyCallback ready = [&](std::size_t done) { copy_range(done); };
    const Backend used = launch(dptr.data(), cs ? ready : Evaluator::ReadyCallback{});
    if (cs) {
        copy_range(n);
        detail::check_cuda(cudaStreamSynchronize(cs), "cudaStreamSynchronize (results)");
    } else {
        for (std::size_t i = 0; i < props.size(); ++i)
            if (chans[i] * n)
                detail::check_cuda(cudaMemcpyAsync(outputs[i], dptr[i], sizeof(double) * chans[i] * n,
                                                   cudaMemcpyDeviceToHost, nullptr),
                                   "cudaMemcpyAsync (results)");
    }
    detail::check_cuda(cudaStreamSynchronize(nullptr), "cudaStreamSynchronize (results)");
    if (precision == Precision::Mixed && kumo_dev::take_pipeline_status() != 0)
        throw std::runtime_error("mixed-precision contraction: a tensor-core pipeline wait timed out");
    return used;
}

struct DevBuf {
    void* p = nullptr;
    explicit DevBuf(std::size_t bytes) { detail::check_cuda(cudaMalloc(&p, std::max<std::size_t>(bytes, 16)), "cudaMalloc"); }
    ~DevBuf() { cudaFree(p); }
    template <typename T>
    T* as() const {
        return static_cast<T*>(p);
    }
};

template <typename T>
[[maybe_unused]] void run_ao_build(const detail::DeviceMolecule& d, const kumo_dev::PointSource& src, long long block_size, int nblocks,
                  int order, int npanel, double threshold, kumo_dev::AoScratch<T> out, long long first_point) {
    kumo_dev::AoBuildParams<T> p{};
    p.basis = d.basis;
    p.src = src;
    p.first_point = first_point;
    p.block_size = block_size;
    p.nblocks = nblocks;
    p.threshold = threshold;
    p.out = out;
    for (int l = 0; l < 3; ++l)
        for (int i = 0; i < 135; ++i) p.pure[l][i] = sizeof(T) == 8 ? static_cast<T>(d.pure_d[l][i]) : static_cast<T>(d.pure_f[l][i]);
    kumo_dev::launch_ao_build<T>(p, order, npanel, nullptr);
    detail::check_cuda(cudaGetLastError(), "ao_build launch");
}

}  // namespace

extern "C" {

void kumo_default_options(kumo_options* opt) {
    if (!opt) return;
    opt->block_size = 128;
    opt->backend = 0;
    opt->screening_threshold = default_screening_threshold;
    opt->potential_tolerance = 1e-8;
    opt->precision = 0;
    opt->fukui_delta = 0.1;
}

int kumo_set_device(int device, char* err, size_t errlen) {
    return guarded(err, errlen, [&] { detail::check_cuda(cudaSetDevice(device), "cudaSetDevice"); });
}

int kumo_preload_kernels(char* err, size_t errlen) {
    return guarded(err, errlen, [&] { kumo_dev::preload_kernels(); });
}

int kumo_registered_kernels(void) { return static_cast<int>(kumo_dev::kernel_registry().size()); }

int kumo_molecule_from_fchk(const char* path, kumo_molecule** out, char* err, size_t errlen) {
    return guarded(err, errlen, [&] {
        if (!path || !out) throw std::invalid_argument("null argument");
        *out = new kumo_molecule{Molecule::from_fchk(path)};
    });
}

int kumo_molecule_from_arrays(int natoms, const int* z, const double* charges, const double* coords, int nshell,
                              const int* shell_types, const int* nprim, const int* shell_atom, const double* exponents,
                              const double* coefs, const double* p_coefs, const double* shell_xyz, int nbasis,
                              const double* packed_total, const double* packed_spin, int nalpha, int nbeta,
                              const double* alpha_mos, int nmo_alpha, const double* beta_mos, int nmo_beta,
                              kumo_molecule** out, char* err, size_t errlen) {
    return guarded(err, errlen, [&] {
        if (!out || natoms <= 0 || nshell <= 0 || nbasis <= 0 || !z || !coords || !shell_types || !nprim ||
            !shell_atom || !exponents || !coefs || !shell_xyz || !packed_total)
            throw std::invalid_argument("invalid molecule arrays");
        std::vector<Atom> atoms;
        for (int i = 0; i < natoms; ++i)
            atoms.push_back({z[i], charges ? charges[i] : static_cast<double>(z[i]),
                             {coords[3 * i], coords[3 * i + 1], coords[3 * i + 2]}});
        std::vector<Shell> shells;
        std::size_t off = 0;
        for (int s = 0; s < nshell; ++s) {
            Shell sh;
            const int t = shell_types[s];
            if (shell_atom[s] < 1 || shell_atom[s] > natoms) throw std::runtime_error("invalid 1-based shell center in fchk");
            if (nprim[s] <= 0) throw std::runtime_error("invalid Number of primitives per shell in fchk");
            sh.center = static_cast<std::size_t>(shell_atom[s] - 1);
            sh.is_sp = t == -1;
            sh.angular_momentum = sh.is_sp ? 1 : std::abs(t);
            sh.representation = (!sh.is_sp && t <= -2) ? ShellRepresentation::Pure : ShellRepresentation::Cartesian;
            sh.origin = {shell_xyz[3 * s], shell_xyz[3 * s + 1], shell_xyz[3 * s + 2]};
            sh.exponents.assign(exponents + off, exponents + off + nprim[s]);
            sh.coefficients.assign(coefs + off, coefs + off + nprim[s]);
            if (p_coefs)
                sh.p_coefficients.assign(p_coefs + off, p_coefs + off + nprim[s]);
            else
                sh.p_coefficients.assign(static_cast<std::size_t>(nprim[s]), 0.0);
            if (sh.is_sp && !p_coefs) throw std::runtime_error("missing P(S=P) coefficients for sp shell");
            off += static_cast<std::size_t>(nprim[s]);
            shells.push_back(std::move(sh));
        }
        BasisSet basis(std::move(shells), static_cast<std::size_t>(nbasis));
        const std::size_t n = static_cast<std::size_t>(nbasis);
        auto unpack = [n](const double* packed) {
            Matrix m(n, n);
            std::size_t q = 0;
            for (std::size_t i = 0; i < n; ++i)
                for (std::size_t j = 0; j <= i; ++j, ++q) m(i, j) = m(j, i) = packed[q];
            return m;
        };
        Matrix total = unpack(packed_total);
        Matrix spin = packed_spin ? unpack(packed_spin) : Matrix(n, n);
        Matrix ca, cb;
        if (alpha_mos && nmo_alpha > 0) {
            ca = Matrix(n, static_cast<std::size_t>(nmo_alpha));
            std::copy(alpha_mos, alpha_mos + n * static_cast<std::size_t>(nmo_alpha), ca.data());
        }
        if (beta_mos && nmo_beta > 0) {
            cb = Matrix(n, static_cast<std::size_t>(nmo_beta));
            std::copy(beta_mos, beta_mos + n * static_cast<std::size_t>(nmo_beta), cb.data());
        }
        *out = new kumo_molecule{Molecule::from_parts(std::move(atoms), std::move(basis), std::move(total), std::move(spin),
                                                      nalpha, nbeta, std::move(ca), std::move(cb), {}, {})};
    });
}

void kumo_molecule_destroy(kumo_molecule* m) { delete m; }

int kumo_molecule_info_get(const kumo_molecule* m, kumo_molecule_info* info) {
    if (!m || !info) return KUMO_INVALID_ARGUMENT;
    const auto& mol = m->mol;
    const auto& e = mol.electronic_structure_info();
    info->natoms = static_cast<int>(mol.atoms().size());
    info->nbasis = static_cast<int>(mol.basis_size());
    info->nalpha = static_cast<int>(mol.occupied_count(SpinChannel::Alpha));
    info->nbeta = static_cast<int>(mol.occupied_count(SpinChannel::Beta));
    info->nmo_alpha = static_cast<int>(mol.orbital_count(SpinChannel::Alpha));
    info->nmo_beta = static_cast<int>(mol.orbital_count(SpinChannel::Beta));
    info->unrestricted = mol.unrestricted() ? 1 : 0;
    info->ao_mo_eligible = e.ao_mo_eligible() ? 1 : 0;
    info->check_errors[0] = e.total_absolute_error;
    info->check_errors[1] = e.total_relative_error;
    info->check_errors[2] = e.spin_absolute_error;
    info->check_errors[3] = e.spin_relative_error;
    info->nblocks = static_cast<int>(mol.blocks().size());
    info->device_bytes = static_cast<long long>(mol.device_bytes());
    return KUMO_OK;
}

int kumo_molecule_atoms(const kumo_molecule* m, int* z, double* charges, double* xyz) {
    if (!m) return KUMO_INVALID_ARGUMENT;
    const auto& atoms = m->mol.atoms();
    for (std::size_t i = 0; i < atoms.size(); ++i) {
        if (z) z[i] = atoms[i].atomic_number;
        if (charges) charges[i] = atoms[i].nuclear_charge;
        if (xyz)
            for (int k = 0; k < 3; ++k) xyz[3 * i + static_cast<std::size_t>(k)] = atoms[i].position[k];
    }
    return KUMO_OK;
}

int kumo_molecule_block(const kumo_molecule* m, int i, int* l, int* nprim, int* offset, int* count, int* pure,
                        double* cutoff_r2) {
    if (!m || i < 0 || static_cast<std::size_t>(i) >= m->mol.blocks().size()) return KUMO_OUT_OF_RANGE;
    const auto& b = m->mol.blocks()[static_cast<std::size_t>(i)];
    *l = b.angular_momentum;
    *nprim = static_cast<int>(b.exponents.size());
    *offset = static_cast<int>(b.offset);
    *count = static_cast<int>(b.count);
    *pure = b.pure ? 1 : 0;
    *cutoff_r2 = b.cutoff_radius2;
    return KUMO_OK;
}

int kumo_evaluate_grid(const kumo_molecule* m, const kumo_options* opt, const kumo_grid* grid, const kumo_property* props,
                       int nprops, double* const* outputs, int* backend_used, char* err, size_t errlen) {
    return guarded(err, errlen, [&] {
        if (!m) throw std::invalid_argument("null molecule");
        const Grid g = to_grid(grid);
        const Request req = to_request(props, nprops);
        const EvaluationOptions o = to_options(opt);
        Evaluator ev(m->mol, o);
        const std::size_t n = detail::validated_point_count(g);
        ev.validate(req);
        if (!outputs && nprops > 0) throw std::invalid_argument("null outputs");
        const Backend b = evaluate_to_host(req, n, outputs, o.precision,
                                           [&](double* const* d, const Evaluator::ReadyCallback& ready) {
                                               return ev.evaluate_device(g, req, d, nullptr, ready);
                                           });
        if (backend_used) *backend_used = static_cast<int>(b);
    });
}

int kumo_evaluate_points(const kumo_molecule* m, const kumo_options* opt, const double* points, long long npoints,
                         const kumo_property* props, int nprops, double* const* outputs, int* backend_used, char* err,
                         size_t errlen) {
    return guarded(err, errlen, [&] {
        if (!m || npoints < 0 || (npoints > 0 && !points)) throw std::invalid_argument("invalid points");
        const Request req = to_request(props, nprops);
        const EvaluationOptions o = to_options(opt);
        Evaluator ev(m->mol, o);
        const std::size_t n = static_cast<std::size_t>(npoints);
        for (std::size_t i = 0; i < 3 * n; ++i)
            if (!std::isfinite(points[i])) throw std::invalid_argument("evaluation points must be finite");
        ev.validate(req);
        if (!outputs && nprops > 0) throw std::invalid_argument("null outputs");
        void* dpts = nullptr;
        detail::check_cuda(cudaMallocAsync(&dpts, sizeof(double) * 3 * std::max<std::size_t>(n, 1), nullptr),
                           "cudaMallocAsync (points)");
        struct Free {
            void* p;
            ~Free() { cudaFreeAsync(p, nullptr); }
        } guard{dpts};
        if (n)
            detail::check_cuda(cudaMemcpyAsync(dpts, points, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, nullptr),
                               "cudaMemcpyAsync (points)");
        const Backend b =
            evaluate_to_host(req, n, outputs, o.precision, [&](double* const* d, const Evaluator::ReadyCallback& ready) {
                return ev.evaluate_device(Points{static_cast<const double*>(dpts), n}, req, d, nullptr, ready);
            });
        if (backend_used) *backend_used = static_cast<int>(b);
    });
}

int kumo_evaluate_grid_device(const kumo_molecule* m, const kumo_options* opt, const kumo_grid* grid,
                              const kumo_property* props, int nprops, double* const* outputs, void* stream,
                              int* backend_used, char* err, size_t errlen) {
    return guarded(err, errlen, [&] {
        if (!m) throw std::invalid_argument("null molecule");
        const Grid g = to_grid(grid);
        const Request req = to_request(props, nprops);
        Evaluator ev(m->mol, to_options(opt));
        const Backend b = ev.evaluate_device(g, req, outputs, stream);
        if (backend_used) *backend_used = static_cast<int>(b);
    });
}

int kumo_evaluate_points_device(const kumo_molecule* m, const kumo_options* opt, const double* device_points,
                                long long npoints, const kumo_property* props, int nprops, double* const* outputs,
                                void* stream, int* backend_used, char* err, size_t errlen) {
    return guarded(err, errlen, [&] {
        if (!m || npoints < 0) throw std::invalid_argument("invalid points");
        const Request req = to_request(props, nprops);
        Evaluator ev(m->mol, to_options(opt));
        const Backend b = ev.evaluate_device(Points{device_points, static_cast<std::size_t>(npoints)}, req, outputs, stream);
        if (backend_used) *backend_used = static_cast<int>(b);
    });
}

int kumo_ao_panels(const kumo_molecule* m, const double* points, int npts, int order, int precision, double* out,
                   char* err, size_t errlen) {
    return guarded(err, errlen, [&] {
        if (!m || !points || !out || npts <= 0 || npts > kumo_dev::kBlockPoints)
            throw std::invalid_argument("kumo_ao_panels needs 1 to 128 points");
        if (order < 0 || order > 2) throw std::invalid_argument("AO derivative order must be 0, 1 or 2");
        const auto& d = m->mol.device();
        const int nao = d.basis.nao;
        const int npanel = order == 0 ? 1 : (order == 1 ? 4 : 10);
        DevBuf pts(sizeof(double) * 3 * static_cast<std::size_t>(npts));
        detail::check_cuda(cudaMemcpy(pts.as<double>(), points, sizeof(double) * 3 * npts, cudaMemcpyHostToDevice), "cudaMemcpy");
        kumo_dev::PointSource src{};
        src.points = pts.as<double>();
        src.count = npts;
        DevBuf kept(sizeof(int) * nao), nkept(sizeof(int));
        const std::size_t cells = static_cast<std::size_t>(npanel) * nao * kumo_dev::kBlockPoints;
        std::vector<double> host(cells);
        if (precision == 0) {
            DevBuf panels(sizeof(double) * cells);
            run_ao_build<double>(d, src, npts, 1, order, npanel, 0.0,
                                 {panels.as<double>(), kept.as<int>(), nkept.as<int>(), nao, npanel}, 0);
            detail::check_cuda(cudaMemcpy(host.data(), panels.as<double>(), sizeof(double) * cells, cudaMemcpyDeviceToHost), "cudaMemcpy");
        } else {
            // Mixed-form AO build: rows of the AO blocks within reach, kept[row] = AO index.
            DevBuf panels(sizeof(float) * cells), rowmax(sizeof(float) * 4 * nao);
            kumo_dev::AoMixedParams p{};
            p.basis = d.basis;
            p.prims = d.mix_prims;
            p.src = src;
            p.block_size = npts;
            p.nblocks = 1;
            std::memcpy(p.tpure, d.tpure_g, sizeof p.tpure);
            std::memcpy(p.gcart, d.gcart, sizeof p.gcart);
            p.out = {panels.as<float>(), kept.as<int>(), nkept.as<int>(), nao, npanel, rowmax.as<float>()};
            kumo_dev::launch_ao_mixed(p, npanel, nullptr);
            detail::check_cuda(cudaGetLastError(), "ao_mixed launch");
            std::vector<float> hf(cells);
            std::vector<int> rows(static_cast<std::size_t>(nao));
            int nrows = 0;
            detail::check_cuda(cudaMemcpy(hf.data(), panels.as<float>(), sizeof(float) * cells, cudaMemcpyDeviceToHost), "cudaMemcpy");
            detail::check_cuda(cudaMemcpy(&nrows, nkept.as<int>(), sizeof(int), cudaMemcpyDeviceToHost), "cudaMemcpy");
            detail::check_cuda(cudaMemcpy(rows.data(), kept.as<int>(), sizeof(int) * nao, cudaMemcpyDeviceToHost), "cudaMemcpy");
            std::fill(host.begin(), host.end(), 0.0);
            for (int c = 0; c < npanel; ++c)
                for (int r = 0; r < nrows; ++r)
                    for (int j = 0; j < kumo_dev::kBlockPoints; ++j)
                        host[(static_cast<std::size_t>(c) * nao + rows[r]) * kumo_dev::kBlockPoints + j] =
                            hf[(static_cast<std::size_t>(c) * nao + r) * kumo_dev::kBlockPoints + j];
        }
        // scratch [c][ao][point] -> out column-major nao x (panels * npts)
        for (int c = 0; c < npanel; ++c)
            for (int a = 0; a < nao; ++a)
                for (int j = 0; j < npts; ++j)
                    out[(static_cast<std::size_t>(c) * npts + j) * nao + a] =
                        host[(static_cast<std::size_t>(c) * nao + a) * kumo_dev::kBlockPoints + j];
    });
}

int kumo_screening_masks(const kumo_molecule* m, const kumo_grid* grid, long long block_size, int ao_order,
                         double threshold, unsigned char* mask, char* err, size_t errlen) {
    return guarded(err, errlen, [&] {
        if (!m || !mask) throw std::invalid_argument("null argument");
        if (block_size <= 0 || block_size > static_cast<long long>(max_block_size))
            throw std::invalid_argument("evaluation block_size must be in [1, " + std::to_string(max_block_size) + "]");
        if (ao_order < 0 || ao_order > 2) throw std::invalid_argument("AO derivative order must be 0, 1 or 2");
        const Grid g = to_grid(grid);
        const long long n = static_cast<long long>(g.counts[0]) * g.counts[1] * g.counts[2];
        const auto& d = m->mol.device();
        const int nao = d.basis.nao;
        const int npanel = ao_order == 0 ? 1 : (ao_order == 1 ? 4 : 10);
        kumo_dev::PointSource src{};
        for (int k = 0; k < 3; ++k) src.origin[k] = g.origin[k];
        for (int i = 0; i < 9; ++i) src.steps[i] = g.steps.m[static_cast<std::size_t>(i)];
        src.ny = g.counts[1];
        src.nz = g.counts[2];
        src.count = n;
        const long long nblocks = (n + block_size - 1) / block_size;
        if (block_size > kumo_dev::kBlockPoints) {
            // Blocks above 128 points: the maximum of each AO over the whole
            // block from chunks of 128 points (the AO build's first screening
            // launch), compared with the threshold here.
            const long long per = (block_size + kumo_dev::kBlockPoints - 1) / kumo_dev::kBlockPoints;
            const long long ws = std::max<long long>(1, 256 / per);
            DevBuf panels(sizeof(double) * static_cast<std::size_t>(npanel) * nao * kumo_dev::kBlockPoints * ws * per);
            DevBuf kept(sizeof(int) * static_cast<std::size_t>(nao) * ws * per), nkept(sizeof(int) * ws * per);
            DevBuf bmax(sizeof(double) * static_cast<std::size_t>(nao) * ws);
            std::vector<double> hm(static_cast<std::size_t>(nao) * ws);
            for (long long b0 = 0; b0 < nblocks; b0 += ws) {
                const long long nb = std::min(ws, nblocks - b0);
                kumo_dev::AoBuildParams<double> p{};
                p.basis = d.basis;
                p.src = src;
                p.first_point = b0 * block_size;
                p.block_size = kumo_dev::kBlockPoints;
                p.screen_block = block_size;
                p.nblocks = static_cast<int>(nb * per);
                p.threshold = threshold;
                p.out = {panels.as<double>(), kept.as<int>(), nkept.as<int>(), nao, npanel};
                p.mask_pass = 1;
                p.block_max = bmax.as<double>();
                for (int l = 0; l < 3; ++l)
                    for (int i = 0; i < 135; ++i) p.pure[l][i] = d.pure_d[l][i];
                detail::check_cuda(cudaMemset(bmax.as<double>(), 0, sizeof(double) * nao * nb), "cudaMemset");
                kumo_dev::launch_ao_build<double>(p, ao_order, npanel, nullptr);
                detail::check_cuda(cudaGetLastError(), "ao_build launch");
                detail::check_cuda(cudaMemcpy(hm.data(), bmax.as<double>(), sizeof(double) * nao * nb, cudaMemcpyDeviceToHost),
                                   "cudaMemcpy");
                for (long long b = 0; b < nb; ++b)
                    for (int a = 0; a < nao; ++a)
                        mask[(b0 + b) * nao + a] = (threshold == 0.0 || hm[static_cast<std::size_t>(b * nao + a)] > threshold) ? 1 : 0;
            }
            return;
        }
        const int W = static_cast<int>(std::min<long long>(nblocks, 256));
        DevBuf panels(sizeof(double) * static_cast<std::size_t>(npanel) * nao * kumo_dev::kBlockPoints * W);
        DevBuf kept(sizeof(int) * static_cast<std::size_t>(nao) * W), nkept(sizeof(int) * W);
        std::vector<int> hk(static_cast<std::size_t>(nao) * W), hn(W);
        std::fill(mask, mask + nblocks * nao, 0);
        for (long long b0 = 0; b0 < nblocks; b0 += W) {
            const int nb = static_cast<int>(std::min<long long>(W, nblocks - b0));
            run_ao_build<double>(d, src, block_size, nb, ao_order, npanel, threshold,
                                 {panels.as<double>(), kept.as<int>(), nkept.as<int>(), nao, npanel}, b0 * block_size);
            detail::check_cuda(cudaMemcpy(hk.data(), kept.as<int>(), sizeof(int) * nao * nb, cudaMemcpyDeviceToHost), "cudaMemcpy");
            detail::check_cuda(cudaMemcpy(hn.data(), nkept.as<int>(), sizeof(int) * nb, cudaMemcpyDeviceToHost), "cudaMemcpy");
            for (int b = 0; b < nb; ++b)
                for (int s = 0; s < hn[b]; ++s) mask[(b0 + b) * nao + hk[static_cast<std::size_t>(b) * nao + s]] = 1;
        }
    });
}

int kumo_boys(const double* t, long long n, int nvalues, double* out, char* err, size_t errlen) {
    return guarded(err, errlen, [&] {
        if (nvalues <= 0 || nvalues > kumo_dev::kBoysMaxOrder + 1) throw std::invalid_argument("unsupported Boys function order");
        for (long long i = 0; i < n; ++i)
            if (!std::isfinite(t[i]) || t[i] < 0.0)
                throw std::invalid_argument("Boys function argument must be finite and nonnegative");
        if (n == 0) return;
        const auto table = kumo_dev::boys_table_host();
        DevBuf dt(sizeof(double) * table.size()), din(sizeof(double) * n), dout(sizeof(double) * n * nvalues);
        detail::check_cuda(cudaMemcpy(dt.as<double>(), table.data(), sizeof(double) * table.size(), cudaMemcpyHostToDevice), "cudaMemcpy");
        detail::check_cuda(cudaMemcpy(din.as<double>(), t, sizeof(double) * n, cudaMemcpyHostToDevice), "cudaMemcpy");
        kumo_dev::launch_boys_f64(dt.as<double>(), din.as<double>(), n, nvalues, dout.as<double>(), nullptr);
        detail::check_cuda(cudaGetLastError(), "boys launch");
        detail::check_cuda(cudaMemcpy(out, dout.as<double>(), sizeof(double) * n * nvalues, cudaMemcpyDeviceToHost), "cudaMemcpy");
    });
}

int kumo_esp_pair_count(const kumo_molecule* m, long long* count, char* err, size_t errlen) {
    return guarded(err, errlen, [&] {
        if (!m || !count) throw std::invalid_argument("null argument");
        kumo_dev::EspDevice e(m->mol, nullptr);
        *count = e.pair_count();
    });
}

int kumo_esp_pairs_evaluated(const kumo_molecule* m, double tolerance, long long* count, char* err, size_t errlen) {
    return guarded(err, errlen, [&] {
        if (!m || !count) throw std::invalid_argument("null argument");
        if (!std::isfinite(tolerance) || tolerance < 0.0)
            throw std::invalid_argument("potential tolerance must be finite and nonnegative");
        auto& dev = m->mol.device();
        *count = dev.esp_state(m->mol, nullptr).view_for(tolerance, nullptr).npairs;
    });
}

int kumo_write_cube(const char* path, const char* comment, const kumo_grid* grid, int natoms, const int* z,
                    const double* charges, const double* xyz, const double* values, long long orbital_index, char* err,
                    size_t errlen) {
    return guarded(err, errlen, [&] {
        if (!path || !values || natoms < 0) throw std::invalid_argument("invalid cube arguments");
        const Grid g = to_grid(grid);
        std::vector<Atom> atoms;
        for (int i = 0; i < natoms; ++i) atoms.push_back({z[i], charges[i], {xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]}});
        const std::size_t n = static_cast<std::size_t>(g.counts[0]) * g.counts[1] * g.counts[2];
        Field f(g, std::move(atoms), std::vector<double>(values, values + n));
        if (orbital_index > 0)
            f.write_orbital_cube(path, static_cast<std::size_t>(orbital_index), comment ? comment : "Molecular orbital amplitude");
        else
            f.write_cube(path, comment ? comment : "Electron density");
    });
}

long long kumo_tile_tuning_report(char* buf, size_t len) {
    std::string r;
    try {
        r = chem::kumo::detail::tile_tuning_report();
    } catch (...) {
        return -1;
    }
    if (buf && len) {
        const size_t n = std::min(len - 1, r.size());
        std::memcpy(buf, r.data(), n);
        buf[n] = '\0';
    }
    return static_cast<long long>(r.size());
}

struct kumo_cube {
    chem::kumo::CubeData data;
};

int kumo_read_cube(const char* path, kumo_cube** out, char* err, size_t errlen) {
    return guarded(err, errlen, [&] {
        if (!path || !out) throw std::invalid_argument("null argument");
        *out = nullptr;
        *out = new kumo_cube{read_cube(path)};
    });
}

int kumo_cube_info(const kumo_cube* c, long long* natoms, kumo_grid* grid, int* angstrom) {
    if (!c) return KUMO_INVALID_ARGUMENT;
    const Grid& g = c->data.field.grid();
    if (natoms) *natoms = static_cast<long long>(c->data.field.atoms().size());
    if (grid) {
        for (int k = 0; k < 3; ++k) grid->origin[k] = g.origin[k];
        for (int i = 0; i < 9; ++i) grid->steps[i] = g.steps.m[static_cast<std::size_t>(i)];
        for (int k = 0; k < 3; ++k) grid->counts[k] = g.counts[k];
    }
    if (angstrom) *angstrom = c->data.metadata.coordinates_in_angstrom ? 1 : 0;
    return KUMO_OK;
}

int kumo_cube_data(const kumo_cube* c, int* z, double* charges, double* xyz, double* values, char* first_comment,
                   size_t first_len, char* second_comment, size_t second_len) {
    if (!c) return KUMO_INVALID_ARGUMENT;
    const auto& atoms = c->data.field.atoms();
    for (std::size_t i = 0; i < atoms.size(); ++i) {
        if (z) z[i] = atoms[i].atomic_number;
        if (charges) charges[i] = atoms[i].nuclear_charge;
        if (xyz)
            for (int k = 0; k < 3; ++k) xyz[3 * i + static_cast<std::size_t>(k)] = atoms[i].position[static_cast<std::size_t>(k)];
    }
    const auto& v = c->data.field.values();
    if (values) std::memcpy(values, v.data(), sizeof(double) * v.size());
    auto put_line = [](char* dst, size_t len, const std::string& src) {
        if (!dst || !len) return;
        const size_t n = std::min(len - 1, src.size());
        std::memcpy(dst, src.data(), n);
        dst[n] = '\0';
    };
    put_line(first_comment, first_len, c->data.metadata.first_comment);
    put_line(second_comment, second_len, c->data.metadata.second_comment);
    return KUMO_OK;
}

void kumo_cube_destroy(kumo_cube* c) { delete c; }

int kumo_write_cube_data(const char* path, const char* first_comment, const char* second_comment, int angstrom,
                         const kumo_grid* grid, long long natoms, const int* z, const double* charges, const double* xyz,
                         const double* values, char* err, size_t errlen) {
    return guarded(err, errlen, [&] {
        if (!path || !grid || !values || natoms < 0 || (natoms > 0 && (!z || !charges || !xyz)))
            throw std::invalid_argument("invalid cube arguments");
        const Grid g = to_grid(grid);
        std::vector<Atom> atoms;
        atoms.reserve(static_cast<std::size_t>(natoms));
        for (long long i = 0; i < natoms; ++i) atoms.push_back({z[i], charges[i], {xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]}});
        const std::size_t n = static_cast<std::size_t>(g.counts[0]) * g.counts[1] * g.counts[2];
        CubeData cube{Field(g, std::move(atoms), std::vector<double>(values, values + n)),
                      {first_comment ? first_comment : "", second_comment ? second_comment : "", angstrom != 0}};
        write_cube(cube, path);
    });
}

int kumo_grid_around(const kumo_molecule* m, double margin, double spacing, kumo_grid* out, char* err, size_t errlen) {
    return guarded(err, errlen, [&] {
        if (!m || !out) throw std::invalid_argument("null argument");
        const Grid g = Grid::around(m->mol.atoms(), margin, spacing);
        for (int k = 0; k < 3; ++k) out->origin[k] = g.origin[k];
        for (int i = 0; i < 9; ++i) out->steps[i] = g.steps.m[static_cast<std::size_t>(i)];
        for (int k = 0; k < 3; ++k) out->counts[k] = g.counts[k];
    });
}

void kumo_profile_enable(int on) {
    try {
        detail::profile_enable(on != 0);
    } catch (...) {
    }
}

void kumo_profile_reset(void) { detail::profile_reset(); }

int kumo_profile_read(kumo_profile_entry* out, int max_entries) {
    int n = 0;
    try {
        for (int k = 0; k < detail::kProfCount && n < max_entries; ++k) {
            const auto s = detail::profile_read(static_cast<detail::ProfileKernel>(k));
            kumo_profile_entry& e = out[n++];
            std::memset(e.name, 0, sizeof e.name);
            std::strncpy(e.name, detail::profile_name(static_cast<detail::ProfileKernel>(k)), sizeof e.name - 1);
            e.launches = s.launches;
            e.ms = s.ms;
            e.kept_rows = s.kept_rows;
            e.units = s.units;
            e.flops = s.flops;
            e.bytes = s.bytes;
        }
    } catch (...) {
        return -1;
    }
    return n;
}


struct kumo_server {
    std::unique_ptr<Server> srv;
};

int kumo_server_create(const kumo_server_options* opt, kumo_server** out, char* err, size_t errlen) {
    return guarded(err, errlen, [&] {
        if (!out) throw std::invalid_argument("null argument");
        ServerOptions o;
        if (opt) {
            o.device = opt->device;
            if (opt->hbm_budget_bytes > 0) o.hbm_budget = static_cast<std::size_t>(opt->hbm_budget_bytes);
            if (opt->max_active > 0) o.max_active = opt->max_active;
            if (opt->graph_points > 0) o.graph_points = static_cast<std::size_t>(opt->graph_points);
            if (opt->graph_points < 0) o.graph_points = 0;  // no graphs
            if (opt->request_scratch_bytes > 0) o.request_scratch = static_cast<std::size_t>(opt->request_scratch_bytes);
            if (opt->staging_bytes > 0) o.staging_bytes = static_cast<std::size_t>(opt->staging_bytes);
            if (opt->staging_bytes < 0) o.staging_bytes = 0;
        }
        auto s = std::make_unique<kumo_server>();
        s->srv = std::make_unique<Server>(o);
        *out = s.release();
    });
}

int kumo_server_destroy(kumo_server* server) {
    if (!server) return KUMO_OK;
    try {
        server->srv->drain();
    } catch (...) {
    }
    delete server;
    return KUMO_OK;
}

namespace {
int server_submit(kumo_server* server, const kumo_molecule* m, const kumo_options* opt, const kumo_grid* grid,
                  const double* points, long long npoints, const kumo_property* props, int nprops,
                  double* const* outputs, unsigned long long* ticket, char* err, size_t errlen) {
    return guarded(err, errlen, [&] {
        if (!server || !m || !ticket || (nprops > 0 && !outputs)) throw std::invalid_argument("null argument");
        ServeRequest r;
        r.molecule = &m->mol;
        r.options = to_options(opt);
        r.request = to_request(props, nprops);
        if (grid) {
            r.grid = to_grid(grid);
        } else {
            if (npoints < 0 || (npoints > 0 && !points)) throw std::invalid_argument("invalid points");
            r.points.assign(points, points + 3 * npoints);
        }
        r.outputs.assign(outputs, outputs + nprops);
        *ticket = server->srv->submit(std::move(r));
    });
}
}  // namespace

int kumo_server_submit_grid(kumo_server* server, const kumo_molecule* m, const kumo_options* opt,
                            const kumo_grid* grid, const kumo_property* props, int nprops,
                            double* const* outputs, unsigned long long* ticket, char* err, size_t errlen) {
    if (!grid) return guarded(err, errlen, [] { throw std::invalid_argument("null grid"); });
    return server_submit(server, m, opt, grid, nullptr, 0, props, nprops, outputs, ticket, err, errlen);
}

int kumo_server_submit_points(kumo_server* server, const kumo_molecule* m, const kumo_options* opt,
                              const double* points, long long npoints, const kumo_property* props, int nprops,
                              double* const* outputs, unsigned long long* ticket, char* err, size_t errlen) {
    return server_submit(server, m, opt, nullptr, points, npoints, props, nprops, outputs, ticket, err, errlen);
}

int kumo_server_wait(kumo_server* server, unsigned long long ticket, double timeout_s, int* done, char* err,
                     size_t errlen) {
    return guarded(err, errlen, [&] {
        if (!server) throw std::invalid_argument("null server");
        const bool d = server->srv->wait(ticket, timeout_s);
        if (done) *done = d ? 1 : 0;
    });
}

int kumo_server_drain(kumo_server* server, char* err, size_t errlen) {
    return guarded(err, errlen, [&] {
        if (!server) throw std::invalid_argument("null server");
        server->srv->drain();
    });
}

int kumo_server_stats_get(kumo_server* server, kumo_server_stats* out, char* err, size_t errlen) {
    return guarded(err, errlen, [&] {
        if (!server || !out) throw std::invalid_argument("null argument");
        const ServeStats s = server->srv->stats();
        out->submitted = static_cast<long long>(s.submitted);
        out->completed = static_cast<long long>(s.completed);
        out->failed = static_cast<long long>(s.failed);
        out->points = static_cast<long long>(s.points);
        out->p50_ms = s.p50_ms;
        out->p99_ms = s.p99_ms;
        out->mean_ms = s.mean_ms;
        out->max_ms = s.max_ms;
        out->busy_s = s.busy_s;
        out->points_per_s = s.points_per_s;
        out->graph_captures = static_cast<long long>(s.graph_captures);
        out->graph_replays = static_cast<long long>(s.graph_replays);
        out->direct_runs = static_cast<long long>(s.direct_runs);
        out->peak_bytes = static_cast<double>(s.peak_bytes);
        out->budget_bytes = static_cast<double>(s.budget_bytes);
        out->launch_s = s.launch_s;
        out->copy_s = s.copy_s;
        out->queue_ms = s.queue_ms;
    });
}

int kumo_server_reset_stats(kumo_server* server, char* err, size_t errlen) {
    return guarded(err, errlen, [&] {
        if (!server) throw std::invalid_argument("null server");
        server->srv->reset_stats();
    });
}

int kumo_density_isosurface(const kumo_molecule* m, double isovalue, double spacing, kumo_surface** out,
                            char* err, size_t errlen) {
    return guarded(err, errlen, [&] {
        if (!m || !out) throw std::invalid_argument("null molecule or output");
        auto s = std::make_unique<kumo_surface>();
        s->mesh = density_isosurface(m->mol, isovalue, spacing);
        *out = s.release();
    });
}

int kumo_potential_surface(const kumo_molecule* m, double isovalue, double spacing, double tolerance,
                           kumo_surface** out, char* err, size_t errlen) {
    return guarded(err, errlen, [&] {
        if (!m || !out) throw std::invalid_argument("null molecule or output");
        SurfaceOptions o;
        o.isovalue = isovalue;
        o.spacing = spacing;
        o.potential_tolerance = tolerance;
        PotentialSurface p = electrostatic_potential_surface(m->mol, o);
        auto s = std::make_unique<kumo_surface>();
        s->mesh = std::move(p.mesh);
        s->values.push_back(std::move(p.potential));
        s->stats.push_back(std::move(p.statistics));
        *out = s.release();
    });
}

int kumo_ionization_energy_surface(const kumo_molecule* m, double isovalue, double spacing, kumo_surface** out,
                                   char* err, size_t errlen) {
    return guarded(err, errlen, [&] {
        if (!m || !out) throw std::invalid_argument("null molecule or output");
        IonizationEnergySurface p = local_ionization_energy_surface(m->mol, isovalue, spacing);
        auto s = std::make_unique<kumo_surface>();
        s->mesh = std::move(p.mesh);
        s->values.push_back(std::move(p.ionization_energy));
        s->stats.push_back(std::move(p.statistics));
        *out = s.release();
    });
}

int kumo_map_on_density_isosurface(const kumo_molecule* m, const kumo_options* opt, const kumo_property* props,
                                   int nprops, double isovalue, double spacing, kumo_surface** out,
                                   int* backend_used, char* err, size_t errlen) {
    return guarded(err, errlen, [&] {
        if (!m || !out) throw std::invalid_argument("null molecule or output");
        const Request req = to_request(props, nprops);
        MappedSurface p = map_on_density_isosurface(m->mol, req.properties(), isovalue, spacing, to_options(opt));
        auto s = std::make_unique<kumo_surface>();
        s->mesh = std::move(p.mesh);
        s->values = std::move(p.values);
        s->stats = std::move(p.statistics);
        if (backend_used) *backend_used = static_cast<int>(p.backend_used);
        *out = s.release();
    });
}

int kumo_average_local_ionization_energy(const kumo_molecule* m, const double* points, long long npoints,
                                         double* out, char* err, size_t errlen) {
    return guarded(err, errlen, [&] {
        if (!m) throw std::invalid_argument("null molecule");
        if (npoints < 0 || (npoints > 0 && (!points || !out))) throw std::invalid_argument("invalid points");
        const auto v = average_local_ionization_energy(m->mol, Points{points, static_cast<std::size_t>(npoints)});
        std::copy(v.begin(), v.end(), out);
    });
}

int kumo_extract_isosurface(const kumo_grid* grid, const double* samples, double isovalue, kumo_scalar_fn fn,
                            void* user, kumo_surface** out, char* err, size_t errlen) {
    return guarded(err, errlen, [&] {
        if (!out || !fn) throw std::invalid_argument("null function or output");
        const Grid g = to_grid(grid);
        detail::validated_point_count(g);
        const detail::ScalarFunction f = [&](const std::vector<Vec3>& pts, std::vector<double>& values,
                                             std::vector<Vec3>& gradients) {
            std::vector<double> grad(3 * pts.size(), 0.0);
            fn(pts.empty() ? nullptr : pts[0].data(), static_cast<long long>(pts.size()), values.data(), grad.data(),
               user);
            for (std::size_t p = 0; p < pts.size(); ++p)
                for (int r = 0; r < 3; ++r) gradients[p][static_cast<std::size_t>(r)] = grad[3 * p + r];
        };
        detail::Isosurface iso = detail::extract_isosurface(g, samples, false, isovalue, f);
        auto s = std::make_unique<kumo_surface>();
        s->mesh = std::move(iso.mesh);
        s->cells = std::move(iso.vertex_cells);
        *out = s.release();
    });
}

void kumo_surface_info(const kumo_surface* s, long long* nvertices, long long* ntriangles, int* nfields) {
    if (nvertices) *nvertices = s ? static_cast<long long>(s->mesh.vertices.size()) : 0;
    if (ntriangles) *ntriangles = s ? static_cast<long long>(s->mesh.triangles.size()) : 0;
    if (nfields) *nfields = s ? static_cast<int>(s->values.size()) : 0;
}

void kumo_surface_mesh(const kumo_surface* s, double* vertices, long long* triangles, int* cells) {
    if (!s) return;
    for (std::size_t v = 0; v < s->mesh.vertices.size(); ++v)
        for (int r = 0; r < 3; ++r) {
            if (vertices) vertices[3 * v + static_cast<std::size_t>(r)] = s->mesh.vertices[v][static_cast<std::size_t>(r)];
            if (cells && v < s->cells.size())
                cells[3 * v + static_cast<std::size_t>(r)] = s->cells[v][static_cast<std::size_t>(r)];
        }
    if (triangles)
        for (std::size_t t = 0; t < s->mesh.triangles.size(); ++t)
            for (int r = 0; r < 3; ++r)
                triangles[3 * t + static_cast<std::size_t>(r)] =
                    static_cast<long long>(s->mesh.triangles[t][static_cast<std::size_t>(r)]);
}

int kumo_surface_field(const kumo_surface* s, int index, double* values, kumo_surface_stats* stats,
                       long long* minima, long long cap_min, long long* maxima, long long cap_max, char* err,
                       size_t errlen) {
    return guarded(err, errlen, [&] {
        if (!s || index < 0 || index >= static_cast<int>(s->values.size()))
            throw std::out_of_range("surface field index out of range");
        const auto& v = s->values[static_cast<std::size_t>(index)];
        if (values) std::copy(v.begin(), v.end(), values);
        fill_stats(s->stats[static_cast<std::size_t>(index)], stats, minima, cap_min, maxima, cap_max);
    });
}

void kumo_surface_destroy(kumo_surface* s) { delete s; }

int kumo_surface_statistics(const double* vertices, long long nvertices, const long long* triangles,
                            long long ntriangles, const double* values, double polar_threshold,
                            kumo_surface_stats* out, long long* minima, long long cap_min, long long* maxima,
                            long long cap_max, char* err, size_t errlen) {
    return guarded(err, errlen, [&] {
        const TriangleMesh mesh = to_mesh(vertices, nvertices, triangles, ntriangles);
        if (nvertices > 0 && !values) throw std::invalid_argument("surface values do not match the mesh vertices");
        const SurfaceStatistics st = surface_statistics(
            mesh, std::span<const double>(values, static_cast<std::size_t>(nvertices)), polar_threshold);
        fill_stats(st, out, minima, cap_min, maxima, cap_max);
    });
}

int kumo_write_ply(const char* path, const double* vertices, long long nvertices, const long long* triangles,
                   long long ntriangles, const char* const* names, const double* const* values, int nfields,
                   const char* const* comments, int ncomments, char* err, size_t errlen) {
    return guarded(err, errlen, [&] {
        if (!path) throw std::invalid_argument("null PLY path");
        const TriangleMesh mesh = to_mesh(vertices, nvertices, triangles, ntriangles);
        if (nfields < 0 || ncomments < 0 || (nfields > 0 && (!names || !values)) || (ncomments > 0 && !comments))
            throw std::invalid_argument("invalid PLY fields or comments");
        std::vector<std::pair<std::string, std::vector<double>>> fields;
        for (int f = 0; f < nfields; ++f) {
            if (!names[f] || (nvertices > 0 && !values[f])) throw std::invalid_argument("invalid PLY field");
            fields.emplace_back(names[f], std::vector<double>(values[f], values[f] + nvertices));
        }
        std::vector<std::string> cs;
        for (int c = 0; c < ncomments; ++c) cs.emplace_back(comments[c] ? comments[c] : "");
        write_ply(path, mesh, fields, cs);
    });
}

}  // extern "C"
