// Molecular surfaces (chem-kumo's src/surface.cpp): the density on a grid and
// the polygonization run on the device; the Newton placement of the vertices
// asks the device evaluator for the density and its gradient at all
// unconverged vertices at once; statistics, triangulation and PLY output are
// host code.
#include "chem/kumo/surface.hpp"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <limits>
#include <numeric>
#include <stdexcept>
#include <string>

#include "../cuda/isosurface.cuh"
#include "device_state.hpp"
#include "grid_geometry.hpp"

namespace chem::kumo {
namespace {

constexpr double kRootTolerance = 1e-10;  // bohr, along the edge (src/surface.cpp:63)
constexpr int kMaxRootIterations = 200;

Vec3 sub3(const Vec3& a, const Vec3& b) { return {a[0] - b[0], a[1] - b[1], a[2] - b[2]}; }
double dot3(const Vec3& a, const Vec3& b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
Vec3 cross3(const Vec3& a, const Vec3& b) {
    return {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
}
double norm3(const Vec3& a) { return std::sqrt(dot3(a, a)); }

// Grid point of a linear index: origin + steps (i, j, k).
Vec3 grid_point(const Grid& g, long long linear) {
    const long long ny = g.counts[1], nz = g.counts[2];
    const double i = static_cast<double>(linear / (ny * nz)), j = static_cast<double>((linear / nz) % ny),
                 k = static_cast<double>(linear % nz);
    Vec3 p;
    for (int r = 0; r < 3; ++r) p[r] = g.origin[r] + ((g.steps(r, 0) * i + g.steps(r, 1) * j) + g.steps(r, 2) * k);
    return p;
}

kumo_dev::IsoGrid iso_grid(const Grid& g) {
    kumo_dev::IsoGrid d{};
    for (int r = 0; r < 3; ++r) d.origin[r] = g.origin[r];
    for (int i = 0; i < 9; ++i) d.steps[i] = g.steps.m[static_cast<std::size_t>(i)];
    for (int a = 0; a < 3; ++a) d.n[a] = g.counts[a];
    return d;
}

struct DeviceBuffer {
    double* p = nullptr;
    explicit DeviceBuffer(std::size_t n) {
        detail::check_cuda(cudaMalloc(reinterpret_cast<void**>(&p), sizeof(double) * std::max<std::size_t>(n, 1)),
                           "cudaMalloc (surface)");
    }
    ~DeviceBuffer() { cudaFree(p); }
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
};

// Root of f - iso on every crossed edge (src/surface.cpp:203-259): start at
// the linear interpolation of the samples, then Newton steps safeguarded by
// bisection, all unconverged vertices evaluated at once.
std::vector<Vec3> place_vertices(const Grid& grid, double iso, const std::vector<kumo_dev::IsoEdge>& edges,
                                 const detail::ScalarFunction& function) {
    const std::size_t nv = edges.size();
    std::vector<double> t(nv), low(nv, 0.0), high(nv, 1.0);
    std::vector<Vec3> a(nv), b(nv);
    for (std::size_t v = 0; v < nv; ++v) {
        const double fa = edges[v].f_inside, fb = edges[v].f_outside;
        t[v] = std::clamp((fa - iso) / (fa - fb), 0.0, 1.0);
        a[v] = grid_point(grid, edges[v].inside);
        b[v] = grid_point(grid, edges[v].outside);
    }
    std::vector<std::size_t> active(nv);
    std::iota(active.begin(), active.end(), std::size_t{0});
    std::vector<Vec3> points, gradients;
    std::vector<double> values;
    for (int iteration = 0; !active.empty(); ++iteration) {
        if (iteration == kMaxRootIterations) throw std::runtime_error("isosurface vertices did not converge");
        points.resize(active.size());
        values.assign(active.size(), 0.0);
        gradients.assign(active.size(), Vec3{0.0, 0.0, 0.0});
        for (std::size_t p = 0; p < active.size(); ++p) {
            const std::size_t v = active[p];
            const Vec3 d = sub3(b[v], a[v]);
            for (int r = 0; r < 3; ++r) points[p][r] = a[v][r] + t[v] * d[r];
        }
        function(points, values, gradients);
        std::vector<std::size_t> next;
        for (std::size_t p = 0; p < active.size(); ++p) {
            const std::size_t v = active[p];
            const double g = values[p] - iso;
            if (!std::isfinite(g) || !std::isfinite(gradients[p][0]) || !std::isfinite(gradients[p][1]) ||
                !std::isfinite(gradients[p][2]))
                throw std::runtime_error("isosurface function is not finite");
            if (g == 0.0) continue;
            (g > 0.0 ? low[v] : high[v]) = t[v];
            const Vec3 d = sub3(b[v], a[v]);
            const double length = norm3(d);
            double step = t[v] - g / dot3(gradients[p], d);
            if (!(step > low[v] && step < high[v])) step = 0.5 * (low[v] + high[v]);
            const double moved = std::abs(step - t[v]) * length;
            t[v] = step;
            if (moved > kRootTolerance && (high[v] - low[v]) * length > kRootTolerance) next.push_back(v);
        }
        active.swap(next);
    }
    std::vector<Vec3> x(nv);
    for (std::size_t v = 0; v < nv; ++v) {
        const Vec3 d = sub3(b[v], a[v]);
        for (int r = 0; r < 3; ++r) x[v][r] = a[v][r] + t[v] * d[r];
    }
    return x;
}

// Quadrilaterals split along their shorter diagonal (src/surface.cpp:262-281).
std::vector<std::array<std::size_t, 3>> triangulate(const std::vector<kumo_dev::IsoPolygon>& polygons,
                                                    const std::vector<Vec3>& x) {
    std::vector<std::array<std::size_t, 3>> tri;
    tri.reserve(polygons.size() * 2);
    const std::size_t nv = x.size();
    for (const auto& poly : polygons) {
        std::size_t p[4];
        for (int c = 0; c < poly.count; ++c) {
            if (poly.vertex[c] < 0 || static_cast<std::size_t>(poly.vertex[c]) >= nv)
                throw std::runtime_error("isosurface polygon refers to a missing vertex");
            p[c] = static_cast<std::size_t>(poly.vertex[c]);
        }
        if (poly.count == 3) {
            tri.push_back({p[0], p[1], p[2]});
        } else {
            const Vec3 d02 = sub3(x[p[0]], x[p[2]]), d13 = sub3(x[p[1]], x[p[3]]);
            if (dot3(d02, d02) <= dot3(d13, d13)) {
                tri.push_back({p[0], p[1], p[2]});
                tri.push_back({p[0], p[2], p[3]});
            } else {
                tri.push_back({p[0], p[1], p[3]});
                tri.push_back({p[1], p[2], p[3]});
            }
        }
    }
    return tri;
}

EvaluationOptions density_options() {
    EvaluationOptions o;
    o.backend = Backend::AO_P;  // the FCHK density matrix, as densities_blocked / density_derivatives_shared
    return o;
}

struct DensitySurface {
    detail::Isosurface surface;
    Grid grid;
};

// src/surface.cpp:329-352: grids of growing margin until the isosurface stays
// inside, the total density on the device, then the isosurface.
DensitySurface density_surface(const Molecule& molecule, double isovalue, double spacing) {
    if (!std::isfinite(isovalue) || isovalue < minimum_density_isovalue)
        throw std::invalid_argument("density isovalue must be finite and at least 1e-8 e/bohr^3");
    if (!std::isfinite(spacing) || spacing <= 0.0)
        throw std::invalid_argument("surface grid spacing must be positive and finite");
    const Evaluator evaluator(molecule, density_options());
    const detail::ScalarFunction density = [&](const std::vector<Vec3>& pts, std::vector<double>& values,
                                               std::vector<Vec3>& gradients) {
        Request r;
        r.add({PropertyKind::Density}).add({PropertyKind::Gradient});
        const Results res = evaluator.evaluate(Points{pts.empty() ? nullptr : pts[0].data(), pts.size()}, r);
        const auto& rho = res.get({PropertyKind::Density});
        const auto& grad = res.get({PropertyKind::Gradient});
        for (std::size_t p = 0; p < pts.size(); ++p) {
            values[p] = rho.components[0][p];
            for (int a = 0; a < 3; ++a) gradients[p][a] = grad.components[static_cast<std::size_t>(a)][p];
        }
    };
    Request rho_request;
    rho_request.add({PropertyKind::Density});
    for (double margin = 4.0; margin <= 16.0; margin += 2.0) {
        const Grid grid = Grid::around(molecule.atoms(), margin, spacing);
        const std::size_t n = detail::validated_point_count(grid);
        DeviceBuffer samples(n);
        double* outs[1] = {samples.p};
        (void)evaluator.evaluate_device(grid, rho_request, outs, nullptr);
        detail::check_cuda(cudaStreamSynchronize(nullptr), "density on the surface grid");
        if (kumo_dev::iso_reaches_boundary(iso_grid(grid), samples.p, isovalue, nullptr)) continue;
        return {detail::extract_isosurface(grid, samples.p, true, isovalue, density), grid};
    }
    throw std::runtime_error(
        "the density isosurface extends more than 16 bohr beyond the atoms; use a larger isovalue");
}

// Part of triangle x (values v, linear in between) where the value is >= level
// (upper) or < level, in triangles: piece(area, w0, w1, w2) for each
// (src/surface.cpp:355-383).
template <typename Piece>
void clip(const std::array<Vec3, 3>& x, const std::array<double, 3>& v, double level, bool upper, Piece&& piece) {
    Vec3 px[4];
    double pv[4];
    int n = 0;
    const auto keep = [&](double value) { return upper ? value >= level : value < level; };
    for (int i = 0; i < 3; ++i) {
        const int j = (i + 1) % 3;
        const bool ki = keep(v[static_cast<std::size_t>(i)]), kj = keep(v[static_cast<std::size_t>(j)]);
        if (ki) {
            px[n] = x[static_cast<std::size_t>(i)];
            pv[n++] = v[static_cast<std::size_t>(i)];
        }
        if (ki != kj) {
            const double s = (level - v[static_cast<std::size_t>(i)]) /
                             (v[static_cast<std::size_t>(j)] - v[static_cast<std::size_t>(i)]);
            const Vec3 d = sub3(x[static_cast<std::size_t>(j)], x[static_cast<std::size_t>(i)]);
            for (int r = 0; r < 3; ++r) px[n][r] = x[static_cast<std::size_t>(i)][r] + s * d[r];
            pv[n++] = level;
        }
    }
    for (int i = 1; i + 1 < n; ++i)
        piece(0.5 * norm3(cross3(sub3(px[i], px[0]), sub3(px[i + 1], px[0]))), pv[0], pv[i], pv[i + 1]);
}

// Integral of (w - s)^2 over a triangle of the given area with w linear.
double square_integral(double area, double w0, double w1, double w2, double s) {
    const double a = w0 - s, b = w1 - s, c = w2 - s;
    return area / 6.0 * (a * a + b * b + c * c + a * b + b * c + c * a);
}

}  // namespace

namespace detail {

Isosurface extract_isosurface(const Grid& grid, const double* samples, bool samples_on_device, double isovalue,
                              const ScalarFunction& function) {
    const std::size_t n = validated_point_count(grid);
    if (grid.counts[0] < 2 || grid.counts[1] < 2 || grid.counts[2] < 2)
        throw std::invalid_argument("isosurface grid needs at least two points along each axis");
    if (!samples) throw std::invalid_argument("isosurface samples do not match the grid");
    if (!std::isfinite(isovalue)) throw std::invalid_argument("isovalue must be finite");
    const double* dev = samples;
    std::unique_ptr<DeviceBuffer> copy;
    if (!samples_on_device) {
        for (std::size_t q = 0; q < n; ++q)
            if (!std::isfinite(samples[q])) throw std::invalid_argument("isosurface samples must be finite");
        copy = std::make_unique<DeviceBuffer>(n);
        check_cuda(cudaMemcpy(copy->p, samples, sizeof(double) * n, cudaMemcpyHostToDevice), "isosurface samples");
        dev = copy->p;
    }
    const kumo_dev::IsoGrid g = iso_grid(grid);
    if (kumo_dev::iso_reaches_boundary(g, dev, isovalue, nullptr))
        throw std::invalid_argument("the isosurface reaches the grid boundary, so it would not be closed");
    std::vector<kumo_dev::IsoEdge> edges;
    std::vector<kumo_dev::IsoPolygon> polygons;
    kumo_dev::iso_polygonize(g, dev, isovalue, edges, polygons, nullptr);
    copy.reset();
    Isosurface s;
    s.mesh.vertices = place_vertices(grid, isovalue, edges, function);
    s.vertex_cells.reserve(edges.size());
    for (const auto& e : edges) s.vertex_cells.push_back({e.cell[0], e.cell[1], e.cell[2]});
    s.mesh.triangles = triangulate(polygons, s.mesh.vertices);
    return s;
}

}  // namespace detail

double TriangleMesh::area() const {
    double total = 0.0;
    for (const auto& t : triangles) {
        const Vec3& a = vertices.at(t[0]);
        total += 0.5 * norm3(cross3(sub3(vertices.at(t[1]), a), sub3(vertices.at(t[2]), a)));
    }
    return total;
}

double TriangleMesh::volume() const {
    if (vertices.empty()) return 0.0;
    Vec3 c{0.0, 0.0, 0.0};
    for (const auto& v : vertices)
        for (int r = 0; r < 3; ++r) c[r] += v[r];
    for (int r = 0; r < 3; ++r) c[r] /= static_cast<double>(vertices.size());
    double total = 0.0;
    for (const auto& t : triangles)
        total += dot3(sub3(vertices.at(t[0]), c), cross3(sub3(vertices.at(t[1]), c), sub3(vertices.at(t[2]), c)));
    return total / 6.0;
}

// src/surface.cpp:417-531.
SurfaceStatistics surface_statistics(const TriangleMesh& mesh, std::span<const double> values, double polar_threshold) {
    const std::size_t nv = mesh.vertices.size();
    if (values.size() != nv) throw std::invalid_argument("surface values do not match the mesh vertices");
    for (double v : values)
        if (!std::isfinite(v)) throw std::invalid_argument("surface values must be finite");
    if (!std::isfinite(polar_threshold) || polar_threshold < 0.0)
        throw std::invalid_argument("polar threshold must be finite and nonnegative");
    for (const auto& t : mesh.triangles)
        if (t[0] >= nv || t[1] >= nv || t[2] >= nv)
            throw std::invalid_argument("surface triangle refers to a missing vertex");
    SurfaceStatistics s;
    const auto corners = [&](const std::array<std::size_t, 3>& t) {
        return std::pair{std::array<Vec3, 3>{mesh.vertices[t[0]], mesh.vertices[t[1]], mesh.vertices[t[2]]},
                         std::array<double, 3>{values[t[0]], values[t[1]], values[t[2]]}};
    };
    const auto mean = [](double a, double b, double c) { return (a + b + c) / 3.0; };
    double pos_int = 0.0, neg_int = 0.0, above = 0.0, below = 0.0;
    for (const auto& t : mesh.triangles) {
        const auto [x, v] = corners(t);
        clip(x, v, 0.0, true, [&](double a, double w0, double w1, double w2) {
            s.positive_area += a;
            pos_int += a * mean(w0, w1, w2);
        });
        clip(x, v, 0.0, false, [&](double a, double w0, double w1, double w2) {
            s.negative_area += a;
            neg_int += a * mean(w0, w1, w2);
        });
        clip(x, v, polar_threshold, true, [&](double a, double, double, double) { above += a; });
        clip(x, v, -polar_threshold, false, [&](double a, double, double, double) { below += a; });
    }
    s.area = s.positive_area + s.negative_area;
    const double integral = pos_int + neg_int;
    if (!(s.area > 0.0) || !std::isfinite(s.area)) throw std::invalid_argument("surface area must be positive");
    const double nan = std::numeric_limits<double>::quiet_NaN();
    s.average = integral / s.area;
    s.positive_average = s.positive_area > 0.0 ? pos_int / s.positive_area : nan;
    s.negative_average = s.negative_area > 0.0 ? neg_int / s.negative_area : nan;
    s.polarity_index = (pos_int - neg_int) / s.area;
    s.nonpolar_area = std::max(0.0, s.area - above - below);
    double pos_sq = 0.0, neg_sq = 0.0, dev = 0.0;
    for (const auto& t : mesh.triangles) {
        const auto [x, v] = corners(t);
        if (s.positive_area > 0.0)
            clip(x, v, 0.0, true, [&](double a, double w0, double w1, double w2) {
                pos_sq += square_integral(a, w0, w1, w2, s.positive_average);
            });
        if (s.negative_area > 0.0)
            clip(x, v, 0.0, false, [&](double a, double w0, double w1, double w2) {
                neg_sq += square_integral(a, w0, w1, w2, s.negative_average);
            });
        clip(x, v, s.average, true,
             [&](double a, double w0, double w1, double w2) { dev += a * (mean(w0, w1, w2) - s.average); });
        clip(x, v, s.average, false,
             [&](double a, double w0, double w1, double w2) { dev += a * (s.average - mean(w0, w1, w2)); });
    }
    s.positive_variance = s.positive_area > 0.0 ? pos_sq / s.positive_area : 0.0;
    s.negative_variance = s.negative_area > 0.0 ? neg_sq / s.negative_area : 0.0;
    s.total_variance = s.positive_variance + s.negative_variance;
    s.balance = s.total_variance > 0.0
                    ? s.positive_variance * s.negative_variance / (s.total_variance * s.total_variance)
                    : nan;
    s.charge_separation = dev / s.area;
    const auto [lo, hi] = std::minmax_element(values.begin(), values.end());
    s.minimum_vertex = static_cast<std::size_t>(lo - values.begin());
    s.maximum_vertex = static_cast<std::size_t>(hi - values.begin());
    s.minimum = *lo;
    s.maximum = *hi;
    // Local extrema: below (above) every neighbour and every neighbour's
    // neighbour along triangle edges.
    std::vector<std::vector<std::size_t>> nb(nv);
    for (const auto& t : mesh.triangles)
        for (int a = 0; a < 3; ++a) {
            nb[t[static_cast<std::size_t>(a)]].push_back(t[static_cast<std::size_t>((a + 1) % 3)]);
            nb[t[static_cast<std::size_t>(a)]].push_back(t[static_cast<std::size_t>((a + 2) % 3)]);
        }
    for (auto& l : nb) {
        std::sort(l.begin(), l.end());
        l.erase(std::unique(l.begin(), l.end()), l.end());
    }
    const auto extremum = [&](std::size_t i, auto beyond) {
        if (nb[i].empty()) return false;
        for (std::size_t j : nb[i]) {
            if (j == i) continue;
            if (!beyond(values[i], values[j])) return false;
            for (std::size_t k : nb[j])
                if (k != i && !beyond(values[i], values[k])) return false;
        }
        return true;
    };
    for (std::size_t i = 0; i < nv; ++i) {
        if (extremum(i, std::less<double>{})) s.local_minima.push_back(i);
        if (extremum(i, std::greater<double>{})) s.local_maxima.push_back(i);
    }
    std::sort(s.local_minima.begin(), s.local_minima.end(),
              [&](std::size_t a, std::size_t b) { return values[a] < values[b] || (values[a] == values[b] && a < b); });
    std::sort(s.local_maxima.begin(), s.local_maxima.end(),
              [&](std::size_t a, std::size_t b) { return values[a] > values[b] || (values[a] == values[b] && a < b); });
    return s;
}

TriangleMesh density_isosurface(const Molecule& molecule, double isovalue, double spacing) {
    return density_surface(molecule, isovalue, spacing).surface.mesh;
}

// src/surface.cpp:537-566: the orbital-energy sums of the occupied orbitals
// (every AO of the shells within reach, no screening); the device pass gives
// 0 where the occupied density vanishes, which is an error here.
std::vector<double> average_local_ionization_energy(const Molecule& molecule, Points points) {
    if (points.count > 0 && !points.data) throw std::invalid_argument("ionization energy points must be finite");
    for (std::size_t q = 0; q < 3 * points.count; ++q)
        if (!std::isfinite(points.data[q])) throw std::invalid_argument("ionization energy points must be finite");
    EvaluationOptions o;
    o.block_size = 128;
    const Evaluator evaluator(molecule, o);
    Request r;
    r.add({PropertyKind::AverageLocalIonizationEnergy});
    const Results res = evaluator.evaluate(points, r);
    std::vector<double> out(res.get({PropertyKind::AverageLocalIonizationEnergy}).components[0]);
    for (double v : out)
        if (!(v != 0.0))
            throw std::invalid_argument("the average local ionization energy is undefined where the density vanishes");
    return out;
}

IonizationEnergySurface local_ionization_energy_surface(const Molecule& molecule, double isovalue, double spacing) {
    (void)average_local_ionization_energy(molecule, Points{nullptr, 0});  // the orbital checks first
    auto surface = density_surface(molecule, isovalue, spacing).surface;
    IonizationEnergySurface result;
    result.ionization_energy = average_local_ionization_energy(
        molecule, Points{surface.mesh.vertices.empty() ? nullptr : surface.mesh.vertices[0].data(),
                         surface.mesh.vertices.size()});
    result.statistics = surface_statistics(surface.mesh, result.ionization_energy);
    result.mesh = std::move(surface.mesh);
    return result;
}

PotentialSurface electrostatic_potential_surface(const Molecule& molecule, const SurfaceOptions& options) {
    if (!std::isfinite(options.potential_tolerance) || options.potential_tolerance < 0.0)
        throw std::invalid_argument("potential tolerance must be finite and nonnegative");
    auto density = density_surface(molecule, options.isovalue, options.spacing);
    auto& mesh = density.surface.mesh;
    EvaluationOptions o;
    o.potential_tolerance = options.potential_tolerance;
    const Evaluator evaluator(molecule, o);
    Request r;
    r.add({PropertyKind::ElectrostaticPotential});
    PotentialSurface result;
    const Results res =
        evaluator.evaluate(Points{mesh.vertices.empty() ? nullptr : mesh.vertices[0].data(), mesh.vertices.size()}, r);
    result.potential = res.get({PropertyKind::ElectrostaticPotential}).components[0];
    result.statistics = surface_statistics(mesh, result.potential);
    result.mesh = std::move(mesh);
    return result;
}

// src/surface.cpp:633-670.
MappedSurface map_on_density_isosurface(const Molecule& molecule, const std::vector<Property>& properties,
                                        double isovalue, double spacing, const EvaluationOptions& options) {
    if (properties.empty()) throw std::invalid_argument("no property to map on the surface");
    MappedSurface result;
    Request request;
    for (const Property& p : properties) {
        if (p.kind == PropertyKind::Gradient || p.kind == PropertyKind::Hessian ||
            p.kind == PropertyKind::OrbitalGradient || p.kind == PropertyKind::OrbitalHessian ||
            p.kind == PropertyKind::TauComponents || p.kind == PropertyKind::HamiltonianKineticEnergyComponents)
            throw std::invalid_argument(
                "only one-component properties can be mapped on a surface (not a gradient, a Hessian or the "
                "Cartesian terms of G or K)");
        if (std::find(result.properties.begin(), result.properties.end(), p) == result.properties.end()) {
            result.properties.push_back(p);
            request.add(p);
        }
    }
    const Evaluator evaluator(molecule, options);
    (void)evaluator.evaluate(Points{nullptr, 0}, request);  // the request checks before the surface
    result.mesh = density_surface(molecule, isovalue, spacing).surface.mesh;
    const auto& v = result.mesh.vertices;
    const Results res = evaluator.evaluate(Points{v.empty() ? nullptr : v[0].data(), v.size()}, request);
    result.backend_used = res.backend_used();
    for (const Property& p : result.properties) {
        result.values.push_back(res.get(p).components[0]);
        result.statistics.push_back(surface_statistics(result.mesh, result.values.back(), 0.0));
    }
    return result;
}

// src/surface.cpp:672-720: ASCII PLY, 10 significant digits.
void write_ply(const std::filesystem::path& path, const TriangleMesh& mesh,
               const std::vector<std::pair<std::string, std::vector<double>>>& fields,
               const std::vector<std::string>& comments) {
    std::vector<std::string> names{"x", "y", "z"};
    for (const auto& [name, vals] : fields) {
        if (name.empty() ||
            !std::all_of(name.begin(), name.end(), [](unsigned char c) { return std::isalnum(c) || c == '_'; }))
            throw std::invalid_argument("invalid PLY property name '" + name + "'");
        if (std::find(names.begin(), names.end(), name) != names.end())
            throw std::invalid_argument("duplicate PLY property name '" + name + "'");
        names.push_back(name);
        if (vals.size() != mesh.vertices.size())
            throw std::invalid_argument("PLY property '" + name + "' needs one value per vertex");
        for (double v : vals)
            if (!std::isfinite(v)) throw std::invalid_argument("nonfinite value in PLY property '" + name + "'");
    }
    for (const auto& c : comments)
        if (c.find_first_of("\r\n") != std::string::npos)
            throw std::invalid_argument("PLY comments must not contain line breaks");
    for (const auto& v : mesh.vertices)
        if (!std::isfinite(v[0]) || !std::isfinite(v[1]) || !std::isfinite(v[2]))
            throw std::invalid_argument("nonfinite PLY vertex");
    for (const auto& t : mesh.triangles)
        for (std::size_t v : t)
            if (v >= mesh.vertices.size()) throw std::invalid_argument("PLY triangle refers to a missing vertex");
    std::string text = "ply\nformat ascii 1.0\n";
    for (const auto& c : comments) text += "comment " + c + "\n";
    text += "element vertex " + std::to_string(mesh.vertices.size()) + "\n";
    for (const auto& n : names) text += "property double " + n + "\n";
    text += "element face " + std::to_string(mesh.triangles.size()) +
            "\nproperty list uchar int vertex_indices\nend_header\n";
    char buf[64];
    for (std::size_t v = 0; v < mesh.vertices.size(); ++v) {
        for (int r = 0; r < 3; ++r) {
            std::snprintf(buf, sizeof buf, r ? " %.9e" : "%.9e", mesh.vertices[v][static_cast<std::size_t>(r)]);
            text += buf;
        }
        for (const auto& f : fields) {
            std::snprintf(buf, sizeof buf, " %.9e", f.second[v]);
            text += buf;
        }
        text += '\n';
    }
    for (const auto& t : mesh.triangles)
        text += "3 " + std::to_string(t[0]) + " " + std::to_string(t[1]) + " " + std::to_string(t[2]) + "\n";
    std::ofstream out(path);
    if (!out) throw std::runtime_error("cannot open PLY output " + path.string());
    out << text;
    out.flush();
    if (!out) throw std::runtime_error("PLY write failed: " + path.string());
}

}  // namespace chem::kumo
