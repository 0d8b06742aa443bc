// Grid constructors and Field (chem-kumo src/grid.cpp:15-117 semantics).
#include <algorithm>
#include <cmath>
#include <limits>
#include <stdexcept>

#include "chem/kumo/density.hpp"
#include "grid_geometry.hpp"

namespace chem::kumo {
namespace {

Vec3 sub(const Vec3& a, const Vec3& b) { return {a[0] - b[0], a[1] - b[1], a[2] - b[2]}; }
double dot(const Vec3& a, const Vec3& b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
double norm(const Vec3& a) { return std::sqrt(dot(a, a)); }
Vec3 scale(const Vec3& a, double s) { return {a[0] * s, a[1] * s, a[2] * s}; }
Vec3 cross(const Vec3& a, const Vec3& b) {
    return {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
}
bool finite(const Vec3& a) { return std::isfinite(a[0]) && std::isfinite(a[1]) && std::isfinite(a[2]); }

void check_margin_spacing(double margin, double spacing) {
    if (!std::isfinite(margin) || margin < 0 || !std::isfinite(spacing) || spacing <= 0)
        throw std::invalid_argument("invalid grid margin or spacing");
}

int points_covering(double length, double spacing) {
    const double steps = std::ceil(length / spacing * (1.0 - 1e-12));
    if (!std::isfinite(steps) || steps + 1 > std::numeric_limits<int>::max())
        throw std::invalid_argument("grid too large");
    return std::max(2, static_cast<int>(steps) + 1);
}

void set_col(Mat3& m, int c, const Vec3& v) {
    for (int r = 0; r < 3; ++r) m(r, c) = v[static_cast<std::size_t>(r)];
}

}  // namespace

Grid Grid::around(const std::vector<Atom>& atoms, double margin, double spacing) {
    if (atoms.empty() || !std::isfinite(margin) || margin < 0 || !std::isfinite(spacing) || spacing <= 0)
        throw std::invalid_argument("invalid grid parameters");
    Vec3 lo = atoms.front().position, hi = lo;
    for (const auto& a : atoms) {
        if (!finite(a.position) || a.atomic_number <= 0) throw std::invalid_argument("invalid atom in grid");
        for (int k = 0; k < 3; ++k) {
            lo[k] = std::min(lo[k], a.position[k]);
            hi[k] = std::max(hi[k], a.position[k]);
        }
    }
    Grid g;
    for (int k = 0; k < 3; ++k) {
        g.origin[k] = lo[k] - margin;
        const double count = std::ceil((hi[k] - lo[k] + 2 * margin) / spacing) + 1;
        if (!std::isfinite(count) || count > std::numeric_limits<int>::max()) throw std::invalid_argument("grid too large");
        g.counts[k] = std::max(2, static_cast<int>(count));
    }
    g.steps = Mat3::scaled_identity(spacing);
    return g;
}

Grid Grid::line(const Vec3& start, const Vec3& end, double margin, double spacing) {
    check_margin_spacing(margin, spacing);
    if (!finite(start) || !finite(end)) throw std::invalid_argument("invalid line: nonfinite end point");
    const double length = norm(sub(end, start));
    if (!(length > 0)) throw std::invalid_argument("invalid line: coincident end points");
    const Vec3 dir = scale(sub(end, start), 1.0 / length);
    int least = 0;
    for (int k = 1; k < 3; ++k)
        if (std::abs(dir[k]) < std::abs(dir[least])) least = k;
    Vec3 unit{0, 0, 0};
    unit[least] = 1.0;
    Vec3 p = cross(dir, unit);
    p = scale(p, 1.0 / norm(p));
    const double total = length + 2 * margin;
    Grid g;
    g.counts = {points_covering(total, spacing), 1, 1};
    g.origin = sub(start, scale(dir, margin));
    set_col(g.steps, 0, scale(dir, total / (g.counts[0] - 1)));
    set_col(g.steps, 1, p);
    set_col(g.steps, 2, cross(dir, p));
    return g;
}

Grid Grid::plane(const Vec3& a, const Vec3& b, const Vec3& c, double margin, double spacing) {
    check_margin_spacing(margin, spacing);
    if (!finite(a) || !finite(b) || !finite(c)) throw std::invalid_argument("invalid plane: nonfinite point");
    const Vec3 ab = sub(b, a), ac = sub(c, a);
    const double sc = norm(ab) * norm(ac);
    if (!(sc > 0) || norm(cross(ab, ac)) <= 1e-8 * sc)
        throw std::invalid_argument("invalid plane: the three points are collinear");
    const Vec3 u = scale(ab, 1.0 / norm(ab));
    Vec3 v = sub(ac, scale(u, dot(ac, u)));
    v = scale(v, 1.0 / norm(v));
    const double cu = dot(ac, u), cv = dot(ac, v);
    const double ulo = std::min(0.0, cu) - margin, uhi = std::max(norm(ab), cu) + margin;
    const double vlo = -margin, vhi = cv + margin;
    Grid g;
    g.counts = {points_covering(uhi - ulo, spacing), points_covering(vhi - vlo, spacing), 1};
    for (int k = 0; k < 3; ++k) g.origin[k] = a[k] + ulo * u[k] + vlo * v[k];
    set_col(g.steps, 0, scale(u, (uhi - ulo) / (g.counts[0] - 1)));
    set_col(g.steps, 1, scale(v, (vhi - vlo) / (g.counts[1] - 1)));
    set_col(g.steps, 2, cross(u, v));
    return g;
}

Field::Field(Grid g, std::vector<Atom> atoms, std::vector<double> v)
    : grid_(std::move(g)), atoms_(std::move(atoms)), values_(std::move(v)) {
    if (values_.size() != detail::validated_point_count(grid_)) throw std::invalid_argument("field size mismatch");
}

double Field::operator()(int i, int j, int k) const {
    if (i < 0 || j < 0 || k < 0 || i >= grid_.counts[0] || j >= grid_.counts[1] || k >= grid_.counts[2])
        throw std::out_of_range("field index");
    const std::size_t idx = (static_cast<std::size_t>(i) * static_cast<std::size_t>(grid_.counts[1]) +
                             static_cast<std::size_t>(j)) *
                                static_cast<std::size_t>(grid_.counts[2]) +
                            static_cast<std::size_t>(k);
    return values_.at(idx);
}

}  // namespace chem::kumo
