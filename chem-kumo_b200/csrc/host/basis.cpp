// Basis set from FCHK shell records and its preparation for evaluation.
//
// The floating-point expressions of the normalisation, the Schlegel-Frisch
// coefficients and the cutoff bound keep the operation order of chem-kumo
// (src/basis_math.cpp:17-25, src/basis_evaluator.cpp:49-127), so that the
// prepared weights, transforms and cutoff radii are bit-identical to the
// reference's; this file is compiled without floating-point contraction.
#include "chem/kumo/basis.hpp"

#include <algorithm>
#include <cmath>
#include <limits>
#include <numbers>
#include <stdexcept>

namespace chem::kumo {
namespace {

std::size_t positive_size(long long v, const char* what) {
    if (v <= 0) throw std::runtime_error(std::string("invalid ") + what + " in fchk");
    return static_cast<std::size_t>(v);
}

double fact(int n) {
    if (n < 0) throw std::runtime_error("negative factorial argument");
    double v = 1.0;
    for (long long i = 2; i <= n; ++i) v *= static_cast<double>(i);
    return v;
}

double odd_double_factorial(int n) {
    double v = 1.0;
    for (int i = n; i >= 1; i -= 2) v *= static_cast<double>(i);
    return v;
}

// Coefficient of x^lx y^ly z^lz in the real solid harmonic (l, m), both
// normalised (H. B. Schlegel and M. J. Frisch, Int. J. Quantum Chem. 54, 83
// (1995)); 0 for components that do not contribute.
double solid_harmonic_coefficient(int l, int m, int lx, int ly) {
    const int lz = l - lx - ly;
    const int am = std::abs(m);
    if (am > l || lz < 0) return 0.0;
    const double norm_ratio = std::sqrt(fact(2 * lx) * fact(2 * ly) * fact(2 * lz) * fact(l) /
                                        (fact(2 * l) * fact(lx) * fact(ly) * fact(lz)));
    const double radial = std::sqrt(fact(l - am) / fact(l + am)) / (std::pow(2.0, l) * fact(l));
    const int half = (l - am - lz) / 2;
    if (2 * half != l - am - lz) return 0.0;
    double sum = 0.0;
    for (int i = 0; i <= (l - am) / 2; ++i) {
        if (half < 0 || half > i) continue;
        const double ci = fact(l) / (fact(i) * fact(l - i)) * fact(2 * l - 2 * i) * std::pow(-1.0, i) /
                          fact(l - am - 2 * i) * fact(i) / (fact(half) * fact(i - half));
        for (int k = 0; k <= half; ++k) {
            if (lx - 2 * k < 0 || lx - 2 * k > am) continue;
            const double dk = fact(half) / (fact(k) * fact(half - k)) * fact(am) /
                              (fact(lx - 2 * k) * fact(am + 2 * k - lx));
            double sign = 0.0;
            if (m == 0 && lx % 2 == 0) sign = std::pow(-1.0, k - lx / 2);
            const int kt = (2 * k + am - lx) / 2;
            if (m > 0 && std::abs(am - lx) % 2 == 0) sign = std::sqrt(2.0) * std::pow(-1.0, kt);
            if (m < 0 && std::abs(am - lx) % 2 == 1) sign = std::sqrt(2.0) * std::pow(-1.0, kt);
            sum += ci * dk * sign;
        }
    }
    return norm_ratio * radial * sum;
}

// Radius beyond which every AO of the block and its first and second
// derivatives are at most `cutoff`: bisection on the bound
// transform_norm * sum_p W_p (1 + l + l^2 + 2 a_p (2l+2) + 4 a_p^2) r^(l+2) exp(-a_p r^2).
double cutoff_radius(const PreparedBlock& b, double transform_norm, double cutoff) {
    const int l = b.angular_momentum;
    const std::size_t np = b.exponents.size();
    const std::size_t nc = b.powers.size();
    std::vector<double> coef(np);
    double start = 1.0;
    for (std::size_t p = 0; p < np; ++p) {
        const double a = b.exponents[p];
        double wmax = std::abs(b.weights[p]);
        for (std::size_t k = 1; k < nc; ++k) wmax = std::max(wmax, std::abs(b.weights[k * np + p]));
        coef[p] = transform_norm * wmax * (1.0 + l + l * l + 2.0 * a * (2.0 * l + 2.0) + 4.0 * a * a);
        start = std::max(start, std::sqrt((l + 2.0) / (2.0 * a)));
    }
    auto bound = [&](double r) {
        double s = 0.0;
        for (std::size_t p = 0; p < np; ++p) s += coef[p] * std::pow(r, l + 2) * std::exp(-b.exponents[p] * r * r);
        return s;
    };
    if (bound(start) <= cutoff) return start;
    double lo = start, hi = 2.0 * start;
    while (bound(hi) > cutoff) hi *= 2.0;
    for (int it = 0; it < 60; ++it) {
        const double mid = 0.5 * (lo + hi);
        if (bound(mid) > cutoff)
            lo = mid;
        else
            hi = mid;
    }
    return hi;
}

}  // namespace

std::size_t Shell::function_count() const {
    if (is_sp) return 4U;
    if (angular_momentum < 0) throw std::runtime_error("negative angular momentum in shell");
    const auto l = static_cast<std::size_t>(angular_momentum);
    if (representation == ShellRepresentation::Pure && angular_momentum >= 2) return 2U * l + 1U;
    return (l + 1U) * (l + 2U) / 2U;
}

BasisSet::BasisSet(std::vector<Shell> shells, std::size_t declared) : shells_(std::move(shells)) {
    for (const auto& s : shells_) function_count_ += s.function_count();
    if (declared && function_count_ != declared)
        throw std::runtime_error("basis size reconstructed from shells does not match fchk");
}

BasisSet::BasisSet(const FormattedCheckpoint& f) {
    const auto& types = f.integers("Shell types");
    const auto& nprim = f.integers("Number of primitives per shell");
    const auto& centers = f.integers("Shell to atom map");
    const auto& exps = f.reals("Primitive exponents");
    const auto& coef = f.reals("Contraction coefficients");
    const bool has_p = f.contains("P(S=P) Contraction coefficients");
    const std::vector<double> none;
    const auto& pcoef = has_p ? f.reals("P(S=P) Contraction coefficients") : none;
    const auto& xyz = f.reals("Coordinates of each shell");
    if (types.size() != nprim.size() || types.size() != centers.size())
        throw std::runtime_error("inconsistent shell arrays in fchk");
    if (xyz.size() != 3U * types.size()) throw std::runtime_error("invalid shell-coordinate array in fchk");
    if (exps.size() != coef.size() || (has_p && exps.size() != pcoef.size()))
        throw std::runtime_error("inconsistent primitive arrays in fchk");
    const auto natoms = positive_size(f.integer("Number of atoms"), "Number of atoms");
    const auto declared = positive_size(f.integer("Number of basis functions"), "Number of basis functions");
    if (!has_p)
        for (auto t : types)
            if (t == -1) throw std::runtime_error("missing P(S=P) coefficients for sp shell");
    std::size_t off = 0;
    for (std::size_t i = 0; i < types.size(); ++i) {
        const long long t = types[i];
        if (t == std::numeric_limits<long long>::min()) throw std::runtime_error("invalid shell type in fchk");
        const bool sp = t == -1;
        const long long lraw = sp ? 1 : (t < 0 ? -t : t);
        if (lraw > std::numeric_limits<int>::max()) throw std::runtime_error("unsupported angular momentum in fchk shell");
        const auto count = positive_size(nprim[i], "Number of primitives per shell");
        if (count > exps.size() - std::min(off, exps.size()))
            throw std::runtime_error("invalid primitive count in fchk shell");
        if (centers[i] <= 0 || static_cast<std::size_t>(centers[i]) > natoms)
            throw std::runtime_error("invalid 1-based shell center in fchk");
        Shell s;
        s.center = static_cast<std::size_t>(centers[i] - 1);
        s.angular_momentum = static_cast<int>(lraw);
        s.is_sp = sp;
        s.representation = (!sp && t <= -2) ? ShellRepresentation::Pure : ShellRepresentation::Cartesian;
        s.origin = {xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]};
        for (double c : s.origin)
            if (!std::isfinite(c)) throw std::runtime_error("non-finite shell coordinate in fchk");
        s.exponents.assign(exps.begin() + off, exps.begin() + off + count);
        s.coefficients.assign(coef.begin() + off, coef.begin() + off + count);
        if (has_p)
            s.p_coefficients.assign(pcoef.begin() + off, pcoef.begin() + off + count);
        else
            s.p_coefficients.assign(count, 0.0);
        for (std::size_t p = 0; p < count; ++p)
            if (!(s.exponents[p] > 0.0) || !std::isfinite(s.exponents[p]) || !std::isfinite(s.coefficients[p]) ||
                !std::isfinite(s.p_coefficients[p]))
                throw std::runtime_error("invalid primitive exponent/coefficient in fchk shell");
        off += count;
        const auto nf = s.function_count();
        if (nf > declared - std::min(function_count_, declared))
            throw std::runtime_error("basis function count exceeds fchk declaration");
        function_count_ += nf;
        shells_.push_back(std::move(s));
    }
    if (off != exps.size()) throw std::runtime_error("unused primitive data after parsing fchk basis");
    if (function_count_ != declared) throw std::runtime_error("basis size reconstructed from shells does not match fchk");
}

std::vector<CartesianPower> gaussian_cartesian_order(int l) {
    if (l < 0) throw std::runtime_error("negative angular momentum");
    switch (l) {
        case 0: return {{0, 0, 0}};
        case 1: return {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
        case 2: return {{2, 0, 0}, {0, 2, 0}, {0, 0, 2}, {1, 1, 0}, {1, 0, 1}, {0, 1, 1}};
        case 3:
            return {{3, 0, 0}, {0, 3, 0}, {0, 0, 3}, {1, 2, 0}, {2, 1, 0},
                    {2, 0, 1}, {1, 0, 2}, {0, 1, 2}, {0, 2, 1}, {1, 1, 1}};
        default: break;
    }
    std::vector<CartesianPower> out;
    for (int x = 0; x <= l; ++x)
        for (int y = 0; y <= l - x; ++y) out.push_back({x, y, l - x - y});
    return out;
}

Matrix gaussian_cartesian_to_pure(int l) {
    if (l < 2) throw std::runtime_error("pure transformation requested below d shell");
    const auto cart = gaussian_cartesian_order(l);
    Matrix t(static_cast<std::size_t>(2 * l + 1), cart.size());
    for (std::size_t g = 0; g < cart.size(); ++g) {
        t(0, g) = solid_harmonic_coefficient(l, 0, cart[g].x, cart[g].y);
        for (int m = 1; m <= l; ++m) {
            t(static_cast<std::size_t>(2 * m - 1), g) = solid_harmonic_coefficient(l, m, cart[g].x, cart[g].y);
            t(static_cast<std::size_t>(2 * m), g) = solid_harmonic_coefficient(l, -m, cart[g].x, cart[g].y);
        }
    }
    return t;
}

double cartesian_primitive_normalization(double alpha, const CartesianPower& p) {
    const int l = p.x + p.y + p.z;
    const double radial = std::pow(2.0 * alpha / std::numbers::pi, 0.75);
    const double angular = std::sqrt(std::pow(4.0 * alpha, static_cast<double>(l)) /
                                     (odd_double_factorial(2 * p.x - 1) * odd_double_factorial(2 * p.y - 1) *
                                      odd_double_factorial(2 * p.z - 1)));
    return radial * angular;
}

std::vector<PreparedBlock> prepare_blocks(const BasisSet& basis) {
    std::vector<PreparedBlock> blocks;
    std::size_t offset = 0;
    auto add = [&](const Shell& s, int l, const std::vector<double>& c, bool pure) {
        PreparedBlock b;
        b.origin = s.origin;
        b.angular_momentum = l;
        b.exponents = s.exponents;
        b.powers = gaussian_cartesian_order(l);
        const std::size_t nc = b.powers.size(), np = b.exponents.size();
        b.weights.resize(nc * np);
        for (std::size_t k = 0; k < nc; ++k)
            for (std::size_t p = 0; p < np; ++p)
                b.weights[k * np + p] = c[p] * cartesian_primitive_normalization(b.exponents[p], b.powers[k]);
        b.pure = pure && l >= 2;
        double tnorm = 1.0;
        if (b.pure) {
            const Matrix t = gaussian_cartesian_to_pure(l);
            tnorm = 0.0;
            for (std::size_t m = 0; m < t.rows(); ++m) {
                double row = std::abs(t(m, 0));
                for (std::size_t k = 1; k < t.cols(); ++k) row += std::abs(t(m, k));
                tnorm = m == 0 ? row : std::max(tnorm, row);
            }
            b.count = t.rows();
        } else {
            b.count = nc;
        }
        b.offset = offset;
        offset += b.count;
        const double r = cutoff_radius(b, tnorm, ao_cutoff);
        b.cutoff_radius2 = r * r;
        blocks.push_back(std::move(b));
    };
    for (const auto& s : basis.shells()) {
        if (s.is_sp) {
            add(s, 0, s.coefficients, false);
            add(s, 1, s.p_coefficients, false);
        } else {
            add(s, s.angular_momentum, s.coefficients, s.representation == ShellRepresentation::Pure);
        }
    }
    if (offset != basis.function_count()) throw std::logic_error("AO blocks do not match the basis size");
    return blocks;
}

}  // namespace chem::kumo
