// Molecule loading and the load-time check of the orbital representation:
// the record order and rules of chem-kumo's src/molecule.cpp:20-180 and the
// decision of src/backend_selection.hpp:43-78.
#include "chem/kumo/density.hpp"
#include "device_state.hpp"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <limits>
#include <stdexcept>
#include <thread>

namespace chem::kumo {
namespace {

Matrix unpack_packed(const std::vector<double>& packed, std::size_t n) {
    if (n > std::numeric_limits<std::size_t>::max() / (n + 1) || packed.size() != n * (n + 1) / 2)
        throw std::runtime_error("invalid packed AO density matrix size");
    Matrix p(n, n);
    std::size_t q = 0;
    for (std::size_t i = 0; i < n; ++i)
        for (std::size_t j = 0; j <= i; ++j, ++q) {
            p(i, j) = packed[q];
            p(j, i) = packed[q];
        }
    for (std::size_t i = 0; i < p.size(); ++i)
        if (!std::isfinite(p.data()[i])) throw std::runtime_error("nonfinite AO density matrix");
    return p;
}

Matrix read_mos(const FormattedCheckpoint& f, const std::string& label, std::size_t n) {
    const auto& flat = f.reals(label);
    if (n == 0 || flat.size() % n != 0 || flat.size() / n > n)
        throw std::runtime_error("invalid MO coefficient dimensions: " + label);
    Matrix c(n, flat.size() / n);
    std::copy(flat.begin(), flat.end(), c.data());  // MO by MO, AO fastest = column-major
    for (std::size_t i = 0; i < c.size(); ++i)
        if (!std::isfinite(c.data()[i])) throw std::runtime_error("nonfinite MO coefficients: " + label);
    return c;
}

std::vector<Atom> read_atoms(const FormattedCheckpoint& f) {
    const auto& z = f.integers("Atomic numbers");
    const auto& xyz = f.reals("Current cartesian coordinates");
    if (xyz.size() != 3 * z.size() || z.empty()) throw std::runtime_error("invalid FCHK geometry");
    const std::vector<double>* charges = nullptr;
    if (f.contains("Nuclear charges")) {
        const auto& c = f.reals("Nuclear charges");
        if (c.size() != z.size()) throw std::runtime_error("invalid FCHK nuclear charge count");
        charges = &c;
    }
    if (!charges)
        for (const char* l : {"ECP-LMax", "ECP-LPSkip", "ECP-RNFroz", "ECP-NLP", "ECP-CLP1", "ECP-CLP2", "ECP-ZLP",
                              "ECP-KFirst", "ECP-KLast"})
            if (f.contains(l))
                throw std::runtime_error(
                    "FCHK has an effective core potential (ECP) but no \"Nuclear charges\" record, so the "
                    "effective nuclear charges are unknown");
    std::vector<Atom> atoms;
    for (std::size_t i = 0; i < z.size(); ++i) {
        if (z[i] <= 0 || z[i] > 118 || !std::isfinite(xyz[3 * i]) || !std::isfinite(xyz[3 * i + 1]) ||
            !std::isfinite(xyz[3 * i + 2]))
            throw std::runtime_error("invalid FCHK atom or coordinates");
        const double q = charges ? (*charges)[i] : static_cast<double>(z[i]);
        if (!std::isfinite(q) || q < 0.0) throw std::runtime_error("invalid FCHK nuclear charge");
        atoms.push_back({static_cast<int>(z[i]), q, {xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]}});
    }
    return atoms;
}

// Frobenius norms of P_total - (Pa + Pb) and P_spin - (Pa - Pb) with
// Pa = Ca,occ Ca,occ^T and Pb likewise, and of the four matrices.  Rows are
// taken in tiles of 32 (each tile of Pa and Pb stays in cache while the
// occupied columns stream past once) spread over the host threads; the
// per-tile sums are added in tile order, so the result does not depend on
// the thread count.
struct CheckNorms {
    double total_err = 0, spin_err = 0, total = 0, rtotal = 0, spin = 0, rspin = 0;
};

CheckNorms check_norms(const Matrix& total, const Matrix& spin, const Matrix& ca, std::size_t na,
                       const Matrix& cb, std::size_t nb) {
    const std::size_t n = total.rows();
    constexpr std::size_t tile = 32;
    const std::size_t ntiles = (n + tile - 1) / tile;
    std::vector<CheckNorms> part(ntiles);
    auto run_tile = [&](std::size_t t, std::vector<double>& pa, std::vector<double>& pb) {
        const std::size_t i0 = t * tile, rows = std::min(tile, n - i0);
        std::fill(pa.begin(), pa.begin() + rows * n, 0.0);
        std::fill(pb.begin(), pb.begin() + rows * n, 0.0);
        auto outer = [&](const Matrix& c, std::size_t nocc, std::vector<double>& p) {
            for (std::size_t o = 0; o < nocc; ++o) {
                const double* col = c.col(o);
                for (std::size_t r = 0; r < rows; ++r) {
                    const double ci = col[i0 + r];
                    double* row = p.data() + r * n;
                    for (std::size_t j = 0; j < n; ++j) row[j] += ci * col[j];
                }
            }
        };
        outer(ca, na, pa);
        outer(cb, nb, pb);
        CheckNorms r;
        for (std::size_t q = 0; q < rows; ++q)
            for (std::size_t j = 0; j < n; ++j) {
                const double rt = pa[q * n + j] + pb[q * n + j], rs = pa[q * n + j] - pb[q * n + j];
                const double tv = total(i0 + q, j), sv = spin(i0 + q, j);
                r.total_err += (tv - rt) * (tv - rt);
                r.spin_err += (sv - rs) * (sv - rs);
                r.total += tv * tv;
                r.rtotal += rt * rt;
                r.spin += sv * sv;
                r.rspin += rs * rs;
            }
        part[t] = r;
    };
    const std::size_t nthreads =
        std::max<std::size_t>(1, std::min<std::size_t>(std::thread::hardware_concurrency(), ntiles));
    std::atomic<std::size_t> next{0};
    auto worker = [&] {
        std::vector<double> pa(tile * n), pb(tile * n);
        for (std::size_t t; (t = next.fetch_add(1)) < ntiles;) run_tile(t, pa, pb);
    };
    std::vector<std::thread> pool;
    for (std::size_t k = 1; k < nthreads; ++k) pool.emplace_back(worker);
    worker();
    for (auto& th : pool) th.join();
    CheckNorms r;
    for (const auto& p : part) {
        r.total_err += p.total_err;
        r.spin_err += p.spin_err;
        r.total += p.total;
        r.rtotal += p.rtotal;
        r.spin += p.spin;
        r.rspin += p.rspin;
    }
    return r;
}

}  // namespace

Molecule::Molecule(Molecule&&) noexcept = default;
Molecule& Molecule::operator=(Molecule&&) noexcept = default;
Molecule::~Molecule() = default;

Molecule Molecule::from_fchk(const std::filesystem::path& path) {
    FormattedCheckpoint f(path);
    Molecule m;
    m.atoms_ = read_atoms(f);
    m.basis_ = BasisSet(f);
    const std::size_t n = m.basis_.function_count();
    m.blocks_ = prepare_blocks(m.basis_);
    m.total_ = unpack_packed(f.reals("Total SCF Density"), n);
    if (f.contains("Spin SCF Density")) {
        m.spin_ = unpack_packed(f.reals("Spin SCF Density"), n);
    } else {
        if (f.contains("Number of alpha electrons") && f.contains("Number of beta electrons") &&
            f.integer("Number of alpha electrons") != f.integer("Number of beta electrons"))
            throw std::runtime_error("open-shell FCHK lacks Spin SCF Density");
        m.spin_ = Matrix(n, n);
    }
    if (!f.contains("Number of alpha electrons") || !f.contains("Number of beta electrons"))
        throw std::runtime_error("missing electron counts in FCHK");
    const long long na = f.integer("Number of alpha electrons"), nb = f.integer("Number of beta electrons");
    if (na < 0 || nb < 0 || na > static_cast<long long>(n) || nb > static_cast<long long>(n))
        throw std::runtime_error("invalid electron counts in FCHK");
    m.nalpha_ = static_cast<int>(na);
    m.nbeta_ = static_cast<int>(nb);
    if (f.contains("Alpha MO coefficients")) m.alpha_mos_ = read_mos(f, "Alpha MO coefficients", n);
    if (f.contains("Beta MO coefficients")) m.beta_mos_ = read_mos(f, "Beta MO coefficients", n);
    m.unrestricted_ = m.beta_mos_.cols() != 0;
    if (m.nalpha_ != m.nbeta_ && !m.unrestricted_) throw std::runtime_error("open-shell FCHK lacks Beta MO coefficients");
    auto energies = [&](const char* label, const Matrix& mos, const char* ch) {
        if (!f.contains(label)) return std::vector<double>{};
        const auto& e = f.reals(label);
        if (mos.cols() && !e.empty() && e.size() != mos.cols())
            throw std::runtime_error(std::string(ch) + " orbital energy count mismatch");
        return e;
    };
    m.alpha_energies_ = energies("Alpha Orbital Energies", m.alpha_mos_, "alpha");
    m.beta_energies_ = energies("Beta Orbital Energies", m.beta_mos_, "beta");
    m.finish();
    return m;
}

Molecule Molecule::from_parts(std::vector<Atom> atoms, BasisSet basis, Matrix total, Matrix spin, int nalpha,
                              int nbeta, Matrix alpha_mos, Matrix beta_mos, std::vector<double> alpha_energies,
                              std::vector<double> beta_energies) {
    Molecule m;
    m.atoms_ = std::move(atoms);
    m.basis_ = std::move(basis);
    const std::size_t n = m.basis_.function_count();
    if (total.rows() != n || total.cols() != n) throw std::invalid_argument("density matrix does not match the basis");
    if (spin.size() == 0) spin = Matrix(n, n);
    if (spin.rows() != n || spin.cols() != n) throw std::invalid_argument("spin density matrix does not match the basis");
    m.blocks_ = prepare_blocks(m.basis_);
    m.total_ = std::move(total);
    m.spin_ = std::move(spin);
    if (nalpha < 0 || nbeta < 0 || nalpha > static_cast<int>(n) || nbeta > static_cast<int>(n))
        throw std::invalid_argument("invalid electron counts");
    m.nalpha_ = nalpha;
    m.nbeta_ = nbeta;
    m.alpha_mos_ = std::move(alpha_mos);
    m.beta_mos_ = std::move(beta_mos);
    m.unrestricted_ = m.beta_mos_.cols() != 0;
    m.alpha_energies_ = std::move(alpha_energies);
    m.beta_energies_ = std::move(beta_energies);
    m.finish();
    return m;
}

void Molecule::finish() {
    const std::size_t n = basis_size();
    ElectronicStructureInfo info;
    info.occupied_alpha = static_cast<std::size_t>(nalpha_);
    info.occupied_beta = static_cast<std::size_t>(nbeta_);
    const bool has_a = alpha_mos_.cols() >= static_cast<std::size_t>(nalpha_) && alpha_mos_.rows() == n;
    const bool has_b = !unrestricted_ ||
                       (beta_mos_.cols() >= static_cast<std::size_t>(nbeta_) && beta_mos_.rows() == n);
    if (has_a && has_b && (unrestricted_ || nalpha_ == nbeta_)) {
        const Matrix& cb = unrestricted_ ? beta_mos_ : alpha_mos_;
        const CheckNorms r = check_norms(total_, spin_, alpha_mos_, static_cast<std::size_t>(nalpha_), cb,
                                         static_cast<std::size_t>(nbeta_));
        const double te = std::sqrt(r.total_err), se = std::sqrt(r.spin_err);
        const double tscale = std::max(std::sqrt(r.total), std::sqrt(r.rtotal));
        const double sscale = std::max({std::sqrt(r.spin), std::sqrt(r.rspin), tscale});
        info.total_absolute_error = te;
        info.spin_absolute_error = se;
        info.total_relative_error = tscale > 0 ? te / tscale : te;
        info.spin_relative_error = sscale > 0 ? se / sscale : se;
        const bool ok = te <= orbital_check_absolute_tolerance + orbital_check_relative_tolerance * tscale &&
                        se <= orbital_check_absolute_tolerance + orbital_check_relative_tolerance * sscale;
        info.orbital_status = ok ? OrbitalRepresentationStatus::Valid : OrbitalRepresentationStatus::Inconsistent;
    } else if (has_a && has_b) {
        info.orbital_status = OrbitalRepresentationStatus::Inconsistent;
    }
    electronic_info_ = info;
}

Matrix Molecule::density_matrix(DensityComponent component) const {
    switch (component) {
        case DensityComponent::Total: return total_;
        case DensityComponent::Difference: return spin_;
        case DensityComponent::Alpha:
        case DensityComponent::Beta: {
            Matrix m(total_.rows(), total_.cols());
            const double sign = component == DensityComponent::Alpha ? 1.0 : -1.0;
            for (std::size_t i = 0; i < m.size(); ++i) m.data()[i] = 0.5 * (total_.data()[i] + sign * spin_.data()[i]);
            return m;
        }
    }
    throw std::invalid_argument("invalid density spin component");
}

const Matrix& Molecule::mo_coefficients(SpinChannel channel) const {
    if (channel != SpinChannel::Alpha && channel != SpinChannel::Beta)
        throw std::invalid_argument("MO spin channel must be alpha or beta");
    return (channel == SpinChannel::Beta && unrestricted_) ? beta_mos_ : alpha_mos_;
}

std::size_t Molecule::orbital_count(SpinChannel channel) const { return mo_coefficients(channel).cols(); }

std::size_t Molecule::occupied_count(SpinChannel channel) const {
    return static_cast<std::size_t>(channel == SpinChannel::Alpha ? nalpha_ : nbeta_);
}

const std::vector<double>& Molecule::orbital_energies(SpinChannel channel) const {
    return (channel == SpinChannel::Beta && unrestricted_) ? beta_energies_ : alpha_energies_;
}

detail::DeviceMolecule& Molecule::device() const {
    std::lock_guard<std::mutex> lock(*device_mutex_);
    int dev = 0;
    detail::check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
    if (!device_ || device_->device != dev) {
        device_.reset();
        device_ = std::make_unique<detail::DeviceMolecule>(*this);
    }
    return *device_;
}

const detail::DeviceMolecule* Molecule::device_if_resident() const {
    std::lock_guard<std::mutex> lock(*device_mutex_);
    int dev = 0;
    detail::check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
    return (device_ && device_->device == dev) ? device_.get() : nullptr;
}

std::size_t Molecule::device_bytes() const {
    std::lock_guard<std::mutex> lock(*device_mutex_);
    return device_ ? device_->bytes : 0;
}

}  // namespace chem::kumo
