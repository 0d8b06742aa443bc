#pragma once
// Molecule, Grid and Field of the B200 grid evaluator, with the names and
// semantics of chem-kumo's include/chem/kumo/density.hpp (Eigen types replaced
// by the small types of types.hpp).

#include "chem/kumo/basis.hpp"
#include "chem/kumo/spin.hpp"
#include "chem/kumo/types.hpp"

#include <cstddef>
#include <filesystem>
#include <functional>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

namespace chem::kumo {

namespace detail {
struct DeviceMolecule;
}

/// include/chem/kumo/density.hpp:28 of chem-kumo.
inline constexpr double default_screening_threshold = 1e-12;
/// include/chem/kumo/density.hpp:32 of chem-kumo.
inline constexpr std::size_t max_block_size = 65536;

/// Progress report: called after each batch of point blocks with the number
/// of points done so far and the total; calls are serialized, `done` never
/// decreases, and an exception thrown by the callback aborts the evaluation
/// and reaches the caller.
using ProgressCallback = std::function<void(std::size_t done, std::size_t total)>;

struct Atom {
    int atomic_number = 0;
    double nuclear_charge = 0.0;
    Vec3 position{0, 0, 0};
};

/// Regular grid r(i, j, k) = origin + steps * (i, j, k), k fastest
/// ("Field order").  steps(r, a) is component r of the step vector of axis a.
struct Grid {
    Vec3 origin{0, 0, 0};
    Mat3 steps = Mat3::identity();
    IVec3 counts{1, 1, 1};
    static Grid around(const std::vector<Atom>& atoms, double margin_bohr, double spacing_bohr);
    static Grid line(const Vec3& start, const Vec3& end, double margin_bohr, double spacing_bohr);
    static Grid plane(const Vec3& a, const Vec3& b, const Vec3& c, double margin_bohr, double spacing_bohr);
};

/// Scalar values on a grid with the atoms, for Cube output.
class Field {
public:
    Field(Grid grid, std::vector<Atom> atoms, std::vector<double> values);
    double operator()(int i, int j, int k) const;
    const std::vector<double>& values() const noexcept { return values_; }
    std::vector<double>& mutable_values() noexcept { return values_; }
    const Grid& grid() const noexcept { return grid_; }
    const std::vector<Atom>& atoms() const noexcept { return atoms_; }
    /// Gaussian Cube file, six significant digits (src/cube.cpp:70-111).
    void write_cube(const std::filesystem::path& path, const std::string& comment = "Electron density") const;
    void write_orbital_cube(const std::filesystem::path& path, std::size_t orbital_index,
                            const std::string& comment = "Molecular orbital amplitude") const;

private:
    Grid grid_;
    std::vector<Atom> atoms_;
    std::vector<double> values_;
};

enum class OrbitalRepresentationStatus { Valid, Inconsistent, Unavailable };

inline constexpr double orbital_check_relative_tolerance = 1e-8;
inline constexpr double orbital_check_absolute_tolerance = 1e-10;

struct ElectronicStructureInfo {
    OrbitalRepresentationStatus orbital_status = OrbitalRepresentationStatus::Unavailable;
    double total_absolute_error = 0.0;
    double total_relative_error = 0.0;
    double spin_absolute_error = 0.0;
    double spin_relative_error = 0.0;
    std::size_t occupied_alpha = 0;
    std::size_t occupied_beta = 0;
    [[nodiscard]] bool ao_mo_eligible() const noexcept {
        return orbital_status == OrbitalRepresentationStatus::Valid;
    }
};

/// Molecule loaded from an FCHK: atoms, basis, SCF density matrices, MOs and
/// energies, with the load-time check of the MOs against the density
/// matrices (src/molecule.cpp:153-180).  Its device copy (AO tables, P, MO
/// coefficients) is created on the first evaluation and kept resident.
class Molecule {
public:
    static Molecule from_fchk(const std::filesystem::path& path);
    /// Molecule from in-memory arrays (the same records as an FCHK); an empty
    /// `spin` means a zero spin-difference matrix.
    static Molecule from_parts(std::vector<Atom> atoms, BasisSet basis, Matrix total, Matrix spin,
                               int nalpha, int nbeta, Matrix alpha_mos, Matrix beta_mos,
                               std::vector<double> alpha_energies, std::vector<double> beta_energies);

    Molecule(Molecule&&) noexcept;
    Molecule& operator=(Molecule&&) noexcept;
    ~Molecule();

    const std::vector<Atom>& atoms() const noexcept { return atoms_; }
    const ElectronicStructureInfo& electronic_structure_info() const noexcept { return electronic_info_; }
    std::size_t basis_size() const noexcept { return basis_.function_count(); }
    const BasisSet& basis() const noexcept { return basis_; }
    const std::vector<PreparedBlock>& blocks() const noexcept { return blocks_; }
    /// AO density matrix of a component: Total and Difference from the FCHK,
    /// Alpha/Beta = (Total +/- Difference) / 2.
    Matrix density_matrix(DensityComponent component = DensityComponent::Total) const;
    bool unrestricted() const noexcept { return unrestricted_; }
    const Matrix& mo_coefficients(SpinChannel channel) const;
    std::size_t orbital_count(SpinChannel channel = SpinChannel::Alpha) const;
    std::size_t occupied_count(SpinChannel channel = SpinChannel::Alpha) const;
    const std::vector<double>& orbital_energies(SpinChannel channel = SpinChannel::Alpha) const;

    /// Device copy of the molecule on the current CUDA device (created on
    /// first use; internal).
    detail::DeviceMolecule& device() const;
    /// Bytes of device memory held by the resident copy (0 before first use).
    std::size_t device_bytes() const;
    /// The device copy on the current CUDA device if it already exists, else
    /// null; never allocates (internal).
    const detail::DeviceMolecule* device_if_resident() const;

private:
    Molecule() = default;
    void finish();
    std::vector<Atom> atoms_;
    BasisSet basis_{std::vector<Shell>{}, 0};
    std::vector<PreparedBlock> blocks_;
    Matrix total_, spin_;
    Matrix alpha_mos_, beta_mos_;
    std::vector<double> alpha_energies_, beta_energies_;
    int nalpha_ = 0, nbeta_ = 0;
    bool unrestricted_ = false;
    ElectronicStructureInfo electronic_info_;
    mutable std::unique_ptr<std::mutex> device_mutex_ = std::make_unique<std::mutex>();
    mutable std::unique_ptr<detail::DeviceMolecule> device_;
};

}  // namespace chem::kumo
