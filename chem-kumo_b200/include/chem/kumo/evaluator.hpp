#pragma once
// Evaluator, Request and Results of the B200 grid evaluator, with the names
// and semantics of chem-kumo's include/chem/kumo/evaluator.hpp.

#include "chem/kumo/density.hpp"

#include <cstddef>
#include <functional>
#include <map>
#include <span>
#include <vector>

namespace chem::kumo {

/// include/chem/kumo/evaluator.hpp:109-153 of chem-kumo (same enumerators, same
/// order, so that the integer values agree).
enum class PropertyKind {
    Density,
    Gradient,
    Hessian,
    Laplacian,
    Tau,
    Orbital,
    Elf,
    ReducedGradient,
    SignLambda2Density,
    ElectrostaticPotential,
    Lol,
    InteractionRegionIndicator,
    DensityOverlapRegionsIndicator,
    HamiltonianKineticEnergy,
    PotentialEnergyDensity,
    EnergyDensity,
    SpinPolarization,
    ShannonEntropyDensity,
    FisherInformationDensity,
    AverageLocalIonizationEnergy,
    LocalElectronAffinity,
    LocalElectronAttachmentEnergy,
    LocalElectronegativity,
    LocalHardness,
    OrbitalGradient,
    OrbitalHessian,
    OrbitalWeightedFukuiPlus,
    OrbitalWeightedFukuiMinus,
    OrbitalWeightedFukuiZero,
    OrbitalWeightedDualDescriptor,
    TauComponents,
    HamiltonianKineticEnergyComponents,
    PotentialKineticRatio,
    EnergyDensityPerElectron,
    KineticEnergyPerElectron,
    ElfTsirelsonStash,
    LolTsirelsonStash
};

inline constexpr double reduced_gradient_cap = 100.0;
inline constexpr double interaction_region_indicator_cap = 100.0;
inline constexpr double potential_cluster_edge = 1.6;

struct Property {
    PropertyKind kind;
    DensityComponent component = DensityComponent::Total;
    SpinChannel channel = SpinChannel::Alpha;
    std::size_t orbital_index = 0;  ///< one-based
    friend bool operator==(const Property&, const Property&) = default;
    friend bool operator<(const Property& a, const Property& b) noexcept {
        if (a.kind != b.kind) return a.kind < b.kind;
        if (a.component != b.component) return a.component < b.component;
        if (a.channel != b.channel) return a.channel < b.channel;
        return a.orbital_index < b.orbital_index;
    }
};

struct DensityDescriptor {
    DensityComponent component;
    constexpr Property value() const { return {PropertyKind::Density, component}; }
    constexpr Property gradient() const { return {PropertyKind::Gradient, component}; }
    constexpr Property hessian() const { return {PropertyKind::Hessian, component}; }
    constexpr Property laplacian() const { return {PropertyKind::Laplacian, component}; }
    constexpr Property tau() const { return {PropertyKind::Tau, component}; }
    constexpr Property elf() const { return {PropertyKind::Elf, component}; }
    constexpr Property reduced_gradient() const { return {PropertyKind::ReducedGradient, component}; }
    constexpr Property sign_lambda2_density() const { return {PropertyKind::SignLambda2Density, component}; }
    constexpr Property electrostatic_potential() const { return {PropertyKind::ElectrostaticPotential, component}; }
    constexpr Property lol() const { return {PropertyKind::Lol, component}; }
    constexpr Property interaction_region_indicator() const {
        return {PropertyKind::InteractionRegionIndicator, component};
    }
    constexpr Property density_overlap_regions_indicator() const {
        return {PropertyKind::DensityOverlapRegionsIndicator, component};
    }
    constexpr Property hamiltonian_kinetic_energy() const { return {PropertyKind::HamiltonianKineticEnergy, component}; }
    constexpr Property potential_energy_density() const { return {PropertyKind::PotentialEnergyDensity, component}; }
    constexpr Property energy_density() const { return {PropertyKind::EnergyDensity, component}; }
    constexpr Property tau_components() const { return {PropertyKind::TauComponents, component}; }
    constexpr Property hamiltonian_kinetic_energy_components() const {
        return {PropertyKind::HamiltonianKineticEnergyComponents, component};
    }
    constexpr Property potential_kinetic_ratio() const { return {PropertyKind::PotentialKineticRatio, component}; }
    constexpr Property energy_density_per_electron() const {
        return {PropertyKind::EnergyDensityPerElectron, component};
    }
    constexpr Property elf_tsirelson_stash() const { return {PropertyKind::ElfTsirelsonStash, component}; }
    constexpr Property lol_tsirelson_stash() const { return {PropertyKind::LolTsirelsonStash, component}; }
    constexpr Property kinetic_energy_per_electron() const {
        return {PropertyKind::KineticEnergyPerElectron, component};
    }
    constexpr Property spin_polarization() const { return {PropertyKind::SpinPolarization, component}; }
    constexpr Property shannon_entropy_density() const { return {PropertyKind::ShannonEntropyDensity, component}; }
    constexpr Property fisher_information_density() const {
        return {PropertyKind::FisherInformationDensity, component};
    }
};

namespace density {
inline constexpr DensityDescriptor total{DensityComponent::Total};
inline constexpr DensityDescriptor alpha{DensityComponent::Alpha};
inline constexpr DensityDescriptor beta{DensityComponent::Beta};
inline constexpr DensityDescriptor difference{DensityComponent::Difference};
}  // namespace density

struct OrbitalDescriptor {
    SpinChannel channel;
    std::size_t index;  ///< one-based
    Property value() const { return {PropertyKind::Orbital, DensityComponent::Total, channel, index}; }
    Property gradient() const { return {PropertyKind::OrbitalGradient, DensityComponent::Total, channel, index}; }
    Property hessian() const { return {PropertyKind::OrbitalHessian, DensityComponent::Total, channel, index}; }
};

namespace orbital {
inline OrbitalDescriptor alpha(std::size_t index) { return {SpinChannel::Alpha, index}; }
inline OrbitalDescriptor beta(std::size_t index) { return {SpinChannel::Beta, index}; }
}  // namespace orbital

class Request {
public:
    Request& add(Property property) {
        properties_.push_back(property);
        return *this;
    }
    const std::vector<Property>& properties() const noexcept { return properties_; }

private:
    std::vector<Property> properties_;
};

enum class Backend { AUTO, AO_P, AO_MO };

/// Arithmetic of the device kernels: FP64 throughout (reproduces the
/// reference), or the mixed-precision form (FP32 AO values, tensor-core
/// contractions with FP32 accumulation, FP64 per-point reductions and fields).
enum class Precision { FP64, Mixed };

struct EvaluationOptions {
    int threads = 0;  ///< accepted for compatibility: 0 or 1
    std::size_t block_size = 128;
    Backend backend = Backend::AUTO;
    double screening_threshold = default_screening_threshold;
    double potential_tolerance = 1e-8;
    double fukui_delta = 0.1;
    ProgressCallback progress = {};
    Precision precision = Precision::FP64;
    /// Device scratch (AO panels) of one evaluation, which sets how many
    /// point blocks run per wave; 0 = 4 GiB (or KUMO_SCRATCH_MB).  The
    /// serving loop sets it per request for its HBM admission.
    std::size_t scratch_bytes = 0;
};

struct PropertyField {
    std::size_t points = 0;
    std::vector<std::vector<double>> components;
    std::span<const double> component(std::size_t index = 0) const { return components.at(index); }
};

class Results {
public:
    const PropertyField& get(Property key) const { return fields_.at(key); }
    bool contains(Property key) const noexcept { return fields_.contains(key); }
    [[nodiscard]] Backend backend_used() const noexcept { return backend_used_; }

private:
    friend class Evaluator;
    std::map<Property, PropertyField> fields_;
    Backend backend_used_ = Backend::AO_P;
};

/// Number of output arrays of a property kind (3, 6 or 1).
std::size_t property_channels(PropertyKind kind);

/// Evaluates the properties of a Request for one molecule on the GPU, on a
/// Grid or at arbitrary points.  The Molecule must outlive the Evaluator.
class Evaluator {
public:
    explicit Evaluator(const Molecule& molecule, EvaluationOptions options = {});
    [[nodiscard]] Results evaluate(const Grid& grid, const Request& request) const;
    [[nodiscard]] Results evaluate(Points points, const Request& request) const;
    [[nodiscard]] Field field(const Grid& grid, Property property) const;

    /// Called by evaluate_device, without synchronizing, each time the work
    /// that completes points [0, done) of every output has been enqueued on
    /// the stream (one pass over the points writes all outputs; requests that
    /// need several passes report only the end).
    using ReadyCallback = std::function<void(std::size_t done)>;

    /// Device-resident form: outputs[i] points to property_channels(kind) x N
    /// device doubles (component-major) for the i-th property of `request`,
    /// written on `stream` (a cudaStream_t); returns the backend used.  The
    /// points of evaluate_device(Points) are a device array.
    Backend evaluate_device(const Grid& grid, const Request& request, double* const* outputs, void* stream,
                            const ReadyCallback& ready = {}) const;
    /// The request checks evaluate() makes before any device work (backend
    /// eligibility, orbital indices, block size, potential tolerance); throws
    /// the same exceptions.
    void validate(const Request& request) const;
    Backend evaluate_device(Points device_points, const Request& request, double* const* outputs, void* stream,
                            const ReadyCallback& ready = {}) const;

private:
    class Run;
    const Molecule* molecule_;
    EvaluationOptions options_;
};

}  // namespace chem::kumo
