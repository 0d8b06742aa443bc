#pragma once
// Molecular surfaces with the names and semantics of chem-kumo's
// include/chem/kumo/surface.hpp: the density isosurface (marching tetrahedra
// on the device, vertices placed on the exact isosurface by Newton steps
// whose density and gradient come from the device evaluator), surface
// statistics, the electrostatic potential, the average local ionization
// energy and any one-component property on it, and PLY output.
#include "chem/kumo/density.hpp"
#include "chem/kumo/evaluator.hpp"

#include <array>
#include <cstddef>
#include <filesystem>
#include <functional>
#include <span>
#include <string>
#include <utility>
#include <vector>

namespace chem::kumo {

/// Hartree in kcal/mol (CODATA 2018).
inline constexpr double hartree_in_kcal_per_mol = 627.5094740631;
/// Hartree in eV (CODATA 2018).
inline constexpr double hartree_in_electronvolt = 27.211386245988;

/// Closed, oriented triangle mesh (bohr); each triangle counter-clockwise
/// seen from outside (include/chem/kumo/surface.hpp:22-35).
struct TriangleMesh {
    std::vector<Vec3> vertices;
    std::vector<std::array<std::size_t, 3>> triangles;
    [[nodiscard]] double area() const;
    [[nodiscard]] double volume() const;
};

/// Politzer-Murray statistics of vertex values interpolated linearly over the
/// triangles (include/chem/kumo/surface.hpp:37-77).
struct SurfaceStatistics {
    double area = 0.0;
    double positive_area = 0.0;
    double negative_area = 0.0;
    double nonpolar_area = 0.0;
    double minimum = 0.0;
    double maximum = 0.0;
    std::size_t minimum_vertex = 0;
    std::size_t maximum_vertex = 0;
    double average = 0.0;
    double positive_average = 0.0;
    double negative_average = 0.0;
    double positive_variance = 0.0;
    double negative_variance = 0.0;
    double total_variance = 0.0;
    double balance = 0.0;
    double charge_separation = 0.0;
    double polarity_index = 0.0;
    std::vector<std::size_t> local_minima;
    std::vector<std::size_t> local_maxima;
};

[[nodiscard]] SurfaceStatistics surface_statistics(const TriangleMesh& mesh, std::span<const double> values,
                                                   double polar_threshold = 10.0 / hartree_in_kcal_per_mol);

/// Smallest density isovalue accepted, e/bohr^3.
inline constexpr double minimum_density_isovalue = 1e-8;

/// Isosurface rho = isovalue of the total density (include/chem/kumo/surface.hpp:101-116).
[[nodiscard]] TriangleMesh density_isosurface(const Molecule& molecule, double isovalue = 1e-3,
                                              double spacing = 0.25);

struct SurfaceOptions {
    double isovalue = 1e-3;
    double spacing = 0.25;
    double potential_tolerance = 1e-8;
};

struct PotentialSurface {
    TriangleMesh mesh;
    std::vector<double> potential;
    SurfaceStatistics statistics;
};

/// Electrostatic potential at the vertices of the density isosurface, with
/// its statistics (polar threshold 10 kcal/mol).  The device evaluates every
/// primitive pair exactly, which meets any potential_tolerance.
[[nodiscard]] PotentialSurface electrostatic_potential_surface(const Molecule& molecule,
                                                               const SurfaceOptions& options = {});

/// Average local ionization energy at points (include/chem/kumo/surface.hpp:135-155).
[[nodiscard]] std::vector<double> average_local_ionization_energy(const Molecule& molecule, Points points);

struct IonizationEnergySurface {
    TriangleMesh mesh;
    std::vector<double> ionization_energy;
    SurfaceStatistics statistics;
};

[[nodiscard]] IonizationEnergySurface local_ionization_energy_surface(const Molecule& molecule,
                                                                      double isovalue = 1e-3, double spacing = 0.25);

struct MappedSurface {
    TriangleMesh mesh;
    std::vector<Property> properties;
    std::vector<std::vector<double>> values;
    std::vector<SurfaceStatistics> statistics;
    Backend backend_used = Backend::AO_P;
};

/// One-component properties at the vertices of the density isosurface
/// (include/chem/kumo/surface.hpp:167-192).
[[nodiscard]] MappedSurface map_on_density_isosurface(const Molecule& molecule,
                                                      const std::vector<Property>& properties,
                                                      double isovalue = 1e-3, double spacing = 0.25,
                                                      const EvaluationOptions& options = {});

/// ASCII PLY output (include/chem/kumo/surface.hpp:194-208).
void write_ply(const std::filesystem::path& path, const TriangleMesh& mesh,
               const std::vector<std::pair<std::string, std::vector<double>>>& fields,
               const std::vector<std::string>& comments = {});

namespace detail {
/// f and its gradient at points (src/isosurface.hpp).
using ScalarFunction =
    std::function<void(const std::vector<Vec3>& points, std::vector<double>& values, std::vector<Vec3>& gradients)>;

struct Isosurface {
    TriangleMesh mesh;
    std::vector<IVec3> vertex_cells;  ///< grid indices of the lower end of each vertex's edge
};

/// Isosurface f = isovalue of samples on a grid (host or device array):
/// marching tetrahedra on the device, vertices moved onto f = isovalue along
/// their edges to 1e-10 bohr (src/surface.cpp:206-320).
Isosurface extract_isosurface(const Grid& grid, const double* samples, bool samples_on_device, double isovalue,
                              const ScalarFunction& function);
}  // namespace detail

}  // namespace chem::kumo
