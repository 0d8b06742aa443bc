#pragma once

#include <filesystem>
#include <string>

#include "chem/kumo/density.hpp"

namespace chem::kumo {

/// Header lines of a Cube file that are not part of the field, and the
/// length unit of its header (include/chem/kumo/cube.hpp of chem-kumo).
struct CubeMetadata {
    std::string first_comment;
    std::string second_comment;
    /// The header was in angstrom (negative grid counts); the Field is in
    /// bohr either way.
    bool coordinates_in_angstrom = false;
};

/// One scalar Cube dataset: its field (bohr) and header information.
struct CubeData {
    Field field;
    CubeMetadata metadata;
};

/// Reads a scalar Gaussian Cube file, plain or gzip-compressed (detected
/// from its first two bytes; the gzip trailer is verified).  Same rules as
/// chem-kumo's read_cube (src/cube.cpp:114-212): a non-negative atom count
/// (orbital Cubes are rejected), an optional NVAL of 1 after the origin,
/// grid counts of at least 2 per axis and 1e9 samples in all, one length unit
/// for all three axes (negative counts: angstrom, converted to bohr), atoms
/// with 0 <= Z <= 118 and finite records, Fortran D exponents, exactly as many
/// finite samples as grid points.  Throws std::runtime_error with the
/// reference's messages.
[[nodiscard]] CubeData read_cube(const std::filesystem::path& path);

/// Writes a Cube file that read_cube reproduces: the metadata's comment lines
/// and length unit, header and values with 13 significant digits, six values
/// per line (src/cube.cpp:215-251).  Throws std::invalid_argument for a
/// comment with a line break, a nonfinite value, an invalid atom or a value
/// count that does not match the grid, std::runtime_error if the file cannot
/// be written.
void write_cube(const CubeData& cube, const std::filesystem::path& path);

}  // namespace chem::kumo
