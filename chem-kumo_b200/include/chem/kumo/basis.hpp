#pragma once

#include "chem/kumo/fchk.hpp"
#include "chem/kumo/types.hpp"

#include <cstddef>
#include <vector>

namespace chem::kumo {

enum class ShellRepresentation { Cartesian, Pure };

/// One contracted shell of an FCHK basis, in file order
/// (include/chem/kumo/basis.hpp of chem-kumo).
struct Shell {
    std::size_t center = 0;
    int angular_momentum = 0;
    ShellRepresentation representation = ShellRepresentation::Cartesian;
    bool is_sp = false;
    Vec3 origin{0, 0, 0};
    std::vector<double> exponents;
    std::vector<double> coefficients;
    std::vector<double> p_coefficients;
    [[nodiscard]] std::size_t function_count() const;
};

/// Basis set rebuilt from the FCHK shell records (src/basis.cpp:21-120).
class BasisSet {
public:
    explicit BasisSet(const FormattedCheckpoint& fchk);
    BasisSet(std::vector<Shell> shells, std::size_t declared_functions);
    [[nodiscard]] const std::vector<Shell>& shells() const noexcept { return shells_; }
    [[nodiscard]] std::size_t function_count() const noexcept { return function_count_; }

private:
    std::vector<Shell> shells_;
    std::size_t function_count_ = 0;
};

/// Powers (i, j, k) of one Cartesian component x^i y^j z^k.
struct CartesianPower {
    int x = 0, y = 0, z = 0;
};

/// Gaussian FCHK order of the Cartesian components of a shell
/// (src/basis_evaluator.cpp:135-152).
[[nodiscard]] std::vector<CartesianPower> gaussian_cartesian_order(int l);
/// (2l+1) x ncart Cartesian-to-pure matrix, rows m = 0, +1, -1, ...
/// (Schlegel and Frisch 1995; src/basis_evaluator.cpp:157-175).
[[nodiscard]] Matrix gaussian_cartesian_to_pure(int l);

/// One normalised AO block (a shell, or half of an SP shell) prepared for
/// evaluation: weights are contraction coefficient times primitive
/// normalisation (src/basis_math.cpp:27-66), and cutoff_radius2 the squared
/// radius beyond which every AO of the block and its first and second
/// derivatives are at most 1e-14 (src/basis_evaluator.cpp:98-127).
struct PreparedBlock {
    Vec3 origin{0, 0, 0};
    int angular_momentum = 0;
    bool pure = false;
    std::vector<double> exponents;
    std::vector<CartesianPower> powers;
    std::vector<double> weights;  ///< ncart x nprim, row-major
    std::size_t offset = 0;
    std::size_t count = 0;
    double cutoff_radius2 = 0.0;
};

/// Shell cutoff: a rigorous bound on every AO and first/second derivative
/// beyond the cutoff radius (BasisEvaluator::ao_cutoff).
inline constexpr double ao_cutoff = 1e-14;

/// Prepared AO blocks of a basis, in AO order.
[[nodiscard]] std::vector<PreparedBlock> prepare_blocks(const BasisSet& basis);

/// Primitive normalisation (2a/pi)^(3/4) sqrt((4a)^l / prod (2n-1)!!)
/// (src/basis_math.cpp:17-25).
[[nodiscard]] double cartesian_primitive_normalization(double alpha, const CartesianPower& power);

}  // namespace chem::kumo
