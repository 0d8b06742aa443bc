#pragma once
// Small fixed-size and dynamic matrix types that stand in for the Eigen types
// of chem-kumo's public API (Eigen::Vector3d, Eigen::Matrix3d,
// Eigen::MatrixXd, 3 x N point matrices).  Storage is column-major, like
// Eigen's default.

#include <array>
#include <cstddef>
#include <stdexcept>
#include <vector>

namespace chem::kumo {

using Vec3 = std::array<double, 3>;
using IVec3 = std::array<int, 3>;

/// 3 x 3 matrix, column-major: m[c * 3 + r] is row r of column c.
struct Mat3 {
    std::array<double, 9> m{1, 0, 0, 0, 1, 0, 0, 0, 1};
    double& operator()(int r, int c) { return m[static_cast<std::size_t>(c * 3 + r)]; }
    double operator()(int r, int c) const { return m[static_cast<std::size_t>(c * 3 + r)]; }
    Vec3 col(int c) const { return {m[c * 3], m[c * 3 + 1], m[c * 3 + 2]}; }
    static Mat3 identity() { return Mat3{}; }
    static Mat3 scaled_identity(double s) {
        Mat3 a;
        a.m = {s, 0, 0, 0, s, 0, 0, 0, s};
        return a;
    }
};

/// Dynamic column-major matrix of doubles.
class Matrix {
public:
    Matrix() = default;
    Matrix(std::size_t rows, std::size_t cols, double fill = 0.0)
        : rows_(rows), cols_(cols), data_(rows * cols, fill) {}
    std::size_t rows() const noexcept { return rows_; }
    std::size_t cols() const noexcept { return cols_; }
    std::size_t size() const noexcept { return data_.size(); }
    double& operator()(std::size_t r, std::size_t c) { return data_[c * rows_ + r]; }
    double operator()(std::size_t r, std::size_t c) const { return data_[c * rows_ + r]; }
    double* data() noexcept { return data_.data(); }
    const double* data() const noexcept { return data_.data(); }
    const double* col(std::size_t c) const { return data_.data() + c * rows_; }

private:
    std::size_t rows_ = 0, cols_ = 0;
    std::vector<double> data_;
};

/// View of a 3 x N matrix of points (bohr), one point per column: point j is
/// (data[3j], data[3j+1], data[3j+2]).
struct Points {
    const double* data = nullptr;
    std::size_t count = 0;
};

}  // namespace chem::kumo
