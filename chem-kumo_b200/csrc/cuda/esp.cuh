// Molecular electrostatic potential on the device (McMurchie-Davidson),
// exact form (tolerance 0) of chem-kumo's detail::ElectrostaticPotential
// (src/electrostatic_potential.cpp:117-360) and its Boys function
// (src/boys_function.cpp:11-76).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <vector>

#include "kumo_device.cuh"

namespace chem::kumo {
class Molecule;
}

namespace kumo_dev {

constexpr int kBoysMaxOrder = 32;
constexpr int kBoysTaylor = 7;
constexpr int kBoysOrders = kBoysMaxOrder + kBoysTaylor;  // 39
constexpr int kBoysPoints = 801;                          // T = 0, 0.05, ..., 40
constexpr int kEspMaxL = 8;                               // la + lb of the device kernel

// One primitive pair: exponent p, product centre Q, order L = la + lb and
// the offset of its C(L+3,3) Hermite coefficients (which include 2 pi / p
// and the density-matrix weights).
struct EspPair {
    double p;
    double qx, qy, qz;
    int order;
    int first;
};

struct EspView {
    const EspPair* pairs = nullptr;
    const double* coef = nullptr;
    long long npairs = 0;
    const double* boys_table = nullptr;  // kBoysPoints x kBoysOrders
    const double4* atoms = nullptr;      // x, y, z, nuclear charge
    int natoms = 0;
    // Hermite triples (t, u, v), t + u + v <= kEspMaxL, ordered by t + u + v
    // as src/electrostatic_potential.cpp:100-107; entry k gives the axis of
    // its recursion step, the entries one and two steps down that axis (-1 if
    // none) and the factor of the second term.
    const int4* recursion = nullptr;
    // Pairs are grouped by order: those of order L are [order_first[L], order_first[L + 1]).
    long long order_first[kEspMaxL + 2] = {};
};

struct EspParams {
    EspView esp;
    PointSource src;
    double* out = nullptr;
    long long out_base = 0;
    // Mixed form: FP32 Hermite recursion, coefficient dot and pair sums;
    // FP64 Boys values, scaling and nuclear-minus-electronic difference.
    bool mixed = false;
};

/// Host setup of the pairs and the Boys table, uploaded to the device.
class EspDevice {
public:
    EspDevice(const chem::kumo::Molecule& m, cudaStream_t stream);
    ~EspDevice();
    EspDevice(const EspDevice&) = delete;
    EspDevice& operator=(const EspDevice&) = delete;
    EspView view() const { return view_; }
    long long pair_count() const { return view_.npairs; }
    std::size_t device_bytes() const { return bytes_; }

private:
    EspView view_;
    std::vector<void*> allocs_;
    std::size_t bytes_ = 0;
};

/// Boys table F_m(T_i), m < kBoysOrders, T_i = 0.05 i (src/boys_function.cpp:23-44).
std::vector<double> boys_table_host();
/// F_0..F_{n-1}(T) on the host from the same table (src/boys_function.cpp:47-76).
void boys_host(const double* table, double T, int n, double* out);

/// Exact potential at the points of p.src: one launch per pair order over
/// (128-point tiles x pair chunks) writing partial sums to stream-ordered
/// scratch, then a fixed-order FP64 reduction with the nuclear term.  FP64
/// throughout, or the mixed form when p.mixed is set.
void launch_esp(const EspParams& p, cudaStream_t stream);
/// F_m(T) for an array of T on the device (test seam of the Boys kernel).
void launch_boys_f64(const double* table, const double* t, long long n, int nvalues, double* out, cudaStream_t stream);

}  // namespace kumo_dev
