// Molecular electrostatic potential on the device (McMurchie-Davidson),
// exact form (tolerance 0) of chem-kumo's detail::ElectrostaticPotential
// (src/electrostatic_potential.cpp:117-360) and its Boys function
// (src/boys_function.cpp:11-76).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <vector>
#include <mutex>
#include <map>

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
    /// The pairs to evaluate for a potential within `tolerance` of the exact
    /// one: every pair for tolerance 0; otherwise the pairs left after
    /// dropping, smallest bound first, those whose bounds sum to at most half
    /// the tolerance (the bound of a pair holds at every point, so the
    /// dropped pairs change no value by more than that).  Built on first use
    /// per tolerance (synchronous copies on `stream`) and kept.
    EspView view_for(double tolerance, cudaStream_t stream);
    /// Bound of |sum_k c_k R_k(p, X)| over all X for each pair (in pair order).
    const std::vector<double>& pair_bounds() const { return bound_; }

private:
    EspView view_;
    std::vector<void*> allocs_;
    std::size_t bytes_ = 0;
    // Host copies of the pairs (order-grouped) and coefficients, for the
    // screened views.
    std::vector<EspPair> pairs_;
    std::vector<double> coef_;
    std::vector<double> bound_;
    std::mutex views_mutex_;
    std::map<double, EspView> views_;
};

/// sup over Y of |d^(t,u,v) F_0(|Y|^2)| (F_0 the zeroth Boys function), from
/// its Fourier form F_0(|Y|^2) = sqrt(pi) / (4 pi^2) int exp(-k^2 / 4) / k^2
/// exp(i k.Y) d^3k: the derivative is bounded by the integral of
/// |k_x^t k_y^u k_z^v| exp(-k^2 / 4) / k^2, which is
/// sqrt(pi) / (4 pi^2) 2^n Gamma((n+1)/2) 2 Gamma((t+1)/2) Gamma((u+1)/2)
/// Gamma((v+1)/2) / Gamma((n+3)/2), n = t + u + v (1 for n = 0, the value at
/// Y = 0).  With R_tuv(p, X) = d^(t,u,v) F_0(p |X|^2) this gives
/// |R_tuv(p, X)| <= p^(n/2) hermite_sup(t, u, v) for all X.
double hermite_sup(int t, int u, int v);

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
