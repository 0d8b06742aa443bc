// Per-point density-derivative records and the derived fields of
// src/evaluator.cpp:117-353, evaluated on the device in the epilogue of the
// contraction kernels.  All of this is FP64, in both precisions.
#pragma once

#include <cuda_runtime.h>

#include "kumo_device.cuh"

namespace kumo_dev {

constexpr int kMaxProps = 40;

// detail::DensityDerivatives (include/chem/kumo/density.hpp:153-160) with the
// symmetric Hessian stored as xx, xy, xz, yy, yz, zz.
struct DevDD {
    double value, grad[3], hess[6], lap, tau, tau_axes[3];
};

__device__ __forceinline__ void dd_zero(DevDD& d) {
    d.value = 0;
    for (int i = 0; i < 3; ++i) d.grad[i] = d.tau_axes[i] = 0;
    for (int i = 0; i < 6; ++i) d.hess[i] = 0;
    d.lap = d.tau = 0;
}

// combine(), src/density.cpp:50-60.  With the full Hessian the Laplacian is
// its trace; in Laplacian-only mode it is combined like the other terms.
__device__ __forceinline__ DevDD dd_combine(const DevDD& a, const DevDD& b, double sign, double scale,
                                            bool full_hessian) {
    DevDD d;
    d.value = scale * (a.value + sign * b.value);
    for (int i = 0; i < 3; ++i) d.grad[i] = scale * (a.grad[i] + sign * b.grad[i]);
    for (int i = 0; i < 6; ++i) d.hess[i] = scale * (a.hess[i] + sign * b.hess[i]);
    d.lap = full_hessian ? (d.hess[0] + d.hess[3]) + d.hess[5] : scale * (a.lap + sign * b.lap);
    d.tau = scale * (a.tau + sign * b.tau);
    for (int i = 0; i < 3; ++i) d.tau_axes[i] = scale * (a.tau_axes[i] + sign * b.tau_axes[i]);
    return d;
}

// One requested property: kind (PropertyKind), component (DensityComponent)
// and its output, channels(kind) arrays of `stride` doubles.
struct OutProp {
    int kind;
    int component;
    double* out;
};

struct FieldSpec {
    int nprops = 0;
    long long stride = 0;       // points per output component array
    long long out_base = 0;     // global index of the point stored at out[0]
    OutProp props[kMaxProps];
    GridTiles tiles;            // evaluation index -> grid index (see GridTiles)
};

__device__ __forceinline__ double fermi_constant() {
    // 0.3 (6 pi^2)^(2/3) as the host's libm rounds it (a literal: the device
    // pow of constant arguments is evaluated at run time, at every point).
    return 4.557799872345596;
}

__device__ __forceinline__ double sq3(const double* g) { return g[0] * g[0] + g[1] * g[1] + g[2] * g[2]; }

// elf(), src/evaluator.cpp:127-140.
__device__ __forceinline__ double dev_elf(const DevDD* const* ch, int n) {
    const double fermi = fermi_constant();
    double pauli = 0.0, uniform = 0.0;
    for (int i = 0; i < n; ++i) {
        const DevDD* d = ch[i];
        if (!(d->value > 0.0)) continue;
        pauli += d->tau - sq3(d->grad) / (8.0 * d->value);
        uniform += fermi * pow(d->value, 5.0 / 3.0);
    }
    if (!(uniform > 0.0)) return 0.0;
    const double chi = pauli / uniform;
    return 1.0 / (1.0 + chi * chi);
}

// lol(), src/evaluator.cpp:168-179.
__device__ __forceinline__ double dev_lol(const DevDD* const* ch, int n) {
    const double fermi = fermi_constant();
    double tau = 0.0, uniform = 0.0;
    for (int i = 0; i < n; ++i) {
        tau += ch[i]->tau;
        if (ch[i]->value > 0.0) uniform += fermi * pow(ch[i]->value, 5.0 / 3.0);
    }
    if (!(uniform > 0.0)) return 0.0;
    if (!(tau > 0.0)) return 1.0;
    return uniform / (tau + uniform);
}

// gradient_expansion_locator(), src/evaluator.cpp:195-215.
__device__ __forceinline__ double dev_gradient_expansion(const DevDD* const* ch, int n, bool lol) {
    const double fermi = fermi_constant();
    double uniform = 0.0, pauli = 0.0, kinetic = 0.0;
    for (int i = 0; i < n; ++i) {
        const DevDD* d = ch[i];
        if (!(d->value > 0.0)) continue;
        const double reference = fermi * pow(d->value, 5.0 / 3.0);
        const double weizsacker = sq3(d->grad) / d->value;
        uniform += reference;
        pauli += reference - weizsacker / 9.0 + d->lap / 6.0;
        kinetic += reference + weizsacker / 72.0 + d->lap / 6.0;
    }
    if (!(uniform > 0.0)) return 0.0;
    if (lol) {
        const double den = kinetic + uniform;
        return den != 0.0 ? uniform / den : 0.0;
    }
    const double chi = pauli / uniform;
    return 1.0 / (1.0 + chi * chi);
}

// reduced_gradient(), src/evaluator.cpp:145-154 (cap 100).
__device__ inline double dev_reduced_gradient(const DevDD& d) {
    const double scale = 6.187335452560272;  // 2 cbrt(3 pi^2), as the host's libm rounds it
    if (!(d.value > 0.0)) return 100.0;
    const double den = scale * pow(d.value, 4.0 / 3.0);
    const double norm = sqrt(sq3(d.grad));
    if (!(den > 0.0) || !(norm < 100.0 * den)) return 100.0;
    return norm / den;
}

// Middle eigenvalue of the symmetric 3x3 Hessian by cyclic Jacobi rotations
// (the sign decides sign(lambda2) rho, src/evaluator.cpp:158-161).
// Hessian entries xx, xy, xz, yy, yz, zz by value: the caller's record then
// need not live in memory.
static __device__ __noinline__ double dev_lambda2(double xx, double xy, double xz, double yy, double yz, double zz) {
    double a[3][3] = {{xx, xy, xz}, {xy, yy, yz}, {xz, yz, zz}};
    for (int sweep = 0; sweep < 64; ++sweep) {
        const double off = fabs(a[0][1]) + fabs(a[0][2]) + fabs(a[1][2]);
        if (off == 0.0) break;
        for (int p = 0; p < 2; ++p)
            for (int q = p + 1; q < 3; ++q) {
                if (a[p][q] == 0.0) continue;
                const double theta = (a[q][q] - a[p][p]) / (2.0 * a[p][q]);
                const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < 3; ++k) {
                    const double akp = a[k][p], akq = a[k][q];
                    a[k][p] = c * akp - s * akq;
                    a[k][q] = s * akp + c * akq;
                }
                for (int k = 0; k < 3; ++k) {
                    const double apk = a[p][k], aqk = a[q][k];
                    a[p][k] = c * apk - s * aqk;
                    a[q][k] = s * apk + c * aqk;
                }
            }
    }
    const double e0 = a[0][0], e1 = a[1][1], e2 = a[2][2];
    if ((e0 >= e1 && e0 <= e2) || (e0 <= e1 && e0 >= e2)) return e0;
    if ((e1 >= e0 && e1 <= e2) || (e1 <= e0 && e1 >= e2)) return e1;
    return e2;
}

// Whether lambda2 < 0 (lambda2 == 0 counts as positive).  The eigenvalues
// l1 <= l2 <= l3 are the roots of det(x I - H); with e1 = l1 + l2 + l3,
// e2 = l1 l2 + l1 l3 + l2 l3 and e3 = l1 l2 l3, l2 < 0 exactly when at least
// two eigenvalues are negative: for e3 < 0 when all three are (e1 < 0 and
// e2 > 0), for e3 > 0 unless all three are positive (e1 > 0 and e2 > 0).
// Where e1, e2 and e3 all stand clear of zero (|e_k| > 1e-8 |H|_F^k, far
// above their rounding errors) the signs are exact and |l2| > 1e-8 |H|_F,
// so the answer is the Jacobi eigenvalue's sign; elsewhere the Jacobi
// eigenvalue decides.  H is first scaled by a power of two (exactly) to
// entries of magnitude below 2, so that no product under- or overflows.
__device__ __forceinline__ bool dev_lambda2_negative(const double* h6) {
    double m = 0.0;
#pragma unroll
    for (int i = 0; i < 6; ++i) m = fmax(m, fabs(h6[i]));
    // (A NaN entry makes the e_k NaN, and the margins then fail.)
    if (!(m > 0.0) || !isfinite(m)) return dev_lambda2(h6[0], h6[1], h6[2], h6[3], h6[4], h6[5]) < 0.0;
    const int ex = ilogb(m);
    const double a = ldexp(h6[0], -ex), b = ldexp(h6[1], -ex), c = ldexp(h6[2], -ex);
    const double d = ldexp(h6[3], -ex), e = ldexp(h6[4], -ex), f = ldexp(h6[5], -ex);
    const double e1 = a + d + f;
    const double e2 = (a * d - b * b) + (a * f - c * c) + (d * f - e * e);
    const double e3 = a * (d * f - e * e) - b * (b * f - c * e) + c * (b * e - c * d);
    const double s2 = (a * a + d * d + f * f) + 2.0 * ((b * b + c * c) + e * e);
    const double k2 = 1e-16;  // (1e-8)^2
    if (e1 * e1 > k2 * s2 && e2 * e2 > k2 * s2 * s2 && e3 * e3 > k2 * s2 * s2 * s2)
        return e3 < 0.0 ? (e1 < 0.0 && e2 > 0.0) : !(e1 > 0.0 && e2 > 0.0);
    return dev_lambda2(h6[0], h6[1], h6[2], h6[3], h6[4], h6[5]) < 0.0;
}

__device__ inline double dev_iri(const DevDD& d) {
    if (!(d.value > 0.0)) return 100.0;
    const double v = sqrt(sq3(d.grad)) / pow(d.value, 1.1);
    return v < 100.0 ? v : 100.0;
}

__device__ inline double dev_dori(const DevDD& d) {
    if (!(d.value > 0.0)) return 0.0;
    const double q[3] = {d.grad[0] / d.value, d.grad[1] / d.value, d.grad[2] / d.value};
    const double q2 = sq3(q);
    if (!(q2 > 0.0)) return 1.0;
    const double H[3][3] = {{d.hess[0], d.hess[1], d.hess[2]},
                            {d.hess[1], d.hess[3], d.hess[4]},
                            {d.hess[2], d.hess[4], d.hess[5]}};
    double w[3];
    for (int a = 0; a < 3; ++a) w[a] = (H[a][0] * q[0] + H[a][1] * q[1] + H[a][2] * q[2]) / d.value - q2 * q[a];
    const double theta = 4.0 * sq3(w) / (q2 * q2 * q2);
    if (!isfinite(theta)) return 1.0;
    return theta / (1.0 + theta);
}

// One property of one component record d (store_block's per-kind cases).
__device__ __forceinline__ void store_one(int kind, const DevDD& d, double* out, long long p, long long S) {
    const DevDD* one[1] = {&d};
    switch (kind) {
        case 0: out[p] = d.value; break;
        case 1:
            for (int a = 0; a < 3; ++a) out[a * S + p] = d.grad[a];
            break;
        case 2:
            for (int h = 0; h < 6; ++h) out[h * S + p] = d.hess[h];
            break;
        case 3: out[p] = d.lap; break;
        case 4: out[p] = d.tau; break;
        case 6: out[p] = dev_elf(one, 1); break;
        case 7: out[p] = dev_reduced_gradient(d); break;
        case 8: out[p] = dev_lambda2_negative(d.hess) ? -d.value : d.value; break;
        case 10: out[p] = dev_lol(one, 1); break;
        case 35: out[p] = dev_gradient_expansion(one, 1, false); break;
        case 36: out[p] = dev_gradient_expansion(one, 1, true); break;
        case 11: out[p] = dev_iri(d); break;
        case 12: out[p] = dev_dori(d); break;
        case 13: out[p] = d.tau - 0.25 * d.lap; break;
        case 14: out[p] = 0.25 * d.lap - 2.0 * d.tau; break;
        case 15: out[p] = 0.25 * d.lap - d.tau; break;
        case 30:
            for (int a = 0; a < 3; ++a) out[a * S + p] = d.tau_axes[a];
            break;
        case 31: {
            const int diag[3] = {0, 3, 5};
            for (int a = 0; a < 3; ++a) out[a * S + p] = d.tau_axes[a] - 0.25 * d.hess[diag[a]];
            break;
        }
        case 32: out[p] = d.tau > 0.0 ? fabs(0.25 * d.lap - 2.0 * d.tau) / d.tau : 0.0; break;
        case 33: out[p] = d.value > 0.0 ? (0.25 * d.lap - d.tau) / d.value : 0.0; break;
        case 34: out[p] = d.value > 0.0 ? d.tau / d.value : 0.0; break;
        case 17: out[p] = d.value > 0.0 ? -d.value * log(d.value) : 0.0; break;
        case 18: out[p] = d.value > 0.0 ? sq3(d.grad) / d.value : 0.0; break;
        default: break;
    }
}

// store_block(), src/evaluator.cpp:248-353, for one point.  alpha and beta
// are the records of DensityComponent Alpha and Beta; rec(c) gives the record
// of Total (c = 0) or Difference (c = 3).  Each record is named in its own
// branch (none is indexed at run time), so the caller's records can stay in
// registers.
template <typename Rec>
__device__ __forceinline__ void store_point_records(const FieldSpec& spec, const DevDD& alpha, const DevDD& beta,
                                                    Rec rec, long long q) {
    if (spec.tiles.on && !tile_to_linear(spec.tiles, q, q)) return;  // tile padding
    const long long p = q - spec.out_base;
    const long long S = spec.stride;
    for (int i = 0; i < spec.nprops; ++i) {
        const int kind = spec.props[i].kind;
        const int cpt = spec.props[i].component;
        double* out = spec.props[i].out;
        if ((kind == 6 || kind == 10 || kind == 35 || kind == 36) && cpt == 0) {
            const DevDD* ch[2] = {&alpha, &beta};
            out[p] = kind == 6 ? dev_elf(ch, 2) : kind == 10 ? dev_lol(ch, 2) : dev_gradient_expansion(ch, 2, kind == 36);
            continue;
        }
        if (kind == 16) {
            const double t = rec(0).value;
            out[p] = t > 0.0 ? rec(3).value / t : 0.0;
            continue;
        }
        switch (cpt) {
            case 0: store_one(kind, rec(0), out, p, S); break;
            case 1: store_one(kind, alpha, out, p, S); break;
            case 2: store_one(kind, beta, out, p, S); break;
            default: store_one(kind, rec(3), out, p, S); break;
        }
    }
}

// From the two channels' records: Total and Difference formed where a
// property asks for them (combine(), src/density.cpp:50-60).
__device__ __forceinline__ void store_point(const FieldSpec& spec, const DevDD& alpha, const DevDD& beta,
                                            bool full_hessian, long long q) {
    store_point_records(
        spec, alpha, beta,
        [&](int c) { return dd_combine(alpha, beta, c == 0 ? 1.0 : -1.0, 1.0, full_hessian); }, q);
}

// With comp[c] the record of DensityComponent c.
__device__ inline void store_point(const FieldSpec& spec, const DevDD* comp, long long q) {
    store_point_records(spec, comp[1], comp[2], [&](int c) { return comp[c]; }, q);
}

}  // namespace kumo_dev
