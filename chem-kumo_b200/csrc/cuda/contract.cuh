// Contraction kernels of the grid-block evaluator (FP64 path):
//  - AO-MO: V_a = C_occ[kept]^T Phi_a[kept] for each stored panel a, reduced
//    per point to rho, grad rho, tau (per axis), the Hessian or Laplacian
//    (Molecule::density_derivatives_mo, src/density.cpp:235-351), then the
//    requested fields (store_block, src/evaluator.cpp:248-353);
//  - MO amplitudes and their derivatives for selected MOs (no screening),
//    Molecule::orbitals (src/orbitals.cpp:66-102) and the orbital pass
//    (src/evaluator.cpp:688-730).
#pragma once

#include "fields.cuh"
#include "kumo_device.cuh"

namespace kumo_dev {

struct MoChannel {
    const double* ct = nullptr;  // [nao][ldc], MO contiguous
    int ldc = 0;                 // multiple of 4
    int nocc = 0;
    int role = 0;                // 1 alpha, 2 beta
};

struct ContractMoParams {
    AoScratch<double> scr;
    long long first_point = 0;
    long long block_size = 128;   // points per CTA chunk (see cta_points)
    long long screen_block = 0;   // points per screening block (0: block_size)
    long long count = 0;
    int nblocks = 0;
    int nchannels = 0;
    MoChannel ch[2];
    int beta_is_alpha = 0;  // beta record is a copy of the alpha record
    int ao_order = 2;
    FieldSpec spec;
};

struct OrbitalParams {
    AoScratch<double> scr;  // threshold 0: every AO of the shells reaching the block, in AO order
    long long first_point = 0;
    long long block_size = 128;
    long long count = 0;
    int nblocks = 0;
    int nao = 0;
    int npanel = 1;         // 1 (values), 4 (gradient) or 10 (Hessian)
    int nsel = 0;
    const double* coef[8];  // MO coefficient columns (length nao)
    double* out[8];         // channels x stride arrays
    int first_channel[8];   // panel of the first output channel (0, 1 or 4)
    int nchan[8];           // 1, 3 or 6
    long long stride = 0;
    long long out_base = 0;
};

// AO-P: Y = P[kept, kept] * Phi[kept, panels 0..3]; per point
// rho = phi.y, grad = 2 phi_a.y, tau_a = phi_a.(P phi_a) / 2,
// H_ac = 2 (phi_ac.y + phi_a.(P phi_c))  (src/density.cpp:26-44,150-229).
// With density_component >= 0 it is the values-only grid density of one
// component (src/density.cpp:366-444): rho = phi.(P_c phi).
struct ContractPParams {
    AoScratch<double> scr;
    long long first_point = 0;
    long long block_size = 128;   // points per CTA chunk (see cta_points)
    long long screen_block = 0;   // points per screening block (0: block_size)
    long long count = 0;
    int nblocks = 0;
    int nao = 0;
    int total_needed = 0;
    int spin_needed = 0;
    int density_component = -1;
    const double* p_total = nullptr;
    const double* p_spin = nullptr;
    int ao_order = 2;
    FieldSpec spec;
};

// Orbital-energy sums (src/orbital_energy_fields.hpp:14-264): with the MO
// columns of each set scaled as the reference scales them (sqrt(n_i) for the
// occupied, sqrt(w) for the attachment, sqrt(g_i) for the Fukui sets), per
// point D_s = sum_(i in s) X_i^2 and E_s = sum_(i in s) e_i X_i^2, X = C_s^T phi
// over every AO (values, shell cutoff only); then the fields of
// store_orbital_energy_block (src/evaluator.cpp:480-516).
constexpr int kOrbitalEnergySets = 5;  // occupied, virtual, attachment, Fukui +, Fukui -
constexpr int kOrbitalEnergyChunk = 128;

struct OrbitalEnergyParams {
    AoScratch<double> scr;  // values, threshold 0 (every AO of the shells reaching the block), AO order
    long long first_point = 0;
    long long block_size = 128;
    long long screen_block = 0;  // unused: no screening (see cta_points)
    long long count = 0;
    int nblocks = 0;
    const double* w = nullptr;           // [nao][ldw]: the sets' columns, each set padded to 128-column chunks
    int ldw = 0;
    int nchunks = 0;
    const int* chunk_set = nullptr;      // set of each chunk
    const double* col_energy = nullptr;  // e_i of each column (0 for padding)
    int have_virtuals = 0;
    int have_fukui = 0;
    int nout = 0;
    int kinds[9];     // PropertyKind of each output
    double* outs[9];
    long long out_base = 0;
};

void launch_orbital_energy_f64(const OrbitalEnergyParams& p, cudaStream_t stream);

void launch_contract_mo_f64(const ContractMoParams& p, int npanel, cudaStream_t stream);
void launch_contract_p_f64(const ContractPParams& p, int npanel, cudaStream_t stream);
void launch_density_values_f64(const ContractPParams& p, cudaStream_t stream);
void launch_orbitals_f64(const OrbitalParams& p, cudaStream_t stream);

}  // namespace kumo_dev
