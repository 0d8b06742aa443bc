#pragma once
// Device-resident copy of a molecule (internal).
#include "chem/kumo/density.hpp"

#include <cuda_runtime.h>

#include <cstddef>
#include <memory>
#include <mutex>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "orbital_energy.hpp"
#include "../cuda/ao_mixed.cuh"
#include "../cuda/kumo_device.cuh"

namespace kumo_dev {
class EspDevice;
}

namespace chem::kumo::detail {

[[noreturn]] void throw_cuda(cudaError_t e, const char* what);
inline void check_cuda(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw_cuda(e, what);
}

/// AO tables, density matrices and MO coefficients of one molecule in HBM.
struct DeviceMolecule {
    int device = -1;
    kumo_dev::DevBasis basis;
    double pure_d[3][135] = {};
    float pure_f[3][135] = {};
    // Mixed-form AO build: per primitive a log2(e), a and the radial factor u
    // (weights = u_p g_k), T[m][k] g_k for pure blocks, g_k for Cartesian ones.
    kumo_dev::MixPrim* mix_prims = nullptr;
    float tpure_g[3][135] = {};
    float gcart[5][15] = {};
    double* p_total = nullptr;  // n x n
    double* p_spin = nullptr;
    // Occupied MOs transposed [AO][MO], rows padded to a multiple of 4.
    double* ct_alpha = nullptr;
    int ldc_alpha = 0, nocc_alpha = 0;
    double* ct_beta = nullptr;
    int ldc_beta = 0, nocc_beta = 0;
    // Occupied MOs of the mixed form as three BF16 pieces (c = c0 + c1 + c2,
    // each the BF16 rounding of what the previous pieces leave), stored
    // [piece][AO][MO] with rows of ldn MOs (a multiple of 16, zero padded).
    // P_total and P_spin for the mixed AO-P form: each element as its three
    // BF16 pieces and a zero, [row][col][4] (one 8-byte load per element).
    // Built on first use by ensure_p_pieces (the AO-MO form never reads them,
    // and splitting a large P costs the host far more than a launch).
    std::uint16_t* p_total_s = nullptr;
    std::uint16_t* p_spin_s = nullptr;
    void ensure_p_pieces(const Molecule& m);
    std::uint16_t* cs_alpha = nullptr;
    std::uint16_t* cs_beta = nullptr;
    int ldn_alpha = 0, ldn_beta = 0;
    // All MO coefficients, one MO per column (n x nmo), for amplitudes.
    double* c_alpha = nullptr;
    int nmo_alpha = 0;
    double* c_beta = nullptr;
    int nmo_beta = 0;
    bool unrestricted = false;
    std::size_t bytes = 0;
    std::vector<void*> allocations;
    // Primitive pairs of the electrostatic potential, built on first use and
    // kept with the molecule (their host set-up costs far more than a launch).
    std::unique_ptr<kumo_dev::EspDevice> esp;
    std::mutex esp_mutex;  // guards every state built on first use
    kumo_dev::EspDevice& esp_state(const Molecule& m, cudaStream_t stream);
    // Scaled MO columns of the orbital-energy sums, one entry per set of
    // needs met so far, built on first use and kept with the molecule.
    struct OrbitalEnergyDevice {
        OrbitalEnergyNeeds needs;
        double* w = nullptr;  // [nao][ldw]
        int ldw = 0;
        int nchunks = 0;
        int* chunk_set = nullptr;
        double* energy = nullptr;
    };
    std::vector<std::unique_ptr<OrbitalEnergyDevice>> orbital_energy;
    const OrbitalEnergyDevice& orbital_energy_state(const Molecule& m, const OrbitalEnergyNeeds& needs,
                                                    const std::string& what);

    explicit DeviceMolecule(const Molecule& m);
    ~DeviceMolecule();
    DeviceMolecule(const DeviceMolecule&) = delete;
    DeviceMolecule& operator=(const DeviceMolecule&) = delete;

    template <typename T>
    T* upload(const T* host, std::size_t count);
};

}  // namespace chem::kumo::detail
