#pragma once
// Host set-up of the orbital-energy fields (internal): the checks of
// src/orbital_energy_fields.hpp:100-196 of chem-kumo, with its messages, and
// the scaled MO columns of each orbital sum laid out for the device kernel
// (every set padded to 128-column chunks, AO-major rows).
#include "chem/kumo/density.hpp"

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <stdexcept>
#include <string>
#include <vector>

namespace chem::kumo::detail {

struct OrbitalEnergyNeeds {
    bool virtuals = false;
    bool fukui = false;
    double fukui_delta = 0.1;
    friend bool operator==(const OrbitalEnergyNeeds&, const OrbitalEnergyNeeds&) = default;
};

/// Sets of the orbital sums, in the order of the device kernel's sums.
enum OrbitalEnergySet { kOccupiedSet = 0, kVirtualSet = 1, kAttachmentSet = 2, kFukuiPlusSet = 3, kFukuiMinusSet = 4 };

struct OrbitalEnergyColumns {
    std::size_t nao = 0;
    std::size_t ldw = 0;              // columns per AO row: chunks x 128
    std::vector<double> w;            // [nao][ldw]
    std::vector<double> energy;       // [ldw], 0 for padding
    std::vector<int> chunk_set;       // set of each 128-column chunk
};

/// Normalized orbital-weighted Fukui weights g_i of the orbitals with the
/// given energies (src/orbital_energy_fields.hpp:77-97): the exponents
/// -((mu - e_i) / delta)^2 are shifted by their largest value before
/// exponentiation.
inline std::vector<double> orbital_weights(const std::vector<double>& energies, double mu, double delta) {
    std::vector<double> ex(energies.size());
    for (std::size_t i = 0; i < energies.size(); ++i) {
        const double x = (mu - energies[i]) / delta;
        ex[i] = -x * x;
    }
    const double top = *std::max_element(ex.begin(), ex.end());
    std::vector<double> g(energies.size());
    double sum = 0.0;
    for (std::size_t i = 0; i < energies.size(); ++i) {
        g[i] = std::exp(ex[i] - top);
        sum += g[i];
    }
    for (double& v : g) v /= sum;
    return g;
}

/// The checks of the OrbitalEnergyFields constructor
/// (src/orbital_energy_fields.hpp:114-143, 192-193, 222-226), in its order and
/// with its messages; `what` names the quantity.
inline void check_orbital_energy_fields(const Molecule& m, const OrbitalEnergyNeeds& needs, const std::string& what) {
    const std::size_t na = m.occupied_count(SpinChannel::Alpha), nb = m.occupied_count(SpinChannel::Beta);
    const bool unrestricted = m.unrestricted();
    if (needs.virtuals && !unrestricted && na != nb)
        throw std::invalid_argument(what + " is not defined for a restricted open-shell calculation");
    if (needs.fukui && (unrestricted || na != nb))
        throw std::invalid_argument(what + " is defined only for a restricted closed-shell calculation");
    if (needs.fukui && (!std::isfinite(needs.fukui_delta) || needs.fukui_delta <= 0.0))
        throw std::invalid_argument(what + ": the Fukui delta must be finite and positive");
    if (!m.electronic_structure_info().ao_mo_eligible())
        throw std::invalid_argument(what +
                                    " needs occupied MOs that reproduce the FCHK density matrices (an SCF calculation)");
    const auto& ea = m.orbital_energies(SpinChannel::Alpha);
    const auto& eb = m.orbital_energies(SpinChannel::Beta);
    const std::size_t ca = m.mo_coefficients(SpinChannel::Alpha).cols();
    const std::size_t cb = unrestricted ? m.mo_coefficients(SpinChannel::Beta).cols() : 0;
    if (ea.size() < ca || (unrestricted && eb.size() < cb) || ea.size() < na || eb.size() < nb)
        throw std::invalid_argument(what + " needs the FCHK orbital energies");
    // Virtual MOs: those above the occupied ones of each channel (restricted:
    // above max(nalpha, nbeta)).
    const std::size_t vir = unrestricted ? (ca > na ? ca - na : 0) + (cb > nb ? cb - nb : 0)
                                         : (ca > std::max(na, nb) ? ca - std::max(na, nb) : 0);
    if (needs.virtuals && vir == 0) throw std::invalid_argument(what + " needs virtual orbitals, and the FCHK has none");
    if (needs.fukui && (na == 0 || na >= ca))
        throw std::invalid_argument(what + " needs occupied and virtual orbitals, and the FCHK lacks one kind");
}

/// The scaled columns of every sum `needs` asks for
/// (src/orbital_energy_fields.hpp:145-196, 219-258): occupied MOs times
/// sqrt(n_i) with energy |e_i|, virtual MOs with e_i, virtual MOs of negative
/// energy times sqrt(w) with e_i (w = 2 restricted, 1 unrestricted), and for
/// the Fukui sums the virtual (f+) and occupied (f-) MOs of the closed shell
/// times sqrt(g_i), leaving out those whose weight underflows to zero.
inline OrbitalEnergyColumns orbital_energy_columns(const Molecule& m, const OrbitalEnergyNeeds& needs,
                                                   const std::string& what) {
    check_orbital_energy_fields(m, needs, what);
    const Matrix& alpha = m.mo_coefficients(SpinChannel::Alpha);
    const std::size_t nao = alpha.rows();
    struct Col {
        const double* c;
        double scale, energy;
    };
    std::vector<Col> sets[5];
    const auto channel = [&](const Matrix& mos, const std::vector<double>& e, std::size_t occupied,
                             std::size_t doubly, double weight) {
        for (std::size_t i = 0; i < mos.cols(); ++i) {
            if (i < occupied) {
                sets[kOccupiedSet].push_back({mos.col(i), std::sqrt(i < doubly ? 2.0 : 1.0), std::abs(e[i])});
            } else if (needs.virtuals) {
                sets[kVirtualSet].push_back({mos.col(i), 1.0, e[i]});
                if (e[i] < 0.0) sets[kAttachmentSet].push_back({mos.col(i), std::sqrt(weight), e[i]});
            }
        }
    };
    const std::size_t na = m.occupied_count(SpinChannel::Alpha), nb = m.occupied_count(SpinChannel::Beta);
    if (m.unrestricted()) {
        channel(alpha, m.orbital_energies(SpinChannel::Alpha), na, 0, 1.0);
        channel(m.mo_coefficients(SpinChannel::Beta), m.orbital_energies(SpinChannel::Beta), nb, 0, 1.0);
    } else {
        channel(alpha, m.orbital_energies(SpinChannel::Alpha), std::max(na, nb), std::min(na, nb), 2.0);
    }
    if (needs.fukui) {
        const auto& e = m.orbital_energies(SpinChannel::Alpha);
        const std::size_t count = alpha.cols(), homo = na;
        const double mu = 0.5 * (e[homo - 1] + e[homo]);
        const auto add = [&](std::size_t first, std::size_t last, std::vector<Col>& out) {
            const std::vector<double> range(e.begin() + static_cast<std::ptrdiff_t>(first),
                                            e.begin() + static_cast<std::ptrdiff_t>(last));
            const auto g = orbital_weights(range, mu, needs.fukui_delta);
            for (std::size_t i = 0; i < range.size(); ++i)
                if (g[i] > 0.0) out.push_back({alpha.col(first + i), std::sqrt(g[i]), 0.0});
        };
        add(homo, count, sets[kFukuiPlusSet]);
        add(0, homo, sets[kFukuiMinusSet]);
    }

    OrbitalEnergyColumns out;
    out.nao = nao;
    std::vector<const Col*> order;
    for (int s = 0; s < 5; ++s) {
        const std::size_t chunks = (sets[s].size() + 127) / 128;
        for (std::size_t c = 0; c < chunks; ++c) out.chunk_set.push_back(s);
        for (std::size_t i = 0; i < chunks * 128; ++i) order.push_back(i < sets[s].size() ? &sets[s][i] : nullptr);
    }
    out.ldw = order.size();
    out.w.assign(nao * out.ldw, 0.0);
    out.energy.assign(out.ldw, 0.0);
    for (std::size_t j = 0; j < order.size(); ++j) {
        if (!order[j]) continue;
        out.energy[j] = order[j]->energy;
        for (std::size_t a = 0; a < nao; ++a) out.w[a * out.ldw + j] = order[j]->scale * order[j]->c[a];
    }
    return out;
}

}  // namespace chem::kumo::detail
