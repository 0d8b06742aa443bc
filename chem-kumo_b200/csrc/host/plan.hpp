#pragma once
// What a Request needs per density component, and the backend choice:
// the semantics of chem-kumo's src/evaluation_plan.hpp:37-273 and
// src/automatic_backend.hpp:38-50 (same rules, same error messages).
#include "chem/kumo/evaluator.hpp"

#include <algorithm>
#include <array>
#include <stdexcept>
#include <string>

namespace chem::kumo::detail {

struct ComponentNeeds {
    bool density = false, gradient = false, hessian = false, laplacian = false, tau = false;
    bool elf_input = false, reduced_gradient = false, sign_lambda2 = false, lol_input = false;
    bool gradient_expansion_input = false, gradient_input = false, hessian_input = false;
    bool energy_input = false, tau_input = false, value_input = false, electrostatic_potential = false;

    bool derivatives() const {
        return gradient || hessian || laplacian || tau || elf_input || reduced_gradient || sign_lambda2 ||
               lol_input || gradient_input || hessian_input || energy_input || tau_input ||
               gradient_expansion_input || value_input;
    }
    int ao_order() const {
        if (hessian || laplacian || sign_lambda2 || hessian_input || energy_input || gradient_expansion_input) return 2;
        if (gradient || tau || elf_input || reduced_gradient || lol_input || gradient_input || tau_input || value_input)
            return 1;
        return density ? 0 : -1;
    }
};

inline bool is_orbital_kind(PropertyKind k) {
    return k == PropertyKind::Orbital || k == PropertyKind::OrbitalGradient || k == PropertyKind::OrbitalHessian;
}

inline bool is_orbital_energy_kind(PropertyKind k) {
    switch (k) {
        case PropertyKind::AverageLocalIonizationEnergy:
        case PropertyKind::LocalElectronAffinity:
        case PropertyKind::LocalElectronAttachmentEnergy:
        case PropertyKind::LocalElectronegativity:
        case PropertyKind::LocalHardness:
        case PropertyKind::OrbitalWeightedFukuiPlus:
        case PropertyKind::OrbitalWeightedFukuiMinus:
        case PropertyKind::OrbitalWeightedFukuiZero:
        case PropertyKind::OrbitalWeightedDualDescriptor: return true;
        default: return false;
    }
}

// Names of the orbital-energy fields in error messages
// (src/evaluation_plan.hpp:112-130).
inline const char* orbital_energy_name(PropertyKind kind) {
    switch (kind) {
        case PropertyKind::AverageLocalIonizationEnergy: return "the average local ionization energy";
        case PropertyKind::LocalElectronAffinity: return "the local electron affinity";
        case PropertyKind::LocalElectronAttachmentEnergy: return "the local electron attachment energy";
        case PropertyKind::LocalElectronegativity: return "the local electronegativity";
        case PropertyKind::LocalHardness: return "the local hardness";
        case PropertyKind::OrbitalWeightedFukuiPlus: return "the orbital-weighted Fukui function f+";
        case PropertyKind::OrbitalWeightedFukuiMinus: return "the orbital-weighted Fukui function f-";
        case PropertyKind::OrbitalWeightedFukuiZero: return "the orbital-weighted Fukui function f0";
        default: return "the orbital-weighted dual descriptor";
    }
}

struct Plan {
    std::array<ComponentNeeds, 4> c{};
    bool orbitals = false;
    bool orbital_energies = false;
    bool virtual_orbitals = false;        // the virtual-orbital sums are needed too
    bool orbital_weighted_fukui = false;  // the orbital-weighted Fukui sums are needed too
    int max_order = -1;

    static std::size_t idx(DensityComponent d) { return static_cast<std::size_t>(d); }

    static void total_only(const Property& p, const char* what) {
        if (p.component != DensityComponent::Total)
            throw std::invalid_argument(std::string(what) + " is defined only for the total density");
    }

    void spin_inputs(const Property& p, bool ComponentNeeds::*input, const char* what) {
        if (p.component == DensityComponent::Difference)
            throw std::invalid_argument(std::string(what) + " is not defined for the spin-difference density");
        if (p.component == DensityComponent::Total) {
            c[idx(DensityComponent::Alpha)].*input = true;
            c[idx(DensityComponent::Beta)].*input = true;
        } else {
            c[idx(p.component)].*input = true;
        }
    }

    static Plan from(const Request& request) {
        Plan plan;
        for (const Property& p : request.properties()) {
            if (is_orbital_kind(p.kind)) {
                if (p.orbital_index == 0) throw std::invalid_argument("orbital indices are one-based");
                plan.orbitals = true;
                plan.max_order = std::max(plan.max_order, 0);
                continue;
            }
            auto& n = plan.c.at(idx(p.component));
            switch (p.kind) {
                case PropertyKind::Density: n.density = true; break;
                case PropertyKind::Gradient: n.gradient = true; break;
                case PropertyKind::Hessian: n.hessian = true; break;
                case PropertyKind::Laplacian: n.laplacian = true; break;
                case PropertyKind::Tau: n.tau = true; break;
                case PropertyKind::Elf: plan.spin_inputs(p, &ComponentNeeds::elf_input, "ELF"); break;
                case PropertyKind::ReducedGradient:
                    total_only(p, "the reduced density gradient");
                    n.reduced_gradient = true;
                    break;
                case PropertyKind::SignLambda2Density:
                    total_only(p, "sign(lambda2) rho");
                    n.sign_lambda2 = true;
                    break;
                case PropertyKind::ElectrostaticPotential:
                    total_only(p, "the electrostatic potential");
                    n.electrostatic_potential = true;
                    break;
                case PropertyKind::Lol: plan.spin_inputs(p, &ComponentNeeds::lol_input, "LOL"); break;
                case PropertyKind::ElfTsirelsonStash:
                    plan.spin_inputs(p, &ComponentNeeds::gradient_expansion_input, "the Tsirelson-Stash ELF");
                    break;
                case PropertyKind::LolTsirelsonStash:
                    plan.spin_inputs(p, &ComponentNeeds::gradient_expansion_input, "the Tsirelson-Stash LOL");
                    break;
                case PropertyKind::InteractionRegionIndicator:
                    total_only(p, "the interaction region indicator");
                    n.gradient_input = true;
                    break;
                case PropertyKind::ShannonEntropyDensity:
                    total_only(p, "the Shannon entropy density");
                    n.gradient_input = true;
                    break;
                case PropertyKind::FisherInformationDensity:
                    total_only(p, "the Fisher information density");
                    n.gradient_input = true;
                    break;
                case PropertyKind::DensityOverlapRegionsIndicator:
                    total_only(p, "the density overlap regions indicator");
                    n.hessian_input = true;
                    break;
                case PropertyKind::HamiltonianKineticEnergy: n.energy_input = true; break;
                case PropertyKind::PotentialEnergyDensity:
                    total_only(p, "the potential energy density");
                    n.energy_input = true;
                    break;
                case PropertyKind::EnergyDensity:
                    total_only(p, "the energy density");
                    n.energy_input = true;
                    break;
                case PropertyKind::HamiltonianKineticEnergyComponents: n.energy_input = true; break;
                case PropertyKind::TauComponents: n.tau_input = true; break;
                case PropertyKind::PotentialKineticRatio:
                    total_only(p, "|V| / G");
                    n.energy_input = true;
                    break;
                case PropertyKind::EnergyDensityPerElectron:
                    total_only(p, "the energy density per electron");
                    n.energy_input = true;
                    break;
                case PropertyKind::KineticEnergyPerElectron:
                    total_only(p, "the kinetic energy per electron");
                    n.tau_input = true;
                    break;
                case PropertyKind::SpinPolarization:
                    if (p.component != DensityComponent::Difference)
                        throw std::invalid_argument("the spin polarization is defined only for the spin component");
                    plan.c[idx(DensityComponent::Total)].value_input = true;
                    n.value_input = true;
                    break;
                case PropertyKind::AverageLocalIonizationEnergy:
                    total_only(p, orbital_energy_name(p.kind));
                    plan.orbital_energies = true;
                    break;
                case PropertyKind::LocalElectronAffinity:
                case PropertyKind::LocalElectronAttachmentEnergy:
                case PropertyKind::LocalElectronegativity:
                case PropertyKind::LocalHardness:
                    total_only(p, orbital_energy_name(p.kind));
                    plan.orbital_energies = true;
                    plan.virtual_orbitals = true;
                    break;
                case PropertyKind::OrbitalWeightedFukuiPlus:
                case PropertyKind::OrbitalWeightedFukuiMinus:
                case PropertyKind::OrbitalWeightedFukuiZero:
                case PropertyKind::OrbitalWeightedDualDescriptor:
                    total_only(p, orbital_energy_name(p.kind));
                    plan.orbital_energies = true;
                    plan.orbital_weighted_fukui = true;
                    break;
                default:
                    throw std::invalid_argument("unknown property kind");
            }
        }
        for (const auto& n : plan.c) plan.max_order = std::max(plan.max_order, n.ao_order());
        return plan;
    }

    bool needs_esp() const { return c[0].electrostatic_potential; }
};

inline Backend choose_backend(Backend requested, bool eligible, const Plan& plan) {
    if (requested == Backend::AO_P) return Backend::AO_P;
    if (requested == Backend::AO_MO) {
        if (!eligible) throw std::invalid_argument("AO_MO requested for ineligible orbital representation");
        return Backend::AO_MO;
    }
    if (requested != Backend::AUTO) throw std::invalid_argument("unknown evaluation backend");
    if (!eligible) return Backend::AO_P;
    for (const auto& n : plan.c)
        if (n.ao_order() >= 0) return Backend::AO_MO;
    return Backend::AO_P;
}

}  // namespace chem::kumo::detail
