#pragma once

namespace chem::kumo {

/// Component of the electron density (include/chem/kumo/spin.hpp of
/// chem-kumo): total, alpha, beta or the spin difference alpha - beta.
enum class DensityComponent { Total, Alpha, Beta, Difference };

/// Spin channel of a molecular orbital.  A restricted calculation has one set
/// of spatial MOs, used for both channels.
enum class SpinChannel { Alpha, Beta };

}  // namespace chem::kumo
