#pragma once
#include "chem/kumo/basis.hpp"
#include "chem/kumo/density.hpp"
#include "chem/kumo/evaluator.hpp"
#include "chem/kumo/fchk.hpp"
#include "chem/kumo/spin.hpp"
#include "chem/kumo/types.hpp"
