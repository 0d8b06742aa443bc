#pragma once
// Kernel timing and algorithmic counters of the evaluation waves (internal).
// When enabled, each launch of a profiled kernel is bracketed by CUDA events
// on its stream, and the kept AO rows of every screening block are summed on
// the device; nothing is synchronized until the statistics are read.
#include <cuda_runtime.h>

#include <string>

namespace chem::kumo::detail {

enum ProfileKernel : int { kProfAoBuild = 0, kProfContractMo, kProfContractMixed, kProfContractP,
                           kProfDensityValues, kProfOrbitals, kProfEsp, kProfCount };

bool profiling_enabled();
void profile_enable(bool on);
void profile_reset();
// Returns an event pair index or -1 when profiling is off.
int profile_begin(ProfileKernel k, cudaStream_t s);
void profile_end(int token, cudaStream_t s);
// Adds sum(nkept[0..n)) to the kept-rows counter of kernel k, and `units`
// (blocks, points or point-pair interactions) and `flops` to its counters.
void profile_count(ProfileKernel k, const int* nkept, int n, double flops_per_kept_row, double units,
                   double flops, double bytes, cudaStream_t s);
// Adds sum(nkept[0..n)) to the kept-rows counter of kernel k and
// flops_per_row_sq * sum(nkept^2) to its FLOPs (products with a kept x kept
// block of a matrix).
void profile_count_sq(ProfileKernel k, const int* nkept, int n, double flops_per_row_sq, cudaStream_t s);

struct ProfileStats {
    int launches;
    double ms;
    double kept_rows;
    double units;
    double flops;
    double bytes;
};
// Synchronizes the recorded events and returns the totals of kernel k.
ProfileStats profile_read(ProfileKernel k);
const char* profile_name(ProfileKernel k);

}  // namespace chem::kumo::detail
