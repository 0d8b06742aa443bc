// Kernel timing and algorithmic counters; see profile.hpp.
#include "profile.hpp"

#include <atomic>
#include <mutex>
#include <vector>

#include "device_state.hpp"

namespace chem::kumo::detail {
namespace {

struct Record {
    int kernel;
    cudaEvent_t start, stop;
};

struct State {
    std::mutex mu;
    std::atomic<bool> on{false};
    std::vector<Record> records;
    double flops[kProfCount] = {};
    double units[kProfCount] = {};
    double bytes[kProfCount] = {};
    // Device counters: kept rows (double) and the FLOPs they imply.
    double* d_counters = nullptr;  // [kProfCount][2]
};

State& state() {
    static State s;
    return s;
}

// counters[0] += sum nkept; counters[1] += sum (flops_per_row nkept +
// flops_per_row_sq nkept^2).
__global__ void sum_kept(const int* nkept, int n, double flops_per_row, double flops_per_row_sq, double* counters) {
    __shared__ double s[256], s2[256];
    double v = 0, v2 = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double k = nkept[i];
        v += k;
        v2 += k * k;
    }
    s[threadIdx.x] = v;
    s2[threadIdx.x] = v2;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            s[threadIdx.x] += s[threadIdx.x + o];
            s2[threadIdx.x] += s2[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        counters[0] += s[0];
        counters[1] += s[0] * flops_per_row + s2[0] * flops_per_row_sq;
    }
}

}  // namespace

bool profiling_enabled() { return state().on.load(); }

void profile_enable(bool on) {
    State& s = state();
    std::lock_guard<std::mutex> l(s.mu);
    if (on && !s.d_counters) {
        check_cuda(cudaMalloc(&s.d_counters, sizeof(double) * 2 * kProfCount), "cudaMalloc (profile)");
        check_cuda(cudaMemset(s.d_counters, 0, sizeof(double) * 2 * kProfCount), "cudaMemset (profile)");
    }
    s.on = on;
}

void profile_reset() {
    State& s = state();
    std::lock_guard<std::mutex> l(s.mu);
    for (auto& r : s.records) {
        cudaEventSynchronize(r.stop);
        cudaEventDestroy(r.start);
        cudaEventDestroy(r.stop);
    }
    s.records.clear();
    for (int k = 0; k < kProfCount; ++k) s.flops[k] = s.units[k] = s.bytes[k] = 0;
    if (s.d_counters) {
        cudaDeviceSynchronize();
        cudaMemset(s.d_counters, 0, sizeof(double) * 2 * kProfCount);
    }
}

int profile_begin(ProfileKernel k, cudaStream_t st) {
    State& s = state();
    if (!s.on) return -1;
    std::lock_guard<std::mutex> l(s.mu);
    Record r{k, nullptr, nullptr};
    check_cuda(cudaEventCreate(&r.start), "cudaEventCreate");
    check_cuda(cudaEventCreate(&r.stop), "cudaEventCreate");
    check_cuda(cudaEventRecord(r.start, st), "cudaEventRecord");
    s.records.push_back(r);
    return static_cast<int>(s.records.size()) - 1;
}

void profile_end(int token, cudaStream_t st) {
    if (token < 0) return;
    State& s = state();
    std::lock_guard<std::mutex> l(s.mu);
    check_cuda(cudaEventRecord(s.records[static_cast<std::size_t>(token)].stop, st), "cudaEventRecord");
}

void profile_count(ProfileKernel k, const int* nkept, int n, double flops_per_row, double units, double flops,
                   double bytes, cudaStream_t st) {
    State& s = state();
    if (!s.on) return;
    std::lock_guard<std::mutex> l(s.mu);
    s.units[k] += units;
    s.flops[k] += flops;
    s.bytes[k] += bytes;
    if (nkept && n > 0) sum_kept<<<1, 256, 0, st>>>(nkept, n, flops_per_row, 0.0, s.d_counters + 2 * k);
}
void profile_count_sq(ProfileKernel k, const int* nkept, int n, double flops_per_row_sq, cudaStream_t st) {
    State& s = state();
    if (!s.on) return;
    std::lock_guard<std::mutex> l(s.mu);
    if (nkept && n > 0) sum_kept<<<1, 256, 0, st>>>(nkept, n, 0.0, flops_per_row_sq, s.d_counters + 2 * k);
}

ProfileStats profile_read(ProfileKernel k) {
    State& s = state();
    std::lock_guard<std::mutex> l(s.mu);
    ProfileStats out{0, 0.0, 0.0, s.units[k], s.flops[k], s.bytes[k]};
    for (auto& r : s.records) {
        if (r.kernel != k) continue;
        check_cuda(cudaEventSynchronize(r.stop), "cudaEventSynchronize (profile)");
        float ms = 0.f;
        check_cuda(cudaEventElapsedTime(&ms, r.start, r.stop), "cudaEventElapsedTime");
        out.ms += ms;
        ++out.launches;
    }
    if (s.d_counters) {
        double c[2];
        check_cuda(cudaMemcpy(c, s.d_counters + 2 * k, sizeof c, cudaMemcpyDeviceToHost), "cudaMemcpy (profile)");
        out.kept_rows = c[0];
        out.flops += c[1];
    }
    return out;
}

const char* profile_name(ProfileKernel k) {
    static const char* names[kProfCount] = {"ao_build", "contract_mo_f64", "contract_mixed", "contract_p",
                                            "density_values_f64", "orbitals_f64", "esp_f64"};
    return names[k];
}

}  // namespace chem::kumo::detail
