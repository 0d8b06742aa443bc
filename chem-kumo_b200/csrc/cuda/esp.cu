// Electrostatic potential: host setup of the primitive pairs and the FP64
// device kernel; see esp.cuh.
#include "esp.cuh"
#include "func_attr.cuh"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <exception>
#include <numbers>
#include <stdexcept>
#include <string>
#include <thread>
#include <type_traits>

#include "../host/device_state.hpp"
#include "chem/kumo/density.hpp"

namespace kumo_dev {
namespace {

constexpr int hermite_count(int s) { return (s + 1) * (s + 2) * (s + 3) / 6; }

struct Triple {
    int t, u, v;
};

std::vector<Triple> hermite_triples(int L) {
    std::vector<Triple> out;
    for (int sum = 0; sum <= L; ++sum)
        for (int t = sum; t >= 0; --t)
            for (int u = sum - t; u >= 0; --u) out.push_back({t, u, sum - t - u});
    return out;
}

// Hermite expansion E^{ij}_t of (x-A)^i (x-B)^j exp(-a (x-A)^2 - b (x-B)^2)
// without the Gaussian prefactor, by the recursions
// E^{i+1,j}_t = E^{ij}_{t-1}/(2p) + X_PA E^{ij}_t + (t+1) E^{ij}_{t+1} and the
// same in j with X_PB, stored [(i*(lb+1)+j)*(la+lb+1)+t].
class Hermite1D {
public:
    Hermite1D(int la, int lb, double p, double pa, double pb)
        : lb_(lb), width_(la + lb + 1), v_(static_cast<std::size_t>((la + 1) * (lb + 1) * (la + lb + 1)), 0.0) {
        const double h = 0.5 / p;
        set(0, 0, 0, 1.0);
        auto step = [&](int si, int sj, int ti, int tj, double shift) {
            for (int t = 0; t <= ti + tj; ++t) {
                double value = shift * get(si, sj, t);
                if (t > 0) value += h * get(si, sj, t - 1);
                if (t + 1 <= si + sj) value += (t + 1) * get(si, sj, t + 1);
                set(ti, tj, t, value);
            }
        };
        for (int i = 0; i < la; ++i) step(i, 0, i + 1, 0, pa);
        for (int i = 0; i <= la; ++i)
            for (int j = 0; j < lb; ++j) step(i, j, i, j + 1, pb);
    }
    double get(int i, int j, int t) const {
        if (t < 0 || t > i + j) return 0.0;
        return v_[static_cast<std::size_t>((i * (lb_ + 1) + j) * width_ + t)];
    }

private:
    void set(int i, int j, int t, double x) { v_[static_cast<std::size_t>((i * (lb_ + 1) + j) * width_ + t)] = x; }
    int lb_, width_;
    std::vector<double> v_;
};

}  // namespace

std::vector<double> boys_table_host() {
    std::vector<double> table(static_cast<std::size_t>(kBoysPoints * kBoysOrders));
    const int top = kBoysOrders - 1;
    for (int i = 0; i < kBoysPoints; ++i) {
        const double T = i * 0.05;
        const double decay = std::exp(-T);
        double term = 1.0 / (2.0 * top + 1.0);
        double sum = term;
        for (int k = 1; k < 10000 && term > 1e-18 * sum; ++k) {
            term *= 2.0 * T / (2.0 * top + 2.0 * k + 1.0);
            sum += term;
        }
        double* row = table.data() + static_cast<std::size_t>(i * kBoysOrders);
        row[top] = decay * sum;
        for (int m = top; m > 0; --m) row[m - 1] = (2.0 * T * row[m] + decay) / (2.0 * m - 1.0);
    }
    return table;
}

void boys_host(const double* table, double T, int n, double* out) {
    const int top = n - 1;
    const double decay = std::exp(-T);
    if (T >= 40.0) {
        out[0] = 0.5 * std::sqrt(std::numbers::pi / T);
        for (int m = 0; m < top; ++m) out[m + 1] = ((2.0 * m + 1.0) * out[m] - decay) / (2.0 * T);
        return;
    }
    const int point = static_cast<int>(std::lround(T / 0.05));
    const double delta = T - point * 0.05;
    const double* row = table + static_cast<std::size_t>(point * kBoysOrders);
    double sum = 0.0, factor = 1.0;
    for (int k = 0; k < kBoysTaylor; ++k) {
        sum += row[top + k] * factor;
        factor *= -delta / (k + 1.0);
    }
    out[top] = sum;
    for (int m = top; m > 0; --m) out[m - 1] = (2.0 * T * out[m] + decay) / (2.0 * m - 1.0);
}

double hermite_sup(int t, int u, int v) {
    const int n = t + u + v;
    const double pi = std::numbers::pi;
    return std::sqrt(pi) / (4.0 * pi * pi) * std::ldexp(1.0, n) * std::tgamma(0.5 * (n + 1)) * 2.0 *
           std::tgamma(0.5 * (t + 1)) * std::tgamma(0.5 * (u + 1)) * std::tgamma(0.5 * (v + 1)) /
           std::tgamma(0.5 * (n + 3));
}

EspDevice::EspDevice(const chem::kumo::Molecule& m, cudaStream_t stream) {
    using chem::kumo::detail::check_cuda;
    const auto& blocks = m.blocks();
    for (const auto& b : blocks)
        if (2 * b.angular_momentum > kEspMaxL)
            throw std::invalid_argument("the B200 electrostatic potential supports shells up to l = 4");
    const chem::kumo::Matrix P = m.density_matrix(chem::kumo::DensityComponent::Total);
    std::vector<chem::kumo::Matrix> transforms(kMaxL + 1);
    for (int l = 2; l <= kMaxL; ++l) transforms[static_cast<std::size_t>(l)] = chem::kumo::gaussian_cartesian_to_pure(l);
    // The pairs of each first block a are built independently (host threads
    // take blocks a from a shared counter) and joined in the order of a, so
    // the pair list is the same as one thread's.
    struct Part {
        std::vector<EspPair> pairs;
        std::vector<double> coef;
    };
    std::vector<Part> parts(blocks.size());
    auto build_a = [&](std::size_t a, std::vector<double>& cart, std::vector<double>& left, std::vector<double>& pc) {
        std::vector<EspPair>& pairs = parts[a].pairs;
        std::vector<double>& coef = parts[a].coef;
        const auto& A = blocks[a];
        for (std::size_t bb = a; bb < blocks.size(); ++bb) {
            const auto& B = blocks[bb];
            const std::size_t na = A.powers.size(), nb = B.powers.size();
            const std::size_t ra = A.count, rb = B.count;
            // Cartesian block TA^T P(A, B) TB, doubled off the diagonal.
            left.assign(na * rb, 0.0);
            for (std::size_t k = 0; k < na; ++k)
                for (std::size_t j = 0; j < rb; ++j) {
                    double s = 0.0;
                    if (A.pure) {
                        const auto& T = transforms[static_cast<std::size_t>(A.angular_momentum)];
                        for (std::size_t i = 0; i < ra; ++i) s += T(i, k) * P(A.offset + i, B.offset + j);
                    } else {
                        s = P(A.offset + k, B.offset + j);
                    }
                    left[k * rb + j] = s;
                }
            cart.assign(na * nb, 0.0);
            for (std::size_t i = 0; i < na; ++i)
                for (std::size_t k = 0; k < nb; ++k) {
                    double s = 0.0;
                    if (B.pure) {
                        const auto& T = transforms[static_cast<std::size_t>(B.angular_momentum)];
                        for (std::size_t j = 0; j < rb; ++j) s += left[i * rb + j] * T(j, k);
                    } else {
                        s = left[i * rb + k];
                    }
                    cart[i * nb + k] = a != bb ? s * 2.0 : s;
                }
            if (std::all_of(cart.begin(), cart.end(), [](double x) { return x == 0.0; })) continue;
            const int la = A.angular_momentum, lb = B.angular_momentum, L = la + lb;
            const auto list = hermite_triples(L);
            double ab2 = 0.0;
            {
                const double dx = A.origin[0] - B.origin[0], dy = A.origin[1] - B.origin[1],
                             dz = A.origin[2] - B.origin[2];
                ab2 = dx * dx + dy * dy + dz * dz;
            }
            const std::size_t npa = A.exponents.size(), npb = B.exponents.size();
            for (std::size_t p = 0; p < npa; ++p)
                for (std::size_t q = 0; q < npb; ++q) {
                    const double alpha = A.exponents[p], beta = B.exponents[q];
                    const double ex = alpha + beta;
                    double c3[3];
                    for (int k = 0; k < 3; ++k) c3[k] = (alpha * A.origin[k] + beta * B.origin[k]) / ex;
                    const double scale = std::exp(-alpha * beta / ex * ab2) * 2.0 * std::numbers::pi / ex;
                    const Hermite1D hx(la, lb, ex, c3[0] - A.origin[0], c3[0] - B.origin[0]);
                    const Hermite1D hy(la, lb, ex, c3[1] - A.origin[1], c3[1] - B.origin[1]);
                    const Hermite1D hz(la, lb, ex, c3[2] - A.origin[2], c3[2] - B.origin[2]);
                    pc.assign(list.size(), 0.0);
                    for (std::size_t i = 0; i < na; ++i) {
                        const auto& pi = A.powers[i];
                        for (std::size_t j = 0; j < nb; ++j) {
                            const auto& pj = B.powers[j];
                            const double w = cart[i * nb + j] * A.weights[i * npa + p] * B.weights[j * npb + q];
                            if (w == 0.0) continue;
                            for (std::size_t k = 0; k < list.size(); ++k) {
                                const Triple& h = list[k];
                                if (h.t > pi.x + pj.x || h.u > pi.y + pj.y || h.v > pi.z + pj.z) continue;
                                pc[k] += w * hx.get(pi.x, pj.x, h.t) * hy.get(pi.y, pj.y, h.u) * hz.get(pi.z, pj.z, h.v);
                            }
                        }
                    }
                    if (std::all_of(pc.begin(), pc.end(), [](double x) { return x == 0.0; })) continue;
                    pairs.push_back({ex, c3[0], c3[1], c3[2], L, static_cast<int>(coef.size())});
                    for (double x : pc) coef.push_back(scale * x);
                }
        }
    };
    {
        const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
        const std::size_t nthreads = blocks.size() < 64 ? 1 : std::min<std::size_t>(hw, 32);
        std::atomic<std::size_t> next{0};
        std::vector<std::exception_ptr> errors(nthreads);
        auto worker = [&](std::size_t t) {
            try {
                std::vector<double> cart, left, pc;
                for (std::size_t a = next++; a < blocks.size(); a = next++) build_a(a, cart, left, pc);
            } catch (...) {
                errors[t] = std::current_exception();
                next = blocks.size();
            }
        };
        std::vector<std::thread> pool;
        for (std::size_t t = 1; t < nthreads; ++t) pool.emplace_back(worker, t);
        worker(0);
        for (auto& th : pool) th.join();
        for (const auto& e : errors)
            if (e) std::rethrow_exception(e);
    }
    std::vector<EspPair> pairs;
    std::vector<double> coef;
    for (auto& part : parts) {
        const int base = static_cast<int>(coef.size());
        for (EspPair pr : part.pairs) {
            pr.first += base;
            pairs.push_back(pr);
        }
        coef.insert(coef.end(), part.coef.begin(), part.coef.end());
        part = Part{};
    }
    // Pairs grouped by order (stable), so that each launch of the device
    // kernel handles one order with its recursion unrolled.
    std::stable_sort(pairs.begin(), pairs.end(), [](const EspPair& x, const EspPair& y) { return x.order < y.order; });
    // Coefficients in pair order, so that a run of pairs has one contiguous
    // run of coefficients (the kernel stages them in batches).
    {
        std::vector<double> ordered;
        ordered.reserve(coef.size());
        for (auto& pr : pairs) {
            const int nt = hermite_count(pr.order);
            const std::size_t f = static_cast<std::size_t>(pr.first);
            pr.first = static_cast<int>(ordered.size());
            ordered.insert(ordered.end(), coef.begin() + static_cast<std::ptrdiff_t>(f),
                           coef.begin() + static_cast<std::ptrdiff_t>(f + nt));
        }
        coef.swap(ordered);
    }
    // Bound of each pair's contribution at any point: sum_k |c_k| p^(n_k/2)
    // hermite_sup(alpha_k), the triples of order L being a prefix of those
    // of order kEspMaxL.
    {
        const auto triples = hermite_triples(kEspMaxL);
        std::vector<double> sup(triples.size());
        std::vector<int> degree(triples.size());
        for (std::size_t k = 0; k < triples.size(); ++k) {
            sup[k] = hermite_sup(triples[k].t, triples[k].u, triples[k].v);
            degree[k] = triples[k].t + triples[k].u + triples[k].v;
        }
        bound_.resize(pairs.size());
        for (std::size_t i = 0; i < pairs.size(); ++i) {
            const EspPair& pr = pairs[i];
            const double sp = std::sqrt(pr.p);
            double b = 0.0;
            for (int k = 0; k < hermite_count(pr.order); ++k)
                b += std::abs(coef[static_cast<std::size_t>(pr.first + k)]) * std::pow(sp, degree[k]) * sup[k];
            bound_[i] = b;
        }
    }
    for (int L = 0; L <= kEspMaxL + 1; ++L)
        view_.order_first[L] = std::lower_bound(pairs.begin(), pairs.end(), L,
                                                [](const EspPair& x, int v) { return x.order < v; }) -
                               pairs.begin();
    // Recursion table of the Hermite triples up to kEspMaxL.
    const auto all = hermite_triples(kEspMaxL);
    auto index_of = [&](int t, int u, int v) {
        for (std::size_t k = 0; k < all.size(); ++k)
            if (all[k].t == t && all[k].u == u && all[k].v == v) return static_cast<int>(k);
        return -1;
    };
    std::vector<int4> rec(all.size());
    for (std::size_t k = 0; k < all.size(); ++k) {
        const Triple& h = all[k];
        if (h.t > 0)
            rec[k] = make_int4(0, index_of(h.t - 1, h.u, h.v), h.t > 1 ? index_of(h.t - 2, h.u, h.v) : -1, h.t - 1);
        else if (h.u > 0)
            rec[k] = make_int4(1, index_of(h.t, h.u - 1, h.v), h.u > 1 ? index_of(h.t, h.u - 2, h.v) : -1, h.u - 1);
        else if (h.v > 0)
            rec[k] = make_int4(2, index_of(h.t, h.u, h.v - 1), h.v > 1 ? index_of(h.t, h.u, h.v - 2) : -1, h.v - 1);
        else
            rec[k] = make_int4(-1, -1, -1, 0);
    }
    std::vector<double4> atoms;
    for (const auto& at : m.atoms())
        atoms.push_back(make_double4(at.position[0], at.position[1], at.position[2], at.nuclear_charge));
    const auto table = boys_table_host();
    auto up = [&](const void* src, std::size_t bytes) {
        void* d = nullptr;
        check_cuda(cudaMalloc(&d, std::max<std::size_t>(bytes, 16)), "cudaMalloc (potential)");
        allocs_.push_back(d);
        bytes_ += std::max<std::size_t>(bytes, 16);
        if (bytes) check_cuda(cudaMemcpyAsync(d, src, bytes, cudaMemcpyHostToDevice, stream), "cudaMemcpyAsync (potential)");
        return d;
    };
    view_.pairs = static_cast<const EspPair*>(up(pairs.data(), sizeof(EspPair) * pairs.size()));
    view_.coef = static_cast<const double*>(up(coef.data(), sizeof(double) * coef.size()));
    view_.npairs = static_cast<long long>(pairs.size());
    view_.boys_table = static_cast<const double*>(up(table.data(), sizeof(double) * table.size()));
    view_.atoms = static_cast<const double4*>(up(atoms.data(), sizeof(double4) * atoms.size()));
    view_.natoms = static_cast<int>(atoms.size());
    view_.recursion = static_cast<const int4*>(up(rec.data(), sizeof(int4) * rec.size()));
    check_cuda(cudaStreamSynchronize(stream), "cudaStreamSynchronize (potential setup)");
    pairs_ = std::move(pairs);
    coef_ = std::move(coef);
}

EspView EspDevice::view_for(double tolerance, cudaStream_t stream) {
    using chem::kumo::detail::check_cuda;
    if (!(tolerance > 0.0) || pairs_.empty()) return view_;
    std::lock_guard<std::mutex> lock(views_mutex_);
    const auto found = views_.find(tolerance);
    if (found != views_.end()) return found->second;
    // Drop the pairs of smallest bound while the dropped bounds sum to at most
    // half the tolerance (the other half is left to rounding).
    std::vector<std::size_t> order(pairs_.size());
    for (std::size_t i = 0; i < order.size(); ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](std::size_t a, std::size_t b) { return bound_[a] < bound_[b]; });
    std::vector<char> drop(pairs_.size(), 0);
    double dropped = 0.0;
    const double budget = 0.5 * tolerance;
    for (const std::size_t i : order) {
        if (dropped + bound_[i] > budget) break;
        dropped += bound_[i];
        drop[i] = 1;
    }
    std::vector<EspPair> kept;
    std::vector<double> coef;
    for (std::size_t i = 0; i < pairs_.size(); ++i) {
        if (drop[i]) continue;
        EspPair pr = pairs_[i];
        const int nt = hermite_count(pr.order);
        coef.insert(coef.end(), coef_.begin() + pr.first, coef_.begin() + pr.first + nt);
        pr.first = static_cast<int>(coef.size()) - nt;
        kept.push_back(pr);
    }
    EspView v = view_;
    if (kept.size() != pairs_.size()) {
        auto up = [&](const void* src, std::size_t bytes) {
            void* d = nullptr;
            check_cuda(cudaMalloc(&d, std::max<std::size_t>(bytes, 16)), "cudaMalloc (potential)");
            allocs_.push_back(d);
            bytes_ += std::max<std::size_t>(bytes, 16);
            if (bytes)
                check_cuda(cudaMemcpyAsync(d, src, bytes, cudaMemcpyHostToDevice, stream), "cudaMemcpyAsync (potential)");
            return d;
        };
        v.pairs = static_cast<const EspPair*>(up(kept.data(), sizeof(EspPair) * kept.size()));
        v.coef = static_cast<const double*>(up(coef.data(), sizeof(double) * coef.size()));
        v.npairs = static_cast<long long>(kept.size());
        for (int L = 0; L <= kEspMaxL + 1; ++L)
            v.order_first[L] = std::lower_bound(kept.begin(), kept.end(), L,
                                                [](const EspPair& x, int o) { return x.order < o; }) -
                               kept.begin();
        check_cuda(cudaStreamSynchronize(stream), "cudaStreamSynchronize (potential screening)");
    }
    views_.emplace(tolerance, v);
    return v;
}

EspDevice::~EspDevice() {
    for (void* p : allocs_) cudaFree(p);
}

__device__ __forceinline__ void boys_device(const double* table, double T, int n, double* out) {
    const int top = n - 1;
    const double decay = exp(-T);
    if (T >= 40.0) {
        out[0] = 0.5 * sqrt(3.141592653589793 / T);
        for (int m = 0; m < top; ++m) out[m + 1] = ((2.0 * m + 1.0) * out[m] - decay) / (2.0 * T);
        return;
    }
    const int point = static_cast<int>(llround(T / 0.05));
    const double delta = T - point * 0.05;
    const double* row = table + point * kBoysOrders;
    double sum = 0.0, factor = 1.0;
#pragma unroll
    for (int k = 0; k < kBoysTaylor; ++k) {
        sum += row[top + k] * factor;
        factor *= -delta / (k + 1.0);
    }
    out[top] = sum;
    for (int m = top; m > 0; --m) out[m - 1] = (2.0 * T * out[m] + decay) / (2.0 * m - 1.0);
}

// Compile-time form of the recursion table (same ordering and steps as the
// host table uploaded in EspView::recursion).
struct HermiteTable {
    int axis[hermite_count(kEspMaxL)];
    int one[hermite_count(kEspMaxL)];
    int two[hermite_count(kEspMaxL)];
    int factor[hermite_count(kEspMaxL)];
};

constexpr HermiteTable make_hermite_table() {
    HermiteTable h{};
    int tt[hermite_count(kEspMaxL)] = {}, uu[hermite_count(kEspMaxL)] = {}, vv[hermite_count(kEspMaxL)] = {};
    int n = 0;
    for (int sum = 0; sum <= kEspMaxL; ++sum)
        for (int t = sum; t >= 0; --t)
            for (int u = sum - t; u >= 0; --u) {
                tt[n] = t;
                uu[n] = u;
                vv[n] = sum - t - u;
                ++n;
            }
    auto index_of = [&](int t, int u, int v) {
        for (int k = 0; k < n; ++k)
            if (tt[k] == t && uu[k] == u && vv[k] == v) return k;
        return -1;
    };
    for (int k = 0; k < n; ++k) {
        const int t = tt[k], u = uu[k], v = vv[k];
        h.axis[k] = -1;
        h.one[k] = -1;
        h.two[k] = -1;
        h.factor[k] = 0;
        if (t > 0) {
            h.axis[k] = 0;
            h.one[k] = index_of(t - 1, u, v);
            h.two[k] = t > 1 ? index_of(t - 2, u, v) : -1;
            h.factor[k] = t - 1;
        } else if (u > 0) {
            h.axis[k] = 1;
            h.one[k] = index_of(t, u - 1, v);
            h.two[k] = u > 1 ? index_of(t, u - 2, v) : -1;
            h.factor[k] = u - 1;
        } else if (v > 0) {
            h.axis[k] = 2;
            h.one[k] = index_of(t, u, v - 1);
            h.two[k] = v > 1 ? index_of(t, u, v - 2) : -1;
            h.factor[k] = v - 1;
        }
    }
    return h;
}

constexpr HermiteTable kHermite = make_hermite_table();

// F_0..F_TOP(T) as boys_device, with exp(-T) only where a recursion needs it.
template <int TOP>
__device__ __forceinline__ void boys_top(const double* table, double T, double (&out)[TOP + 1]) {
    if (T >= 40.0) {
        out[0] = 0.5 * sqrt(3.141592653589793 / T);
        if constexpr (TOP > 0) {
            const double decay = exp(-T);
#pragma unroll
            for (int m = 0; m < TOP; ++m) out[m + 1] = ((2.0 * m + 1.0) * out[m] - decay) / (2.0 * T);
        }
        return;
    }
    const int point = static_cast<int>(llround(T / 0.05));
    const double delta = T - point * 0.05;
    const double* row = table + point * kBoysOrders;
    double sum = 0.0, factor = 1.0;
#pragma unroll
    for (int k = 0; k < kBoysTaylor; ++k) {
        sum += row[TOP + k] * factor;
        factor *= -delta / (k + 1.0);
    }
    out[TOP] = sum;
    if constexpr (TOP > 0) {
        const double decay = exp(-T);
#pragma unroll
        for (int m = TOP; m > 0; --m) out[m - 1] = (2.0 * T * out[m] + decay) / (2.0 * m - 1.0);
    }
}

// One level of the Hermite recursion: R^(n) from R^(n+1) in place, entries
// K = NT-1 down to 1 of the first `live` (each entry reads lower-index entries
// of the level above, which a descending sweep has not overwritten yet).
// R is double in the FP64 form and float in the mixed one.
template <int K, int NT, typename R_t>
__device__ __forceinline__ void hermite_level(R_t (&R)[NT], int live, R_t pcx, R_t pcy, R_t pcz) {
    if constexpr (K >= 1) {
        if (K < live) {
            constexpr int ax = kHermite.axis[K];
            constexpr int one = kHermite.one[K];
            constexpr int two = kHermite.two[K];
            constexpr R_t f = static_cast<R_t>(kHermite.factor[K]);
            const R_t X = ax == 0 ? pcx : (ax == 1 ? pcy : pcz);
            R_t v = X * R[one];
            if constexpr (two >= 0) v += f * R[two];
            R[K] = v;
        }
        hermite_level<K - 1, NT>(R, live, pcx, pcy, pcz);
    }
}

// Pairs of order L: thread = point of a 128-point tile, blockIdx.y = chunk of
// the order's pairs; the partial sum of the chunk goes to
// part[(slot0 + chunk) * ld + point].  The chunk's pairs and their
// coefficients (contiguous, in pair order) are staged in shared memory in
// batches by the whole CTA with coalesced loads, so the per-pair loop reads
// them with broadcast shared loads instead of dependent global ones.
//
// MIXED = false: FP64 throughout (src/electrostatic_potential.cpp:231-348).
// MIXED = true: the Boys values F_0..F_L(T), their (-2p)^n scaling and the
// point-to-centre vector stay FP64; the Hermite recursion, the dot with the
// coefficients and the sum over the chunk's pairs are FP32, the sum
// compensated (Kahan) so that its rounding does not grow with the chunk's
// length.  The nuclear term and the subtraction of the partial sums stay
// FP64 (esp_reduce_kernel).
template <int L, bool MIXED>
__global__ void __launch_bounds__(128) esp_order_kernel(const __grid_constant__ EspParams prm, long long first,
                                                       long long count, long long chunk, int slot0, double* part,
                                                       long long ld) {
    using R_t = std::conditional_t<MIXED, float, double>;
    constexpr int NT = hermite_count(L);
    constexpr int BATCH = (2048 / NT) < 128 ? (2048 / NT) : 128;
    __shared__ double s_p[BATCH], s_q[BATCH][3];
    __shared__ R_t s_c[BATCH * NT];
    const long long q = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    const bool valid = q < prm.src.count;
    double x = 0.0, y = 0.0, z = 0.0;
    if (valid) point_at(prm.src, q, x, y, z);
    const EspView& e = prm.esp;
    const long long i0 = first + static_cast<long long>(blockIdx.y) * chunk;
    const long long i1 = min(first + count, i0 + chunk);
    R_t sum = 0, comp = 0;
    for (long long b0 = i0; b0 < i1; b0 += BATCH) {
        const int nb = static_cast<int>(min(static_cast<long long>(BATCH), i1 - b0));
        __syncthreads();  // the previous batch is no longer read
        for (int t = threadIdx.x; t < nb; t += blockDim.x) {
            const EspPair pr = e.pairs[b0 + t];
            s_p[t] = pr.p;
            s_q[t][0] = pr.qx;
            s_q[t][1] = pr.qy;
            s_q[t][2] = pr.qz;
        }
        const double* cbase = e.coef + e.pairs[b0].first;
        for (int t = threadIdx.x; t < nb * NT; t += blockDim.x) s_c[t] = static_cast<R_t>(cbase[t]);
        __syncthreads();
        for (int ib = 0; ib < nb; ++ib) {
            const double pcx = s_q[ib][0] - x, pcy = s_q[ib][1] - y, pcz = s_q[ib][2] - z;
            const double pp = s_p[ib];
            double F[L + 1];
            boys_top<L>(e.boys_table, pp * (pcx * pcx + pcy * pcy + pcz * pcz), F);
            double power = 1.0;
#pragma unroll
            for (int k = 1; k <= L; ++k) {
                power *= -2.0 * pp;
                F[k] *= power;
            }
            const R_t rx = static_cast<R_t>(pcx), ry = static_cast<R_t>(pcy), rz = static_cast<R_t>(pcz);
            R_t R[NT];
#pragma unroll
            for (int n = L; n >= 0; --n) {
                hermite_level<NT - 1, NT>(R, hermite_count(L - n), rx, ry, rz);
                R[0] = static_cast<R_t>(F[n]);
            }
            const R_t* c = s_c + ib * NT;
            R_t s = 0;
#pragma unroll
            for (int k = 0; k < NT; ++k) s += c[k] * R[k];
            if constexpr (MIXED) {
                const R_t yk = s - comp;
                const R_t t = sum + yk;
                comp = (t - sum) - yk;
                sum = t;
            } else {
                sum += s;
            }
        }
    }
    if (valid) {
        double total = static_cast<double>(sum);
        if constexpr (MIXED) total -= static_cast<double>(comp);
        part[static_cast<long long>(slot0 + blockIdx.y) * ld + q] = total;
    }
}

// out = nuclear term - the partial sums in slot order.
__global__ void __launch_bounds__(128) esp_reduce_kernel(const __grid_constant__ EspParams prm, const double* part,
                                                        int nslots, long long ld) {
    const long long q = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q >= prm.src.count) return;
    double x, y, z;
    point_at(prm.src, q, x, y, z);
    const EspView& e = prm.esp;
    double nuclear = 0.0;
    for (int a = 0; a < e.natoms; ++a) {
        const double4 at = e.atoms[a];
        const double dx = at.x - x, dy = at.y - y, dz = at.z - z;
        const double d = sqrt(dx * dx + dy * dy + dz * dz);
        if (at.w == 0.0 || d < 1e-8) continue;
        nuclear += at.w / d;
    }
    double sum = 0.0;
    for (int s = 0; s < nslots; ++s) sum += part[static_cast<long long>(s) * ld + q];
    prm.out[q - prm.out_base] = nuclear - sum;
}

template <int L>
void launch_order(const EspParams& p, long long first, long long count, long long chunk, int chunks, int slot0,
                  double* part, long long ld, unsigned tiles, cudaStream_t stream) {
    KUMO_REGISTER_KERNEL(esp_order_kernel<L, true>);
    KUMO_REGISTER_KERNEL(esp_order_kernel<L, false>);
    if (p.mixed) {
        esp_order_kernel<L, true><<<dim3(tiles, static_cast<unsigned>(chunks)), 128, 0, stream>>>(
            p, first, count, chunk, slot0, part, ld);
        return;
    }
    esp_order_kernel<L, false><<<dim3(tiles, static_cast<unsigned>(chunks)), 128, 0, stream>>>(p, first, count, chunk, slot0,
                                                                                       part, ld);
}

void launch_esp(const EspParams& p, cudaStream_t stream) {
    using chem::kumo::detail::check_cuda;
    const long long n = p.src.count;
    if (n <= 0) return;
    const unsigned tiles = static_cast<unsigned>((n + 127) / 128);
    const EspView& e = p.esp;
    // Chunks per order: each order's launch (they run one after another)
    // gets about 8 CTAs per SM, with at least 64 pairs a chunk.
    constexpr long long kTargetCtas = 8 * 148;
    int chunks[kEspMaxL + 1] = {};
    long long chunk_size[kEspMaxL + 1] = {};
    int nslots = 0;
    for (int L = 0; L <= kEspMaxL; ++L) {
        const long long count = e.order_first[L + 1] - e.order_first[L];
        if (count <= 0) continue;
        long long want = (kTargetCtas + tiles - 1) / tiles;
        want = std::max<long long>(1, std::min<long long>(want, (count + 63) / 64));
        chunk_size[L] = (count + want - 1) / want;
        chunks[L] = static_cast<int>((count + chunk_size[L] - 1) / chunk_size[L]);
        nslots += chunks[L];
    }
    double* part = nullptr;
    const long long ld = n;
    if (nslots > 0)
        check_cuda(cudaMallocAsync(reinterpret_cast<void**>(&part), sizeof(double) * static_cast<size_t>(nslots) * n,
                                   stream),
                   "cudaMallocAsync (potential partial sums)");
    int slot = 0;
    for (int L = 0; L <= kEspMaxL; ++L) {
        if (!chunks[L]) continue;
        const long long first = e.order_first[L], count = e.order_first[L + 1] - first;
        const long long cs = chunk_size[L];
        const int nc = chunks[L];
        switch (L) {
            case 0: launch_order<0>(p, first, count, cs, nc, slot, part, ld, tiles, stream); break;
            case 1: launch_order<1>(p, first, count, cs, nc, slot, part, ld, tiles, stream); break;
            case 2: launch_order<2>(p, first, count, cs, nc, slot, part, ld, tiles, stream); break;
            case 3: launch_order<3>(p, first, count, cs, nc, slot, part, ld, tiles, stream); break;
            case 4: launch_order<4>(p, first, count, cs, nc, slot, part, ld, tiles, stream); break;
            case 5: launch_order<5>(p, first, count, cs, nc, slot, part, ld, tiles, stream); break;
            case 6: launch_order<6>(p, first, count, cs, nc, slot, part, ld, tiles, stream); break;
            case 7: launch_order<7>(p, first, count, cs, nc, slot, part, ld, tiles, stream); break;
            default: launch_order<8>(p, first, count, cs, nc, slot, part, ld, tiles, stream); break;
        }
        slot += nc;
    }
    KUMO_REGISTER_KERNEL(esp_reduce_kernel);
    esp_reduce_kernel<<<tiles, 128, 0, stream>>>(p, part, nslots, ld);
    if (part) cudaFreeAsync(part, stream);
}

__global__ void boys_kernel(const double* table, const double* t, long long n, int nvalues, double* out) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double v[kBoysMaxOrder + 1];
    boys_device(table, t[i], nvalues, v);
    for (int m = 0; m < nvalues; ++m) out[i * nvalues + m] = v[m];
}

void launch_boys_f64(const double* table, const double* t, long long n, int nvalues, double* out, cudaStream_t stream) {
    KUMO_REGISTER_KERNEL(boys_kernel);
    if (n <= 0) return;
    boys_kernel<<<(unsigned)((n + 127) / 128), 128, 0, stream>>>(table, t, n, nvalues, out);
}

}  // namespace kumo_dev
