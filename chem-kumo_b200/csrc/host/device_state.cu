// Upload of a molecule's AO tables, density matrices and MO coefficients.
#include "device_state.hpp"

#include "../cuda/esp.cuh"
#include "../cuda/mixed.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>

namespace chem::kumo::detail {

void throw_cuda(cudaError_t e, const char* what) {
    throw std::runtime_error(std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e));
}

namespace {

// BF16 (8-bit significand) rounding of a double, to nearest with ties to even,
// in two steps: to FP32 with round-to-odd (so the second rounding cannot
// double-round), then to BF16 by integer rounding of the FP32 bits.
std::uint16_t bf16_bits(double x) {
    float f = static_cast<float>(x);
    if (std::isfinite(f) && static_cast<double>(f) != x) {
        std::uint32_t u;
        std::memcpy(&u, &f, 4);
        // Round to odd: truncate toward zero, then set the last bit.
        const float t = std::fabs(static_cast<double>(f)) > std::fabs(x) ? std::nextafter(f, 0.0f) : f;
        std::memcpy(&u, &t, 4);
        u |= 1u;
        std::memcpy(&f, &u, 4);
    }
    std::uint32_t u;
    std::memcpy(&u, &f, 4);
    if ((u & 0x7f800000u) == 0x7f800000u) return static_cast<std::uint16_t>(u >> 16);
    u += 0x7fffu + ((u >> 16) & 1u);
    return static_cast<std::uint16_t>(u >> 16);
}

double bf16_value(std::uint16_t h) {
    const std::uint32_t u = static_cast<std::uint32_t>(h) << 16;
    float f;
    std::memcpy(&f, &u, 4);
    return static_cast<double>(f);
}

}  // namespace

template <typename T>
T* DeviceMolecule::upload(const T* host, std::size_t count) {
    if (count == 0) count = 1;
    void* p = nullptr;
    check_cuda(cudaMalloc(&p, sizeof(T) * count), "cudaMalloc (molecule)");
    allocations.push_back(p);
    bytes += sizeof(T) * count;
    if (host) check_cuda(cudaMemcpy(p, host, sizeof(T) * count, cudaMemcpyHostToDevice), "cudaMemcpy (molecule)");
    return static_cast<T*>(p);
}

DeviceMolecule::DeviceMolecule(const Molecule& m) {
    check_cuda(cudaGetDevice(&device), "cudaGetDevice");
    const auto& blocks = m.blocks();
    const std::size_t n = m.basis_size();
    std::vector<double4> origin(blocks.size());
    std::vector<int4> info(blocks.size());
    std::vector<double> exps, weights;
    int max_l = 0, max_count = 0;
    for (std::size_t i = 0; i < blocks.size(); ++i) {
        const auto& b = blocks[i];
        const int l = b.angular_momentum;
        const int np = static_cast<int>(b.exponents.size());
        if (l > kumo_dev::kMaxL)
            throw std::invalid_argument("the B200 evaluator supports shells up to l = 4 (g)");
        if (np > kumo_dev::kMaxPrim)
            throw std::invalid_argument("the B200 evaluator supports at most 16 primitives per shell");
        origin[i] = make_double4(b.origin[0], b.origin[1], b.origin[2], b.cutoff_radius2);
        info[i] = make_int4(l | (b.pure ? 1 << 8 : 0) | (np << 16), static_cast<int>(exps.size()),
                            static_cast<int>(weights.size()), static_cast<int>(b.offset));
        exps.insert(exps.end(), b.exponents.begin(), b.exponents.end());
        weights.insert(weights.end(), b.weights.begin(), b.weights.end());
        max_l = std::max(max_l, l);
        max_count = std::max(max_count, static_cast<int>(b.count));
    }
    std::vector<float> exps_f(exps.begin(), exps.end()), weights_f(weights.begin(), weights.end());
    // g_k = ((2x-1)!!(2y-1)!!(2z-1)!!)^(-1/2) of each Cartesian component; the
    // first component of every order (x^l, or z^l for l >= 4) has g = ((2l-1)!!)^(-1/2).
    auto odd_df = [](int n) {
        double r = 1.0;
        for (int k = n; k > 1; k -= 2) r *= k;
        return r;
    };
    std::vector<kumo_dev::MixPrim> mix(exps.size());
    for (const auto& b : blocks) {
        const auto& pw = b.powers;
        const double g0 = 1.0 / std::sqrt(odd_df(2 * pw[0].x - 1) * odd_df(2 * pw[0].y - 1) * odd_df(2 * pw[0].z - 1));
        const std::size_t np = b.exponents.size();
        const std::size_t first = static_cast<std::size_t>(&b - blocks.data());
        const std::size_t p0 = static_cast<std::size_t>(info[first].y);
        for (std::size_t p = 0; p < np; ++p) {
            const double a = b.exponents[p];
            mix[p0 + p] = {a * 1.4426950408889634, static_cast<float>(a), static_cast<float>(b.weights[p] / g0)};
        }
    }
    mix_prims = upload(mix.data(), mix.size());
    double g64[kumo_dev::kMaxL + 1][15] = {};
    for (int l = 0; l <= kumo_dev::kMaxL; ++l) {
        const auto cart = gaussian_cartesian_order(l);
        for (std::size_t k = 0; k < cart.size(); ++k) {
            g64[l][k] = 1.0 / std::sqrt(odd_df(2 * cart[k].x - 1) * odd_df(2 * cart[k].y - 1) * odd_df(2 * cart[k].z - 1));
            gcart[l][k] = static_cast<float>(g64[l][k]);
        }
    }
    basis.nblocks = static_cast<int>(blocks.size());
    basis.nao = static_cast<int>(n);
    basis.max_l = max_l;
    basis.max_count = max_count;
    basis.origin_r2 = upload(origin.data(), origin.size());
    basis.info = upload(info.data(), info.size());
    basis.exps = upload(exps.data(), exps.size());
    basis.weights = upload(weights.data(), weights.size());
    basis.exps_f = upload(exps_f.data(), exps_f.size());
    basis.weights_f = upload(weights_f.data(), weights_f.size());
    std::vector<int> ao_block(n);
    for (std::size_t i = 0; i < blocks.size(); ++i)
        for (std::size_t c = 0; c < blocks[i].count; ++c)
            ao_block[blocks[i].offset + c] = static_cast<int>(i) * 32 + static_cast<int>(c);
    basis.ao_block = upload(ao_block.data(), ao_block.size());
    double tg64[3][135] = {};
    for (int l = 2; l <= kumo_dev::kMaxL; ++l) {
        const Matrix t = gaussian_cartesian_to_pure(l);
        for (std::size_t r = 0; r < t.rows(); ++r)
            for (std::size_t c = 0; c < t.cols(); ++c) {
                pure_d[l - 2][r * t.cols() + c] = t(r, c);
                pure_f[l - 2][r * t.cols() + c] = static_cast<float>(t(r, c));
                tg64[l - 2][r * t.cols() + c] = t(r, c) * g64[l][c];
                tpure_g[l - 2][r * t.cols() + c] = static_cast<float>(tg64[l - 2][r * t.cols() + c]);
                // The mixed AO kernel skips the entries this predicate calls zero.
                const auto cart = gaussian_cartesian_order(l);
                if (t(r, c) != 0.0 && !kumo_dev::solid_harmonic_nonzero(l, static_cast<int>(r), cart[c].x, cart[c].y))
                    throw std::logic_error("Cartesian-to-pure pattern mismatch");
            }
    }
    // The exact rows' FP64 tables are the same for every basis: once per device.
    {
        static std::mutex mu;
        static bool done[64] = {};
        std::lock_guard<std::mutex> lock(mu);
        if (device < 0 || device >= 64 || !done[device]) {
            kumo_dev::upload_exact_tables(g64, tg64);
            if (device >= 0 && device < 64) done[device] = true;
        }
    }
    const Matrix pt = m.density_matrix(DensityComponent::Total);
    const Matrix ps = m.density_matrix(DensityComponent::Difference);
    p_total = upload(pt.data(), pt.size());
    p_spin = upload(ps.data(), ps.size());
    unrestricted = m.unrestricted();
    const Matrix& ca = m.mo_coefficients(SpinChannel::Alpha);
    const Matrix& cb = m.mo_coefficients(SpinChannel::Beta);
    nmo_alpha = static_cast<int>(ca.cols());
    nmo_beta = static_cast<int>(cb.cols());
    if (nmo_alpha) c_alpha = upload(ca.data(), ca.size());
    if (unrestricted && nmo_beta) c_beta = upload(cb.data(), cb.size());
    if (!unrestricted) c_beta = c_alpha;
    auto transpose_occ = [&](const Matrix& c, int nocc, int& ld, double*& dst, int& ldn, std::uint16_t*& dst_s) {
        // Rows padded to a multiple of 4 so that every 16-byte chunk of a row
        // (2 doubles, 4 floats) lies inside the row.
        ld = std::max(4, (nocc + 3) / 4 * 4);
        std::vector<double> t(n * static_cast<std::size_t>(ld), 0.0);
        for (int o = 0; o < nocc && static_cast<std::size_t>(o) < c.cols(); ++o)
            for (std::size_t a = 0; a < n; ++a) t[a * static_cast<std::size_t>(ld) + static_cast<std::size_t>(o)] = c(a, static_cast<std::size_t>(o));
        dst = upload(t.data(), t.size());
        ldn = std::max(16, (nocc + 15) / 16 * 16);
        std::vector<std::uint16_t> pieces(3 * n * static_cast<std::size_t>(ldn), 0);
        for (std::size_t a = 0; a < n; ++a)
            for (int o = 0; o < nocc && static_cast<std::size_t>(o) < c.cols(); ++o) {
                double rest = c(a, static_cast<std::size_t>(o));
                for (int k = 0; k < 3; ++k) {
                    const std::uint16_t h = bf16_bits(rest);
                    pieces[(k * n + a) * static_cast<std::size_t>(ldn) + static_cast<std::size_t>(o)] = h;
                    rest -= bf16_value(h);
                }
            }
        dst_s = upload(pieces.data(), pieces.size());
    };
    nocc_alpha = static_cast<int>(m.occupied_count(SpinChannel::Alpha));
    nocc_beta = static_cast<int>(m.occupied_count(SpinChannel::Beta));
    if (nmo_alpha) {
        transpose_occ(ca, nocc_alpha, ldc_alpha, ct_alpha, ldn_alpha, cs_alpha);
        transpose_occ(unrestricted ? cb : ca, nocc_beta, ldc_beta, ct_beta, ldn_beta, cs_beta);
    }
}

void DeviceMolecule::ensure_p_pieces(const Molecule& m) {
    std::lock_guard<std::mutex> lock(esp_mutex);
    if (p_total_s) return;
    const std::size_t n = m.basis_size();
    auto split_matrix = [&](const Matrix& a) {
        std::vector<std::uint16_t> pieces(4 * n * n, 0);
        for (std::size_t r = 0; r < n; ++r)
            for (std::size_t c = 0; c < n; ++c) {
                double rest = a(r, c);
                for (int k = 0; k < 3; ++k) {
                    const std::uint16_t h = bf16_bits(rest);
                    pieces[(r * n + c) * 4 + static_cast<std::size_t>(k)] = h;
                    rest -= bf16_value(h);
                }
            }
        return upload(pieces.data(), pieces.size());
    };
    std::uint16_t* spin = split_matrix(m.density_matrix(DensityComponent::Difference));
    p_spin_s = spin;
    p_total_s = split_matrix(m.density_matrix(DensityComponent::Total));
}

kumo_dev::EspDevice& DeviceMolecule::esp_state(const Molecule& m, cudaStream_t stream) {
    std::lock_guard<std::mutex> lock(esp_mutex);
    if (!esp) {
        esp = std::make_unique<kumo_dev::EspDevice>(m, stream);
        bytes += esp->device_bytes();
    }
    return *esp;
}

const DeviceMolecule::OrbitalEnergyDevice& DeviceMolecule::orbital_energy_state(const Molecule& m,
                                                                                const OrbitalEnergyNeeds& needs,
                                                                                const std::string& what) {
    std::lock_guard<std::mutex> lock(esp_mutex);
    for (const auto& e : orbital_energy)
        if (e->needs == needs) return *e;
    const OrbitalEnergyColumns cols = orbital_energy_columns(m, needs, what);
    auto e = std::make_unique<OrbitalEnergyDevice>();
    e->needs = needs;
    e->ldw = static_cast<int>(cols.ldw);
    e->nchunks = static_cast<int>(cols.chunk_set.size());
    e->w = upload(cols.w.data(), cols.w.size());
    e->energy = upload(cols.energy.data(), cols.energy.size());
    e->chunk_set = upload(cols.chunk_set.data(), cols.chunk_set.size());
    orbital_energy.push_back(std::move(e));
    return *orbital_energy.back();
}

DeviceMolecule::~DeviceMolecule() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (cur != device) cudaSetDevice(device);
    esp.reset();
    for (void* p : allocations) cudaFree(p);
    if (cur != device && cur >= 0) cudaSetDevice(cur);
}

}  // namespace chem::kumo::detail
