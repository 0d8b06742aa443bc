// Gaussian Cube writer of Field: the fixed-width layout of chem-kumo's
// src/cube.cpp:70-111 (six decimals in the header, %13.5e values, six per
// line and a break after every run along the third axis).
#include <algorithm>
#include <charconv>
#include <cinttypes>
#include <cmath>
#include <cstdio>
#include <memory>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "chem/kumo/density.hpp"

#ifndef KUMO_B200_VERSION
#define KUMO_B200_VERSION "2.1.0"
#endif

namespace chem::kumo {
namespace {

struct FileCloser {
    void operator()(std::FILE* f) const {
        if (f) std::fclose(f);
    }
};

void write_field_cube(const std::filesystem::path& path, const std::string& comment, const Grid& grid,
                      const std::vector<Atom>& atoms, const std::vector<double>& values, std::size_t orbital) {
    const bool is_orbital = orbital != 0;
    if (!std::all_of(values.begin(), values.end(), [](double v) { return std::isfinite(v); }))
        throw std::invalid_argument("nonfinite Cube sample");
    std::unique_ptr<std::FILE, FileCloser> f(std::fopen(path.string().c_str(), "w"));
    if (!f) throw std::runtime_error(is_orbital ? "cannot open orbital cube output" : "cannot open cube output");
    std::FILE* o = f.get();
    std::fprintf(o, "chem-kumo %s\n%s\n", KUMO_B200_VERSION, comment.c_str());
    const long long na = static_cast<long long>(atoms.size());
    std::fprintf(o, "%5lld", is_orbital ? -na : na);
    for (int k = 0; k < 3; ++k) std::fprintf(o, "%13.6f", grid.origin[k]);
    std::fprintf(o, "\n");
    for (int a = 0; a < 3; ++a) {
        std::fprintf(o, "%5d", grid.counts[a]);
        for (int k = 0; k < 3; ++k) std::fprintf(o, "%13.6f", grid.steps(k, a));
        std::fprintf(o, "\n");
    }
    for (const auto& a : atoms) {
        std::fprintf(o, "%5d%13.6f", a.atomic_number, a.nuclear_charge);
        for (int k = 0; k < 3; ++k) std::fprintf(o, "%13.6f", a.position[k]);
        std::fprintf(o, "\n");
    }
    if (is_orbital) std::fprintf(o, "%5d%5zu\n", 1, orbital);
    const std::size_t nz = static_cast<std::size_t>(grid.counts[2]);
    // The values: %13.5e (std::to_chars gives the same correctly rounded
    // digits as printf), a break after every sixth value of the whole array
    // and after each run along the third axis; formatted on all host threads,
    // each taking a contiguous range of runs, then written in order.
    const std::size_t runs = nz ? values.size() / nz : 0;
    const std::size_t nthreads =
        std::max<std::size_t>(1, std::min<std::size_t>(std::thread::hardware_concurrency(), runs / 64 + 1));
    std::vector<std::string> parts(nthreads);
    auto format = [&](std::size_t t) {
        const std::size_t r0 = runs * t / nthreads, r1 = runs * (t + 1) / nthreads;
        std::string& buf = parts[t];
        buf.reserve((r1 - r0) * nz * 14 + (r1 - r0) + 16);
        char tmp[32];
        for (std::size_t i = r0 * nz; i < r1 * nz; ++i) {
            const auto res = std::to_chars(tmp, tmp + sizeof tmp, values[i], std::chars_format::scientific, 5);
            const std::size_t len = static_cast<std::size_t>(res.ptr - tmp);
            if (len < 13) buf.append(13 - len, ' ');
            buf.append(tmp, len);
            if ((i + 1) % 6 == 0 || (i + 1) % nz == 0) buf.push_back('\n');
        }
    };
    std::vector<std::thread> pool;
    for (std::size_t t = 1; t < nthreads; ++t) pool.emplace_back(format, t);
    format(0);
    for (auto& th : pool) th.join();
    for (const auto& b : parts) std::fwrite(b.data(), 1, b.size(), o);
    if (std::ferror(o)) throw std::runtime_error(is_orbital ? "orbital cube write failed" : "cube write failed");
}

}  // namespace

void Field::write_cube(const std::filesystem::path& path, const std::string& comment) const {
    write_field_cube(path, comment, grid_, atoms_, values_, 0);
}

void Field::write_orbital_cube(const std::filesystem::path& path, std::size_t orbital_index,
                               const std::string& comment) const {
    if (orbital_index == 0 || orbital_index > 9999) throw std::invalid_argument("invalid orbital index for a Cube file");
    write_field_cube(path, comment, grid_, atoms_, values_, orbital_index);
}

}  // namespace chem::kumo
