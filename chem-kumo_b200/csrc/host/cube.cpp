// Gaussian Cube files.  The writer of Field: the fixed-width layout of
// chem-kumo's src/cube.cpp:70-111 (six decimals in the header, %13.5e values,
// six per line and a break after every run along the third axis).  The
// reader and the full-precision writer of CubeData: the rules of
// src/cube.cpp:114-251 (see chem/kumo/cube.hpp).
#include <zlib.h>

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

#include "chem/kumo/cube.hpp"
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

// ---------------------------------------------------------------------------
// CubeData reader and writer.
//
// The file is read whole (inflated through zlib when it starts with the gzip
// magic; gzread checks the member's CRC and length at its end).  Header lines
// are split into whitespace tokens, each read in full; the samples after the
// header are split into as many contiguous text ranges as there are host
// threads (cut at whitespace) and parsed in parallel with from_chars.

namespace {

constexpr double kAngstromToBohr = 1.8897261246257702;
constexpr long long kMaxAtoms = 1000000;
constexpr long long kMaxAxisCount = 1000000000LL;
constexpr std::size_t kMaxSamples = 1000000000ULL;

[[noreturn]] void cube_error(const char* what) { throw std::runtime_error(what); }

bool cube_space(char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == '\v' || c == '\f'; }

std::string slurp(const std::filesystem::path& path) {
    std::unique_ptr<std::FILE, FileCloser> f(std::fopen(path.string().c_str(), "rb"));
    if (!f) throw std::runtime_error("cannot open Cube input: " + path.string());
    std::string bytes;
    char chunk[1 << 16];
    std::size_t n;
    while ((n = std::fread(chunk, 1, sizeof chunk, f.get())) > 0) bytes.append(chunk, n);
    if (std::ferror(f.get())) cube_error("Cube input read failure");
    if (bytes.size() < 2 || static_cast<unsigned char>(bytes[0]) != 0x1f || static_cast<unsigned char>(bytes[1]) != 0x8b)
        return bytes;
    gzFile g = gzopen(path.string().c_str(), "rb");
    if (!g) throw std::runtime_error("cannot open Cube input: " + path.string());
    std::string text;
    for (;;) {
        const int m = gzread(g, chunk, sizeof chunk);
        if (m < 0) {
            int code = 0;
            const char* why = gzerror(g, &code);
            const std::string msg = std::string("gzip decoding failed for Cube: ") + (why ? why : "error");
            gzclose(g);
            throw std::runtime_error(msg);
        }
        if (m == 0) break;
        text.append(chunk, static_cast<std::size_t>(m));
    }
    // A member cut short (no CRC and length trailer) ends the reads early
    // with a buffer error instead of a negative count.
    int code = Z_OK;
    const char* why = gzerror(g, &code);
    if (code != Z_OK) {
        const std::string msg = std::string("gzip decoding failed for Cube: ") + (why ? why : "error");
        gzclose(g);
        throw std::runtime_error(msg);
    }
    gzclose(g);
    return text;
}

// Whitespace tokens of one header line, D/d exponents read as E/e.
class HeaderRow {
public:
    explicit HeaderRow(std::string line) : line_(std::move(line)) {
        for (char& c : line_) {
            if (c == 'D') c = 'E';
            if (c == 'd') c = 'e';
        }
    }
    bool next(std::string_view& tok) {
        while (at_ < line_.size() && cube_space(line_[at_])) ++at_;
        if (at_ >= line_.size()) return false;
        const std::size_t from = at_;
        while (at_ < line_.size() && !cube_space(line_[at_])) ++at_;
        tok = std::string_view(line_).substr(from, at_ - from);
        return true;
    }
    template <class T>
    bool read(T& v) {
        std::string_view tok;
        if (!next(tok)) return false;
        const char* b = tok.data();
        if (*b == '+') ++b;  // as strtod / stream extraction accept
        const auto r = std::from_chars(b, tok.data() + tok.size(), v);
        return r.ec == std::errc() && r.ptr == tok.data() + tok.size();
    }
    bool at_end() {
        std::string_view tok;
        return !next(tok);
    }

private:
    std::string line_;
    std::size_t at_ = 0;
};

struct LineReader {
    std::string_view text;
    std::size_t at = 0;
    bool line(std::string& out) {
        if (at >= text.size()) return false;
        const std::size_t end = text.find('\n', at);
        const std::size_t stop = end == std::string_view::npos ? text.size() : end;
        out.assign(text.substr(at, stop - at));
        if (!out.empty() && out.back() == '\r') out.pop_back();
        at = end == std::string_view::npos ? text.size() : end + 1;
        return true;
    }
    HeaderRow row() {
        std::string l;
        if (!line(l)) cube_error("truncated Cube header");
        return HeaderRow(std::move(l));
    }
};

bool valid_cube_atom(const Atom& a) {
    return a.atomic_number >= 0 && a.atomic_number <= 118 && std::isfinite(a.nuclear_charge) &&
           std::isfinite(a.position[0]) && std::isfinite(a.position[1]) && std::isfinite(a.position[2]);
}

// Samples of text[from, to): appends them to out; false on a malformed or
// nonfinite token.
bool parse_samples(std::string_view text, std::vector<double>& out) {
    std::size_t i = 0;
    std::string tok;
    while (true) {
        while (i < text.size() && cube_space(text[i])) ++i;
        if (i >= text.size()) return true;
        const std::size_t from = i;
        while (i < text.size() && !cube_space(text[i])) ++i;
        tok.assign(text.substr(from, i - from));
        for (char& c : tok) {
            if (c == 'D') c = 'E';
            if (c == 'd') c = 'e';
        }
        const char* b = tok.data();
        if (*b == '+') ++b;
        double v = 0.0;
        const auto r = std::from_chars(b, tok.data() + tok.size(), v);
        if (r.ec != std::errc() || r.ptr != tok.data() + tok.size() || !std::isfinite(v)) return false;
        out.push_back(v);
    }
}

}  // namespace

CubeData read_cube(const std::filesystem::path& path) {
    const std::string bytes = slurp(path);
    LineReader in{bytes};
    CubeMetadata meta;
    if (!in.line(meta.first_comment) || !in.line(meta.second_comment)) cube_error("missing Cube comments");

    Grid grid;
    HeaderRow first = in.row();
    long long natoms = 0;
    if (!first.read(natoms) || !first.read(grid.origin[0]) || !first.read(grid.origin[1]) || !first.read(grid.origin[2]) ||
        natoms < 0 || natoms > kMaxAtoms)
        cube_error("invalid Cube atom count or unsupported orbital Cube");
    {
        std::string_view tok;
        HeaderRow rest = first;
        if (rest.next(tok)) {
            int nval = 0;
            if (!first.read(nval) || nval != 1) cube_error("only scalar Cube NVAL=1 is supported");
            if (!first.at_end()) cube_error("malformed Cube header");
        }
    }
    std::size_t samples = 1;
    for (int a = 0; a < 3; ++a) {
        HeaderRow r = in.row();
        long long n = 0;
        double st[3];
        if (!r.read(n) || !r.read(st[0]) || !r.read(st[1]) || !r.read(st[2]) || n < -kMaxAxisCount ||
            n > kMaxAxisCount || (n >= -1 && n <= 1))
            cube_error("invalid Cube grid axis");
        if (!r.at_end()) cube_error("malformed Cube header");
        if (a == 0) meta.coordinates_in_angstrom = n < 0;
        if ((n < 0) != meta.coordinates_in_angstrom) cube_error("mixed Cube coordinate units");
        const long long c = n < 0 ? -n : n;
        if (static_cast<std::size_t>(c) > kMaxSamples / samples) cube_error("invalid Cube dimensions");
        samples *= static_cast<std::size_t>(c);
        grid.counts[a] = static_cast<int>(c);
        for (int k = 0; k < 3; ++k) grid.steps(k, a) = st[k];
    }
    std::vector<Atom> atoms(static_cast<std::size_t>(natoms));
    for (auto& at : atoms) {
        HeaderRow r = in.row();
        if (!r.read(at.atomic_number) || !r.read(at.nuclear_charge) || !r.read(at.position[0]) ||
            !r.read(at.position[1]) || !r.read(at.position[2]))
            cube_error("invalid Cube atom record");
        if (!r.at_end()) cube_error("malformed Cube header");
        if (!valid_cube_atom(at)) cube_error("invalid Cube atom");
    }
    if (meta.coordinates_in_angstrom) {
        for (int k = 0; k < 3; ++k) grid.origin[k] *= kAngstromToBohr;
        for (double& v : grid.steps.m) v *= kAngstromToBohr;
        for (auto& at : atoms)
            for (int k = 0; k < 3; ++k) at.position[k] *= kAngstromToBohr;
    }

    // The samples, in parallel ranges cut at whitespace.
    const std::string_view body = std::string_view(bytes).substr(in.at);
    const std::size_t nthreads = std::max<std::size_t>(
        1, std::min<std::size_t>(std::thread::hardware_concurrency(), body.size() / (1u << 20) + 1));
    std::vector<std::size_t> cut(nthreads + 1, body.size());
    cut[0] = 0;
    for (std::size_t t = 1; t < nthreads; ++t) {
        std::size_t c = std::max(cut[t - 1], body.size() * t / nthreads);
        while (c < body.size() && !cube_space(body[c])) ++c;
        cut[t] = c;
    }
    std::vector<std::vector<double>> parts(nthreads);
    std::vector<char> ok(nthreads, 1);
    auto work = [&](std::size_t t) {
        parts[t].reserve(samples / nthreads + 16);
        ok[t] = parse_samples(body.substr(cut[t], cut[t + 1] - cut[t]), parts[t]) ? 1 : 0;
    };
    std::vector<std::thread> pool;
    for (std::size_t t = 1; t < nthreads; ++t) pool.emplace_back(work, t);
    work(0);
    for (auto& th : pool) th.join();
    // Errors in file order: the first range that holds a bad token, unless
    // the ranges before it already hold more samples than the grid.
    std::size_t total = 0;
    for (std::size_t t = 0; t < nthreads; ++t) {
        if (total + parts[t].size() > samples) cube_error("extra Cube samples");
        if (!ok[t]) cube_error("invalid Cube sample");
        total += parts[t].size();
    }
    if (total != samples) cube_error("truncated Cube samples");
    std::vector<double> values;
    values.reserve(samples);
    for (auto& p : parts) values.insert(values.end(), p.begin(), p.end());
    return {Field(std::move(grid), std::move(atoms), std::move(values)), std::move(meta)};
}

void write_cube(const CubeData& cube, const std::filesystem::path& path) {
    const CubeMetadata& meta = cube.metadata;
    if (meta.first_comment.find_first_of("\r\n") != std::string::npos ||
        meta.second_comment.find_first_of("\r\n") != std::string::npos)
        throw std::invalid_argument("Cube comments must be single lines");
    const Grid& grid = cube.field.grid();
    const auto& atoms = cube.field.atoms();
    const auto& values = cube.field.values();
    std::size_t expect = 1;
    for (int a = 0; a < 3; ++a) expect *= static_cast<std::size_t>(std::max(grid.counts[a], 0));
    if (values.size() != expect) throw std::invalid_argument("inconsistent Cube field size");
    for (const auto& at : atoms)
        if (!valid_cube_atom(at)) throw std::invalid_argument("invalid Cube atom");
    if (!std::all_of(values.begin(), values.end(), [](double v) { return std::isfinite(v); }))
        throw std::invalid_argument("nonfinite Cube sample");
    const double f = meta.coordinates_in_angstrom ? 1.0 / kAngstromToBohr : 1.0;
    std::unique_ptr<std::FILE, FileCloser> out(std::fopen(path.string().c_str(), "w"));
    if (!out) throw std::runtime_error("cannot open Cube output: " + path.string());
    std::FILE* o = out.get();
    std::fprintf(o, "%s\n%s\n%zu", meta.first_comment.c_str(), meta.second_comment.c_str(), atoms.size());
    for (int k = 0; k < 3; ++k) std::fprintf(o, " %.12e", grid.origin[k] * f);
    std::fprintf(o, "\n");
    for (int a = 0; a < 3; ++a) {
        std::fprintf(o, "%d", meta.coordinates_in_angstrom ? -grid.counts[a] : grid.counts[a]);
        for (int k = 0; k < 3; ++k) std::fprintf(o, " %.12e", grid.steps(k, a) * f);
        std::fprintf(o, "\n");
    }
    for (const auto& at : atoms) {
        std::fprintf(o, "%d %.12e", at.atomic_number, at.nuclear_charge);
        for (int k = 0; k < 3; ++k) std::fprintf(o, " %.12e", at.position[k] * f);
        std::fprintf(o, "\n");
    }
    std::string buf;
    buf.reserve(values.size() * 20 + 16);
    char tmp[40];
    for (std::size_t i = 0; i < values.size(); ++i) {
        const auto r = std::to_chars(tmp, tmp + sizeof tmp, values[i], std::chars_format::scientific, 12);
        buf.append(tmp, static_cast<std::size_t>(r.ptr - tmp));
        buf.push_back((i + 1) % 6 == 0 ? '\n' : ' ');
    }
    if (values.size() % 6 != 0) buf.push_back('\n');
    std::fwrite(buf.data(), 1, buf.size(), o);
    if (std::fflush(o) != 0 || std::ferror(o)) throw std::runtime_error("Cube output write failed");
}

}  // namespace chem::kumo
