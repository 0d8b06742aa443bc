// Gaussian formatted checkpoint reader; record rules of chem-kumo's
// src/fchk.cpp:78-187 (label columns 0-42, type at column 43, "N=" arrays,
// only I and R records, Fortran D exponents, duplicate records must agree).
#include "chem/kumo/fchk.hpp"

#include <zlib.h>

#include <cmath>
#include <fstream>
#include <limits>
#include <sstream>
#include <stdexcept>

namespace chem::kumo {
namespace {

std::string trim_right(std::string s) {
    while (!s.empty() && (s.back() == ' ' || s.back() == '\t' || s.back() == '\r')) s.pop_back();
    return s;
}

long long parse_integer(const std::string& token, const std::string& label) {
    std::size_t used = 0;
    long long v = 0;
    try {
        v = std::stoll(token, &used);
    } catch (const std::exception&) {
        throw std::runtime_error("invalid integer token in fchk record " + label + ": " + token);
    }
    if (used != token.size())
        throw std::runtime_error("trailing characters in integer token in fchk record " + label + ": " + token);
    return v;
}

double parse_real(const std::string& raw, const std::string& label) {
    std::string token = raw;
    for (auto& c : token)
        if (c == 'D' || c == 'd') c = 'E';
    std::size_t used = 0;
    double v = 0.0;
    try {
        v = std::stod(token, &used);
    } catch (const std::exception&) {
        throw std::runtime_error("invalid real token in fchk record " + label + ": " + raw);
    }
    if (used != token.size() || !std::isfinite(v))
        throw std::runtime_error("invalid real token in fchk record " + label + ": " + raw);
    return v;
}

bool has_gzip_magic(const std::filesystem::path& path) {
    std::ifstream f(path, std::ios::binary);
    unsigned char m[2] = {0, 0};
    f.read(reinterpret_cast<char*>(m), 2);
    return f.gcount() == 2 && m[0] == 0x1f && m[1] == 0x8b;
}

std::string read_gzip(const std::filesystem::path& path) {
    gzFile g = gzopen(path.string().c_str(), "rb");
    if (!g) throw std::runtime_error("cannot open gzip formatted checkpoint: " + path.string());
    std::string out;
    std::vector<char> buf(1 << 20);
    for (;;) {
        const int n = gzread(g, buf.data(), static_cast<unsigned>(buf.size()));
        if (n < 0) {
            int code = 0;
            const char* msg = gzerror(g, &code);
            std::string m = msg ? msg : "gzip error";
            gzclose(g);
            throw std::runtime_error("gzip decoding failed for formatted checkpoint: " + m);
        }
        if (n == 0) break;
        out.append(buf.data(), static_cast<std::size_t>(n));
    }
    gzclose(g);
    return out;
}

}  // namespace

FormattedCheckpoint::FormattedCheckpoint(const std::filesystem::path& path) {
    std::error_code ec;
    const auto size = std::filesystem::file_size(path, ec);
    if (ec) throw std::runtime_error("cannot stat formatted checkpoint: " + path.string());
    if (has_gzip_magic(path)) {
        std::string text = read_gzip(path);
        std::istringstream in(text);
        parse(in, text.size(), path.string());
        return;
    }
    std::ifstream in(path, std::ios::binary);
    if (!in) throw std::runtime_error("cannot open formatted checkpoint: " + path.string());
    parse(in, static_cast<std::size_t>(size), path.string());
}

FormattedCheckpoint FormattedCheckpoint::from_text(const std::string& text, std::size_t logical_size) {
    FormattedCheckpoint f;
    std::istringstream in(text);
    f.parse(in, logical_size, "<memory>");
    return f;
}

void FormattedCheckpoint::parse(std::istream& input, std::size_t logical_size, const std::string& name) {
    std::string line;
    if (!std::getline(input, line) || !std::getline(input, line))
        throw std::runtime_error("formatted checkpoint is missing its two-line header: " + name);
    while (std::getline(input, line)) {
        if (line.size() < 44U) continue;
        const std::string label = trim_right(line.substr(0, 43));
        if (label.empty()) continue;
        std::istringstream meta(line.substr(43));
        char type = '\0';
        meta >> type;
        if (type != 'I' && type != 'R') continue;
        std::string marker;
        if (!(meta >> marker)) throw std::runtime_error("malformed fchk record metadata: " + label);
        Record rec;
        if (marker == "N=") {
            long long n = 0;
            if (!(meta >> n) || n < 0) throw std::runtime_error("invalid array size in fchk: " + label);
            if (static_cast<unsigned long long>(n) > static_cast<unsigned long long>(logical_size))
                throw std::runtime_error("unreasonable array size in fchk: " + label);
            const auto count = static_cast<std::size_t>(n);
            std::string token;
            if (type == 'I') {
                rec.kind = Kind::IntegerArray;
                rec.integer_array.reserve(count);
            } else {
                rec.kind = Kind::RealArray;
                rec.real_array.reserve(count);
            }
            for (std::size_t i = 0; i < count; ++i) {
                if (!(input >> token)) throw std::runtime_error("truncated array in fchk: " + label);
                if (type == 'I')
                    rec.integer_array.push_back(parse_integer(token, label));
                else
                    rec.real_array.push_back(parse_real(token, label));
            }
            std::string rest;
            std::getline(input, rest);
            if (rest.find_first_not_of(" \t\r") != std::string::npos)
                throw std::runtime_error("too many values on final array line in fchk: " + label);
        } else if (type == 'I') {
            rec.kind = Kind::IntegerScalar;
            rec.integer_scalar = parse_integer(marker, label);
        } else {
            rec.kind = Kind::RealScalar;
            rec.real_scalar = parse_real(marker, label);
        }
        auto it = records_.find(label);
        if (it != records_.end()) {
            const Record& a = it->second;
            bool same = a.kind == rec.kind;
            if (same) {
                switch (a.kind) {
                    case Kind::IntegerScalar: same = a.integer_scalar == rec.integer_scalar; break;
                    case Kind::RealScalar: same = a.real_scalar == rec.real_scalar; break;
                    case Kind::IntegerArray: same = a.integer_array == rec.integer_array; break;
                    case Kind::RealArray: same = a.real_array == rec.real_array; break;
                }
            }
            if (!same) throw std::runtime_error("conflicting duplicate fchk record: " + label);
            continue;
        }
        records_.emplace(label, std::move(rec));
    }
}

const FormattedCheckpoint::Record& FormattedCheckpoint::record(const std::string& label) const {
    auto it = records_.find(label);
    if (it == records_.end()) throw std::runtime_error("missing fchk record: " + label);
    return it->second;
}

bool FormattedCheckpoint::contains(const std::string& label) const { return records_.count(label) != 0; }

long long FormattedCheckpoint::integer(const std::string& label) const {
    const auto& r = record(label);
    if (r.kind != Kind::IntegerScalar) throw std::runtime_error("fchk record is not an integer scalar: " + label);
    return r.integer_scalar;
}

double FormattedCheckpoint::real(const std::string& label) const {
    const auto& r = record(label);
    if (r.kind != Kind::RealScalar) throw std::runtime_error("fchk record is not a real scalar: " + label);
    return r.real_scalar;
}

const std::vector<long long>& FormattedCheckpoint::integers(const std::string& label) const {
    const auto& r = record(label);
    if (r.kind != Kind::IntegerArray) throw std::runtime_error("fchk record is not an integer array: " + label);
    return r.integer_array;
}

const std::vector<double>& FormattedCheckpoint::reals(const std::string& label) const {
    const auto& r = record(label);
    if (r.kind != Kind::RealArray) throw std::runtime_error("fchk record is not a real array: " + label);
    return r.real_array;
}

}  // namespace chem::kumo
