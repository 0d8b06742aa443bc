// Gaussian formatted checkpoint reader.
//
// Design: the whole file (inflated first when it starts with the gzip magic)
// is held in one buffer and scanned once by a cursor that hands out lines and
// whitespace-separated tokens as string_views; records land in a map from
// label to a variant of the four record shapes.
//
// Record rules (chem-kumo's src/fchk.cpp:78-187): two header lines; a record
// header has its label in columns 0-42 (trailing blanks dropped) and its type
// letter as the first non-blank character from column 43; only I and R
// records are kept (C, L and H records and every data line are skipped by the
// same test); "N=" introduces an array whose count is bounded by the file's
// uncompressed size, whose values are the next `count` tokens wherever the
// line breaks fall, and whose last data line must hold nothing after them
// (for count 0 that is the whole next line); reals accept Fortran D
// exponents and must be finite; a label met twice must carry the same record.
// Error messages are the reference's, since its callers match on them.
#include "chem/kumo/fchk.hpp"

#include <zlib.h>

#include <cctype>
#include <cerrno>
#include <cmath>
#include <cstdlib>
#include <fstream>
#include <iterator>
#include <optional>
#include <stdexcept>
#include <string_view>

namespace chem::kumo {
namespace {

[[noreturn]] void fail(const std::string& what) { throw std::runtime_error(what); }

bool is_blank(char c) { return std::isspace(static_cast<unsigned char>(c)) != 0; }

// Lines and tokens of an in-memory file.  `line()` behaves like getline (a
// final line without '\n' still counts; nothing left means no line);
// `token()` skips any whitespace, newlines included, like `stream >> word`.
class Cursor {
public:
    explicit Cursor(std::string_view text) : s_(text) {}

    std::optional<std::string_view> line() {
        if (at_ >= s_.size()) return std::nullopt;
        const std::size_t end = s_.find('\n', at_);
        const std::size_t stop = end == std::string_view::npos ? s_.size() : end;
        std::string_view out = s_.substr(at_, stop - at_);
        at_ = end == std::string_view::npos ? s_.size() : end + 1;
        return out;
    }

    std::optional<std::string_view> token() {
        while (at_ < s_.size() && is_blank(s_[at_])) ++at_;
        if (at_ >= s_.size()) return std::nullopt;
        const std::size_t from = at_;
        while (at_ < s_.size() && !is_blank(s_[at_])) ++at_;
        return s_.substr(from, at_ - from);
    }

private:
    std::string_view s_;
    std::size_t at_ = 0;
};

// Tokens of one header line after column 43 (the type letter, "N=" or the
// scalar value, the array count).
std::vector<std::string_view> split_fields(std::string_view tail) {
    std::vector<std::string_view> out;
    Cursor c(tail);
    while (auto t = c.token()) out.push_back(*t);
    return out;
}

std::string_view without_trailing_blanks(std::string_view s) {
    while (!s.empty() && (s.back() == ' ' || s.back() == '\t' || s.back() == '\r')) s.remove_suffix(1);
    return s;
}

// Whole-token integer: optional sign and digits, nothing after them.
long long to_integer(std::string_view tok, const std::string& label) {
    const std::string z(tok);
    char* end = nullptr;
    errno = 0;
    const long long v = std::strtoll(z.c_str(), &end, 10);
    if (end == z.c_str() || errno == ERANGE)
        fail("invalid integer token in fchk record " + label + ": " + z);
    if (*end != '\0') fail("trailing characters in integer token in fchk record " + label + ": " + z);
    return v;
}

// Whole-token finite real; 'D'/'d' exponents read as 'E'.  Out-of-range
// values (overflow or underflow) are rejected like std::stod rejects them.
double to_real(std::string_view tok, const std::string& label) {
    std::string z(tok);
    for (char& c : z)
        if (c == 'D' || c == 'd') c = 'E';
    char* end = nullptr;
    errno = 0;
    const double v = std::strtod(z.c_str(), &end);
    if (end == z.c_str() || errno == ERANGE || *end != '\0' || !std::isfinite(v))
        fail("invalid real token in fchk record " + label + ": " + std::string(tok));
    return v;
}

// Leading integer of the array-count field, as `istream >> long long` reads it.
std::optional<long long> leading_count(std::string_view tok) {
    const std::string z(tok);
    char* end = nullptr;
    errno = 0;
    const long long v = std::strtoll(z.c_str(), &end, 10);
    if (end == z.c_str() || errno == ERANGE) return std::nullopt;
    return v;
}

bool starts_with_gzip_magic(const std::string& bytes) {
    return bytes.size() >= 2 && static_cast<unsigned char>(bytes[0]) == 0x1f &&
           static_cast<unsigned char>(bytes[1]) == 0x8b;
}

std::string inflate_file(const std::filesystem::path& path) {
    gzFile g = gzopen(path.string().c_str(), "rb");
    if (!g) fail("cannot open gzip formatted checkpoint: " + path.string());
    std::string out;
    char chunk[1 << 16];
    for (;;) {
        const int n = gzread(g, chunk, sizeof chunk);
        if (n < 0) {
            int code = 0;
            const char* why = gzerror(g, &code);
            const std::string m = why ? why : "gzip error";
            gzclose(g);
            fail("gzip decoding failed for formatted checkpoint: " + m);
        }
        if (n == 0) break;
        out.append(chunk, static_cast<std::size_t>(n));
    }
    // A member cut short (no CRC and length trailer) ends the reads early
    // with a buffer error instead of a negative count.
    int code = Z_OK;
    const char* why = gzerror(g, &code);
    if (code != Z_OK) {
        const std::string m = why ? why : "gzip error";
        gzclose(g);
        fail("gzip decoding failed for formatted checkpoint: " + m);
    }
    gzclose(g);
    return out;
}

}  // namespace

FormattedCheckpoint::FormattedCheckpoint(const std::filesystem::path& path) {
    std::error_code ec;
    (void)std::filesystem::file_size(path, ec);
    if (ec) fail("cannot stat formatted checkpoint: " + path.string());
    std::ifstream file(path, std::ios::binary);
    if (!file) fail("cannot open formatted checkpoint: " + path.string());
    std::string bytes((std::istreambuf_iterator<char>(file)), std::istreambuf_iterator<char>());
    file.close();
    if (starts_with_gzip_magic(bytes)) bytes = inflate_file(path);
    load(bytes, bytes.size(), path.string());
}

FormattedCheckpoint FormattedCheckpoint::from_text(const std::string& text, std::size_t logical_size) {
    FormattedCheckpoint f;
    f.load(text, logical_size, "<memory>");
    return f;
}

void FormattedCheckpoint::load(std::string_view text, std::size_t logical_size, const std::string& name) {
    Cursor cur(text);
    if (!cur.line() || !cur.line()) fail("formatted checkpoint is missing its two-line header: " + name);

    while (auto ln = cur.line()) {
        if (ln->size() < 44U) continue;
        const std::string label(without_trailing_blanks(ln->substr(0, 43)));
        if (label.empty()) continue;
        const auto fields = split_fields(ln->substr(43));
        if (fields.empty() || (fields[0][0] != 'I' && fields[0][0] != 'R')) continue;
        const bool is_int = fields[0][0] == 'I';
        // The type letter may run into the next field ("Ifoo"): only its first
        // character is the type and the rest is the marker.
        std::string_view marker;
        std::size_t next = 1;
        if (fields[0].size() > 1) {
            marker = fields[0].substr(1);
        } else if (fields.size() > 1) {
            marker = fields[1];
            next = 2;
        } else {
            fail("malformed fchk record metadata: " + label);
        }

        Value value;
        if (marker == "N=") {
            const auto count = next < fields.size() ? leading_count(fields[next]) : std::nullopt;
            if (!count || *count < 0) fail("invalid array size in fchk: " + label);
            if (static_cast<unsigned long long>(*count) > static_cast<unsigned long long>(logical_size))
                fail("unreasonable array size in fchk: " + label);
            const auto n = static_cast<std::size_t>(*count);
            if (is_int) {
                std::vector<long long> v(n);
                for (auto& x : v) {
                    const auto t = cur.token();
                    if (!t) fail("truncated array in fchk: " + label);
                    x = to_integer(*t, label);
                }
                value = std::move(v);
            } else {
                std::vector<double> v(n);
                for (auto& x : v) {
                    const auto t = cur.token();
                    if (!t) fail("truncated array in fchk: " + label);
                    x = to_real(*t, label);
                }
                value = std::move(v);
            }
            // What follows the last value on its line (or, for an empty
            // array, the whole next line) must be blank.
            if (const auto rest = cur.line())
                for (char c : *rest)
                    if (c != ' ' && c != '\t' && c != '\r') fail("too many values on final array line in fchk: " + label);
        } else if (is_int) {
            value = to_integer(marker, label);
        } else {
            value = to_real(marker, label);
        }

        const auto [slot, fresh] = records_.try_emplace(label, value);
        if (!fresh && !(slot->second == value)) fail("conflicting duplicate fchk record: " + label);
    }
}

template <class T>
const T& FormattedCheckpoint::get(const std::string& label, const char* what) const {
    const auto it = records_.find(label);
    if (it == records_.end()) fail("missing fchk record: " + label);
    const T* v = std::get_if<T>(&it->second);
    if (!v) fail(std::string("fchk record is not ") + what + ": " + label);
    return *v;
}

bool FormattedCheckpoint::contains(const std::string& label) const { return records_.find(label) != records_.end(); }

long long FormattedCheckpoint::integer(const std::string& label) const {
    return get<long long>(label, "an integer scalar");
}

double FormattedCheckpoint::real(const std::string& label) const { return get<double>(label, "a real scalar"); }

const std::vector<long long>& FormattedCheckpoint::integers(const std::string& label) const {
    return get<std::vector<long long>>(label, "an integer array");
}

const std::vector<double>& FormattedCheckpoint::reals(const std::string& label) const {
    return get<std::vector<double>>(label, "a real array");
}

}  // namespace chem::kumo
