#pragma once

#include <cstddef>
#include <filesystem>
#include <string>
#include <map>
#include <string_view>
#include <variant>
#include <vector>

namespace chem::kumo {

/// Reader of the named integer and real records (scalars and arrays) of a
/// Gaussian formatted checkpoint file, plain or gzip-compressed (detected
/// from its content).  Same rules as chem-kumo's FormattedCheckpoint
/// (src/fchk.cpp:78-187): label in columns 0-42, type letter at column 43,
/// "N=" arrays, Fortran D exponents accepted, C/L/H records skipped, identical
/// duplicates accepted and conflicting ones rejected.  Errors throw
/// std::runtime_error with the reference's messages.
class FormattedCheckpoint {
public:
    explicit FormattedCheckpoint(const std::filesystem::path& path);
    /// Parse FCHK text that is already in memory.
    static FormattedCheckpoint from_text(const std::string& text, std::size_t logical_size);

    [[nodiscard]] bool contains(const std::string& label) const;
    [[nodiscard]] long long integer(const std::string& label) const;
    [[nodiscard]] double real(const std::string& label) const;
    [[nodiscard]] const std::vector<long long>& integers(const std::string& label) const;
    [[nodiscard]] const std::vector<double>& reals(const std::string& label) const;

private:
    FormattedCheckpoint() = default;
    // One record: integer scalar, real scalar, integer array or real array.
    using Value = std::variant<long long, double, std::vector<long long>, std::vector<double>>;
    void load(std::string_view text, std::size_t logical_size, const std::string& name);
    template <class T>
    [[nodiscard]] const T& get(const std::string& label, const char* what) const;
    std::map<std::string, Value, std::less<>> records_;
};

}  // namespace chem::kumo
