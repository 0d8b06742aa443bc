#pragma once

#include <cstddef>
#include <filesystem>
#include <string>
#include <unordered_map>
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
    void parse(std::istream& input, std::size_t logical_size, const std::string& name);
    enum class Kind { IntegerScalar, RealScalar, IntegerArray, RealArray };
    struct Record {
        Kind kind{};
        long long integer_scalar = 0;
        double real_scalar = 0.0;
        std::vector<long long> integer_array;
        std::vector<double> real_array;
    };
    [[nodiscard]] const Record& record(const std::string& label) const;
    std::unordered_map<std::string, Record> records_;
};

}  // namespace chem::kumo
