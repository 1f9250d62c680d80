// Test infrastructure only (oracle build). Minimal stand-in for the harness
// header that LINPACK/src/host/linpack_data.cpp includes, so that the
// reference's gefa_ref / gesl_ref / gefa_ref_nopvt / gesl_ref_nopvt compile
// unmodified from their own source file without MPI, OpenCL or cxxopts.
// Only the names that linpack_data.{hpp,cpp} touch are provided:
//   cl_int, uint, STR(), MPI_Comm_rank/size, cxxopts::ParseResult,
//   hpcc_base::BaseSettings (LINPACK/src/host/linpack_data.cpp:37-66).
#ifndef ORACLE_REFSTUB_HPCC_BENCHMARK_HPP
#define ORACLE_REFSTUB_HPCC_BENCHMARK_HPP

#include <cmath>
#include <cstdint>
#include <iostream>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

typedef int32_t cl_int;
typedef unsigned int uint;

#define STR_EXPAND(tok) #tok
#define STR(tok) STR_EXPAND(tok)

typedef int MPI_Comm;
#define MPI_COMM_WORLD 0
inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return 0; }
inline int MPI_Comm_size(MPI_Comm, int* s) { *s = 1; return 0; }

namespace cxxopts {
struct OptionValue {
    unsigned v = 0;
    template <class T> T as() const { return static_cast<T>(v); }
};
struct ParseResult {
    std::map<std::string, OptionValue> values;
    OptionValue operator[](const std::string& k) const {
        auto it = values.find(k);
        return it == values.end() ? OptionValue{} : it->second;
    }
    size_t count(const std::string& k) const { return values.count(k); }
};
}  // namespace cxxopts

namespace hpcc_base {
class BaseSettings {
public:
    explicit BaseSettings(cxxopts::ParseResult&) {}
    virtual ~BaseSettings() = default;
    virtual std::map<std::string, std::string> getSettingsMap() { return {}; }
};
}  // namespace hpcc_base

#endif
