// LinpackBenchmark on one CUDA device: the reference's LinpackProgramSettings,
// LinpackData and LinpackBenchmark (LINPACK/src/host/linpack_data.hpp:48-214,
// linpack_data.cpp:37-66, linpack_benchmark.hpp:50-578) over the C ABI of
// liblpcuda.so.  Options, console tables, result keys and the validation
// criterion are the reference's; additions are marked as such.
#pragma once

#include <cfloat>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <iomanip>
#include <iostream>
#include <limits>
#include <memory>
#include <string>
#include <vector>

#include "hpcc_benchmark.hpp"

namespace linpack {

using hpcc_base::check_lp;
using hpcc_base::CommunicationType;
using hpcc_base::HpccResult;

// linpack_data.hpp:48-114, linpack_data.cpp:37-66
class LinpackProgramSettings : public hpcc_base::BaseSettings {
public:
    unsigned matrixSize;
    unsigned blockSize;
    bool isDiagonallyDominant;
    bool isEmulationKernel;
    int torus_row = 0, torus_col = 0, torus_width = 1, torus_height = 1;
    // Additions of this build: trailing-update precision, input generator.
    std::string precision;
    std::string generator;
    unsigned seed;
    double margin;
    int maxRefinements;

    explicit LinpackProgramSettings(const hpcc_base::Options::Result& r)
        : hpcc_base::BaseSettings(r),
          matrixSize((unsigned)r.integer("m") * (1u << (unsigned)r.integer("b"))),
          blockSize(1u << (unsigned)r.integer("b")),
          isDiagonallyDominant(r.count("uniform") == 0),
          isEmulationKernel(r.count("emulation") > 0),
          torus_width((int)r.integer("p")),
          precision(r.str("precision")),
          generator(r.str("generator")),
          seed((unsigned)r.integer("seed")),
          margin(r.real("margin")),
          maxRefinements((int)r.integer("max-refinements")) {
        const int mpi_size = 1;
        if (torus_width <= 0 || mpi_size % torus_width != 0)
            throw std::runtime_error("MPI size not dividable by P=" + std::to_string(torus_width) + "!");
        torus_height = mpi_size / torus_width;
        if (precision != "f32" && precision != "bf16" && precision != "fp8" && precision != "f32_bf16x6" &&
            precision != "f64")
            throw std::runtime_error("Unknown precision '" + precision + "' (f32, bf16, fp8, f32_bf16x6, f64)");
        if (generator != "reference" && generator != "baseline")
            throw std::runtime_error("Unknown generator '" + generator + "' (reference, baseline)");
    }

    std::map<std::string, std::string> getSettingsMap() override {
        auto map = hpcc_base::BaseSettings::getSettingsMap();
        map["Matrix Size"] = std::to_string(matrixSize);
        map["Block Size"] = std::to_string(blockSize);
        map["Emulate"] = isEmulationKernel ? "Yes" : "No";
        map["Diagonally Dominant"] = isDiagonallyDominant ? "Yes" : "No";
        map["Data Type"] = precision == "f64" ? "double" : "float";
        map["FPGA Torus"] = "P=" + std::to_string(torus_width) + ", Q=" + std::to_string(torus_height);
        map["Precision"] = precision;
        map["Generator"] = generator;
        return map;
    }
};

// linpack_data.hpp:120-214: host buffers, page-locked through lp_host_alloc
// when a device is present (the reference uses posix_memalign(4096)).
class LinpackData {
public:
    float* A = nullptr;
    float* b = nullptr;
    int* ipvt = nullptr;
    std::vector<double> b64;  // FP64 right-hand side of the seeded generator (addition)
    double* A64 = nullptr;    // the double build's matrix and right-hand side (--precision f64)
    double* bd = nullptr;
    double norma64 = 0.0, normb64 = 0.0;
    void use_f64() {
        A64 = static_cast<double*>(alloc(sizeof(double) * matrix_width * matrix_height));
        bd = static_cast<double*>(alloc(sizeof(double) * matrix_width));
    }
    size_t matrix_width, matrix_height;
    float norma = 0.0f, normb = 0.0f;

    LinpackData(size_t width, size_t height) : matrix_width(width), matrix_height(height) {
        A = static_cast<float*>(alloc(sizeof(float) * width * height));
        b = static_cast<float*>(alloc(sizeof(float) * width));
        ipvt = static_cast<int*>(alloc(sizeof(int) * height));
    }
    ~LinpackData() {
        release(A);
        release(b);
        release(ipvt);
        if (A64 != nullptr) release(A64);
        if (bd != nullptr) release(bd);
    }
    LinpackData(const LinpackData&) = delete;
    LinpackData& operator=(const LinpackData&) = delete;

private:
    std::vector<std::pair<void*, bool>> owned_;
    void* alloc(size_t bytes) {
        void* p = nullptr;
        if (lp_host_alloc(bytes, &p) == LP_OK) {
            owned_.push_back({p, true});
            return p;
        }
        if (posix_memalign(&p, 4096, bytes) != 0) throw std::bad_alloc();
        owned_.push_back({p, false});
        return p;
    }
    void release(void* p) {
        for (auto& o : owned_)
            if (o.first == p) {
                if (o.second)
                    lp_host_free(p);
                else
                    std::free(p);
                o.first = nullptr;
            }
    }
};

namespace execution {
namespace cuda {
// The CUDA execution backend, in place of execution::pcie::calculate
// (execution_types/execution_pcie.hpp:53-728): returns {"gefa", "gesl"}
// timings per repetition; data.A becomes the factors, data.b the solution.
inline std::map<std::string, std::vector<double>> calculate(
    const hpcc_base::ExecutionSettings<LinpackProgramSettings>& config, LinpackData& data) {
    const auto& s = *config.programSettings;
    std::vector<double> gefa(s.numRepetitions), gesl(s.numRepetitions);
    check_lp(lp_calculate(config.context, (int)s.matrixSize, (int)data.matrix_width, (int)s.blockSize,
                          (int)s.numRepetitions, data.A, data.b, gefa.data(), gesl.data()),
             "lp_calculate");
    return {{"gefa", gefa}, {"gesl", gesl}};
}

// Matrices without diagonal dominance (--uniform): partial pivoting with
// the reference's gefa_ref / gesl_ref convention (linpack_data.cpp:72-156);
// data.ipvt receives the pivots.
inline std::map<std::string, std::vector<double>> calculate_pvt(
    const hpcc_base::ExecutionSettings<LinpackProgramSettings>& config, LinpackData& data) {
    const auto& s = *config.programSettings;
    std::vector<double> gefa(s.numRepetitions), gesl(s.numRepetitions);
    check_lp(lp_calculate_pvt(config.context, (int)s.matrixSize, (int)data.matrix_width, (int)s.numRepetitions, data.A,
                              data.b, data.ipvt, gefa.data(), gesl.data()),
             "lp_calculate_pvt");
    return {{"gefa", gefa}, {"gesl", gesl}};
}

// The reference's double build (DATA_TYPE double): factors and solution in
// double (data.A64, data.bd); FP64 block size 256 (128 for -b 7, 64 for -b 6).
inline std::map<std::string, std::vector<double>> calculate_f64(
    const hpcc_base::ExecutionSettings<LinpackProgramSettings>& config, LinpackData& data) {
    const auto& s = *config.programSettings;
    const int bs = s.blockSize >= 256 ? 256 : s.blockSize >= 128 ? 128 : (int)s.blockSize;
    std::vector<double> gefa(s.numRepetitions), gesl(s.numRepetitions);
    check_lp(lp_calculate_f64(config.context, (int)s.matrixSize, (int)data.matrix_width, bs, (int)s.numRepetitions,
                              data.A64, data.bd, gefa.data(), gesl.data()),
             "lp_calculate_f64");
    return {{"gefa", gefa}, {"gesl", gesl}};
}

// Mixed precision (addition): tensor-core trailing updates, FP64 refinement.
inline std::map<std::string, std::vector<double>> calculate_mixed(
    const hpcc_base::ExecutionSettings<LinpackProgramSettings>& config, LinpackData& data, int* iters,
    double* hpl_resid) {
    const auto& s = *config.programSettings;
    const int prec = s.precision == "bf16" ? LP_BF16_IR : s.precision == "fp8" ? LP_FP8_IR : LP_F32_BF16X6;
    const int n = (int)s.matrixSize;
    std::vector<double> b64(n), x(n);
    for (int i = 0; i < n; i++) b64[i] = data.b64.empty() ? (double)data.b[i] : data.b64[i];
    std::vector<double> gefa, gesl;
    for (unsigned rep = 0; rep < s.numRepetitions; rep++) {
        lp_timing t;
        check_lp(lp_solve_host(config.context, prec, n, (int)s.blockSize, data.A, (int)data.matrix_width, b64.data(),
                               1, x.data(), s.maxRefinements, &t),
                 "lp_solve_host");
        gefa.push_back(t.gefa_s);
        gesl.push_back(t.gesl_s + t.ir_s);
        *iters = t.ir_iters;
        *hpl_resid = t.hpl_resid;
    }
    for (int i = 0; i < n; i++) data.b[i] = (float)x[i];
    return {{"gefa", gefa}, {"gesl", gesl}};
}
}  // namespace cuda
}  // namespace execution

class LinpackBenchmark : public hpcc_base::HpccFpgaBenchmark<LinpackProgramSettings, LinpackData> {
    int ir_iterations_ = -1;
    double hpl_resid_ = -1.0;

protected:
    std::string programName() const override { return "LINPACK"; }
    std::string programDescription() const override {
        return "Implementation of the LINPACK benchmark proposed in the HPCC benchmark suite for FPGA.\n"
               "Version: " HPCC_VERSION "\n";
    }

    // linpack_benchmark.hpp:60-71 (+ additions after --emulation)
    void addAdditionalParseOptions(hpcc_base::Options& o) override {
        o.value("m", "Global matrix size in number of blocks in one dimension. Local matrix sizes will be determined by "
                     "PQ grid.",
                "2")
            .value("b", "Log2 of the block size in number of values in one dimension", "5")
            .value("p", "Width of the FPGA grid. The heigth (Q) will be calculated from mpi_size / P.", "1")
            .flag("uniform", "Generate a uniform matrix instead of a diagonally dominant. This has to be supported by "
                             "the FPGA kernel!")
            .flag("emulation", "Use kernel arguments for emulation. This may be necessary to simulate persistent local "
                               "memory on the FPGA")
            .value("precision",
                   "Trailing-update precision: f32, bf16, fp8 (bf16/fp8 refine in FP64), f32_bf16x6 (FP32 emulated "
                   "on the BF16 tensor cores; refines only if --max-refinements > 0 and needed) or f64 (the "
                   "reference's double build: input, factors and solution in double)",
                   "f32")
            .value("generator", "Input generator: reference (mt19937(0), U(0,1)) or baseline (seeded, U[-0.5,0.5))",
                   "reference")
            .value("seed", "Seed of the baseline generator", "42")
            .value("margin", "Diagonal-dominance margin of the baseline generator", "1")
            .value("max-refinements", "Maximum FP64 refinement iterations (bf16/fp8)", "50");
    }

public:
    // linpack_benchmark.hpp:211-297 (one rank)
    std::unique_ptr<LinpackData> generateInputData() override {
        const auto& s = *executionSettings->programSettings;
        const int n = (int)s.matrixSize;
        std::unique_ptr<LinpackData> d(new LinpackData(n, n));
        if (s.generator == "reference") {
            check_lp(lp_generate_reference(d->A, d->b, n, s.isDiagonallyDominant ? 1 : 0, &d->norma, &d->normb),
                     "lp_generate_reference");
        } else {
            d->b64.resize(n);
            check_lp(lp_generate_baseline(d->A, d->b64.data(), d->b, n, s.seed, s.margin), "lp_generate_baseline");
            d->normb = 0.0f;
            for (int i = 0; i < n; i++) d->normb = d->b[i] > d->normb ? d->b[i] : d->normb;
        }
        for (int i = 0; i < n; i++) d->ipvt[i] = i;
        if (s.precision == "f64") {  // the double build's own input
            d->use_f64();
            if (s.generator == "reference") {
                check_lp(lp_generate_reference_f64(d->A64, d->bd, n, s.isDiagonallyDominant ? 1 : 0, &d->norma64,
                                                   &d->normb64),
                         "lp_generate_reference_f64");
            } else {
                d->normb64 = 0.0;
                for (size_t i = 0; i < (size_t)n * n; i++) d->A64[i] = d->A[i];
                for (int i = 0; i < n; i++) {
                    d->bd[i] = d->b64[i];
                    d->normb64 = d->bd[i] > d->normb64 ? d->bd[i] : d->normb64;
                }
            }
        }
        return d;
    }

    // linpack_benchmark.hpp:306-324
    void executeKernel(LinpackData& data) override {
        const auto& s = *executionSettings->programSettings;
        if (!s.isDiagonallyDominant && s.precision != "f32")
            throw std::runtime_error("Uniform (non diagonally dominant) matrices are solved with partial pivoting in "
                                     "FP32 only (--precision f32)");
        switch (s.communicationType) {
            case CommunicationType::cuda:
                if (s.precision == "f64") {
                    this->timings = execution::cuda::calculate_f64(*executionSettings, data);
                    break;
                }
                if (!s.isDiagonallyDominant)
                    this->timings = execution::cuda::calculate_pvt(*executionSettings, data);
                else if (s.precision == "f32")
                    this->timings = execution::cuda::calculate(*executionSettings, data);
                else
                    this->timings = execution::cuda::calculate_mixed(*executionSettings, data, &ir_iterations_,
                                                                     &hpl_resid_);
                break;
            default:
                throw std::runtime_error("No calculate method implemented for communication type " +
                                         hpcc_base::commToString(s.communicationType));
        }
        // The substitution ran on the device: data.b already holds x (the
        // reference's distributed_gesl_nopvt_ref, :321-323, is not needed).
    }

    // linpack_benchmark.hpp:334-469 (DISTRIBUTED_VALIDATION, one rank)
    bool validateOutput(LinpackData& data) override {
        const unsigned n = executionSettings->programSettings->matrixSize;
        const bool f64 = data.bd != nullptr;
        double resid = 0.0;
        for (size_t i = 0; i < data.matrix_width; i++) {
            const double e = std::abs((f64 ? data.bd[i] : (double)data.b[i]) - 1.0);
            resid = resid > e ? resid : e;
        }
        const double normx = f64 ? data.normb64 : data.normb;
        const double eps = f64 ? std::numeric_limits<double>::epsilon() : std::numeric_limits<float>::epsilon();
        const double residn = resid / (static_cast<double>(n) * normx * eps);
        errors.emplace("epsilon", eps);
        errors.emplace("residual", resid);
        errors.emplace("residual_norm", residn);
        if (hpl_resid_ >= 0.0) errors.emplace("hpl_resid_norm", hpl_resid_);
        return residn < 1;
    }

    void printError() override {
        std::cout << std::setw(ENTRY_SPACE) << " norm. residual" << std::setw(ENTRY_SPACE) << " res. error"
                  << std::setw(ENTRY_SPACE) << " mach. eps" << std::endl;
        std::cout << std::setw(ENTRY_SPACE) << errors.at("residual_norm") << std::setw(ENTRY_SPACE)
                  << errors.at("residual") << std::setw(ENTRY_SPACE) << errors.at("epsilon") << std::endl;
    }

    // linpack_benchmark.hpp:480-538 (+ gesl_GBps, ir_iterations for the mixed forms)
    void collectResults() override {
        const auto& lu_t = timings["gefa"];
        const auto& sl_t = timings["gesl"];
        double t = 0, tlu = 0, tsl = 0;
        double tmin = std::numeric_limits<double>::max(), lu_min = tmin, sl_min = tmin;
        const double nn = executionSettings->programSettings->matrixSize;
        const double gflop_lu = ((2.0e0 * nn * nn * nn) / 3.0) / 1.0e9;
        const double gflop_sl = (2.0 * (nn * nn)) / 1.0e9;
        for (size_t i = 0; i < lu_t.size(); i++) {
            const double cur = lu_t[i] + sl_t[i];
            t += cur;
            tlu += lu_t[i];
            tsl += sl_t[i];
            tmin = cur < tmin ? cur : tmin;
            lu_min = lu_t[i] < lu_min ? lu_t[i] : lu_min;
            sl_min = sl_t[i] < sl_min ? sl_t[i] : sl_min;
        }
        const double reps = (double)lu_t.size();
        results.emplace("t_mean", HpccResult(t / reps, "s"));
        results.emplace("t_min", HpccResult(tmin, "s"));
        results.emplace("tlu_mean", HpccResult(tlu / reps, "s"));
        results.emplace("tlu_min", HpccResult(lu_min, "s"));
        results.emplace("tsl_mean", HpccResult(tsl / reps, "s"));
        results.emplace("tsl_min", HpccResult(sl_min, "s"));
        results.emplace("gflops", HpccResult((gflop_lu + gflop_sl) / tmin, "GFLOP/s"));
        results.emplace("gflops_lu", HpccResult(gflop_lu / lu_min, "GFLOP/s"));
        results.emplace("gflops_sl", HpccResult(gflop_sl / sl_min, "GFLOP/s"));
        if (executionSettings->programSettings->precision == "f32")
            results.emplace("gesl_GBps", HpccResult(4.0 * nn * nn / sl_min / 1e9, "GB/s"));
        if (ir_iterations_ >= 0) results.emplace("ir_iterations", HpccResult(ir_iterations_, ""));
    }

    // linpack_benchmark.hpp:540-561
    void printResults() override {
        std::cout << std::left << std::setw(ENTRY_SPACE) << " Method" << std::setw(ENTRY_SPACE) << " best"
                  << std::setw(ENTRY_SPACE) << " mean" << std::setw(ENTRY_SPACE) << " GFLOPS" << std::endl;
        std::cout << std::left << std::setw(ENTRY_SPACE) << " total" << results.at("t_min") << results.at("t_mean")
                  << results.at("gflops") << std::endl;
        std::cout << std::left << std::setw(ENTRY_SPACE) << " GEFA" << results.at("tlu_min") << results.at("tlu_mean")
                  << results.at("gflops_lu") << std::endl;
        std::cout << std::left << std::setw(ENTRY_SPACE) << " GESL" << results.at("tsl_min") << results.at("tsl_mean")
                  << results.at("gflops_sl") << std::right << std::endl;
    }

    LinpackBenchmark(int argc, char* argv[]) { this->setupBenchmark(argc, argv); }
};

}  // namespace linpack
