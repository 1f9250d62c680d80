// The benchmark harness of HPCC_FPGA re-implemented for one CUDA device:
// the same virtual interface (generateInputData / executeKernel /
// validateOutput / printError / collectResults / printResults /
// checkInputParameters), the same base command-line options, the same
// control flow and console messages of executeBenchmark, and the same JSON
// dump layout.  Reference: shared/include/hpcc_benchmark.hpp:101-755,
// shared/include/hpcc_settings.hpp, shared/hpcc_settings.cpp:15-86,
// shared/include/communication_types.hpp:35-133.
// MPI, OpenCL and XRT are gone: one process drives one GPU through the C ABI
// of liblpcuda.so (include/lpcuda.h).
#pragma once

#include <chrono>
#include <cstdlib>
#include <ctime>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "cli.hpp"
#include "json_writer.hpp"
#include "lpcuda.h"

#define VALUE_SPACE 11
#define UNIT_SPACE 8
#define ENTRY_SPACE (VALUE_SPACE + UNIT_SPACE + 1)
#define HLINE "-------------------------------------------------------------\n"
#define HPCC_VERSION "2.6"

namespace hpcc_base {

// communication_types.hpp:35-133, plus the CUDA backend of this build.
enum class CommunicationType { intel_external_channels, pcie_mpi, accl, cpu_only, udp, aurora, cuda, unsupported, automatic };

inline const std::map<std::string, CommunicationType>& comm_map() {
    static const std::map<std::string, CommunicationType> m{
        {"IEC", CommunicationType::intel_external_channels}, {"PCIE", CommunicationType::pcie_mpi},
        {"ACCL", CommunicationType::accl}, {"CPU", CommunicationType::cpu_only},
        {"UNSUPPORTED", CommunicationType::unsupported}, {"UDP", CommunicationType::udp},
        {"AURORA", CommunicationType::aurora}, {"CUDA", CommunicationType::cuda},
        {"AUTO", CommunicationType::automatic}};
    return m;
}

inline std::string commToString(CommunicationType c) {
    for (const auto& e : comm_map())
        if (e.second == c) return e.first;
    throw std::runtime_error("Communication type could not be converted to string!");
}

inline CommunicationType retrieveCommunicationType(const std::string& name, const std::string& kernel_file) {
    auto it = comm_map().find(name);
    if (it == comm_map().end())
        throw std::runtime_error("Communication type could not be converted from string: " + name);
    if (it->second != CommunicationType::automatic) return it->second;
    for (const auto& e : comm_map())
        if (kernel_file.find(e.first) != std::string::npos) return e.second;
    throw std::runtime_error("Communication type could not be autodetected from kernel_filename: " + kernel_file);
}

class SetupException : public std::runtime_error {
public:
    using std::runtime_error::runtime_error;
};

// HpccResult (hpcc_benchmark.hpp:70-92): value and unit, printed in fixed columns.
class HpccResult {
public:
    double value;
    std::string unit;
    HpccResult(double v, std::string u) : value(v), unit(std::move(u)) {}
    friend std::ostream& operator<<(std::ostream& os, const HpccResult& r) {
        os << std::setw(VALUE_SPACE) << r.value << " " << std::left << std::setw(UNIT_SPACE) << r.unit << std::right;
        return os;
    }
};

// BaseSettings (hpcc_settings.hpp, hpcc_settings.cpp:15-86).
class BaseSettings {
public:
    unsigned numRepetitions = 10;
    bool useMemoryInterleaving = true;
    bool skipValidation = false;
    int defaultPlatform = -1;
    std::string platformString;
    int defaultDevice = -1;
    std::string kernelFileName;
    unsigned kernelReplications = 1;
    bool testOnly = false;
    std::string dumpfilePath;
    CommunicationType communicationType = CommunicationType::cuda;

    explicit BaseSettings(const Options::Result& r)
        : numRepetitions((unsigned)r.integer("n")), skipValidation(r.count("skip-validation") > 0),
          defaultPlatform((int)r.integer("platform")), platformString(r.str("platform_str")),
          defaultDevice((int)r.integer("device")), kernelFileName(r.str("f")),
          kernelReplications(r.count("r") > 0 ? (unsigned)r.integer("r") : 1), testOnly(r.count("test") > 0),
          dumpfilePath(r.str("dump-json")),
          communicationType(retrieveCommunicationType(r.str("comm-type"), r.str("f"))) {}
    virtual ~BaseSettings() = default;

    virtual std::map<std::string, std::string> getSettingsMap() {
        return {{"Repetitions", std::to_string(numRepetitions)},
                {"Kernel Replications", std::to_string(kernelReplications)},
                {"Kernel File", kernelFileName},
                {"MPI Ranks", "1"},
                {"Test Mode", testOnly ? "Yes" : "No"},
                {"Communication Type", commToString(communicationType)}};
    }
};

// ExecutionSettings (hpcc_settings.hpp): the parsed settings and the device.
template <class TSettings>
class ExecutionSettings {
public:
    std::unique_ptr<TSettings> programSettings;
    lp_ctx* context = nullptr;
    std::string deviceName;

    ExecutionSettings(std::unique_ptr<TSettings> s, lp_ctx* ctx, std::string name)
        : programSettings(std::move(s)), context(ctx), deviceName(std::move(name)) {}
    ~ExecutionSettings() {
        if (context != nullptr) lp_ctx_destroy(context);
    }
    ExecutionSettings(const ExecutionSettings&) = delete;
    ExecutionSettings& operator=(const ExecutionSettings&) = delete;
    std::string getDeviceName() const { return programSettings->testOnly ? "TEST RUN: Not selected!" : deviceName; }
};

template <class TSettings>
std::ostream& operator<<(std::ostream& os, const ExecutionSettings<TSettings>& es) {
    os << std::left;
    for (const auto& k : es.programSettings->getSettingsMap()) os << std::setw(2 * ENTRY_SPACE) << k.first << k.second << std::endl;
    os << std::setw(2 * ENTRY_SPACE) << "Device" << es.getDeviceName() << std::endl;
    os << std::right;
    return os;
}

// Throws std::runtime_error for a non-zero lpcuda status (the reference's
// ASSERT_CL -> exception convention, shared/include/setup/fpga_setup.hpp:80,125).
inline void check_lp(int status, const std::string& where) {
    if (status != LP_OK)
        throw std::runtime_error(where + ": " + lp_strerror(status) + " (" + std::to_string(status) +
                                 "): " + lp_last_error());
}

template <class TSettings, class TData>
class HpccFpgaBenchmark {
private:
    bool benchmark_setup_succeeded = false;

protected:
    std::unique_ptr<ExecutionSettings<TSettings>> executionSettings;
    int mpi_comm_rank = 0;
    int mpi_comm_size = 1;
    std::map<std::string, std::vector<double>> timings;
    std::map<std::string, HpccResult> results;
    std::map<std::string, double> errors;
    bool validated = false;

    virtual void addAdditionalParseOptions(Options& options) = 0;
    virtual std::string programName() const = 0;
    virtual std::string programDescription() const = 0;

public:
    virtual std::unique_ptr<TData> generateInputData() = 0;
    virtual void executeKernel(TData& data) = 0;
    virtual bool validateOutput(TData& data) = 0;
    virtual void printError() = 0;
    virtual void collectResults() = 0;
    virtual void printResults() = 0;
    virtual bool checkInputParameters() { return true; }

    // hpcc_benchmark.hpp:243-325
    std::unique_ptr<TSettings> parseProgramParameters(int argc, char const* const* argv) {
        std::stringstream ss;
        ss << programDescription() << "Config. Time: " << __DATE__ << " " << __TIME__ << std::endl
           << "Git Commit:   " << gitCommit() << std::endl;
        Options options(argv[0], ss.str());
        options.value("f,file", "Kernel file name")
            .value("n", "Number of repetitions", "10")
            .flag("i", "Use memory Interleaving")
            .flag("skip-validation",
                  "Skip the validation of the output data. This will speed up execution and helps when working with "
                  "special data types.")
            .value("device",
                   "Index of the device that has to be used. If not given you will be asked which device to use if "
                   "there are multiple devices available.",
                   "-1")
            .value("platform",
                   "Index of the platform that has to be used. If not given you will be asked which platform to use "
                   "if there are multiple platforms available.",
                   "-1")
            .value("platform_str", "Name of the platform that has to be used", "")
            .value("r", "Number of used kernel replications", "1")
            .value("comm-type", "Used communication type for inter-FPGA communication", "CUDA")
            .value("dump-json", "dump benchmark configuration and results to this file in json format", "")
            .flag("test", "Only test given configuration and skip execution and validation")
            .flag("h,help", "Print this help");
        addAdditionalParseOptions(options);
        try {
            Options::Result result = options.parse(argc, argv);
            if (result.count("h")) {
                std::cout << options.help() << std::endl;
                std::exit(0);
            }
            if (result.count("f") <= 0)
                throw SetupException("Mandatory option is missing! Use -h to show all available options. ERROR: "
                                     "Kernel file must be given with option -f!");
            return std::unique_ptr<TSettings>(new TSettings(result));
        } catch (const OptionError& e) {
            throw SetupException("Input parameters could not be parsed! Use -h to show all available options. ERROR: " +
                                 std::string(e.what()));
        }
    }

    void printFinalConfiguration() {
        std::cout << programDescription();
        std::cout << "Config. Time: " << __DATE__ << " " << __TIME__ << std::endl;
        std::cout << "Git Commit:   " << gitCommit() << std::endl << std::endl;
        std::cout << "Summary:" << std::endl;
        std::cout << *executionSettings << std::endl;
    }

    static std::string gitCommit() {
        const char* g = std::getenv("LP_GIT_COMMIT");
        return g != nullptr ? g : "unknown";
    }

    Json getTimingsJson() {
        Json j = Json::object();
        for (const auto& key : timings) {
            Json list = Json::array();
            for (double t : key.second) {
                Json e = Json::object();
                e["unit"] = Json::string("s");
                e["value"] = Json::number(t);
                list.push_back(e);
            }
            j[key.first] = list;
        }
        return j;
    }

    Json getResultsJson() {
        Json j = Json::object();
        for (const auto& r : results) {
            Json e = Json::object();
            e["unit"] = Json::string(r.second.unit);
            e["value"] = Json::number(r.second.value);
            j[r.first] = e;
        }
        return j;
    }

    static Json parseFPGATorusString(const std::string& str) {
        Json j = Json::object();
        const size_t space = str.find(' ');
        const std::string p = str.substr(0, space), q = str.substr(space);
        j["P"] = Json::integer(std::stoi(p.substr(p.find('=') + 1, p.find(','))));
        j["Q"] = Json::integer(std::stoi(q.substr(q.find('=') + 1)));
        return j;
    }

    // hpcc_benchmark.hpp:439-472.  The reference's condition chain ends in
    // `|| "Dist. Buffers"` (a non-null pointer, always true), so every
    // setting that is not an integer is written as the boolean value=="Yes";
    // the layout is kept identical, quirk included.
    static Json jsonifySettingsMap(const std::map<std::string, std::string>& m) {
        Json j = Json::object();
        for (const auto& item : m) {
            try {
                size_t pos = 0;
                const int v = std::stoi(item.second, &pos);
                j[item.first] = Json::integer(v);
            } catch (const std::invalid_argument&) {
                if (item.first == "FPGA Torus")
                    j[item.first] = parseFPGATorusString(item.second);
                else
                    j[item.first] = Json::boolean(item.second == "Yes");
            }
        }
        return j;
    }

    static std::string getCurrentTime() {
        std::time_t t = std::time(nullptr);
        std::ostringstream oss;
        oss << std::put_time(std::gmtime(&t), "%a %b %d %T UTC %Y");
        return oss.str();
    }

    // hpcc_benchmark.hpp:490-516
    void dumpConfigurationAndResults(const std::string& file_path) {
        std::ofstream fs(file_path);
        if (!fs.is_open()) {
            std::cout << "Unable to open file for dumping configuration and results" << std::endl;
            return;
        }
        Json dump = Json::object();
        dump["name"] = Json::string(programName());
        dump["config_time"] = Json::string(std::string(__DATE__) + " " + __TIME__);
        dump["execution_time"] = Json::string(getCurrentTime());
        dump["git_commit"] = Json::string(gitCommit());
        dump["version"] = Json::string(HPCC_VERSION);
        dump["device"] = Json::string(executionSettings->getDeviceName());
        dump["settings"] = jsonifySettingsMap(executionSettings->programSettings->getSettingsMap());
        dump["timings"] = getTimingsJson();
        dump["results"] = getResultsJson();
        Json errs = Json::object();
        for (const auto& e : errors) errs[e.first] = Json::number(e.second);
        dump["errors"] = errs;
        dump["validated"] = Json::boolean(validated);
        Json env = Json::object();
        const char* ld = std::getenv("LD_LIBRARY_PATH");
        env["LD_LIBRARY_PATH"] = Json::string(ld != nullptr ? ld : "");
        dump["environment"] = env;
        fs << dump.dump();
    }

    // hpcc_benchmark.hpp:529-611: parse, select the device, print the configuration.
    bool setupBenchmark(int argc, char const* const* argv) {
        bool success = true;
        try {
            std::unique_ptr<TSettings> settings = parseProgramParameters(argc, argv);
            lp_ctx* ctx = nullptr;
            std::string name;
            if (!settings->testOnly) {
                const int dev = settings->defaultDevice < 0 ? 0 : settings->defaultDevice;
                check_lp(lp_ctx_create(dev, &ctx), "lp_ctx_create");
                char buf[256];
                check_lp(lp_ctx_device_name(ctx, buf, sizeof(buf)), "lp_ctx_device_name");
                name = buf;
            }
            executionSettings.reset(new ExecutionSettings<TSettings>(std::move(settings), ctx, name));
            if (mpi_comm_rank == 0) {
                if (!checkInputParameters()) {
                    std::cerr << "ERROR: Input parameter check failed!" << std::endl;
                    throw std::runtime_error("Input parameter check failed!");
                }
                printFinalConfiguration();
            }
        } catch (std::exception& e) {
            std::cerr << "An error occured while setting up the benchmark: " << std::endl;
            std::cerr << "\t" << e.what() << std::endl;
            success = false;
        }
        benchmark_setup_succeeded = success;
        return success;
    }

    // hpcc_benchmark.hpp:620-701
    bool executeBenchmark() {
        if (!benchmark_setup_succeeded) {
            std::cerr << "Benchmark execution started without successfully running the benchmark setup!" << std::endl;
            return false;
        }
        if (executionSettings->programSettings->testOnly) {
            std::cout << "TEST MODE ENABLED: SKIP DATA GENERATION, EXECUTION, AND VALIDATION!" << std::endl;
            std::cout << "SUCCESSFULLY parsed input parameters!" << std::endl;
            return benchmark_setup_succeeded;
        }
        std::cout << HLINE << "Start benchmark using the given configuration. Generating data..." << std::endl << HLINE;
        try {
            auto gen_start = std::chrono::high_resolution_clock::now();
            std::unique_ptr<TData> data = generateInputData();
            std::chrono::duration<double> gen_time = std::chrono::high_resolution_clock::now() - gen_start;
            std::cout << "Generation Time: " << gen_time.count() << " s" << std::endl;
            std::cout << HLINE << "Execute benchmark kernel..." << std::endl << HLINE;
            auto exe_start = std::chrono::high_resolution_clock::now();
            executeKernel(*data);
            std::chrono::duration<double> exe_time = std::chrono::high_resolution_clock::now() - exe_start;
            std::cout << "Execution Time: " << exe_time.count() << " s" << std::endl;
            std::cout << HLINE << "Validate output..." << std::endl << HLINE;
            if (!executionSettings->programSettings->skipValidation) {
                auto eval_start = std::chrono::high_resolution_clock::now();
                validated = validateOutput(*data);
                printError();
                std::chrono::duration<double> eval_time = std::chrono::high_resolution_clock::now() - eval_start;
                std::cout << "Validation Time: " << eval_time.count() << " s" << std::endl;
            }
            std::cout << HLINE << "Collect results..." << std::endl << HLINE;
            collectResults();
            if (executionSettings->programSettings->dumpfilePath.size() > 0)
                dumpConfigurationAndResults(executionSettings->programSettings->dumpfilePath);
            printResults();
            if (!validated)
                std::cerr << HLINE << "ERROR: VALIDATION OF OUTPUT DATA FAILED!" << std::endl;
            else
                std::cout << HLINE << "Validation: SUCCESS!" << std::endl;
            return validated;
        } catch (const std::exception& e) {
            std::cerr << "An error occured while executing the benchmark: " << std::endl;
            std::cerr << "\t" << e.what() << std::endl;
            return false;
        }
    }

    ExecutionSettings<TSettings>& getExecutionSettings() { return *executionSettings; }
    std::map<std::string, std::vector<double>>& getTimingsMap() { return timings; }

    // setupEnvironmentAndClocks (shared/setup/fpga_setup.cpp:320-322): numbers
    // on the console in 5-digit scientific notation.
    HpccFpgaBenchmark() { std::cout << std::setprecision(5) << std::scientific; }
    virtual ~HpccFpgaBenchmark() = default;
};

}  // namespace hpcc_base
