// Control-flow tests of the harness with mock benchmarks, after
// shared/tests/hpcc_base_benchmark_test.cpp:20-351: setup, test-only mode,
// failed validation, exceptions in a stage, option errors, the JSON dump.
// Built and run by tests/test_harness.py (no GPU needed: the mocks are set up
// in --test mode, which creates no device context).
#include <cstdio>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "hpcc_benchmark.hpp"

using hpcc_base::BaseSettings;

class MockBenchmark : public hpcc_base::HpccFpgaBenchmark<BaseSettings, int> {
protected:
    void addAdditionalParseOptions(hpcc_base::Options&) override {}
    std::string programName() const override { return "MOCK"; }
    std::string programDescription() const override { return "Mock benchmark\n"; }

public:
    bool returnInputData = true, returnExecuteKernel = true, returnValidate = true, configurationCheckSucceeds = true;
    int generateInputDatacalled = 0, executeKernelcalled = 0, validateOutputcalled = 0;

    std::unique_ptr<int> generateInputData() override {
        if (!returnInputData) throw std::runtime_error("Test input data failed");
        generateInputDatacalled++;
        return std::unique_ptr<int>(new int(0));
    }
    void executeKernel(int&) override {
        if (!returnExecuteKernel) throw std::runtime_error("Test execute kernel failed");
        executeKernelcalled++;
        timings["kernel"] = {0.5, 0.25};
    }
    bool validateOutput(int&) override {
        validateOutputcalled++;
        errors["residual"] = 1e-7;
        return returnValidate;
    }
    void printError() override {}
    bool checkInputParameters() override { return configurationCheckSucceeds; }
    void collectResults() override { results.emplace("gflops", hpcc_base::HpccResult(1.5, "GFLOP/s")); }
    void printResults() override {}

    bool setup(std::vector<std::string> args) {
        std::vector<const char*> argv{"mock"};
        for (auto& a : args) argv.push_back(a.c_str());
        return setupBenchmark((int)argv.size(), argv.data());
    }
};

static int failures = 0;
#define CHECK(cond)                                                                     \
    do {                                                                                \
        if (!(cond)) {                                                                  \
            std::cerr << "FAIL " << __func__ << ":" << __LINE__ << ": " #cond << "\n"; \
            failures++;                                                                 \
        }                                                                               \
    } while (0)

static void SetupSucceedsInTestMode() {
    MockBenchmark bm;
    CHECK(bm.setup({"-f", "kernel_CUDA.bin", "--test"}));
    CHECK(bm.getExecutionSettings().programSettings->kernelFileName == "kernel_CUDA.bin");
    CHECK(bm.getExecutionSettings().programSettings->numRepetitions == 10);
}

static void NothingExecutedWhenTestOnly() {
    MockBenchmark bm;
    bm.setup({"-f", "k", "--test"});
    CHECK(bm.executeBenchmark());
    CHECK(bm.generateInputDatacalled == 0 && bm.executeKernelcalled == 0 && bm.validateOutputcalled == 0);
}

static void AllExecutedWhenNotTestOnly() {
    MockBenchmark bm;
    bm.setup({"-f", "k", "--test"});
    bm.getExecutionSettings().programSettings->testOnly = false;
    CHECK(bm.executeBenchmark());
    CHECK(bm.generateInputDatacalled == 1 && bm.executeKernelcalled == 1 && bm.validateOutputcalled == 1);
}

static void SkipValidation() {
    MockBenchmark bm;
    bm.setup({"-f", "k", "--test", "--skip-validation"});
    bm.getExecutionSettings().programSettings->testOnly = false;
    bm.returnValidate = true;
    CHECK(!bm.executeBenchmark());  // not validated -> reported as failure, as in the reference
    CHECK(bm.validateOutputcalled == 0);
}

static void SuccessfulExeFailedVal() {
    MockBenchmark bm;
    bm.setup({"-f", "k", "--test"});
    bm.getExecutionSettings().programSettings->testOnly = false;
    bm.returnValidate = false;
    CHECK(!bm.executeBenchmark());
}

static void ExceptionInStageFailsExecution() {
    MockBenchmark a, b;
    a.setup({"-f", "k", "--test"});
    a.getExecutionSettings().programSettings->testOnly = false;
    a.returnInputData = false;
    CHECK(!a.executeBenchmark());
    b.setup({"-f", "k", "--test"});
    b.getExecutionSettings().programSettings->testOnly = false;
    b.returnExecuteKernel = false;
    CHECK(!b.executeBenchmark());
    CHECK(b.validateOutputcalled == 0);
}

static void ExecutionFailsWhenSetupFails() {
    MockBenchmark bm;
    bm.configurationCheckSucceeds = false;
    CHECK(!bm.setup({"-f", "k", "--test"}));
    CHECK(!bm.executeBenchmark());
}

static void OptionErrors() {
    MockBenchmark missing, unknown, badint, badcomm;
    CHECK(!missing.setup({"--test"}));
    CHECK(!unknown.setup({"-f", "k", "--test", "--no-such-option"}));
    CHECK(!badint.setup({"-f", "k", "--test", "-n", "ten"}));
    CHECK(!badcomm.setup({"-f", "k", "--test", "--comm-type", "NOPE"}));
}

static void CommTypeAutoDetect() {
    MockBenchmark a, b;
    CHECK(a.setup({"-f", "hpl_torus_PCIE.aocx", "--test", "--comm-type", "AUTO"}));
    CHECK(a.getExecutionSettings().programSettings->communicationType == hpcc_base::CommunicationType::pcie_mpi);
    CHECK(b.setup({"-f", "liblpcuda_CUDA", "--test", "--comm-type", "AUTO"}));
    CHECK(b.getExecutionSettings().programSettings->communicationType == hpcc_base::CommunicationType::cuda);
}

static void JsonDump(const std::string& dir) {
    MockBenchmark bm;
    const std::string path = dir + "/mock.json";
    bm.setup({"-f", "k", "--test", "--dump-json", path});
    bm.getExecutionSettings().programSettings->testOnly = false;
    CHECK(bm.executeBenchmark());
    std::ifstream in(path);
    std::stringstream ss;
    ss << in.rdbuf();
    const std::string j = ss.str();
    for (const char* key : {"\"name\":\"MOCK\"", "\"timings\":{\"kernel\":[{\"unit\":\"s\",\"value\":0.5}",
                            "\"results\":{\"gflops\":{\"unit\":\"GFLOP/s\",\"value\":1.5}}", "\"errors\":{",
                            "\"validated\":true", "\"settings\":{", "\"Repetitions\":10", "\"config_time\"",
                            "\"execution_time\"", "\"git_commit\"", "\"version\"", "\"device\"", "\"environment\""})
        CHECK(j.find(key) != std::string::npos);
}

int main(int argc, char** argv) {
    const std::string dir = argc > 1 ? argv[1] : ".";
    std::streambuf* old = std::cout.rdbuf();
    std::ostringstream sink;
    std::cout.rdbuf(sink.rdbuf());  // the harness's progress messages
    SetupSucceedsInTestMode();
    NothingExecutedWhenTestOnly();
    AllExecutedWhenNotTestOnly();
    SkipValidation();
    SuccessfulExeFailedVal();
    ExceptionInStageFailsExecution();
    ExecutionFailsWhenSetupFails();
    OptionErrors();
    CommTypeAutoDetect();
    JsonDump(dir);
    std::cout.rdbuf(old);
    std::cout << (failures == 0 ? "ALL PASSED" : "FAILURES: " + std::to_string(failures)) << std::endl;
    return failures == 0 ? 0 : 1;
}
