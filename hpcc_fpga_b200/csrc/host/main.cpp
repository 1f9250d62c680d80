// Program entry point (LINPACK/src/host/main.cpp:12-33): construct the
// benchmark from the command line, run it, exit 0 on validated results.
#include "linpack_benchmark.hpp"

int main(int argc, char* argv[]) {
    linpack::LinpackBenchmark bm(argc, argv);
    const bool success = bm.executeBenchmark();
    return success ? 0 : 1;
}
