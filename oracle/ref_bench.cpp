// ORACLE — test infrastructure only (see oracle/oracle.c).
//
// CPU baseline driver: times the reference's own gefa_ref_nopvt +
// gesl_ref_nopvt (LINPACK/src/host/linpack_data.cpp:166-229, compiled
// unmodified by oracle/Makefile) on one host core, on inputs from the
// oracle's restated generators, and prints one JSON object.  The GFLOP/s
// formula is the reference's (LINPACK/src/host/linpack_benchmark.hpp:509-535):
// gflop_lu = 2n^3/3/1e9, gflop_sl = 2n^2/1e9.
//
//   ref_bench --n N [--mode baseline|reference] [--reps R] [--seed S] [--margin M]
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "linpack_data.hpp"

extern "C" {
void orc_gen_reference_f32(float* A, float* b, int n, int diag_dominant, float* norma, float* normb);
void orc_gen_baseline(float* A, double* b64, float* b32, int n, unsigned seed, double margin);
}

int main(int argc, char** argv) {
    int n = 1024, reps = 1;
    unsigned seed = 42;
    double margin = 1.0;
    std::string mode = "baseline";
    for (int i = 1; i < argc; i++) {
        std::string a = argv[i];
        auto next = [&](void) -> const char* {
            if (i + 1 >= argc) { std::fprintf(stderr, "missing value for %s\n", a.c_str()); std::exit(2); }
            return argv[++i];
        };
        if (a == "--n") n = std::atoi(next());
        else if (a == "--reps") reps = std::atoi(next());
        else if (a == "--seed") seed = (unsigned)std::strtoul(next(), nullptr, 10);
        else if (a == "--margin") margin = std::atof(next());
        else if (a == "--mode") mode = next();
        else { std::fprintf(stderr, "unknown option %s\n", a.c_str()); return 2; }
    }
    if (n <= 0 || reps <= 0) { std::fprintf(stderr, "bad size\n"); return 2; }

    std::vector<float> A0((size_t)n * n), b0(n);
    std::vector<double> b64(n);
    float normb = 0.0f;
    if (mode == "reference") {
        float norma = 0.0f;
        orc_gen_reference_f32(A0.data(), b0.data(), n, 1, &norma, &normb);
    } else {
        orc_gen_baseline(A0.data(), b64.data(), b0.data(), n, seed, margin);
        for (int i = 0; i < n; i++) normb = b0[i] > normb ? b0[i] : normb;
    }

    std::vector<float> A((size_t)n * n), b(n);
    std::vector<double> tlu, tsl;
    double resid = 0.0;
    for (int r = 0; r < reps; r++) {
        std::memcpy(A.data(), A0.data(), sizeof(float) * A.size());
        std::memcpy(b.data(), b0.data(), sizeof(float) * b.size());
        auto t0 = std::chrono::steady_clock::now();
        linpack::gefa_ref_nopvt(A.data(), n, n);
        auto t1 = std::chrono::steady_clock::now();
        linpack::gesl_ref_nopvt(A.data(), b.data(), n, n);
        auto t2 = std::chrono::steady_clock::now();
        tlu.push_back(std::chrono::duration<double>(t1 - t0).count());
        tsl.push_back(std::chrono::duration<double>(t2 - t1).count());
    }
    for (int i = 0; i < n; i++) resid = std::fmax(resid, std::fabs((double)b[i] - 1.0));
    const double eps = 1.1920928955078125e-07;
    const double residn = resid / ((double)n * (double)normb * eps);

    double tmin = 1e300, lumin = 1e300, slmin = 1e300;
    for (int r = 0; r < reps; r++) {
        tmin = std::fmin(tmin, tlu[r] + tsl[r]);
        lumin = std::fmin(lumin, tlu[r]);
        slmin = std::fmin(slmin, tsl[r]);
    }
    const double nn = (double)n;
    const double gflop_lu = 2.0 * nn * nn * nn / 3.0 / 1e9;
    const double gflop_sl = 2.0 * nn * nn / 1e9;
    std::printf("{\"n\": %d, \"mode\": \"%s\", \"reps\": %d, \"t_min\": %.9g, \"tlu_min\": %.9g, "
                "\"tsl_min\": %.9g, \"gflops\": %.9g, \"gflops_lu\": %.9g, \"gflops_sl\": %.9g, "
                "\"residual\": %.9g, \"residual_norm\": %.9g, \"threads\": 1}\n",
                n, mode.c_str(), reps, tmin, lumin, slmin, (gflop_lu + gflop_sl) / tmin, gflop_lu / lumin,
                gflop_sl / slmin, resid, residn);
    return 0;
}
