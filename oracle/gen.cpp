// ORACLE — test infrastructure only (see oracle/oracle.c).
//
// Restatement of the two input generators the LINPACK path is run on.
//
// 1. reference mode: LINPACK/src/host/linpack_benchmark.hpp:211-297
//    (generateInputData) for one rank (P = Q = 1): std::mt19937(rank 0),
//    std::uniform_real_distribution<double>(0,1) narrowed to float, filled in
//    storage-row order; for a diagonally dominant matrix each storage-row
//    diagonal is first zeroed and then set to the float sum of its row; b is
//    the float sum of each storage column, so b = M * ones under M = S^T.
// 2. baseline mode: the seeded workload generator of the benchmark configs:
//    mt19937(seed), one 32-bit draw per entry mapped to the float
//    (u >> 8) * 2^-24 - 0.5 in [-0.5, 0.5); storage-row diagonal =
//    sum |off-diagonal| (in double) + margin, rounded to float; b = M * ones
//    formed in double (exact for these entries) and rounded to float for the
//    single-precision right-hand side.
#include <cmath>
#include <cstdint>
#include <random>

extern "C" {

void orc_gen_reference_f32(float* A, float* b, int n, int diag_dominant, float* norma_out,
                           float* normb_out) {
    std::mt19937 gen(0);
    std::uniform_real_distribution<> dis(0.0, 1.0);
    float norma = 0.0f, normb = 0.0f;
    for (int j = 0; j < n; j++) {
        for (int i = 0; i < n; i++) {
            float v = dis(gen);
            A[(size_t)n * j + i] = v;
            norma = (v > norma) ? v : norma;
        }
    }
    if (diag_dominant) {
        for (int r = 0; r < n; r++) {
            A[(size_t)n * r + r] = 0.0f;
            float s = 0.0f;
            for (int i = 0; i < n; i++) s += A[(size_t)n * r + i];
            norma = (s > norma) ? s : norma;
            A[(size_t)n * r + r] = s;
        }
    }
    for (int j = 0; j < n; j++) {
        float s = 0.0f;
        for (int i = 0; i < n; i++) s += A[(size_t)n * i + j];
        b[j] = s;
        normb = (s > normb) ? s : normb;
    }
    if (norma_out) *norma_out = norma;
    if (normb_out) *normb_out = normb;
}

void orc_gen_baseline(float* A, double* b64, float* b32, int n, unsigned seed, double margin) {
    std::mt19937 gen(seed);
    const double scale = 1.0 / 16777216.0;  // 2^-24
    for (int r = 0; r < n; r++) {
        double offsum = 0.0;
        for (int c = 0; c < n; c++) {
            uint32_t u = gen();
            float v = (float)((double)(u >> 8) * scale - 0.5);
            A[(size_t)n * r + c] = v;
            if (c != r) offsum += std::fabs((double)v);
        }
        A[(size_t)n * r + r] = (float)(offsum + margin);
    }
    for (int c = 0; c < n; c++) b64[c] = 0.0;
    for (int r = 0; r < n; r++)
        for (int c = 0; c < n; c++) b64[c] += (double)A[(size_t)n * r + c];
    for (int c = 0; c < n; c++) b32[c] = (float)b64[c];
}

}  // extern "C"
