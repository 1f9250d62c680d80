// Host-only entry points of liblpcuda.so: input generation (no GPU needed).
//
// lp_generate_reference restates LinpackBenchmark::generateInputData
// (LINPACK/src/host/linpack_benchmark.hpp:211-297) for a single rank
// (P = Q = 1, so every MPI_Reduce/Allreduce is the identity):
//   std::mt19937 gen(rank = 0); std::uniform_real_distribution<> dis(0, 1);
//   A filled in storage-row order with the double draw narrowed to float;
//   diagonally dominant: each storage-row diagonal zeroed, then set to the
//   float sum of the row (summed in index order);
//   b[j] = float sum of storage column j (index order): b = M * ones.
// Using the same <random> engine and distribution, the same order of draws
// and the same float accumulation makes the matrix bit-identical to the
// reference's.
//
// lp_generate_baseline is the seeded workload generator: one mt19937 draw
// per entry, mapped to the float (u >> 8) * 2^-24 - 0.5 (exact, in
// [-0.5, 0.5)); diagonal = sum |off-diagonal| (double) + margin, rounded to
// float; b64 = M * ones in double — exact, since every entry is a multiple of
// 2^-24 below 2^24 in magnitude — so the solution of (M, b64) is all ones.
#include <cmath>
#include <cstdint>
#include <random>

#include "../../include/lpcuda.h"

extern "C" {

// The same generator as the reference's double build (HOST_DATA_TYPE double:
// the draws are not narrowed, the sums are in double).
int lp_generate_reference_f64(double* A, double* b, int n, int diag_dominant, double* norma_out, double* normb_out) {
    if (A == nullptr || b == nullptr || n <= 0) return LP_E_INVALID;
    std::mt19937 gen(0);
    std::uniform_real_distribution<> dis(0.0, 1.0);
    double norma = 0.0, normb = 0.0;
    const size_t w = (size_t)n;
    for (size_t r = 0; r < w; r++) {
        double* row = A + r * w;
        for (size_t c = 0; c < w; c++) {
            const double v = dis(gen);
            row[c] = v;
            norma = (v > norma) ? v : norma;
        }
    }
    if (diag_dominant) {
        for (size_t r = 0; r < w; r++) {
            double* row = A + r * w;
            row[r] = 0.0;
            double s = 0.0;
            for (size_t c = 0; c < w; c++) s += row[c];
            norma = (s > norma) ? s : norma;
            row[r] = s;
        }
    }
    for (size_t c = 0; c < w; c++) b[c] = 0.0;
    for (size_t r = 0; r < w; r++) {
        const double* row = A + r * w;
        for (size_t c = 0; c < w; c++) b[c] += row[c];
    }
    for (size_t c = 0; c < w; c++) normb = (b[c] > normb) ? b[c] : normb;
    if (norma_out != nullptr) *norma_out = norma;
    if (normb_out != nullptr) *normb_out = normb;
    return LP_OK;
}

int lp_generate_reference(float* A, float* b, int n, int diag_dominant, float* norma_out, float* normb_out) {
    if (A == nullptr || b == nullptr || n <= 0) return LP_E_INVALID;
    std::mt19937 gen(0);
    std::uniform_real_distribution<> dis(0.0, 1.0);
    float norma = 0.0f, normb = 0.0f;
    const size_t w = (size_t)n;
    for (size_t r = 0; r < w; r++) {
        float* row = A + r * w;
        for (size_t c = 0; c < w; c++) {
            const float v = dis(gen);
            row[c] = v;
            norma = (v > norma) ? v : norma;
        }
    }
    if (diag_dominant) {
        for (size_t r = 0; r < w; r++) {
            float* row = A + r * w;
            row[r] = 0.0f;
            float s = 0.0f;
            for (size_t c = 0; c < w; c++) s += row[c];
            norma = (s > norma) ? s : norma;
            row[r] = s;
        }
    }
    for (size_t c = 0; c < w; c++) b[c] = 0.0f;
    for (size_t r = 0; r < w; r++) {
        const float* row = A + r * w;
        for (size_t c = 0; c < w; c++) b[c] += row[c];
    }
    for (size_t c = 0; c < w; c++) normb = (b[c] > normb) ? b[c] : normb;
    if (norma_out != nullptr) *norma_out = norma;
    if (normb_out != nullptr) *normb_out = normb;
    return LP_OK;
}

int lp_generate_baseline(float* A, double* b64, float* b32, int n, unsigned seed, double margin) {
    if (A == nullptr || n <= 0) return LP_E_INVALID;
    std::mt19937 gen(seed);
    const double scale = 1.0 / 16777216.0;
    const size_t w = (size_t)n;
    for (size_t r = 0; r < w; r++) {
        float* row = A + r * w;
        double off = 0.0;
        for (size_t c = 0; c < w; c++) {
            const uint32_t u = gen();
            const float v = (float)((double)(u >> 8) * scale - 0.5);
            row[c] = v;
            off += std::fabs((double)v);
        }
        off -= std::fabs((double)row[r]);
        row[r] = (float)(off + margin);
    }
    if (b64 != nullptr || b32 != nullptr) {
        double* acc = b64;
        double* tmp = nullptr;
        if (acc == nullptr) acc = tmp = new double[w];
        for (size_t c = 0; c < w; c++) acc[c] = 0.0;
        for (size_t r = 0; r < w; r++) {
            const float* row = A + r * w;
            for (size_t c = 0; c < w; c++) acc[c] += (double)row[c];
        }
        if (b32 != nullptr)
            for (size_t c = 0; c < w; c++) b32[c] = (float)acc[c];
        delete[] tmp;
    }
    return LP_OK;
}

}  // extern "C"
