// Internal declarations shared by the lpcuda translation units.
#pragma once

#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>
#include <string>

#include "../../include/lpcuda.h"

namespace lp {

// Records `msg` as the calling thread's last error and returns `status`.
int fail(int status, const std::string& msg);
int cuda_fail(cudaError_t e, const char* what, const char* file, int line);

#define LP_CUDA(call)                                                          \
    do {                                                                       \
        cudaError_t lp_e_ = (call);                                            \
        if (lp_e_ != cudaSuccess) return ::lp::cuda_fail(lp_e_, #call, __FILE__, __LINE__); \
    } while (0)

#define LP_CHECK(expr)                                                         \
    do {                                                                       \
        int lp_s_ = (expr);                                                    \
        if (lp_s_ != LP_OK) return lp_s_;                                      \
    } while (0)

inline bool is_pow2(int x) { return x > 0 && (x & (x - 1)) == 0; }

// Process-wide count of kernels launched through the library.
void count_launch(long long n = 1);
long long launch_count();
inline bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

#ifdef __CUDACC__
// 4-byte asynchronous global -> shared copy (any float address), and the wait
// for all of the calling thread's outstanding copies.
__device__ __forceinline__ void cp_async4(float* smem, const float* gmem) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }
#endif

// ---- kernel launchers (each returns LP_OK or an error status) ------------
// Diagonal block LU for bs <= 128, whole block in shared memory.
int launch_lu_small(float* a, int lda, int bs, cudaStream_t s);
// Triangular block updates (top: column-independent; left: row-independent).
int launch_trsm_top(const float* lu, int ldlu, float* t, int ldt, int bs, int ncols, cudaStream_t s);
int launch_trsm_left(const float* lu, int ldlu, float* l, int ldl, int bs, int nrows, float* lt, int ldlt,
                     cudaStream_t s);
// FP32 SIMT trailing update C(m x n) += Lt^T (bs x m) * T (bs x n).
int launch_sgemm_update(float* c, int ldc, const float* lt, int ldlt, const float* t, int ldt, int m, int n,
                        int k, cudaStream_t s);
int launch_transpose(const float* src, int lds, float* dst, int ldd, int rows, int cols, cudaStream_t s);
// Forward + back substitution for nrhs rows of b (see k_gesl.cu).
int launch_gesl(const float* a, int lda, int n, float* b, int ldb, int nrhs, float* work, cudaStream_t s);
size_t gesl_work_floats(int n, int nrhs);
// The same with precomputed inverses of the 128 x 128 diagonal blocks (k_gesl_inv.cu).
int launch_diag_inverses(const float* a, int lda, int n, float* inv, cudaStream_t s);
int launch_gesl_inv(const float* a, int lda, int n, float* b, int ldb, int nrhs, float* work, const float* inv,
                    int* sync, cudaStream_t s);
size_t gesl_sync_ints(int n);
size_t gesl_inv_floats(int n);
int gesl_inv_init_attrs();
// FP64 refinement pieces (see k_ir.cu).
int launch_residual_f64(const float* a, int lda, int n, const double* x, int ldx, const double* b, int ldb,
                        double* r, int ldr, int nrhs, cudaStream_t s);
int launch_colabs(const float* a, int lda, int n, double* out, cudaStream_t s);
// out[q] = max_i |v[q*ld + i]| (as the bits of a non-negative double), +inf if any is not finite.
int launch_rhs_absmax(const double* v, int n, int ld, int nrhs, unsigned long long* out, cudaStream_t s);
int launch_axpy_f64(double* x, const float* d, size_t n, cudaStream_t s);
int launch_f64_to_f32(float* y, const double* v, size_t n, cudaStream_t s);
int launch_f32_to_f64(double* y, const float* v, size_t n, cudaStream_t s);
// Per-device one-time kernel attribute setup (large dynamic shared memory).
int lu_init_attrs();
int trsm_init_attrs();
int sgemm_init_attrs();
int gesl_init_attrs();

}  // namespace lp
