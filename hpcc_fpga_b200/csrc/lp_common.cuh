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
// 8-byte copy of one double.
__device__ __forceinline__ void cp_async8(double* smem, const double* gmem) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
// 16-byte copy (both addresses 16-byte aligned).
__device__ __forceinline__ void cp_async_vec16(void* smem, const void* gmem) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_elem(float* smem, const float* gmem) { cp_async4(smem, gmem); }
__device__ __forceinline__ void cp_async_elem(double* smem, const double* gmem) { cp_async8(smem, gmem); }

// Separately rounded product and sum, and -1/x correctly rounded, in the
// element type: the reference's host arithmetic without fused multiply-add
// (for float, -1.0/x divided in double and rounded to float equals the
// correctly rounded float reciprocal, negated).
template <typename T>
struct Rn;
template <>
struct Rn<float> {
    static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
    static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
    static __device__ __forceinline__ float neg_rcp(float a) { return -__frcp_rn(a); }
};
template <>
struct Rn<double> {
    static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
    static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
    static __device__ __forceinline__ double neg_rcp(double a) { return -__drcp_rn(a); }
};

// Four consecutive elements from 16-byte aligned shared memory.
template <typename T>
struct Quad {
    T x, y, z, w;
};
__device__ __forceinline__ Quad<float> ld_quad(const float* p) {
    const float4 v = *reinterpret_cast<const float4*>(p);
    return {v.x, v.y, v.z, v.w};
}
__device__ __forceinline__ Quad<double> ld_quad(const double* p) {
    const double2 a = *reinterpret_cast<const double2*>(p);
    const double2 b = *reinterpret_cast<const double2*>(p + 2);
    return {a.x, a.y, b.x, b.y};
}
#endif

// ---- kernel launchers (each returns LP_OK or an error status) ------------
// Diagonal block LU for bs <= 128, whole block in shared memory.
int launch_lu_small(float* a, int lda, int bs, cudaStream_t s);
// The same kernels on FP64 blocks (bs 64 or 128): the reference's _DP build.
int launch_lu_small_f64(double* a, int lda, int bs, cudaStream_t s);
int launch_top_chunk_f64(const double* lu, int ldlu, double* t, int ldt, int bs, int ncols, cudaStream_t s);
int launch_left_chunk_f64(const double* lu, int ldlu, double* l, int ldl, int bs, int nrows, double* lt, int ldlt,
                          cudaStream_t s);
// Triangular block updates (top: column-independent; left: row-independent).
int launch_trsm_top(const float* lu, int ldlu, float* t, int ldt, int bs, int ncols, cudaStream_t s);
int launch_trsm_left(const float* lu, int ldlu, float* l, int ldl, int bs, int nrows, float* lt, int ldlt,
                     cudaStream_t s);
// FP32 SIMT trailing update C(m x n) += Lt^T (bs x m) * T (bs x n).
int launch_sgemm_update(float* c, int ldc, const float* lt, int ldlt, const float* t, int ldt, int m, int n,
                        int k, cudaStream_t s);
// FP64 SIMT trailing update, the same operand layout (k_dgemm.cu).
int launch_dgemm_update(double* c, int ldc, const double* lt, int ldlt, const double* t, int ldt, int m, int n, int k,
                        cudaStream_t s);
int dgemm_init_attrs();
int launch_transpose(const float* src, int lds, float* dst, int ldd, int rows, int cols, cudaStream_t s);
int launch_transpose_f64(const double* src, int lds, double* dst, int ldd, int rows, int cols, cudaStream_t s);
// Forward + back substitution for nrhs rows of b with the encoded factors:
// two persistent sweeps per 16 right-hand sides, each finisher CTA inverting
// its own diagonal block, the long source ranges split into chunks of `chunk`
// source tiles (0: no chunks) streamed by other CTAs (k_gesl_inv.cu).
// pub: gesl_pub_pairs(n, nrhs, chunk) 64-bit words, tickets: 2 ints, err: an
// error word the caller zeroes and reads.
int launch_gesl_inv(const float* a, int lda, int n, float* b, int ldb, int nrhs, unsigned long long* pub,
                    int* tickets, int* err, bool stall, int chunk, cudaStream_t st);
size_t gesl_pub_pairs(int n, int nrhs, int chunk);
// Chunk size of the substitution sweeps when the caller's workspace allows it.
constexpr int kGeslChunk = 32;
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

}  // namespace lp
