// FP64 form of the path — the reference's _DP build (DATA_TYPE / HOST_DATA_TYPE
// double, LINPACK/src/host/parameters.h.in; CI's double-precision variant):
// the same blocked right-looking LU without pivoting (lu / top / left / inner,
// gefa_ref_nopvt's encoding) and the same substitution, in double.
//
// lu, top and left are the float kernels instantiated for double
// (k_lu.cu, k_trsm.cu: reference operation order, bit-identical on one
// block); inner is k_dgemm_update.  The substitution below is blocked by 64
// unknowns, one launch per block and direction: every CTA stages the diagonal
// block, solves it redundantly (one warp per right-hand side), then updates
// its share of the other unknowns with the block's rows (a GEMV over
// contiguous rows, each factor element read once per sweep).
#include <string>

#include "lp_ctx.cuh"

namespace lp {
namespace {

constexpr int SB = 64;       // substitution block
constexpr int GT = 256;      // threads per CTA; one unknown per thread in the update
constexpr int RMAX = 16;     // right-hand sides per pass

// The kb x kb diagonal block into shared memory, every copy in flight before
// the wait; entries outside it are zero.  FP32 factors (the substitution in
// FP64 arithmetic on FP32 factors, used by the GMRES refinement) are widened
// exactly as they are read.
__device__ __forceinline__ void stage_block(double (*dg)[SB + 1], const double* __restrict__ a, int lda, int k0,
                                            int kb) {
    for (int idx = threadIdx.x; idx < SB * SB; idx += GT) {
        const int r = idx / SB, c = idx - r * SB;
        if (r < kb && c < kb)
            cp_async8(&dg[r][c], a + (size_t)(k0 + r) * lda + k0 + c);
        else
            dg[r][c] = 0.0;
    }
    cp_async_wait_all();
}
__device__ __forceinline__ void stage_block(double (*dg)[SB + 1], const float* __restrict__ a, int lda, int k0,
                                            int kb) {
    float v[SB * SB / GT];
#pragma unroll
    for (int q = 0; q < SB * SB / GT; q++) {  // all loads in flight before the first store
        const int idx = threadIdx.x + q * GT, r = idx / SB, c = idx - r * SB;
        v[q] = (r < kb && c < kb) ? __ldg(a + (size_t)(k0 + r) * lda + k0 + c) : 0.0f;
    }
#pragma unroll
    for (int q = 0; q < SB * SB / GT; q++) {
        const int idx = threadIdx.x + q * GT, r = idx / SB, c = idx - r * SB;
        dg[r][c] = (double)v[q];
    }
}

// acc[r] = sum_{k < kb} coef[r][k] * S[k0 + k][c]: the block's column c, read
// 16 rows at a time with all 16 loads in flight before they are used.
template <typename FT>
__device__ __forceinline__ void block_gemv(const FT* __restrict__ a, int lda, int k0, int kb, int c,
                                           const double (*coef)[SB], int nrhs, double (&acc)[RMAX]) {
#pragma unroll
    for (int r = 0; r < RMAX; r++) acc[r] = 0.0;
    const FT* col = a + (size_t)k0 * lda + c;
    for (int kc = 0; kc < kb; kc += 16) {
        double v[16];
#pragma unroll
        for (int j = 0; j < 16; j++) v[j] = kc + j < kb ? (double)__ldg(col + (size_t)(kc + j) * lda) : 0.0;
#pragma unroll
        for (int r = 0; r < RMAX; r++)
            if (r < nrhs)
#pragma unroll
                for (int j = 0; j < 16; j++)
                    if (kc + j < kb) acc[r] = fma(coef[r][kc + j], v[j], acc[r]);
    }
}

// forward: y_i += y_k S[k][i] (i > k).  w1: accumulating values (all
// unknowns), w2: solved values of the block.
template <typename FT>
__global__ void __launch_bounds__(GT) k_gesl64_fwd(const FT* __restrict__ a, int lda, int n, double* w1,
                                                   double* w2, int ldw, int nrhs, int k0) {
    __shared__ double dg[SB][SB + 1];
    __shared__ double ys[RMAX][SB];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int kb = min(SB, n - k0);
    stage_block(dg, a, lda, k0, kb);
    __syncthreads();
    for (int r = warp; r < nrhs; r += GT / 32) {
        double v0 = lane < kb ? w1[(size_t)r * ldw + k0 + lane] : 0.0;
        double v1 = lane + 32 < kb ? w1[(size_t)r * ldw + k0 + lane + 32] : 0.0;
        for (int k = 0; k < kb; k++) {
            const double yk = __shfl_sync(0xffffffffu, k < 32 ? v0 : v1, k & 31);
            if (lane > k) v0 = fma(yk, dg[k][lane], v0);
            if (lane + 32 > k) v1 = fma(yk, dg[k][lane + 32], v1);
        }
        ys[r][lane] = v0;
        ys[r][lane + 32] = v1;
        if (blockIdx.x == 0) {
            if (lane < kb) w2[(size_t)r * ldw + k0 + lane] = v0;
            if (lane + 32 < kb) w2[(size_t)r * ldw + k0 + lane + 32] = v1;
        }
    }
    __syncthreads();
    const int c = k0 + kb + blockIdx.x * GT + threadIdx.x;
    if (c >= n) return;
    double acc[RMAX];
    block_gemv(a, lda, k0, kb, c, ys, nrhs, acc);
#pragma unroll
    for (int r = 0; r < RMAX; r++)
        if (r < nrhs) w1[(size_t)r * ldw + c] += acc[r];
}

// backward: s = y_k S[k][k]; x_k = -s; y_i += s S[k][i] (i < k).  w2: values
// (updated in place for the unknowns before the block), out: solutions.
template <typename FT>
__global__ void __launch_bounds__(GT) k_gesl64_bwd(const FT* __restrict__ a, int lda, int n, double* w2, int ldw,
                                                   double* out, int ldo, int nrhs, int k0) {
    __shared__ double dg[SB][SB + 1];
    __shared__ double ss[RMAX][SB];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int kb = min(SB, n - k0);
    stage_block(dg, a, lda, k0, kb);
    __syncthreads();
    for (int r = warp; r < nrhs; r += GT / 32) {
        double v0 = lane < kb ? w2[(size_t)r * ldw + k0 + lane] : 0.0;
        double v1 = lane + 32 < kb ? w2[(size_t)r * ldw + k0 + lane + 32] : 0.0;
        for (int k = kb - 1; k >= 0; k--) {
            const double yk = __shfl_sync(0xffffffffu, k < 32 ? v0 : v1, k & 31);
            const double s = yk * dg[k][k];
            if (lane == (k & 31)) {
                if (k < 32)
                    v0 = -s;
                else
                    v1 = -s;
                ss[r][k] = s;
            }
            if (lane < k) v0 = fma(s, dg[k][lane], v0);
            if (lane + 32 < k) v1 = fma(s, dg[k][lane + 32], v1);
        }
        if (blockIdx.x == 0) {
            if (lane < kb) out[(size_t)r * ldo + k0 + lane] = v0;
            if (lane + 32 < kb) out[(size_t)r * ldo + k0 + lane + 32] = v1;
        }
    }
    __syncthreads();
    const int c = blockIdx.x * GT + threadIdx.x;
    if (c >= k0) return;
    double acc[RMAX];
    block_gemv(a, lda, k0, kb, c, ss, nrhs, acc);
#pragma unroll
    for (int r = 0; r < RMAX; r++)
        if (r < nrhs) w2[(size_t)r * ldw + c] += acc[r];
}

double event_s64(cudaEvent_t a, cudaEvent_t b) {
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, a, b);
    return 1e-3 * ms;
}

int validate64(const void* a, int n, int lda, int bs, const char* who) {
    if (a == nullptr) return fail(LP_E_INVALID, std::string(who) + ": null matrix pointer");
    if (n <= 0 || lda < n) return fail(LP_E_INVALID, std::string(who) + ": need n > 0 and lda >= n");
    if (bs != 64 && bs != 128 && bs != 256)
        return fail(LP_E_INVALID, std::string(who) + ": FP64 block size must be 64, 128 or 256");
    if (n % bs != 0) return fail(LP_E_INVALID, std::string(who) + ": n must be a multiple of the block size");
    if (lda % 2 != 0 || !aligned16(a))
        return fail(LP_E_INVALID, std::string(who) + ": matrix must be 16-byte aligned with an even lda");
    return LP_OK;
}

}  // namespace

// Blocks wider than 128 (256): the same blocked algorithm inside the block
// with 128-wide inner blocks, as the FP32 path does for its 512 blocks — the
// lu of the diagonal block recursively, top and left as 128-row / -column
// exact chunks plus FP64 GEMM updates of the rest.  `dt` holds one transposed
// 128-wide sub-block (128 x 128) of the diagonal block.
static int lu_stage64(double* d, int lda, int bs, double* lti, cudaStream_t st) {
    if (bs <= 128) return launch_lu_small_f64(d, lda, bs, st);
    const int ib = 128;
    for (int kk = 0; kk < bs / ib; kk++) {
        double* dd = d + (size_t)kk * ib * lda + (size_t)kk * ib;
        LP_CHECK(launch_lu_small_f64(dd, lda, ib, st));
        const int r = bs - (kk + 1) * ib;
        if (r <= 0) break;
        LP_CHECK(launch_top_chunk_f64(dd, lda, dd + ib, lda, ib, r, st));
        LP_CHECK(launch_left_chunk_f64(dd, lda, dd + (size_t)ib * lda, lda, ib, r, lti, r, st));
        LP_CHECK(launch_dgemm_update(dd + (size_t)ib * lda + ib, lda, lti, r, dd + ib, lda, r, r, ib, st));
    }
    return LP_OK;
}

static int top_blocked64(const double* d, int lda, double* t, int ldt, int bs, int ncols, double* dt,
                         cudaStream_t st) {
    if (bs <= 128) return launch_top_chunk_f64(d, lda, t, ldt, bs, ncols, st);
    const int ib = 128;
    for (int kk = 0; kk < bs / ib; kk++) {
        const double* dkk = d + (size_t)kk * ib * lda + (size_t)kk * ib;
        double* tk = t + (size_t)kk * ib * ldt;
        LP_CHECK(launch_top_chunk_f64(dkk, lda, tk, ldt, ib, ncols, st));
        const int m2 = bs - (kk + 1) * ib;
        if (m2 <= 0) break;
        // T[below] += D[below][chunk] * T[chunk]: D's sub-block transposed into the k-major operand
        LP_CHECK(launch_transpose_f64(dkk + (size_t)ib * lda, lda, dt, m2, m2, ib, st));
        LP_CHECK(launch_dgemm_update(tk + (size_t)ib * ldt, ldt, dt, m2, tk, ldt, m2, ncols, ib, st));
    }
    return LP_OK;
}

static int left_blocked64(const double* d, int lda, double* l, int ldl, int bs, int nrows, double* lt, int ldlt,
                          cudaStream_t st) {
    if (bs <= 128) return launch_left_chunk_f64(d, lda, l, ldl, bs, nrows, lt, ldlt, st);
    const int ib = 128;
    for (int kk = 0; kk < bs / ib; kk++) {
        const double* dkk = d + (size_t)kk * ib * lda + (size_t)kk * ib;
        double* lk = l + (size_t)kk * ib;
        double* ltk = lt + (size_t)kk * ib * ldlt;
        LP_CHECK(launch_left_chunk_f64(dkk, lda, lk, ldl, ib, nrows, ltk, ldlt, st));
        const int m2 = bs - (kk + 1) * ib;
        if (m2 <= 0) break;
        // L[:, after] += L[:, chunk] * D[chunk][after]
        LP_CHECK(launch_dgemm_update(lk + ib, ldl, ltk, ldlt, dkk + ib, lda, nrows, m2, ib, st));
    }
    return LP_OK;
}

int gefa_f64(lp_ctx* c, double* a, int n, int lda, int bs, cudaStream_t st) {
    LP_CHECK(c->f64lt.ensure(sizeof(double) * ((size_t)bs * n + (bs > 128 ? 2 * (size_t)128 * bs : 0))));
    double* lt = static_cast<double*>(c->f64lt.ptr);
    double* scratch = lt + (size_t)bs * n;  // bs > 128: inner Lt of the lu stage, then transposed D sub-blocks
    for (int k0 = 0; k0 < n; k0 += bs) {
        double* d = a + (size_t)k0 * lda + k0;
        const int rest = n - k0 - bs;
        int e = prof_begin(c, st);
        LP_CHECK(lu_stage64(d, lda, bs, scratch, st));
        LP_CHECK(prof_end(c, st, LP_STAGE_LU, e, 2.0 * bs * bs * bs / 3.0, 16.0 * bs * bs));
        if (rest <= 0) break;
        e = prof_begin(c, st);
        LP_CHECK(top_blocked64(d, lda, d + bs, lda, bs, rest, scratch, st));
        LP_CHECK(prof_end(c, st, LP_STAGE_TOP, e, (double)bs * bs * rest, 16.0 * bs * rest));
        e = prof_begin(c, st);
        LP_CHECK(left_blocked64(d, lda, d + (size_t)bs * lda, lda, bs, rest, lt, rest, st));
        LP_CHECK(prof_end(c, st, LP_STAGE_LEFT, e, (double)bs * bs * rest, 24.0 * bs * rest));
        e = prof_begin(c, st);
        LP_CHECK(launch_dgemm_update(d + (size_t)bs * lda + bs, lda, lt, rest, d + bs, lda, rest, rest, bs, st));
        LP_CHECK(prof_end(c, st, LP_STAGE_INNER, e, 2.0 * rest * rest * bs,
                          8.0 * (2.0 * rest * rest + 2.0 * bs * rest)));
    }
    return LP_OK;
}

template <typename FT>
static int gesl64_any(lp_ctx* c, const FT* a, int n, int lda, double* b, int nrhs, int ldb, cudaStream_t st) {
    const int g0 = nrhs < RMAX ? nrhs : RMAX;
    LP_CHECK(c->f64w.ensure(sizeof(double) * 2 * (size_t)n * g0));
    double* w1 = static_cast<double*>(c->f64w.ptr);
    double* w2 = w1 + (size_t)n * g0;
    const int e = prof_begin(c, st);
    const int nblk = (n + SB - 1) / SB;
    for (int r0 = 0; r0 < nrhs; r0 += RMAX) {
        const int g = nrhs - r0 < RMAX ? nrhs - r0 : RMAX;
        double* bb = b + (size_t)r0 * ldb;
        LP_CUDA(cudaMemcpy2DAsync(w1, sizeof(double) * n, bb, sizeof(double) * ldb, sizeof(double) * n, g,
                                  cudaMemcpyDeviceToDevice, st));
        for (int K = 0; K < nblk; K++) {
            const int k0 = K * SB, rest = n - k0 - std::min(SB, n - k0);
            const int grid = rest > 0 ? (rest + GT - 1) / GT : 1;
            k_gesl64_fwd<FT><<<grid, GT, 0, st>>>(a, lda, n, w1, w2, n, g, k0);
            count_launch();
        }
        for (int K = nblk - 1; K >= 0; K--) {
            const int k0 = K * SB;
            const int grid = k0 > 0 ? (k0 + GT - 1) / GT : 1;
            k_gesl64_bwd<FT><<<grid, GT, 0, st>>>(a, lda, n, w2, n, bb, ldb, g, k0);
            count_launch();
        }
        LP_CUDA(cudaGetLastError());
    }
    return prof_end(c, st, LP_STAGE_GESL, e, 2.0 * n * n * nrhs,
                    (double)sizeof(FT) * n * n * ((nrhs + RMAX - 1) / RMAX));
}

int gesl_f64(lp_ctx* c, const double* a, int n, int lda, double* b, int nrhs, int ldb, cudaStream_t st) {
    return gesl64_any(c, a, n, lda, b, nrhs, ldb, st);
}

int gesl_f64_on_f32(lp_ctx* c, const float* a, int n, int lda, double* b, int nrhs, int ldb, cudaStream_t st) {
    return gesl64_any(c, a, n, lda, b, nrhs, ldb, st);
}

}  // namespace lp

using namespace lp;

extern "C" {

int lp_gefa_f64_dev(lp_ctx* c, double* dA, int n, int lda, int bs) {
    if (c == nullptr) return fail(LP_E_INVALID, "lp_gefa_f64_dev: null context");
    LP_CHECK(validate64(dA, n, lda, bs, "lp_gefa_f64_dev"));
    LP_CUDA(cudaSetDevice(c->device));
    return gefa_f64(c, dA, n, lda, bs, c->stream);
}

int lp_gesl_f64_dev(lp_ctx* c, const double* dLU, int n, int lda, double* dB, int nrhs, int ldb) {
    if (c == nullptr || dLU == nullptr || dB == nullptr) return fail(LP_E_INVALID, "lp_gesl_f64_dev: null argument");
    if (n <= 0 || lda < n || nrhs <= 0 || ldb < n) return fail(LP_E_INVALID, "lp_gesl_f64_dev: bad sizes");
    LP_CUDA(cudaSetDevice(c->device));
    return gesl_f64(c, dLU, n, lda, dB, nrhs, ldb, c->stream);
}

int lp_calculate_f64(lp_ctx* c, int n, int lda, int bs, int repetitions, double* A, double* b, double* gefa_times,
                     double* gesl_times) {
    if (c == nullptr || A == nullptr || b == nullptr || gefa_times == nullptr || gesl_times == nullptr)
        return fail(LP_E_INVALID, "lp_calculate_f64: null argument");
    if (repetitions <= 0) return fail(LP_E_INVALID, "lp_calculate_f64: repetitions must be positive");
    if (n <= 0 || lda < n || lda % 2 != 0 || (bs != 64 && bs != 128 && bs != 256) || n % bs != 0)
        return fail(LP_E_INVALID, "lp_calculate_f64: n a multiple of bs (64, 128 or 256), lda >= n and even");
    LP_CUDA(cudaSetDevice(c->device));
    const size_t abytes = sizeof(double) * (size_t)n * lda;
    LP_CHECK(c->f64a.ensure(abytes));
    LP_CHECK(c->f64b.ensure(sizeof(double) * (size_t)n));
    double* dA = static_cast<double*>(c->f64a.ptr);
    double* dB = static_cast<double*>(c->f64b.ptr);
    cudaStream_t st = c->stream;
    for (int rep = 0; rep < repetitions; rep++) {
        LP_CUDA(cudaMemcpyAsync(dA, A, abytes, cudaMemcpyHostToDevice, st));
        LP_CUDA(cudaMemcpyAsync(dB, b, sizeof(double) * n, cudaMemcpyHostToDevice, st));
        LP_CUDA(cudaEventRecord(c->ev[0], st));
        LP_CHECK(gefa_f64(c, dA, n, lda, bs, st));
        LP_CUDA(cudaEventRecord(c->ev[1], st));
        LP_CHECK(gesl_f64(c, dA, n, lda, dB, 1, n, st));
        LP_CUDA(cudaEventRecord(c->ev[2], st));
        LP_CUDA(cudaStreamSynchronize(st));
        gefa_times[rep] = event_s64(c->ev[0], c->ev[1]);
        gesl_times[rep] = event_s64(c->ev[1], c->ev[2]);
    }
    LP_CUDA(cudaMemcpyAsync(A, dA, abytes, cudaMemcpyDeviceToHost, st));
    LP_CUDA(cudaMemcpyAsync(b, dB, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    LP_CUDA(cudaStreamSynchronize(st));
    return LP_OK;
}

}  // extern "C"
