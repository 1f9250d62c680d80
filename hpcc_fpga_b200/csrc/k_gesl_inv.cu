// gesl with inverted diagonal blocks — the substitution of the factorization
// paths (the reference's gesl_ref_nopvt, LINPACK/src/host/linpack_data.cpp:199-229).
//
// For every 128 x 128 diagonal block D of the encoded factors two dense
// operators are formed once per solve, all blocks in one launch:
//   Y = (I - U)^-1             by the left recurrence on an identity (U: D's
//                              strict upper storage triangle, the negated
//                              multipliers);
//   X = (diag(D_kk)^-1 - L)^-1 by the top recurrence on an identity (D_kk =
//                              -1/d as stored; L: D's strict lower storage
//                              triangle, the U factor of M).
// Within a block the forward sweep is then y = Y^T acc and the backward sweep
// s = X^T acc, x = -s: a 128 x 128 matrix-vector product over all 256 threads
// instead of a 128-step sequential chain.  Blocks are still visited in order,
// one launch per block and direction; step (b), the update of the remaining
// unknowns with the block's row panel, is the shared panel_gemv.
#include "gesl_common.cuh"

namespace lp {
namespace {

using namespace gesl;

constexpr int ICH = 32;       // chunk of the inverse recurrences
constexpr int IST = 64;       // strip width of the inverse kernels
constexpr int BLK2 = SB * SB; // floats per operator
constexpr size_t kInvTopSmem = sizeof(float) * (SB * IST + SB * ICH);
constexpr size_t kInvLeftSmem = sizeof(float) * (IST * (SB + 1) + ICH * SB);

// X of diagonal block blockIdx.y, columns [64*blockIdx.x, +64).
__global__ void __launch_bounds__(256) k_inv_top(const float* __restrict__ a, int lda, int n, float* __restrict__ inv) {
    extern __shared__ float ism[];
    float* strip = ism;            // SB x IST
    float* dch = ism + SB * IST;   // SB x ICH
    const int tid = threadIdx.x;
    const int b = blockIdx.y, k0 = b * SB, kb = min(SB, n - k0);
    const int c0 = blockIdx.x * IST;
    const float* d = a + (size_t)k0 * lda + k0;
    for (int idx = tid; idx < SB * IST; idx += 256) {
        const int r = idx / IST, c = idx - r * IST;
        strip[idx] = (r == c0 + c) ? 1.0f : 0.0f;
    }
    for (int r0 = 0; r0 < SB; r0 += ICH) {
        const int nr = SB - r0;
        for (int idx = tid; idx < nr * ICH; idx += 256) {
            const int rr = idx / ICH, kk = idx - rr * ICH;
            const int r = r0 + rr, k = r0 + kk;
            dch[idx] = (r < kb && k < kb) ? d[(size_t)r * lda + k] : (r == k ? 1.0f : 0.0f);
        }
        __syncthreads();
        if (tid < IST) {
            float x[ICH];
#pragma unroll
            for (int k = 0; k < ICH; k++) x[k] = strip[(r0 + k) * IST + tid];
#pragma unroll
            for (int k = 0; k < ICH; k++) {
                const float xk = x[k] * dch[k * ICH + k];
                x[k] = xk;
#pragma unroll
                for (int j = k + 1; j < ICH; j++) x[j] = fmaf(xk, dch[j * ICH + k], x[j]);
            }
#pragma unroll
            for (int k = 0; k < ICH; k++) strip[(r0 + k) * IST + tid] = x[k];
        }
        __syncthreads();
        if (nr > ICH) {
            const int c = tid & (IST - 1), g = tid / IST;
            float x[ICH];
#pragma unroll
            for (int k = 0; k < ICH; k++) x[k] = strip[(r0 + k) * IST + c];
            for (int r = r0 + ICH + g; r < SB; r += 256 / IST) {
                float acc = strip[r * IST + c];
                const float* drow = dch + (r - r0) * ICH;
#pragma unroll
                for (int k = 0; k < ICH; k++) acc = fmaf(x[k], drow[k], acc);
                strip[r * IST + c] = acc;
            }
        }
        __syncthreads();
    }
    float* out = inv + (size_t)b * 2 * BLK2;
    for (int idx = tid; idx < SB * IST; idx += 256) {
        const int r = idx / IST, c = idx - r * IST;
        out[r * SB + c0 + c] = strip[idx];
    }
}

// Y of diagonal block blockIdx.y, rows [64*blockIdx.x, +64).
__global__ void __launch_bounds__(256) k_inv_left(const float* __restrict__ a, int lda, int n, float* __restrict__ inv) {
    constexpr int SL = SB + 1;
    extern __shared__ float ism[];
    float* strip = ism;            // IST x (SB + 1)
    float* dch = ism + IST * SL;   // ICH x SB
    const int tid = threadIdx.x;
    const int b = blockIdx.y, k0 = b * SB, kb = min(SB, n - k0);
    const int r0s = blockIdx.x * IST;
    const float* d = a + (size_t)k0 * lda + k0;
    for (int idx = tid; idx < IST * SB; idx += 256) {
        const int rr = idx / SB, c = idx - rr * SB;
        strip[rr * SL + c] = (r0s + rr == c) ? 1.0f : 0.0f;
    }
    for (int c0 = 0; c0 < SB; c0 += ICH) {
        const int nc = SB - c0;
        for (int idx = tid; idx < ICH * nc; idx += 256) {
            const int kk = idx / nc, cc = idx - kk * nc;
            const int k = c0 + kk, c = c0 + cc;
            dch[idx] = (k < kb && c < kb) ? d[(size_t)k * lda + c] : 0.0f;
        }
        __syncthreads();
        if (tid < IST) {
            float x[ICH];
            float* row = strip + tid * SL + c0;
#pragma unroll
            for (int k = 0; k < ICH; k++) x[k] = row[k];
#pragma unroll
            for (int k = 0; k < ICH; k++)
#pragma unroll
                for (int i = k + 1; i < ICH; i++) x[i] = fmaf(x[k], dch[k * nc + i], x[i]);
#pragma unroll
            for (int k = 0; k < ICH; k++) row[k] = x[k];
        }
        __syncthreads();
        for (int ci = ICH + tid; ci < nc; ci += 256) {
            float dv[ICH];
#pragma unroll
            for (int k = 0; k < ICH; k++) dv[k] = dch[k * nc + ci];
            for (int rr = 0; rr < IST; rr++) {
                const float* row = strip + rr * SL + c0;
                float acc = row[ci];
#pragma unroll
                for (int k = 0; k < ICH; k++) acc = fmaf(row[k], dv[k], acc);
                strip[rr * SL + c0 + ci] = acc;
            }
        }
        __syncthreads();
    }
    float* out = inv + (size_t)b * 2 * BLK2 + BLK2;
    for (int idx = tid; idx < IST * SB; idx += 256) {
        const int rr = idx / SB, c = idx - rr * SB;
        out[(r0s + rr) * SB + c] = strip[rr * SL + c];
    }
}

// coef[r][i] = sum_k M[k][i] * acc[r][k] for the block at k0 (M = Y or X of
// that block); all 256 threads: thread (h, i) sums k in [64h, 64h+64).
template <int NR>
__device__ __forceinline__ void block_matvec(const float* __restrict__ M, const float* acc, float* part, float* coef) {
    const int i = threadIdx.x & (SB - 1), h = threadIdx.x >> 7;
    float p[NR];
#pragma unroll
    for (int r = 0; r < NR; r++) p[r] = 0.0f;
#pragma unroll 16
    for (int kk = 0; kk < SB / 2; kk++) {
        const int k = h * (SB / 2) + kk;
        const float m = M[k * SB + i];
#pragma unroll
        for (int r = 0; r < NR; r++) p[r] = fmaf(m, acc[r * SB + k], p[r]);
    }
#pragma unroll
    for (int r = 0; r < NR; r++) part[(h * NR + r) * SB + i] = p[r];
    __syncthreads();
    for (int idx = threadIdx.x; idx < NR * SB; idx += GT) {
        const int r = idx / SB, ii = idx - r * SB;
        coef[idx] = part[r * SB + ii] + part[(NR + r) * SB + ii];
    }
    __syncthreads();
}

template <int NR>
__device__ __forceinline__ void load_acc(float* acc, const float* __restrict__ w, int ldw, int nrhs, int k0, int kb) {
    for (int idx = threadIdx.x; idx < NR * SB; idx += GT) {
        const int r = idx / SB, i = idx - r * SB;
        acc[idx] = (r < nrhs && i < kb) ? w[(size_t)r * ldw + k0 + i] : 0.0f;
    }
    __syncthreads();
}

template <int NR>
__global__ void __launch_bounds__(GT) k_gesl_fwd_inv(const float* __restrict__ a, int lda, int n,
                                                     const float* __restrict__ inv, float* __restrict__ w1,
                                                     float* __restrict__ w2, int ldw, int nrhs, int k0) {
    extern __shared__ float smem[];
    float* red = smem;                       // 8 x NR x 128 (panel_gemv)
    float* acc = red + 8 * NR * SB;          // NR x 128
    float* part = acc + NR * SB;             // 2 x NR x 128
    float* ys = part + 2 * NR * SB;          // NR x 128
    const int kb = min(SB, n - k0);
    load_acc<NR>(acc, w1, ldw, nrhs, k0, kb);
    block_matvec<NR>(inv + (size_t)(k0 / SB) * 2 * BLK2 + BLK2, acc, part, ys);
    if (blockIdx.x == 0)
        for (int idx = threadIdx.x; idx < NR * SB; idx += GT) {
            const int r = idx / SB, i = idx - r * SB;
            if (r < nrhs && i < kb) w2[(size_t)r * ldw + k0 + i] = ys[idx];
        }
    const int col0 = k0 + kb + blockIdx.x * GCOLS;
    if (col0 < n) panel_gemv<NR>(a, lda, k0, kb, col0, n, ys, red, w1, ldw, nrhs);
}

template <int NR>
__global__ void __launch_bounds__(GT) k_gesl_bwd_inv(const float* __restrict__ a, int lda, int n,
                                                     const float* __restrict__ inv, float* __restrict__ w2,
                                                     float* __restrict__ out, int ldo, int ldw, int nrhs, int k0) {
    extern __shared__ float smem[];
    float* red = smem;
    float* acc = red + 8 * NR * SB;
    float* part = acc + NR * SB;
    float* ss = part + 2 * NR * SB;
    const int kb = min(SB, n - k0);
    load_acc<NR>(acc, w2, ldw, nrhs, k0, kb);
    block_matvec<NR>(inv + (size_t)(k0 / SB) * 2 * BLK2, acc, part, ss);
    if (blockIdx.x == 0)
        for (int idx = threadIdx.x; idx < NR * SB; idx += GT) {
            const int r = idx / SB, i = idx - r * SB;
            if (r < nrhs && i < kb) out[(size_t)r * ldo + k0 + i] = -ss[idx];
        }
    const int col0 = blockIdx.x * GCOLS;
    if (col0 < k0) panel_gemv<NR>(a, lda, k0, kb, col0, k0, ss, red, w2, ldw, nrhs);
}

template <int NR>
constexpr size_t inv_smem() {
    return sizeof(float) * (8 * NR + 4 * NR) * (size_t)SB;
}

template <int NR>
int sweeps_inv(const float* a, int lda, int n, float* b, int ldb, int nrhs, float* w1, float* w2, const float* inv,
               cudaStream_t st) {
    const int nblk = (n + SB - 1) / SB;
    for (int K = 0; K < nblk; K++) {
        const int k0 = K * SB;
        const int rest = n - k0 - min(SB, n - k0);
        const int grid = rest > 0 ? (rest + GCOLS - 1) / GCOLS : 1;
        k_gesl_fwd_inv<NR><<<grid, GT, inv_smem<NR>(), st>>>(a, lda, n, inv, w1, w2, n, nrhs, k0);
    }
    for (int K = nblk - 1; K >= 0; K--) {
        const int k0 = K * SB;
        const int grid = k0 > 0 ? (k0 + GCOLS - 1) / GCOLS : 1;
        k_gesl_bwd_inv<NR><<<grid, GT, inv_smem<NR>(), st>>>(a, lda, n, inv, w2, b, ldb, n, nrhs, k0);
    }
    count_launch(2 * nblk);
    LP_CUDA(cudaGetLastError());
    return LP_OK;
}

template <int NR>
int inv_attrs() {
    LP_CUDA(cudaFuncSetAttribute(k_gesl_fwd_inv<NR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)inv_smem<NR>()));
    LP_CUDA(cudaFuncSetAttribute(k_gesl_bwd_inv<NR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)inv_smem<NR>()));
    return LP_OK;
}

}  // namespace

int gesl_inv_init_attrs() {
    LP_CUDA(cudaFuncSetAttribute(k_inv_top, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kInvTopSmem));
    LP_CUDA(cudaFuncSetAttribute(k_inv_left, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kInvLeftSmem));
    LP_CHECK(inv_attrs<1>());
    LP_CHECK(inv_attrs<4>());
    LP_CHECK(inv_attrs<16>());
    return LP_OK;
}

size_t gesl_inv_floats(int n) { return (size_t)((n + SB - 1) / SB) * 2 * BLK2; }

// X and Y of every diagonal block of the factors (inv: gesl_inv_floats(n)).
int launch_diag_inverses(const float* a, int lda, int n, float* inv, cudaStream_t st) {
    const int nblk = (n + SB - 1) / SB;
    if (nblk > 65535) return fail(LP_E_INVALID, "gesl: too many blocks");
    const dim3 grid(SB / IST, nblk);
    k_inv_top<<<grid, 256, kInvTopSmem, st>>>(a, lda, n, inv);
    k_inv_left<<<grid, 256, kInvLeftSmem, st>>>(a, lda, n, inv);
    count_launch(2);
    LP_CUDA(cudaGetLastError());
    return LP_OK;
}

// Forward + back substitution with precomputed block inverses.
int launch_gesl_inv(const float* a, int lda, int n, float* b, int ldb, int nrhs, float* work, const float* inv,
                    cudaStream_t st) {
    if (n <= 0 || nrhs <= 0) return LP_OK;
    for (int r0 = 0; r0 < nrhs; r0 += 16) {
        const int g = (nrhs - r0) < 16 ? (nrhs - r0) : 16;
        float* bb = b + (size_t)r0 * ldb;
        float* w1 = work;
        float* w2 = work + (size_t)n * g;
        LP_CUDA(cudaMemcpy2DAsync(w1, sizeof(float) * n, bb, sizeof(float) * ldb, sizeof(float) * n, g,
                                  cudaMemcpyDeviceToDevice, st));
        if (g == 1)
            LP_CHECK(sweeps_inv<1>(a, lda, n, bb, ldb, g, w1, w2, inv, st));
        else if (g <= 4)
            LP_CHECK(sweeps_inv<4>(a, lda, n, bb, ldb, g, w1, w2, inv, st));
        else
            LP_CHECK(sweeps_inv<16>(a, lda, n, bb, ldb, g, w1, w2, inv, st));
    }
    return LP_OK;
}

}  // namespace lp
