// gesl: forward and back substitution with the encoded factors on the device
// (the reference runs gesl_ref_nopvt on the host, linpack_data.cpp:199-229,
// and times an empty region for it, execution_pcie.hpp:663-669).
//
// Storage terms (S[r][c] = a[r*lda + c]):
//   forward   y_i += y_k * S[k][i]            for i > k   (unit, negated multipliers)
//   backward  s = y_k * S[k][k]; x_k = -s;  y_i += s * S[k][i]  for i < k
// Blocked by SB = 128 unknowns.  One launch per block and direction:
//   (a) every CTA stages the SB x SB diagonal block in shared memory and
//       solves it redundantly in warps (one warp per right-hand side, values
//       passed by warp shuffles, no global load on the sequential chain),
//   (b) then updates its share of the remaining unknowns with the block's
//       row panel S[block rows][other columns] (a GEMV over contiguous rows,
//       each factor element read once per sweep, for all right-hand sides).
// The accumulating vector and the solved vector are separate buffers, so
// step (a) of launch K never reads what step (b) of launch K writes.
#include "lp_common.cuh"

namespace lp {
namespace {

constexpr int SB = 128;
constexpr int GT = 256;            // threads per CTA
constexpr int GCOLS = GT;          // columns per CTA in step (b)

__device__ __forceinline__ float pick4(const float (&y)[4], int q) {
    return q == 0 ? y[0] : (q == 1 ? y[1] : (q == 2 ? y[2] : y[3]));
}

__device__ __forceinline__ void stage_diag(float* dg, const float* __restrict__ a, int lda, int k0, int kb) {
    for (int idx = threadIdx.x; idx < kb * SB; idx += GT) {
        const int r = idx >> 7, c = idx & (SB - 1);
        dg[idx] = (c < kb) ? a[(size_t)(k0 + r) * lda + k0 + c] : 0.0f;
    }
}

template <int NR>
__global__ void __launch_bounds__(GT) k_gesl_fwd(const float* __restrict__ a, int lda, int n,
                                                 float* __restrict__ w1, float* __restrict__ w2, int ldw, int nrhs,
                                                 int k0) {
    extern __shared__ float smem[];
    float* dg = smem;               // SB x SB diagonal block
    float* ys = smem + SB * SB;     // NR x SB solved values
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int kb = min(SB, n - k0);
    stage_diag(dg, a, lda, k0, kb);
    __syncthreads();
    for (int r = warp; r < nrhs; r += GT / 32) {
        float y[4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int i = lane + 32 * q;
            y[q] = (i < kb) ? w1[(size_t)r * ldw + k0 + i] : 0.0f;
        }
        for (int k = 0; k < kb; k++) {
            const float yk = __shfl_sync(0xffffffffu, pick4(y, k >> 5), k & 31);
            const float* row = dg + k * SB;
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int i = lane + 32 * q;
                if (i > k && i < kb) y[q] = fmaf(yk, row[i], y[q]);
            }
        }
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int i = lane + 32 * q;
            if (i < kb) {
                ys[r * SB + i] = y[q];
                if (blockIdx.x == 0) w2[(size_t)r * ldw + k0 + i] = y[q];
            }
        }
    }
    __syncthreads();
    const int i = k0 + kb + blockIdx.x * GCOLS + threadIdx.x;
    if (i < n) {
        float acc[NR];
#pragma unroll
        for (int r = 0; r < NR; r++) acc[r] = 0.0f;
        const float* col = a + (size_t)k0 * lda + i;
#pragma unroll 4
        for (int k = 0; k < kb; k++) {
            const float v = col[(size_t)k * lda];
#pragma unroll
            for (int r = 0; r < NR; r++) acc[r] = fmaf(ys[r * SB + k], v, acc[r]);
        }
#pragma unroll
        for (int r = 0; r < NR; r++)
            if (r < nrhs) w1[(size_t)r * ldw + i] += acc[r];
    }
}

template <int NR>
__global__ void __launch_bounds__(GT) k_gesl_bwd(const float* __restrict__ a, int lda, int n,
                                                 float* __restrict__ w2, float* __restrict__ out, int ldo, int ldw,
                                                 int nrhs, int k0) {
    extern __shared__ float smem[];
    float* dg = smem;
    float* ss = smem + SB * SB;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int kb = min(SB, n - k0);
    stage_diag(dg, a, lda, k0, kb);
    __syncthreads();
    for (int r = warp; r < nrhs; r += GT / 32) {
        float y[4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int i = lane + 32 * q;
            y[q] = (i < kb) ? w2[(size_t)r * ldw + k0 + i] : 0.0f;
        }
        for (int k = kb - 1; k >= 0; k--) {
            const int qk = k >> 5;
            const float yk = __shfl_sync(0xffffffffu, pick4(y, qk), k & 31);
            const float* row = dg + k * SB;
            const float s = yk * row[k];
            if (lane == (k & 31)) {
#pragma unroll
                for (int q = 0; q < 4; q++)
                    if (q == qk) y[q] = -s;
                ss[r * SB + k] = s;
            }
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int i = lane + 32 * q;
                if (i < k) y[q] = fmaf(s, row[i], y[q]);
            }
        }
        if (blockIdx.x == 0) {
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int i = lane + 32 * q;
                if (i < kb) out[(size_t)r * ldo + k0 + i] = y[q];
            }
        }
    }
    __syncthreads();
    const int i = blockIdx.x * GCOLS + threadIdx.x;
    if (i < k0) {
        float acc[NR];
#pragma unroll
        for (int r = 0; r < NR; r++) acc[r] = 0.0f;
        const float* col = a + (size_t)k0 * lda + i;
#pragma unroll 4
        for (int k = 0; k < kb; k++) {
            const float v = col[(size_t)k * lda];
#pragma unroll
            for (int r = 0; r < NR; r++) acc[r] = fmaf(ss[r * SB + k], v, acc[r]);
        }
#pragma unroll
        for (int r = 0; r < NR; r++)
            if (r < nrhs) w2[(size_t)r * ldw + i] += acc[r];
    }
}

template <int NR>
constexpr size_t gesl_smem() {
    return sizeof(float) * ((size_t)SB * SB + (size_t)NR * SB);
}

template <int NR>
int gesl_sweeps(const float* a, int lda, int n, float* b, int ldb, int nrhs, float* w1, float* w2, cudaStream_t st) {
    const int nblk = (n + SB - 1) / SB;
    for (int K = 0; K < nblk; K++) {
        const int k0 = K * SB;
        const int kb = min(SB, n - k0);
        const int rest = n - k0 - kb;
        const int grid = rest > 0 ? (rest + GCOLS - 1) / GCOLS : 1;
        k_gesl_fwd<NR><<<grid, GT, gesl_smem<NR>(), st>>>(a, lda, n, w1, w2, n, nrhs, k0);
        count_launch();
    }
    for (int K = nblk - 1; K >= 0; K--) {
        const int k0 = K * SB;
        const int grid = k0 > 0 ? (k0 + GCOLS - 1) / GCOLS : 1;
        k_gesl_bwd<NR><<<grid, GT, gesl_smem<NR>(), st>>>(a, lda, n, w2, b, ldb, n, nrhs, k0);
        count_launch();
    }
    LP_CUDA(cudaGetLastError());
    return LP_OK;
}

template <int NR>
int gesl_attrs() {
    LP_CUDA(cudaFuncSetAttribute(k_gesl_fwd<NR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)gesl_smem<NR>()));
    LP_CUDA(cudaFuncSetAttribute(k_gesl_bwd<NR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)gesl_smem<NR>()));
    return LP_OK;
}

}  // namespace

int gesl_init_attrs() {
    LP_CHECK(gesl_attrs<1>());
    LP_CHECK(gesl_attrs<4>());
    LP_CHECK(gesl_attrs<16>());
    return LP_OK;
}

size_t gesl_work_floats(int n, int nrhs) {
    const int g = nrhs < 16 ? nrhs : 16;
    return 2 * (size_t)n * (size_t)g;
}

int launch_gesl(const float* a, int lda, int n, float* b, int ldb, int nrhs, float* work, cudaStream_t st) {
    if (n <= 0 || nrhs <= 0) return LP_OK;
    for (int r0 = 0; r0 < nrhs; r0 += 16) {
        const int g = (nrhs - r0) < 16 ? (nrhs - r0) : 16;
        float* bb = b + (size_t)r0 * ldb;
        float* w1 = work;
        float* w2 = work + (size_t)n * g;
        LP_CUDA(cudaMemcpy2DAsync(w1, sizeof(float) * n, bb, sizeof(float) * ldb, sizeof(float) * n, g,
                                  cudaMemcpyDeviceToDevice, st));
        if (g == 1)
            LP_CHECK(gesl_sweeps<1>(a, lda, n, bb, ldb, g, w1, w2, st));
        else if (g <= 4)
            LP_CHECK(gesl_sweeps<4>(a, lda, n, bb, ldb, g, w1, w2, st));
        else
            LP_CHECK(gesl_sweeps<16>(a, lda, n, bb, ldb, g, w1, w2, st));
    }
    return LP_OK;
}

}  // namespace lp
