// Shared pieces of the substitution kernels (k_gesl.cu, k_gesl_inv.cu).
#pragma once

#include "lp_common.cuh"

namespace lp {
namespace gesl {

constexpr int SB = 128;
constexpr int GT = 256;            // threads per CTA
constexpr int GCOLS = 128;         // columns per CTA in step (b)

// Step (b): w[r][c] += sum_{k<kb} coef[r][k] * a[(k0+k)*lda + c] for the
// CTA's 128 columns c in [col0, colend).  Warp w takes rows 16w..16w+15 of
// the block, each lane 4 adjacent columns (16-byte loads, 16 independent
// loads in flight per thread); the 8 warps' partial sums meet in shared
// memory (`red`, 8 x NR x 128 floats, the diagonal block's buffer reused).
template <int NR>
__device__ __forceinline__ void panel_gemv(const float* __restrict__ a, int lda, int k0, int kb, int col0,
                                           int colend, const float* coef, float* red, float* __restrict__ w,
                                           int ldw, int nrhs) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int c = col0 + lane * 4;
    float acc[NR][4];
#pragma unroll
    for (int r = 0; r < NR; r++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[r][j] = 0.0f;
    const int kbeg = warp * 16;
    if (c + 3 < colend) {
#pragma unroll
        for (int kk = 0; kk < 16; kk++) {
            const int k = kbeg + kk;
            if (k < kb) {
                const float4 v = *reinterpret_cast<const float4*>(a + (size_t)(k0 + k) * lda + c);
#pragma unroll
                for (int r = 0; r < NR; r++) {
                    const float s = coef[r * SB + k];
                    acc[r][0] = fmaf(s, v.x, acc[r][0]);
                    acc[r][1] = fmaf(s, v.y, acc[r][1]);
                    acc[r][2] = fmaf(s, v.z, acc[r][2]);
                    acc[r][3] = fmaf(s, v.w, acc[r][3]);
                }
            }
        }
    } else if (c < colend) {
        for (int kk = 0; kk < 16; kk++) {
            const int k = kbeg + kk;
            if (k >= kb) break;
            const float* row = a + (size_t)(k0 + k) * lda + c;
#pragma unroll
            for (int j = 0; j < 4; j++)
                if (c + j < colend) {
                    const float v = row[j];
#pragma unroll
                    for (int r = 0; r < NR; r++) acc[r][j] = fmaf(coef[r * SB + k], v, acc[r][j]);
                }
        }
    }
    __syncthreads();  // the caller's use of `red` (the diagonal block) is over
#pragma unroll
    for (int r = 0; r < NR; r++)
#pragma unroll
        for (int j = 0; j < 4; j++) red[(warp * NR + r) * GCOLS + lane * 4 + j] = acc[r][j];
    __syncthreads();
    for (int idx = threadIdx.x; idx < NR * GCOLS; idx += GT) {
        const int r = idx / GCOLS, cc = idx - r * GCOLS;
        if (r < nrhs && col0 + cc < colend) {
            float s = 0.0f;
#pragma unroll
            for (int q = 0; q < GT / 32; q++) s += red[(q * NR + r) * GCOLS + cc];
            w[(size_t)r * ldw + col0 + cc] += s;
        }
    }
}

}  // namespace gesl
}  // namespace lp
