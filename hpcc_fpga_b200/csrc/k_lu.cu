// lu stage: LU without pivoting of one diagonal block (bs <= 128), the block
// resident in shared memory, one CTA.
//
// Arithmetic follows gefa_ref_nopvt (LINPACK/src/host/linpack_data.cpp:166-196)
// operation for operation, with no fused multiply-add, so the block result is
// bit-identical to the reference's host routine:
//   d = -1/a_kk  (double division, rounded to float)
//   a_ki = a_ki * d                       (i > k)
//   a_ji = a_ji + a_ki * a_jk             (j > k, i > k)
// The scaled pivot row is not stored before the update: every thread forms
// a_ki * d itself (same rounding), and row k is written back during step k+1,
// when no thread reads it any more.  One barrier per step.
#include "lp_common.cuh"

namespace lp {
namespace {

constexpr int kLuThreads = 512;

__global__ void __launch_bounds__(kLuThreads) k_lu_small(float* __restrict__ a, int lda, int bs, int log2bs) {
    extern __shared__ float s[];  // bs x bs, row-major
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    constexpr int nw = kLuThreads / 32;

    for (int idx = tid; idx < bs * bs; idx += kLuThreads) {
        const int r = idx >> log2bs, c = idx & (bs - 1);
        s[idx] = a[(size_t)r * lda + c];
    }
    __syncthreads();

    float inv_prev = 0.0f;
    for (int k = 0; k < bs; k++) {
        const float inv = (float)(-1.0 / (double)s[k * bs + k]);
        // Finalize the previous pivot row: store -1/d and the scaled row.
        if (k > 0) {
            float* rp = s + (k - 1) * bs;
            for (int i = k + tid; i < bs; i += kLuThreads) rp[i] = __fmul_rn(rp[i], inv_prev);
            if (tid == 0) rp[k - 1] = inv_prev;
        }
        // Rank-1 update of the trailing part with the (on-the-fly scaled) row k.
        const float* rk = s + k * bs;
        float sc[4];
        int ii[4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            ii[q] = k + 1 + lane + 32 * q;
            sc[q] = (ii[q] < bs) ? __fmul_rn(rk[ii[q]], inv) : 0.0f;
        }
        for (int j = k + 1 + warp; j < bs; j += nw) {
            float* rj = s + j * bs;
            const float sjk = rj[k];
#pragma unroll
            for (int q = 0; q < 4; q++)
                if (ii[q] < bs) rj[ii[q]] = __fadd_rn(rj[ii[q]], __fmul_rn(sc[q], sjk));
        }
        inv_prev = inv;
        __syncthreads();
    }
    if (tid == 0) s[(bs - 1) * bs + (bs - 1)] = inv_prev;
    __syncthreads();

    for (int idx = tid; idx < bs * bs; idx += kLuThreads) {
        const int r = idx >> log2bs, c = idx & (bs - 1);
        a[(size_t)r * lda + c] = s[idx];
    }
}

}  // namespace

int launch_lu_small(float* a, int lda, int bs, cudaStream_t st) {
    if (!is_pow2(bs) || bs > 128 || bs < 1) return fail(LP_E_INVALID, "lu_small: bs must be a power of two <= 128");
    int log2bs = 0;
    while ((1 << log2bs) < bs) log2bs++;
    const size_t smem = sizeof(float) * (size_t)bs * bs;
    k_lu_small<<<1, kLuThreads, smem, st>>>(a, lda, bs, log2bs);
    count_launch();
    LP_CUDA(cudaGetLastError());
    return LP_OK;
}

int lu_init_attrs() {
    LP_CUDA(cudaFuncSetAttribute(k_lu_small, cudaFuncAttributeMaxDynamicSharedMemorySize, 128 * 128 * 4));
    return LP_OK;
}

}  // namespace lp
