// top and left stages: the triangular block updates of the blocked LU.
//
// top (hpl_torus_PCIE.cl:452-582; host loop
// LINPACK/tests/test_kernel_communication.cpp:776-789) acts on the bs x ncols
// block row right of a factored diagonal block D.  Every column is
// independent:   for k: t_k *= D_kk;  for j > k: t_j += t_k * D_jk.
// A CTA owns a strip of 64 columns (all bs rows) in shared memory and walks
// the rows in chunks of CH: (1) two warps solve the CH x CH diagonal chunk,
// one thread per column; (2) all threads apply the solved chunk to the rows
// below it.  Every element receives its updates in ascending k, exactly as
// the host loop does, and with no fused multiply-add, so the result is
// bit-identical to the reference loop.
//
// left (hpl_torus_PCIE.cl:588-709; host loop
// test_kernel_communication.cpp:624-631) acts on the nrows x bs block column
// below D.  Every row is independent:  for k, i > k: l_i += l_k * D_ki.
// A CTA owns 64 rows (all bs columns, row length padded to bs+1 against
// bank conflicts) and walks the columns in chunks of CH the same way.  It
// writes the rows back in place and, optionally, transposed into Lt — the
// k-major operand layout of the trailing update (the reference keeps the
// same transposed copy, left_block, hpl_torus_PCIE.cl:697-708).
#include "lp_common.cuh"

namespace lp {
namespace {

constexpr int kTrsmThreads = 256;
constexpr int kStrip = 64;

template <int CH>
__global__ void __launch_bounds__(kTrsmThreads) k_trsm_top(const float* __restrict__ lu, int ldlu,
                                                         float* __restrict__ t, int ldt, int bs, int ncols) {
    extern __shared__ float sm[];
    float* strip = sm;                // bs x 64
    float* dch = sm + bs * kStrip;    // (bs - r0) x CH
    const int tid = threadIdx.x;
    const int c0 = blockIdx.x * kStrip;

    for (int idx = tid; idx < bs * kStrip; idx += kTrsmThreads) {
        const int r = idx >> 6, c = idx & 63;
        strip[idx] = (c0 + c < ncols) ? t[(size_t)r * ldt + c0 + c] : 0.0f;
    }
    for (int r0 = 0; r0 < bs; r0 += CH) {
        const int nr = bs - r0;
        for (int idx = tid; idx < nr * CH; idx += kTrsmThreads) {
            const int rr = idx / CH, kk = idx - rr * CH;
            dch[idx] = lu[(size_t)(r0 + rr) * ldlu + r0 + kk];
        }
        __syncthreads();
        if (tid < kStrip) {
            float x[CH];
#pragma unroll
            for (int k = 0; k < CH; k++) x[k] = strip[(r0 + k) * kStrip + tid];
#pragma unroll
            for (int k = 0; k < CH; k++) {
                const float xk = __fmul_rn(x[k], dch[k * CH + k]);
                x[k] = xk;
#pragma unroll
                for (int j = k + 1; j < CH; j++) x[j] = __fadd_rn(x[j], __fmul_rn(xk, dch[j * CH + k]));
            }
#pragma unroll
            for (int k = 0; k < CH; k++) strip[(r0 + k) * kStrip + tid] = x[k];
        }
        __syncthreads();
        if (nr > CH) {
            const int c = tid & 63, g = tid >> 6;
            float x[CH];
#pragma unroll
            for (int k = 0; k < CH; k++) x[k] = strip[(r0 + k) * kStrip + c];
            for (int r = r0 + CH + g; r < bs; r += kTrsmThreads / kStrip) {
                float acc = strip[r * kStrip + c];
                const float* drow = dch + (r - r0) * CH;
#pragma unroll
                for (int k = 0; k < CH; k++) acc = __fadd_rn(acc, __fmul_rn(x[k], drow[k]));
                strip[r * kStrip + c] = acc;
            }
        }
        __syncthreads();
    }
    for (int idx = tid; idx < bs * kStrip; idx += kTrsmThreads) {
        const int r = idx >> 6, c = idx & 63;
        if (c0 + c < ncols) t[(size_t)r * ldt + c0 + c] = strip[idx];
    }
}

template <int CH>
__global__ void __launch_bounds__(kTrsmThreads) k_trsm_left(const float* __restrict__ lu, int ldlu,
                                                          float* __restrict__ l, int ldl, int bs, int log2bs,
                                                          int nrows, float* __restrict__ lt, int ldlt) {
    extern __shared__ float sm[];
    const int sl = bs + 1;
    float* strip = sm;               // 64 x (bs+1)
    float* dch = sm + kStrip * sl;   // CH x (bs - c0)
    const int tid = threadIdx.x;
    const int r0 = blockIdx.x * kStrip;

    for (int idx = tid; idx < kStrip * bs; idx += kTrsmThreads) {
        const int rr = idx >> log2bs, c = idx & (bs - 1);
        strip[rr * sl + c] = (r0 + rr < nrows) ? l[(size_t)(r0 + rr) * ldl + c] : 0.0f;
    }
    for (int c0 = 0; c0 < bs; c0 += CH) {
        const int nc = bs - c0;
        for (int idx = tid; idx < CH * nc; idx += kTrsmThreads) {
            const int kk = idx / nc, cc = idx - kk * nc;
            dch[idx] = lu[(size_t)(c0 + kk) * ldlu + c0 + cc];
        }
        __syncthreads();
        if (tid < kStrip) {
            float x[CH];
            float* row = strip + tid * sl + c0;
#pragma unroll
            for (int k = 0; k < CH; k++) x[k] = row[k];
#pragma unroll
            for (int k = 0; k < CH; k++) {
#pragma unroll
                for (int i = k + 1; i < CH; i++) x[i] = __fadd_rn(x[i], __fmul_rn(x[k], dch[k * nc + i]));
            }
#pragma unroll
            for (int k = 0; k < CH; k++) row[k] = x[k];
        }
        __syncthreads();
        for (int ci = CH + tid; ci < nc; ci += kTrsmThreads) {
            float d[CH];
#pragma unroll
            for (int k = 0; k < CH; k++) d[k] = dch[k * nc + ci];
            for (int rr = 0; rr < kStrip; rr++) {
                const float* row = strip + rr * sl + c0;
                float acc = row[ci];
#pragma unroll
                for (int k = 0; k < CH; k++) acc = __fadd_rn(acc, __fmul_rn(row[k], d[k]));
                strip[rr * sl + c0 + ci] = acc;
            }
        }
        __syncthreads();
    }
    for (int idx = tid; idx < kStrip * bs; idx += kTrsmThreads) {
        const int rr = idx >> log2bs, c = idx & (bs - 1);
        if (r0 + rr < nrows) l[(size_t)(r0 + rr) * ldl + c] = strip[rr * sl + c];
    }
    if (lt != nullptr) {
        for (int idx = tid; idx < kStrip * bs; idx += kTrsmThreads) {
            const int c = idx >> 6, rr = idx & 63;
            if (r0 + rr < nrows) lt[(size_t)c * ldlt + r0 + rr] = strip[rr * sl + c];
        }
    }
}

int log2i(int x) {
    int r = 0;
    while ((1 << r) < x) r++;
    return r;
}

size_t top_smem(int bs, int ch) { return sizeof(float) * ((size_t)bs * kStrip + (size_t)bs * ch); }
size_t left_smem(int bs, int ch) { return sizeof(float) * ((size_t)kStrip * (bs + 1) + (size_t)ch * bs); }

}  // namespace

int trsm_init_attrs() {
    const int max_smem = (int)left_smem(512, 32);
    LP_CUDA(cudaFuncSetAttribute(k_trsm_top<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)top_smem(512, 32)));
    LP_CUDA(cudaFuncSetAttribute(k_trsm_top<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)top_smem(512, 16)));
    LP_CUDA(cudaFuncSetAttribute(k_trsm_left<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, max_smem));
    LP_CUDA(cudaFuncSetAttribute(k_trsm_left<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)left_smem(512, 16)));
    return LP_OK;
}

int launch_trsm_top(const float* lu, int ldlu, float* t, int ldt, int bs, int ncols, cudaStream_t st) {
    if (!is_pow2(bs) || bs < 16 || bs > 512) return fail(LP_E_INVALID, "top_update: bs must be a power of two in [16, 512]");
    if (ncols <= 0) return LP_OK;
    const dim3 grid((ncols + kStrip - 1) / kStrip);
    if (bs >= 32)
        k_trsm_top<32><<<grid, kTrsmThreads, top_smem(bs, 32), st>>>(lu, ldlu, t, ldt, bs, ncols);
    else
        k_trsm_top<16><<<grid, kTrsmThreads, top_smem(bs, 16), st>>>(lu, ldlu, t, ldt, bs, ncols);
    count_launch();
    LP_CUDA(cudaGetLastError());
    return LP_OK;
}

int launch_trsm_left(const float* lu, int ldlu, float* l, int ldl, int bs, int nrows, float* lt, int ldlt,
                     cudaStream_t st) {
    if (!is_pow2(bs) || bs < 16 || bs > 512) return fail(LP_E_INVALID, "left_update: bs must be a power of two in [16, 512]");
    if (nrows <= 0) return LP_OK;
    const dim3 grid((nrows + kStrip - 1) / kStrip);
    const int lg = log2i(bs);
    if (bs >= 32)
        k_trsm_left<32><<<grid, kTrsmThreads, left_smem(bs, 32), st>>>(lu, ldlu, l, ldl, bs, lg, nrows, lt, ldlt);
    else
        k_trsm_left<16><<<grid, kTrsmThreads, left_smem(bs, 16), st>>>(lu, ldlu, l, ldl, bs, lg, nrows, lt, ldlt);
    count_launch();
    LP_CUDA(cudaGetLastError());
    return LP_OK;
}

}  // namespace lp
