// inner stage, FP32: C(m x n) += At^T * B on k-major operands
// (At: k x m, B: k x n, rows of contiguous floats).
//
// The trailing update of one block step runs as one or a few launches over
// the whole trailing matrix (the reference issues one inner_update_mm task
// per b x b block, hpl_torus_PCIE.cl:711-865, execution_pcie.hpp:523-583):
// C += L * T with L given transposed.  The blocked top/left stages use the
// same kernel for their chunk-to-rest updates.
//
// Both operands are k-major, so every tile load is a run of 16-byte cp.async
// copies into a STAGES-deep shared-memory ring.  128 x 128 x 16 tiles, 256
// threads, 8 x 8 FP32 accumulators per thread (two 4-row and two 4-column
// groups, conflict-free float4 shared loads), held as 8 x 4 pairs and updated
// with Blackwell's packed FP32 FMA (FFMA2, fma.rn.f32x2: two independent
// correctly rounded fused multiply-adds per issued instruction, so each
// element is computed exactly as fmaf would).  One FFMA2 per pair halves the
// FMA instructions of the FFMA form, whose issue rate was the limit.  C is
// read and written once per launch.
#include "lp_common.cuh"

namespace lp {
namespace {

constexpr int BM = 128, BN = 128, BK = 16, STAGES = 4, NT = 256;

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, int src_bytes) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

__global__ void __launch_bounds__(NT, 2) k_sgemm_update(float* __restrict__ C, int ldc, const float* __restrict__ At,
                                                        int ldat, const float* __restrict__ B, int ldb, int M, int N,
                                                        int K) {
    extern __shared__ __align__(16) float sm[];
    float* As = sm;
    float* Bs = sm + STAGES * BK * BM;
    const int tid = threadIdx.x;
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    const int ty = tid >> 4, tx = tid & 15;

    auto load_stage = [&](int stage, int kt) {
#pragma unroll
        for (int i = 0; i < 2; i++) {
            const int idx = tid + i * NT;
            const int row = idx >> 5, col = (idx & 31) * 4;
            const int kr = kt * BK + row;
            const bool oka = (m0 + col) < M;
            const float* srca = oka ? At + (size_t)kr * ldat + m0 + col : At;
            cp_async16(&As[(stage * BK + row) * BM + col], srca, oka ? 16 : 0);
            const bool okb = (n0 + col) < N;
            const float* srcb = okb ? B + (size_t)kr * ldb + n0 + col : B;
            cp_async16(&Bs[(stage * BK + row) * BN + col], srcb, okb ? 16 : 0);
        }
    };

    // acc[i][h] holds the pair of columns (2h, 2h + 1) of row i of the thread's 8 x 8 tile
    float2 acc[8][4];
#pragma unroll
    for (int i = 0; i < 8; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = make_float2(0.0f, 0.0f);

    const int KT = K / BK;
#pragma unroll
    for (int s = 0; s < STAGES - 1; s++) {
        if (s < KT) load_stage(s, s);
        cp_async_commit();
    }
    for (int kt = 0; kt < KT; kt++) {
        cp_async_wait<STAGES - 2>();
        __syncthreads();
        const int nk = kt + STAGES - 1;
        if (nk < KT) load_stage(nk % STAGES, nk);
        cp_async_commit();
        const float* as = As + (kt % STAGES) * BK * BM;
        const float* bsm = Bs + (kt % STAGES) * BK * BN;
#pragma unroll
        for (int k = 0; k < BK; k++) {
            const float4 a0 = *reinterpret_cast<const float4*>(&as[k * BM + ty * 4]);
            const float4 a1 = *reinterpret_cast<const float4*>(&as[k * BM + 64 + ty * 4]);
            const float4 b0 = *reinterpret_cast<const float4*>(&bsm[k * BN + tx * 4]);
            const float4 b1 = *reinterpret_cast<const float4*>(&bsm[k * BN + 64 + tx * 4]);
            const float a[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
            const float2 b[4] = {make_float2(b0.x, b0.y), make_float2(b0.z, b0.w), make_float2(b1.x, b1.y),
                                 make_float2(b1.z, b1.w)};
#pragma unroll
            for (int i = 0; i < 8; i++) {
                const float2 ai = make_float2(a[i], a[i]);
#pragma unroll
                for (int j = 0; j < 4; j++) acc[i][j] = __ffma2_rn(ai, b[j], acc[i][j]);
            }
        }
    }
    cp_async_wait<0>();

#pragma unroll
    for (int i = 0; i < 8; i++) {
        const int r = m0 + ((i < 4) ? ty * 4 + i : 64 + ty * 4 + (i - 4));
        if (r >= M) continue;
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int c = n0 + h * 64 + tx * 4;
            if (c >= N) continue;
            float4* p = reinterpret_cast<float4*>(C + (size_t)r * ldc + c);
            float4 v = *p;
            v.x += acc[i][2 * h].x;
            v.y += acc[i][2 * h].y;
            v.z += acc[i][2 * h + 1].x;
            v.w += acc[i][2 * h + 1].y;
            *p = v;
        }
    }
}

constexpr size_t kSgemmSmem = sizeof(float) * STAGES * BK * (BM + BN);

}  // namespace

int sgemm_init_attrs() {
    LP_CUDA(cudaFuncSetAttribute(k_sgemm_update, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSgemmSmem));
    return LP_OK;
}

int launch_sgemm_update(float* c, int ldc, const float* lt, int ldlt, const float* t, int ldt, int m, int n, int k,
                        cudaStream_t st) {
    if (m <= 0 || n <= 0) return LP_OK;
    if (k % BK != 0 || m % 4 != 0 || n % 4 != 0 || ldc % 4 != 0 || ldlt % 4 != 0 || ldt % 4 != 0 || !aligned16(c) ||
        !aligned16(lt) || !aligned16(t))
        return fail(LP_E_INVALID, "inner_update: k must be a multiple of 16; m, n, leading dimensions multiples of 4; "
                                  "pointers 16-byte aligned");
    if ((m + BM - 1) / BM > 65535) return fail(LP_E_INVALID, "inner_update: m too large");
    const dim3 grid((n + BN - 1) / BN, (m + BM - 1) / BM);
    k_sgemm_update<<<grid, NT, kSgemmSmem, st>>>(c, ldc, lt, ldlt, t, ldt, m, n, k);
    count_launch();
    LP_CUDA(cudaGetLastError());
    return LP_OK;
}

}  // namespace lp
