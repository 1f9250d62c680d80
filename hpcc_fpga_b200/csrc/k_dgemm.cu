// inner stage, FP64 (the reference's _DP build, DATA_TYPE double): C(m x n) +=
// At^T * B on k-major operands (At: k x m, B: k x n, rows of contiguous
// doubles) — inner_update_mm (hpl_torus_PCIE.cl:711-865) in double.
//
// FP64 runs on the SIMT FMA pipe (tcgen05 has no FP64 kind; the FP64 tensor
// rate of this part equals its DFMA rate).  128 x 64 x 8 tiles, 256 threads,
// 8 x 4 FP64 accumulators per thread (two 4-row groups, one 4-column group),
// operands staged by 16-byte cp.async into a 4-deep shared-memory ring; C is
// read and written once per launch.
#include "lp_common.cuh"

namespace lp {
namespace {

constexpr int BM = 128, BN = 64, BK = 8, STAGES = 4, NT = 256;

__device__ __forceinline__ void cp_async16z(void* smem, const void* gmem, int src_bytes) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes));
}

__global__ void __launch_bounds__(NT, 2) k_dgemm_update(double* __restrict__ C, int ldc,
                                                        const double* __restrict__ At, int ldat,
                                                        const double* __restrict__ B, int ldb, int M, int N, int K) {
    extern __shared__ __align__(16) double dsm[];
    double* As = dsm;                       // STAGES x BK x BM
    double* Bs = dsm + STAGES * BK * BM;    // STAGES x BK x BN
    const int tid = threadIdx.x;
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    const int ty = tid >> 4, tx = tid & 15;

    auto load_stage = [&](int stage, int kt) {
#pragma unroll
        for (int i = 0; i < 2; i++) {  // A: BK rows of 128 doubles = 512 pairs
            const int idx = tid + i * NT;
            const int row = idx >> 6, col = (idx & 63) * 2;
            const bool ok = (m0 + col) < M;
            const double* src = ok ? At + (size_t)(kt * BK + row) * ldat + m0 + col : At;
            cp_async16z(&As[(stage * BK + row) * BM + col], src, ok ? 16 : 0);
        }
        {  // B: BK rows of 64 doubles = 256 pairs
            const int row = tid >> 5, col = (tid & 31) * 2;
            const bool ok = (n0 + col) < N;
            const double* src = ok ? B + (size_t)(kt * BK + row) * ldb + n0 + col : B;
            cp_async16z(&Bs[(stage * BK + row) * BN + col], src, ok ? 16 : 0);
        }
    };

    double acc[8][4];
#pragma unroll
    for (int i = 0; i < 8; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = 0.0;

    const int KT = K / BK;
#pragma unroll
    for (int s = 0; s < STAGES - 1; s++) {
        if (s < KT) load_stage(s, s);
        asm volatile("cp.async.commit_group;\n" ::);
    }
    for (int kt = 0; kt < KT; kt++) {
        asm volatile("cp.async.wait_group %0;\n" ::"n"(STAGES - 2));
        __syncthreads();
        const int nk = kt + STAGES - 1;
        if (nk < KT) load_stage(nk % STAGES, nk);
        asm volatile("cp.async.commit_group;\n" ::);
        const double* as = As + (kt % STAGES) * BK * BM;
        const double* bs = Bs + (kt % STAGES) * BK * BN;
#pragma unroll
        for (int k = 0; k < BK; k++) {
            const Quad<double> a0 = ld_quad(as + k * BM + ty * 4);
            const Quad<double> a1 = ld_quad(as + k * BM + 64 + ty * 4);
            const Quad<double> b0 = ld_quad(bs + k * BN + tx * 4);
            const double a[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
            const double b[4] = {b0.x, b0.y, b0.z, b0.w};
#pragma unroll
            for (int i = 0; i < 8; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) acc[i][j] = fma(a[i], b[j], acc[i][j]);
        }
    }
    asm volatile("cp.async.wait_group 0;\n" ::);

    const int c = n0 + tx * 4;
    if (c >= N) return;
#pragma unroll
    for (int i = 0; i < 8; i++) {
        const int r = m0 + ((i < 4) ? ty * 4 + i : 64 + ty * 4 + (i - 4));
        if (r >= M) continue;
        double2* p = reinterpret_cast<double2*>(C + (size_t)r * ldc + c);
        double2 u = p[0], v = p[1];
        u.x += acc[i][0];
        u.y += acc[i][1];
        v.x += acc[i][2];
        v.y += acc[i][3];
        p[0] = u;
        p[1] = v;
    }
}

constexpr size_t kDgemmSmem = sizeof(double) * STAGES * BK * (BM + BN);

}  // namespace

int dgemm_init_attrs() {
    LP_CUDA(cudaFuncSetAttribute(k_dgemm_update, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDgemmSmem));
    return LP_OK;
}

int launch_dgemm_update(double* c, int ldc, const double* lt, int ldlt, const double* t, int ldt, int m, int n, int k,
                        cudaStream_t st) {
    if (m <= 0 || n <= 0) return LP_OK;
    if (k % BK != 0 || m % 4 != 0 || n % 4 != 0 || ldc % 2 != 0 || ldlt % 2 != 0 || ldt % 2 != 0 || !aligned16(c) ||
        !aligned16(lt) || !aligned16(t))
        return fail(LP_E_INVALID, "FP64 inner update: k a multiple of 8; m, n multiples of 4; leading dimensions "
                                  "even; pointers 16-byte aligned");
    if ((m + BM - 1) / BM > 65535) return fail(LP_E_INVALID, "FP64 inner update: m too large");
    const dim3 grid((n + BN - 1) / BN, (m + BM - 1) / BM);
    k_dgemm_update<<<grid, NT, kDgemmSmem, st>>>(c, ldc, lt, ldlt, t, ldt, m, n, k);
    count_launch();
    LP_CUDA(cudaGetLastError());
    return LP_OK;
}

}  // namespace lp
