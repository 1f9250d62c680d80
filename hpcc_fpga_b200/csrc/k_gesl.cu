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
#include <mutex>

#include "gesl_common.cuh"

namespace lp {
namespace {

using namespace gesl;

__device__ __forceinline__ float pick4(const float (&y)[4], int q) {
    return q == 0 ? y[0] : (q == 1 ? y[1] : (q == 2 ? y[2] : y[3]));
}


// The kb x kb diagonal block into shared memory (row length SB): 16-byte
// loads, all of a thread's 16 loads issued before any is consumed.
__device__ __forceinline__ void stage_diag(float* dg, const float* __restrict__ a, int lda, int k0, int kb) {
#pragma unroll
    for (int it = 0; it < SB * SB / 4 / GT; it++) {
        const int idx = threadIdx.x + it * GT;
        const int r = idx >> 5, c = (idx & 31) * 4;
        float4 v = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if (r < kb) {
            const float* src = a + (size_t)(k0 + r) * lda + k0 + c;
            if (c + 3 < kb) {
                v = *reinterpret_cast<const float4*>(src);
            } else {
                if (c < kb) v.x = src[0];
                if (c + 1 < kb) v.y = src[1];
                if (c + 2 < kb) v.z = src[2];
            }
        }
        *reinterpret_cast<float4*>(dg + r * SB + c) = v;
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
    const int col0 = k0 + kb + blockIdx.x * GCOLS;
    if (col0 < n) panel_gemv<NR>(a, lda, k0, kb, col0, n, ys, dg, w1, ldw, nrhs);
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
    const int col0 = blockIdx.x * GCOLS;
    if (col0 < k0) panel_gemv<NR>(a, lda, k0, kb, col0, k0, ss, dg, w2, ldw, nrhs);
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

// ---- allocation-free variant (lp_gesl_dev_noalloc) ---------------------------
// Its two work vectors live in this fixed device array instead of a context
// workspace: 2^20 floats (4 MiB), enough for 2 * n * min(nrhs, 16) <= 2^20.
// Every GPU that loads the library holds the array until the process exits.
// Host code only sees a host-side stand-in for the array's name; the device
// address is looked up once per device with cudaGetSymbolAddress.
constexpr size_t kNoAllocScratchFloats = size_t(1) << 20;
static __device__ __align__(256) float g_gesl_scratch[kNoAllocScratchFloats];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
float* g_noalloc_ptr[kMaxDevices] = {nullptr};

// Once per device, with that device current: attributes of the substitution
// kernels and the scratch array's device address.
int noalloc_setup(int dev, float** out) {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (g_noalloc_ptr[dev] == nullptr) {
        LP_CHECK(gesl_init_attrs());
        void* p = nullptr;
        LP_CUDA(cudaGetSymbolAddress(&p, g_gesl_scratch));
        g_noalloc_ptr[dev] = static_cast<float*>(p);
    }
    *out = g_noalloc_ptr[dev];
    return LP_OK;
}
}  // namespace

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

extern "C" int lp_gesl_dev_noalloc(const float* dLU, int n, int lda, float* dB, int nrhs, int ldb, void* stream) {
    using namespace lp;
    if (dLU == nullptr || dB == nullptr) return fail(LP_E_INVALID, "lp_gesl_dev_noalloc: null argument");
    if (n <= 0 || lda < n || nrhs <= 0 || ldb < n) return fail(LP_E_INVALID, "lp_gesl_dev_noalloc: bad sizes");
    if (lda % 4 != 0 || !aligned16(dLU))
        return fail(LP_E_INVALID, "lp_gesl_dev_noalloc: factors must be 16-byte aligned with lda a multiple of 4");
    if (gesl_work_floats(n, nrhs) > kNoAllocScratchFloats)
        return fail(LP_E_INVALID, "lp_gesl_dev_noalloc: 2 * n * min(nrhs, 16) exceeds the fixed scratch of 1048576 "
                                  "floats (4 MiB); use lp_gesl_dev for larger systems");
    int dev = 0;
    LP_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return fail(LP_E_INVALID, "lp_gesl_dev_noalloc: device index out of range");
    float* scratch = nullptr;
    LP_CHECK(noalloc_setup(dev, &scratch));
    return launch_gesl(dLU, lda, n, dB, ldb, nrhs, scratch, static_cast<cudaStream_t>(stream));
}
