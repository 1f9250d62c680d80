// Mixed-precision factorization: the block schedule of gefa_f32 (one step of
// look-ahead) with the trailing update on the tensor cores (k_umma.cu), and
// the panel's top and left stages as tensor-core products with the inverted
// triangles of the FP32 diagonal block (panel_tc).  After each panel its left block column L and top
// block row T are rounded to the tensor-core operand type:
//   BF16:  Lq[m][k] = bf16(L[m][k]),  Tq[n][k] = bf16(T[k][n]);
//   E4M3:  one absmax scale per 512 x 512 block: per 512-row block of L and
//          512-wide K segment, per 512-column block of T and K segment
//          (s = absmax / 448), Lq = e4m3(L / s_L), Tq = e4m3(T^T / s_T), and
//          the update adds sum_seg s_L(seg) * s_T(seg) * (Lq_seg Tq_seg^T) in
//          FP32 (k_umma.cu accumulates every segment on its own).
// The FP32 factors the substitution uses are these rounded-update factors;
// accuracy is recovered by FP64 iterative refinement (lp_solve.cu).
//   BF16x6 (FP32 emulation): every element x of L and T is split exactly into
//          three BF16 terms x1 = bf16(x), x2 = bf16(x - x1), x3 = x - x1 - x2
//          (8 + 8 + 8 significant bits = the 24 of an FP32), and the operands
//          become six K-segments so that one tensor-core GEMM with K = 6 bs
//          accumulates x3 t1 + x2 t2 + x1 t3 + x2 t1 + x1 t2 + x1 t1 in FP32
//          (small terms first).  The three dropped products (x2 t3, x3 t2,
//          x3 t3) are below 2^-24 of x1 t1: the update has FP32 accuracy.
#include <cuda_bf16.h>
#include <cuda_fp8.h>

#include "lp_ctx.cuh"

namespace lp {
namespace {

constexpr float kE4M3Max = 448.0f;

__device__ __forceinline__ void atomic_max_nonneg(float* addr, float v) {
    atomicMax(reinterpret_cast<int*>(addr), __float_as_int(v));  // non-negative floats order as ints
}

// amax[seg * nblk + r / 512] = max |L[r][512 seg .. 512 seg + 512)| over each
// 512-row block (blockIdx.y = seg).
__global__ void k_absmax_rows(const float* __restrict__ L, int ldl, int rows, int k, int nblk,
                              float* __restrict__ amax) {
    const int r = blockIdx.x, seg = blockIdx.y;
    const int c1 = min(k, 512 * (seg + 1));
    float m = 0.0f;
    for (int c = 512 * seg + threadIdx.x; c < c1; c += blockDim.x) m = fmaxf(m, fabsf(L[(size_t)r * ldl + c]));
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomic_max_nonneg(&amax[seg * nblk + (r >> 9)], m);
}

// amax[seg * nblk + c / 512] = max |T[512 seg .. 512 seg + 512)[c]| over each
// 512-column block.
__global__ void k_absmax_cols(const float* __restrict__ T, int ldt, int k, int cols, int nblk,
                              float* __restrict__ amax) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cols) return;
    for (int seg = 0; 512 * seg < k; seg++) {
        float m = 0.0f;
        const int r1 = min(k, 512 * (seg + 1));
        for (int r = 512 * seg; r < r1; r++) m = fmaxf(m, fabsf(T[(size_t)r * ldt + c]));
        atomic_max_nonneg(&amax[seg * nblk + (c >> 9)], m);
    }
}

// scale = amax / 448 (1 for an all-zero block); inv = 1 / scale.
__global__ void k_scales(const float* __restrict__ amax, float* __restrict__ scale, float* __restrict__ inv, int nb) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nb) return;
    const float a = amax[i];
    const float s = a > 0.0f ? a / kE4M3Max : 1.0f;
    scale[i] = s;
    inv[i] = 1.0f / s;
}

template <bool FP8>
__global__ void k_quant_rows(const float* __restrict__ L, int ldl, uint8_t* __restrict__ out, int rows, int k,
                             const float* __restrict__ inv, int nblk) {
    const size_t total = (size_t)rows * k / 4;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const size_t e = i * 4;
        const int r = (int)(e / k), c = (int)(e - (size_t)r * k);
        float4 v = *reinterpret_cast<const float4*>(L + (size_t)r * ldl + c);
        if (FP8) {
            const float s = inv[(c >> 9) * nblk + (r >> 9)];  // the four columns share a 512-wide K segment
            __nv_fp8x4_e4m3 q(make_float4(v.x * s, v.y * s, v.z * s, v.w * s));
            *reinterpret_cast<__nv_fp8x4_e4m3*>(out + e) = q;
        } else {
            __nv_bfloat162 lo = __floats2bfloat162_rn(v.x, v.y), hi = __floats2bfloat162_rn(v.z, v.w);
            __nv_bfloat162* o = reinterpret_cast<__nv_bfloat162*>(out + e * 2);
            o[0] = lo;
            o[1] = hi;
        }
    }
}

// out[c][r] = q(T[r][c]) for r < k, c < cols: 32 x 32 tiles through shared memory.
template <bool FP8>
__global__ void __launch_bounds__(256) k_quant_trans(const float* __restrict__ T, int ldt, uint8_t* __restrict__ out,
                                                     int k, int cols, const float* __restrict__ inv, int nblk) {
    __shared__ float tile[32][33];
    const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < 32; j += 8) {
        const int r = r0 + ty + j, c = c0 + tx;
        tile[ty + j][tx] = (r < k && c < cols) ? T[(size_t)r * ldt + c] : 0.0f;
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < 32; j += 8) {
        const int c = c0 + ty + j, r = r0 + tx;
        if (r < k && c < cols) {
            const float v = tile[tx][ty + j];
            if (FP8) {
                __nv_fp8_e4m3 q(v * inv[(r >> 9) * nblk + (c >> 9)]);
                out[(size_t)c * k + r] = *reinterpret_cast<uint8_t*>(&q);
            } else {
                __nv_bfloat16 q = __float2bfloat16_rn(v);
                reinterpret_cast<__nv_bfloat16*>(out)[(size_t)c * k + r] = q;
            }
        }
    }
}

// Exact three-term BF16 split of an FP32 value (each remainder is exact in FP32).
__device__ __forceinline__ void split3(float x, __nv_bfloat16& a, __nv_bfloat16& b, __nv_bfloat16& c) {
    a = __float2bfloat16_rn(x);
    const float r1 = x - __bfloat162float(a);
    b = __float2bfloat16_rn(r1);
    c = __float2bfloat16_rn(r1 - __bfloat162float(b));
}

// Segment s of the K = nseg k operand pairs L-term lterm(s) with T-term
// tterm(s) (term 0 = x1, the largest).  nseg 6: x3 t1 + x2 t2 + x1 t3 +
// x2 t1 + x1 t2 + x1 t1 (FP32 accuracy); nseg 3: x2 t1 + x1 t2 + x1 t1
// (about 2^-16 relative, the three-term split's first two terms); nseg 1:
// x1 t1 (plain BF16 operands).
template <int NSEG>
__host__ __device__ constexpr int lterm(int s) {
    return NSEG == 6 ? (s == 0 ? 2 : (s == 1 || s == 3) ? 1 : 0) : NSEG == 3 ? (s == 0 ? 1 : 0) : 0;
}
template <int NSEG>
__host__ __device__ constexpr int tterm(int s) {
    return NSEG == 6 ? (s == 2 ? 2 : (s == 1 || s == 4) ? 1 : 0) : NSEG == 3 ? (s == 1 ? 1 : 0) : 0;
}

// out[r][s*k + c] = term lterm(s) of L[r][c]: rows x (NSEG k) BF16.
template <int NSEG>
__global__ void k_split_rows(const float* __restrict__ L, int ldl, __nv_bfloat16* __restrict__ out, int rows, int k) {
    const size_t total = (size_t)rows * k;
    const size_t kq = NSEG * (size_t)k;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const int r = (int)(e / k), c = (int)(e - (size_t)r * k);
        __nv_bfloat16 t[3];
        split3(L[(size_t)r * ldl + c], t[0], t[1], t[2]);
        __nv_bfloat16* o = out + (size_t)r * kq + c;
#pragma unroll
        for (int s = 0; s < NSEG; s++) o[(size_t)s * k] = t[lterm<NSEG>(s)];
    }
}

// out[c][s*k + r] = term tterm(s) of T[r][c]: cols x (NSEG k) BF16, through a
// 32 x 32 shared-memory transpose.
template <int NSEG>
__global__ void __launch_bounds__(256) k_split_trans(const float* __restrict__ T, int ldt,
                                                     __nv_bfloat16* __restrict__ out, int k, int cols) {
    __shared__ float tile[32][33];
    const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < 32; j += 8) {
        const int r = r0 + ty + j, c = c0 + tx;
        tile[ty + j][tx] = (r < k && c < cols) ? T[(size_t)r * ldt + c] : 0.0f;
    }
    __syncthreads();
    const size_t kq = NSEG * (size_t)k;
#pragma unroll
    for (int j = 0; j < 32; j += 8) {
        const int c = c0 + ty + j, r = r0 + tx;
        if (r < k && c < cols) {
            __nv_bfloat16 t[3];
            split3(tile[tx][ty + j], t[0], t[1], t[2]);
            __nv_bfloat16* o = out + (size_t)c * kq + r;
#pragma unroll
            for (int s = 0; s < NSEG; s++) o[(size_t)s * k] = t[tterm<NSEG>(s)];
        }
    }
}

// x[i][i] += v for i < n (an n x n block, leading dimension n).
__global__ void k_add_diag(float* __restrict__ x, int n, float v) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[(size_t)i * n + i] += v;
}

// x = identity (two n x n blocks, leading dimension n).
__global__ void k_eye2(float* __restrict__ x, float* __restrict__ y, int n) {
    const size_t total = (size_t)n * n;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const float v = (e / n == e % n) ? 1.0f : 0.0f;
        x[e] = v;
        y[e] = v;
    }
}

}  // namespace

// The split-BF16 operands of a block step (nseg 6, 3 or 1 K-segments):
// aq: rows_l x nseg k, bq: cols_t x nseg k.
int split_panel(const float* L, int ldl, const float* T, int ldt, int rows_l, int cols_t, int k, uint8_t* aq,
                uint8_t* bq, cudaStream_t st, int nseg) {
    if (rows_l <= 0 || cols_t <= 0) return LP_OK;
    if (nseg != 6 && nseg != 3 && nseg != 1) return fail(LP_E_INVALID, "split_panel: 1, 3 or 6 segments");
    const size_t total = (size_t)rows_l * k;
    const int grid = (int)((total + 255) / 256 < 4736 ? (total + 255) / 256 : 4736);
    const dim3 tgrid((cols_t + 31) / 32, (k + 31) / 32);
    auto* a = reinterpret_cast<__nv_bfloat16*>(aq);
    auto* b = reinterpret_cast<__nv_bfloat16*>(bq);
    if (nseg == 6) {
        k_split_rows<6><<<grid, 256, 0, st>>>(L, ldl, a, rows_l, k);
        k_split_trans<6><<<tgrid, 256, 0, st>>>(T, ldt, b, k, cols_t);
    } else if (nseg == 3) {
        k_split_rows<3><<<grid, 256, 0, st>>>(L, ldl, a, rows_l, k);
        k_split_trans<3><<<tgrid, 256, 0, st>>>(T, ldt, b, k, cols_t);
    } else {
        k_split_rows<1><<<grid, 256, 0, st>>>(L, ldl, a, rows_l, k);
        k_split_trans<1><<<tgrid, 256, 0, st>>>(T, ldt, b, k, cols_t);
    }
    count_launch(2);
    LP_CUDA(cudaGetLastError());
    return LP_OK;
}

// Rounds the panel of a block step to the tensor-core operand type.
// L: rows_l x k (ld ldl), T: k x cols_t (ld ldt); aq: rows_l x k, bq:
// cols_t x k; sc: 3 arrays of kseg(k) * nblk floats (absmax, scale, 1/scale,
// indexed seg * nblk + block) for L, then 3 for T (nblk >=
// ceil(max(rows_l, cols_t) / 512)).
int quantize_panel(const float* L, int ldl, const float* T, int ldt, int rows_l, int cols_t, int k, bool fp8,
                   uint8_t* aq, uint8_t* bq, float* sc, int nblk, cudaStream_t st) {
    if (rows_l <= 0 || cols_t <= 0) return LP_OK;
    const size_t q4 = (size_t)rows_l * k / 4;
    const int qgrid = (int)((q4 + 255) / 256 < 2368 ? (q4 + 255) / 256 : 2368);
    const dim3 tgrid((cols_t + 31) / 32, (k + 31) / 32);
    if (fp8) {
        const int ns = kseg(k) * nblk;
        float* amax_a = sc;
        float* scale_a = sc + ns;
        float* inv_a = sc + 2 * ns;
        float* amax_b = sc + 3 * ns;
        float* scale_b = sc + 4 * ns;
        float* inv_b = sc + 5 * ns;
        LP_CUDA(cudaMemsetAsync(amax_a, 0, sizeof(float) * ns, st));
        LP_CUDA(cudaMemsetAsync(amax_b, 0, sizeof(float) * ns, st));
        k_absmax_rows<<<dim3(rows_l, kseg(k)), 128, 0, st>>>(L, ldl, rows_l, k, nblk, amax_a);
        k_absmax_cols<<<(cols_t + 255) / 256, 256, 0, st>>>(T, ldt, k, cols_t, nblk, amax_b);
        k_scales<<<(ns + 127) / 128, 128, 0, st>>>(amax_a, scale_a, inv_a, ns);
        k_scales<<<(ns + 127) / 128, 128, 0, st>>>(amax_b, scale_b, inv_b, ns);
        k_quant_rows<true><<<qgrid, 256, 0, st>>>(L, ldl, aq, rows_l, k, inv_a, nblk);
        k_quant_trans<true><<<tgrid, 256, 0, st>>>(T, ldt, bq, k, cols_t, inv_b, nblk);
        count_launch(6);
    } else {
        k_quant_rows<false><<<qgrid, 256, 0, st>>>(L, ldl, aq, rows_l, k, nullptr, nblk);
        k_quant_trans<false><<<tgrid, 256, 0, st>>>(T, ldt, bq, k, cols_t, nullptr, nblk);
        count_launch(2);
    }
    LP_CUDA(cudaGetLastError());
    return LP_OK;
}

// One trailing (sub)update of the mixed schedule: rows [m_off, m_off+m) and
// columns [n_off, n_off+n) of the trailing matrix at c11.
static int mixed_update(lp_ctx* c, float* c11, int lda, const uint8_t* aq, const uint8_t* bq, int rest, int m_off,
                        int n_off, int m, int n, int kq, bool fp8, const float* sc, int nblk, cudaStream_t st) {
    const int ns = kseg(kq) * nblk;
    const float* scale_a = fp8 ? sc + ns : nullptr;
    const float* scale_b = fp8 ? sc + 4 * ns : nullptr;
    return launch_umma_update(c11, lda, aq, rest, bq, rest, m_off, n_off, m, n, kq, fp8, scale_a, scale_b, nblk,
                              static_cast<int*>(c->err.ptr), st);
}

// Panel of block step K for the tensor-core schedules.  lu of the diagonal
// block D as in the FP32 schedule.  top and left are triangular solves with
// D's two triangles (storage indices, k_trsm.cu):
//   top:  each column t of the block row satisfies t_k = D_kk (t0_k + sum_{i<k} D_ki t_i),
//         i.e. t = W^-1 t0 with W = diag(D)^-1 - strict-lower(D);
//   left: each row l of the block column satisfies l_i = l0_i + sum_{k<i} l_k D_ki,
//         i.e. l = l0 V with V = (I - strict-upper(D))^-1.
// W^-1 and V are the two recurrences applied to a bs x bs identity (the exact
// kernels over the nonzero triangle only, a small problem); then T = W^-1 T0
// (into the zeroed block row) and
// L += L (V - I) run as split-BF16 tensor-core products (nseg K-segments), so
// the n bs^2 flops of the recurrences per step leave the FMA pipe.  V is unit
// triangular, so L keeps its exact identity part; W^-1 is not (its diagonal
// is D_kk = -1/u_kk), and T0 + (W^-1 - I) T0 would cancel nearly all of T0.
static int panel_tc(lp_ctx* c, float* dA, int n, int lda, int bs, int K, int nseg, cudaStream_t s) {
    float* d = dA + (size_t)K * bs * lda + (size_t)K * bs;
    const double b = bs;
    const int rest = n - (K + 1) * bs;
    const size_t bb = (size_t)bs * bs, kq = (size_t)nseg * bs;
    float* winv = static_cast<float*>(c->tri.ptr);
    float* vinv = winv + bb;
    float* vlt = vinv + bb;
    // bs > 128: W^-1 and V are built 128 rows / columns behind the lu stage on
    // two side streams (lu_stage), rather than after it.  Measured on one B200,
    // factorization alone, n = 32768, block 1024: BF16 55.3 -> 51.5 ms, E4M3
    // 59.3 -> 54.5 ms; n = 65536, block 2048: unchanged.  Not for the emulated
    // FP32 form (six segments), whose tensor-bound update only loses SMs to the
    // side streams (143 -> 148 ms).
    const bool beside = rest > 0 && bs > 128 && nseg < 6;
    if (beside) {
        k_eye2<<<(int)((bb + 255) / 256 < 1184 ? (bb + 255) / 256 : 1184), 256, 0, s>>>(winv, vinv, bs);
        count_launch();
        LP_CUDA(cudaGetLastError());
    }
    const TriInverses inv{winv, vinv, vlt};
    int e = prof_begin(c, s);
    LP_CHECK(lu_stage(c, d, lda, bs, s, beside ? &inv : nullptr));
    LP_CHECK(prof_end(c, s, LP_STAGE_LU, e, 2.0 * b * b * b / 3.0, 8.0 * b * b));
    if (rest <= 0) return LP_OK;
    const double r = rest;
    __nv_bfloat16* tq = static_cast<__nv_bfloat16*>(c->tq.ptr);
    uint8_t* a_top = reinterpret_cast<uint8_t*>(tq);                    // bs x kq: W^-1
    uint8_t* b_left = reinterpret_cast<uint8_t*>(tq + bb * nseg);       // bs x kq: (V - I)^T
    uint8_t* b_top = reinterpret_cast<uint8_t*>(tq + 2 * bb * nseg);    // rest x kq: T^T
    uint8_t* a_left = reinterpret_cast<uint8_t*>(tq + 2 * bb * nseg + (size_t)n * kq);  // rest x kq: L
    int* err = static_cast<int*>(c->err.ptr);

    e = prof_begin(c, s);
    if (!beside) {
        k_eye2<<<(int)((bb + 255) / 256 < 1184 ? (bb + 255) / 256 : 1184), 256, 0, s>>>(winv, vinv, bs);
        count_launch();
        LP_CUDA(cudaGetLastError());
        LP_CUDA(cudaEventRecord(c->ev_side, s));
        LP_CUDA(cudaStreamWaitEvent(c->aux2, c->ev_side, 0));
        LP_CHECK(left_blocked(d, lda, vinv, bs, bs, bs, vlt, bs, c->aux2, true));
        LP_CUDA(cudaEventRecord(c->ev_side_done, c->aux2));
        LP_CHECK(top_blocked(c, d, lda, winv, bs, bs, bs, s, true));
        LP_CUDA(cudaStreamWaitEvent(s, c->ev_side_done, 0));
    }
    k_add_diag<<<(bs + 127) / 128, 128, 0, s>>>(vinv, bs, -1.0f);
    count_launch();
    LP_CUDA(cudaGetLastError());
    float* t = d + bs;
    float* l = d + (size_t)bs * lda;
    LP_CHECK(split_panel(winv, bs, t, lda, bs, rest, bs, a_top, b_top, s, nseg));
    LP_CUDA(cudaMemset2DAsync(t, sizeof(float) * (size_t)lda, 0, sizeof(float) * (size_t)rest, bs, s));
    LP_CHECK(launch_umma_update(t, lda, a_top, bs, b_top, rest, 0, 0, bs, rest, (int)kq, false, nullptr, nullptr, 0,
                                err, s));
    LP_CHECK(prof_end(c, s, LP_STAGE_TOP, e, b * b * r, 8.0 * b * r));
    e = prof_begin(c, s);
    LP_CHECK(split_panel(l, lda, vinv, bs, rest, bs, bs, a_left, b_left, s, nseg));
    LP_CHECK(launch_umma_update(l, lda, a_left, rest, b_left, bs, 0, 0, rest, bs, (int)kq, false, nullptr, nullptr, 0,
                                err, s));
    return prof_end(c, s, LP_STAGE_LEFT, e, b * b * r, 8.0 * b * r);
}

int gefa_mixed(lp_ctx* c, int precision, float* dA, int n, int lda, int bs, cudaStream_t st) {
    const bool fp8 = precision == LP_FP8_IR;
    const bool x6 = precision == LP_F32_BF16X6;
    if (bs < 128 || bs % 128 != 0) return fail(LP_E_INVALID, "mixed precision needs a block size >= 128");
    const size_t esz = fp8 ? 1 : 2;
    const int kq = x6 ? 6 * bs : bs;  // K of the tensor-core update
    const size_t pan = (size_t)kq * n;      // one tensor-core operand
    const int nblk = (n + 511) / 512;
    if (bs > 128) {
        LP_CHECK(c->lti.ensure(2 * sizeof(float) * (size_t)128 * bs));
        LP_CHECK(c->dsub.ensure(2 * sizeof(float) * (size_t)128 * bs));
    }
    LP_CHECK(c->q.ensure(4 * esz * pan));
    LP_CHECK(c->qs.ensure(2 * 6 * sizeof(float) * (size_t)kseg(bs) * nblk));
    LP_CHECK(c->err.ensure(sizeof(int)));
    // the top / left products: FP32 accuracy (six segments) for the emulated-FP32
    // form.  For BF16 / E4M3 (the panel is rounded to them for the update anyway)
    // three segments, and plain BF16 operands from block 2048 on, where the panel
    // chain is the critical path: the products cost about 9 bs / n of the update's
    // flops per three segments.  Measured on one B200 (BF16+IR): n = 65536, block
    // 2048: 582 -> 638 TFLOP/s, one refinement either way; n = 32768, block 1024: no
    // gain, the plainer factors needing a second refinement.
    const int nseg = x6 ? 6 : bs >= 2048 ? 1 : 3;
    LP_CHECK(c->tri.ensure(3 * sizeof(float) * (size_t)bs * bs));
    LP_CHECK(c->tq.ensure(2 * sizeof(__nv_bfloat16) * (size_t)nseg * bs * ((size_t)bs + n)));
    LP_CUDA(cudaMemsetAsync(c->err.ptr, 0, sizeof(int), st));
    uint8_t* q = static_cast<uint8_t*>(c->q.ptr);
    uint8_t* aqb[2] = {q, q + 2 * esz * pan};
    uint8_t* bqb[2] = {q + esz * pan, q + 3 * esz * pan};
    float* scb[2] = {static_cast<float*>(c->qs.ptr), static_cast<float*>(c->qs.ptr) + 6 * (size_t)kseg(bs) * nblk};
    const int nb = n / bs;
    const double b = bs;

    auto panel_q = [&](int K, cudaStream_t s) -> int {
        LP_CHECK(panel_tc(c, dA, n, lda, bs, K, nseg, s));
        const int rest = n - (K + 1) * bs;
        if (rest <= 0) return LP_OK;
        float* d = dA + (size_t)K * bs * lda + (size_t)K * bs;
        const int e = prof_begin(c, s);
        if (x6)
            LP_CHECK(split_panel(d + (size_t)bs * lda, lda, d + bs, lda, rest, rest, bs, aqb[K & 1], bqb[K & 1], s));
        else
            LP_CHECK(quantize_panel(d + (size_t)bs * lda, lda, d + bs, lda, rest, rest, bs, fp8, aqb[K & 1],
                                    bqb[K & 1], scb[K & 1], nblk, s));
        return prof_end(c, s, LP_STAGE_OTHER, e, 0.0, 2.0 * 4.0 * b * rest + 2.0 * esz * b * rest);
    };

    LP_CHECK(panel_q(0, st));
    for (int K = 0; K + 1 < nb; K++) {
        const int rest = n - (K + 1) * bs;
        const double r = rest;
        float* c11 = dA + (size_t)(K + 1) * bs * lda + (size_t)(K + 1) * bs;
        const uint8_t* aq = aqb[K & 1];
        const uint8_t* bq = bqb[K & 1];
        const float* sc = scb[K & 1];
        int e = prof_begin(c, st);
        LP_CHECK(mixed_update(c, c11, lda, aq, bq, rest, 0, 0, bs, rest, kq, fp8, sc, nblk, st));
        if (rest > bs) LP_CHECK(mixed_update(c, c11, lda, aq, bq, rest, bs, 0, rest - bs, bs, kq, fp8, sc, nblk, st));
        LP_CHECK(prof_end(c, st, LP_STAGE_INNER, e, 2.0 * b * r * b + 2.0 * (r - b) * b * b,
                          8.0 * (b * r + (r - b) * b)));
        LP_CUDA(cudaEventRecord(c->ev_fork, st));
        LP_CUDA(cudaStreamWaitEvent(c->aux, c->ev_fork, 0));
        LP_CHECK(panel_q(K + 1, c->aux));
        LP_CUDA(cudaEventRecord(c->ev_join, c->aux));
        if (rest > bs) {
            const double r2 = rest - bs;
            e = prof_begin(c, st);
            LP_CHECK(mixed_update(c, c11, lda, aq, bq, rest, bs, bs, rest - bs, rest - bs, kq, fp8, sc, nblk, st));
            LP_CHECK(prof_end(c, st, LP_STAGE_INNER, e, 2.0 * r2 * r2 * b, 8.0 * r2 * r2));
        }
        LP_CUDA(cudaStreamWaitEvent(st, c->ev_join, 0));
    }
    int herr = 0;
    LP_CUDA(cudaMemcpyAsync(&herr, c->err.ptr, sizeof(int), cudaMemcpyDeviceToHost, st));
    LP_CHECK(wait_stream(c, st));
    if (herr != 0)
        return fail(LP_E_TIMEOUT, "tensor-core trailing update: a bounded wait expired (code " +
                                      std::to_string(herr) + "); the update was abandoned");
    return LP_OK;
}

}  // namespace lp
