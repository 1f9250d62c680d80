// Batched factor + solve of many independent systems in ONE persistent launch.
//
// Each system i is an n_i x n_i matrix in the reference encoding
// (LINPACK/src/host/linpack_data.cpp:166-229: factored in place, diagonal
// -1/u_kk, negated multipliers in storage rows, U in storage columns) with
// nrhs_i right-hand sides stored as rows of B_i, overwritten by the
// solutions.  CTAs pull systems from an atomic counter over a list sorted by
// decreasing n (largest first: the slowest systems start first, the small
// ones fill the tail), so one launch balances any size mix.
//
// Per system, one CTA of 256 threads:
//   n <= small_n_max (<= 128): the whole matrix and right-hand sides in
//     shared memory; right-looking LU with one barrier per step, then the
//     forward and back sweeps.
//   larger n: blocked right-looking LU with panel width NB (16 or 32, per
//     size bucket, chosen by the autotuner): the diagonal block factored by
//     one warp in registers (pivots and columns by shuffles); the top block
//     row (column-independent) and left block column (row-independent) by
//     their recurrences in registers; the trailing update per 128-row block,
//     its left panel resident in shared memory, the 64-column top tiles
//     streamed in with cp.async one tile ahead, each thread's 8 x 4 piece of
//     C loaded into registers while its products run.  (Panel widths 16 and 32 keep a recurrence in registers.)
//     Then blocked forward/back sweeps with the right-hand sides resident in
//     shared memory and each diagonal block staged before its sequential solve.
// Arithmetic uses fused multiply-add: results agree with the reference to
// rounding (checked against the oracle in tests/test_gpu_batch.py).
#include <cuda_bf16.h>
#include <cfloat>

#include "lp_ctx.cuh"

namespace lp {
namespace {

constexpr int BT = 256;
constexpr int SMALL_MAX = 128;
constexpr int RHS_MAX = 16;
constexpr int NBUCKETS = 5;
// Flag in BatchSys::nrhs (server use only; the public entry points accept
// nrhs <= 16): the matrix already holds its factors, solve only.
constexpr int kSolveOnly = kBatchSolveOnly;

struct BatchSys {
    int n, nrhs, lda, ldb;
    long long a_off, b_off;
};
static_assert(sizeof(BatchSys) == sizeof(lp_system), "lp_system layout");

struct Tune {
    int small_n_max;
    int nb[NBUCKETS];
    int absolute;  // a_off / b_off are device addresses (bytes), not offsets into A / B
};

constexpr size_t kSmallFloats = (size_t)SMALL_MAX * (SMALL_MAX + 1) + (size_t)RHS_MAX * SMALL_MAX;
constexpr size_t kBlockedFloats = (size_t)RHS_MAX * 1024;  // right-hand sides of n <= 1024 in the solve phase
constexpr size_t kBatchSmem = sizeof(float) * (kSmallFloats > kBlockedFloats ? kSmallFloats : kBlockedFloats);
// factor_blocked<32, BF16>: diagonal block, left panel (128 rows), 2 top tiles (stride 68 in the BF16 form)
static_assert(sizeof(float) * (32 * 33 + 32 * 132 + 2 * 32 * 68) <= kBatchSmem, "blocked smem");

__device__ __forceinline__ int bucket_of(int n) {
    return n <= 64 ? 0 : n <= 128 ? 1 : n <= 256 ? 2 : n <= 512 ? 3 : 4;
}

// In-place LU (reference encoding) of an m x m matrix in shared memory with
// row stride ld, all threads of the CTA; one barrier per step.
__device__ void smem_lu(float* S, int ld, int m) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    float inv_prev = 0.0f;
    for (int k = 0; k < m; k++) {
        const float inv = (float)(-1.0 / (double)S[k * ld + k]);
        if (k > 0) {
            float* rp = S + (k - 1) * ld;
            for (int i = k + tid; i < m; i += BT) rp[i] *= inv_prev;
            if (tid == 0) rp[k - 1] = inv_prev;
        }
        const float* rk = S + k * ld;
        for (int i0 = k + 1; i0 < m; i0 += 32) {
            const int i = i0 + lane;
            const float sc = (i < m) ? rk[i] * inv : 0.0f;
            for (int j = k + 1 + warp; j < m; j += BT / 32) {
                float* rj = S + j * ld;
                if (i < m) rj[i] = fmaf(sc, rj[k], rj[i]);
            }
        }
        inv_prev = inv;
        __syncthreads();
    }
    if (tid == 0 && m > 0) S[(m - 1) * ld + (m - 1)] = inv_prev;
    __syncthreads();
}

// Forward/back sweeps on right-hand sides Y (nrhs rows of length m, stride m)
// with the factors in shared memory (row stride ld).
__device__ void smem_solve(const float* S, int ld, int m, float* Y, int nrhs, float* sc) {
    const int tid = threadIdx.x;
    for (int k = 0; k + 1 < m; k++) {
        for (int idx = tid; idx < nrhs * m; idx += BT) {
            const int q = idx / m, i = idx - q * m;
            if (i > k) Y[idx] = fmaf(Y[q * m + k], S[k * ld + i], Y[idx]);
        }
        __syncthreads();
    }
    for (int k = m - 1; k >= 0; k--) {
        if (tid < nrhs) sc[tid] = Y[tid * m + k] * S[k * ld + k];
        __syncthreads();
        for (int idx = tid; idx < nrhs * m; idx += BT) {
            const int q = idx / m, i = idx - q * m;
            if (i < k)
                Y[idx] = fmaf(sc[q], S[k * ld + i], Y[idx]);
            else if (i == k)
                Y[idx] = -sc[q];
        }
        __syncthreads();
    }
}

__device__ __noinline__ void solve_small(float* a, int lda, int n, float* b, int ldb, int nrhs, bool factor, float* sm) {
    const int ld = n | 1;  // odd stride: column reads hit distinct banks
    float* S = sm;
    float* Y = sm + SMALL_MAX * (SMALL_MAX + 1);
    __shared__ float sc[RHS_MAX];
    for (int idx = threadIdx.x; idx < n * n; idx += BT) {
        const int r = idx / n, c = idx - r * n;
        S[r * ld + c] = a[(size_t)r * lda + c];
    }
    for (int idx = threadIdx.x; idx < nrhs * n; idx += BT) {
        const int q = idx / n, i = idx - q * n;
        Y[idx] = b[(size_t)q * ldb + i];
    }
    __syncthreads();
    if (factor) smem_lu(S, ld, n);
    smem_solve(S, ld, n, Y, nrhs, sc);
    if (factor)
        for (int idx = threadIdx.x; idx < n * n; idx += BT) {
            const int r = idx / n, c = idx - r * n;
            a[(size_t)r * lda + c] = S[r * ld + c];
        }
    for (int idx = threadIdx.x; idx < nrhs * n; idx += BT) {
        const int q = idx / n, i = idx - q * n;
        b[(size_t)q * ldb + i] = Y[idx];
    }
    __syncthreads();
}

// LU of the kb x kb diagonal block at d (kb <= NB), warp 0 only: lane c
// holds column c in registers, the pivot and column k are shuffled from lane
// k.  Writes the factors to d and to Ds (row stride DL).  Out of line: inlined
// into the persistent loop its register array is not fully unrolled.
template <int NB, int DL>
__device__ __noinline__ void warp_diag_lu(float* d, int lda, int kb, float* Ds) {
    // A partial last block is padded with the identity: diag(D, I) factors as
    // diag(LU_D, I), so every step runs unconditionally (no per-step branches
    // between the shuffles) and only the kb x kb part is written back.
    const int lane = threadIdx.x & 31;
    float x[NB];
#pragma unroll
    for (int j = 0; j < NB; j++)
        x[j] = (lane < kb && j < kb) ? d[(size_t)j * lda + lane] : (j == lane ? 1.0f : 0.0f);
#pragma unroll
    for (int k = 0; k < NB; k++) {
        // -1/pivot correctly rounded in float (equal to the double quotient rounded to float)
        const float inv = -__frcp_rn(__shfl_sync(0xffffffffu, x[k], k));
        if (lane > k)
            x[k] *= inv;
        else if (lane == k)
            x[k] = inv;
#pragma unroll
        for (int j = k + 1; j < NB; j++) {
            const float sjk = __shfl_sync(0xffffffffu, x[j], k);
            if (lane > k) x[j] = fmaf(x[k], sjk, x[j]);
        }
    }
    if (lane < NB) {
#pragma unroll
        for (int j = 0; j < NB; j++) {
            Ds[j * DL + lane] = x[j];
            if (lane < kb && j < kb) d[(size_t)j * lda + lane] = x[j];
        }
    }
}

// Two floats rounded to BF16 (round to nearest even) in one register, the
// first in the low half: the operand order of the warp-level MMA fragments.
__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&v);
}

// D (16 x 8, FP32) += A (16 x 16, BF16, row-major fragments) * B (16 x 8, BF16).
__device__ __forceinline__ void mma_bf16_16816(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                               uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// The BF16 form of one 128 x 64 trailing tile: C[m0.., c0..] += L * T with L
// (Lt, k-major, row stride LS) and T (k-major, row stride TNS) rounded to
// BF16 and the products accumulated in FP32 on the tensor cores (warp-level
// m16n8k16 MMA).  Warp w owns rows 16w..16w+15 and all 64 columns, in two
// passes of four 16 x 8 accumulators; a pass's C values are loaded before its
// products run.
// Fragment reads from shared memory are bank-conflict free: Lt's stride 132
// and T's stride 68 put lane (g, t) of a fragment load on bank 8t + g (+ const).
template <int NB, int LS, int TNS>
__device__ __noinline__ void tile_update_bf16(float* a, int lda, int n, int m0, int c0, const float* Lt,
                                             const float* T) {
    constexpr int NT = 4;  // 8-column MMA tiles per pass: two passes of 32 columns keep C and the sums in registers
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane >> 2, t4 = lane & 3;
    const int rA = m0 + warp * 16 + g;  // rows rA and rA + 8
    asm volatile("cp.async.wait_group 1;\n" ::: "memory");  // this top tile (earlier group)
    __syncthreads();
#pragma unroll
    for (int half = 0; half < 2; half++) {
        float cv[NT][4];
#pragma unroll
        for (int nt = 0; nt < NT; nt++) {
            const int col = c0 + (half * NT + nt) * 8 + 2 * t4;
#pragma unroll
            for (int hh = 0; hh < 2; hh++) {
                const int r = rA + 8 * hh;
                const float* src = a + (size_t)r * lda + col;
                cv[nt][2 * hh] = (r < n && col < n) ? __ldcg(src) : 0.0f;
                cv[nt][2 * hh + 1] = (r < n && col + 1 < n) ? __ldcg(src + 1) : 0.0f;
            }
        }
        float acc[NT][4];
#pragma unroll
        for (int nt = 0; nt < NT; nt++)
#pragma unroll
            for (int e = 0; e < 4; e++) acc[nt][e] = 0.0f;
#pragma unroll
        for (int kq = 0; kq < NB; kq += 16) {
            const float* L0 = Lt + (kq + 2 * t4) * LS + warp * 16 + g;
            const uint32_t a0 = pack_bf16(L0[0], L0[LS]);
            const uint32_t a1 = pack_bf16(L0[8], L0[LS + 8]);
            const uint32_t a2 = pack_bf16(L0[8 * LS], L0[9 * LS]);
            const uint32_t a3 = pack_bf16(L0[8 * LS + 8], L0[9 * LS + 8]);
#pragma unroll
            for (int nt = 0; nt < NT; nt++) {
                const float* T0 = T + (kq + 2 * t4) * TNS + (half * NT + nt) * 8 + g;
                mma_bf16_16816(acc[nt], a0, a1, a2, a3, pack_bf16(T0[0], T0[TNS]),
                               pack_bf16(T0[8 * TNS], T0[9 * TNS]));
            }
        }
#pragma unroll
        for (int nt = 0; nt < NT; nt++) {
            const int col = c0 + (half * NT + nt) * 8 + 2 * t4;
#pragma unroll
            for (int hh = 0; hh < 2; hh++) {
                const int r = rA + 8 * hh;
                float* dst = a + (size_t)r * lda + col;
                if (r < n && col < n) dst[0] = cv[nt][2 * hh] + acc[nt][2 * hh];
                if (r < n && col + 1 < n) dst[1] = cv[nt][2 * hh + 1] + acc[nt][2 * hh + 1];
            }
        }
    }
}

// Blocked factorization of one system in global memory (see file comment).
// Trailing update per row block of 128 rows: the block's left panel (k-major)
// stays in shared memory, the 64-column top tiles stream through a cp.async
// double buffer, and each thread loads its 8 x 4 piece of C into registers
// before the rank-NB products, which hide the load.
template <int NB, bool BF16>
__device__ __noinline__ void factor_blocked(float* a, int lda, int n, float* sm) {
    constexpr int TM = 128, TN = 64;   // trailing-update tile
    constexpr int DL = NB + 1, LS = TM + 4;
    constexpr int TNS = BF16 ? TN + 4 : TN;  // top-tile row stride (conflict-free MMA fragments)
    float* Ds = sm;                    // NB x DL diagonal block
    float* Lt = Ds + NB * DL;          // NB x LS: left panel of one row block, k-major
    float* Tb = Lt + NB * LS;          // 2 x NB x TNS: top tiles
    const int tid = threadIdx.x;
    for (int k0 = 0; k0 < n; k0 += NB) {
        const int kb = min(NB, n - k0);
        const int r0 = k0 + kb, rem = n - r0;
        float* d = a + (size_t)k0 * lda + k0;
        if (tid < 32) warp_diag_lu<NB, DL>(d, lda, kb, Ds);
        __syncthreads();
        if (rem <= 0) break;
        // (rem > 0: this block is full, kb == NB)
        // The recurrences read D through a volatile view: its NB^2 / 2 values are the
        // same for every column / row, and hoisting them out of the loop into
        // registers would spill.
        const volatile float* Dv = Ds;
        // top: every column c of the block row, t_k *= D_kk; t_j += t_k D_jk (j > k)
#pragma unroll 1
        for (int c = r0 + tid; c < n; c += BT) {
            float x[NB];
#pragma unroll
            for (int i = 0; i < NB; i++) x[i] = a[(size_t)(k0 + i) * lda + c];
#pragma unroll
            for (int k = 0; k < NB; k++) {
                const float xk = x[k] * Dv[k * DL + k];
                x[k] = xk;
#pragma unroll
                for (int j = k + 1; j < NB; j++) x[j] = fmaf(xk, Dv[j * DL + k], x[j]);
            }
#pragma unroll
            for (int i = 0; i < NB; i++) a[(size_t)(k0 + i) * lda + c] = x[i];
        }
        // left: every row rr of the block column, l_i += l_k D_ki (i > k)
        const bool vec = ((lda & 3) == 0) && ((reinterpret_cast<uintptr_t>(a) & 15) == 0);
#pragma unroll 1
        for (int rr = r0 + tid; rr < n; rr += BT) {
            float x[NB];
            float* row = a + (size_t)rr * lda + k0;
            if (vec) {  // k0 is a multiple of NB: the row segment is 16-byte aligned
#pragma unroll
                for (int i = 0; i < NB; i += 4) {
                    const float4 v = *reinterpret_cast<const float4*>(row + i);
                    x[i] = v.x, x[i + 1] = v.y, x[i + 2] = v.z, x[i + 3] = v.w;
                }
            } else {
#pragma unroll
                for (int i = 0; i < NB; i++) x[i] = row[i];
            }
#pragma unroll
            for (int k = 0; k < NB; k++)
#pragma unroll
                for (int i = k + 1; i < NB; i++) x[i] = fmaf(x[k], Dv[k * DL + i], x[i]);
            if (vec) {
#pragma unroll
                for (int i = 0; i < NB; i += 4)
                    *reinterpret_cast<float4*>(row + i) = make_float4(x[i], x[i + 1], x[i + 2], x[i + 3]);
            } else {
#pragma unroll
                for (int i = 0; i < NB; i++) row[i] = x[i];
            }
        }
        __syncthreads();
        // inner: C[r0:n, r0:n] += L * T in 128 x 64 tiles, 8 x 4 per thread.  Per tile the
        // C piece and the next top tile are in flight while the current tile's products run.
        const int ty = tid >> 4, tx = tid & 15;
        const int tiles_m = (rem + TM - 1) / TM, tiles_n = (rem + TN - 1) / TN;
        auto issue_top = [&](int tj, int buf) {
            const int c0 = r0 + tj * TN;
            float* T = Tb + buf * (NB * TNS);
            for (int idx = tid; idx < kb * TN / 4; idx += BT) {
                const int k = idx / (TN / 4), j = (idx - k * (TN / 4)) * 4;
                const float* src = a + (size_t)(k0 + k) * lda + c0 + j;
                float* dst = T + k * TNS + j;
                if (vec && ((c0 + j) & 3) == 0 && c0 + j + 3 < n) {
                    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
                    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
                } else {
#pragma unroll
                    for (int e = 0; e < 4; e++) {
                        if (c0 + j + e < n)
                            cp_async4(dst + e, src + e);
                        else
                            dst[e] = 0.0f;
                    }
                }
            }
        };
        for (int ti = 0; ti < tiles_m; ti++) {
            const int m0 = r0 + ti * TM;
            for (int idx = tid; idx < TM * kb; idx += BT) {
                const int i = idx / kb, k = idx - i * kb;
                if (m0 + i < n)
                    cp_async4(Lt + k * LS + i, a + (size_t)(m0 + i) * lda + k0 + k);
                else
                    Lt[k * LS + i] = 0.0f;
            }
            issue_top(0, 0);
            asm volatile("cp.async.commit_group;\n" ::: "memory");  // left panel + first top tile
            for (int tj = 0; tj < tiles_n; tj++) {
                const int c0 = r0 + tj * TN;
                if (tj + 1 < tiles_n) issue_top(tj + 1, (tj + 1) & 1);
                asm volatile("cp.async.commit_group;\n" ::: "memory");  // the next top tile
                if constexpr (BF16) {
                    tile_update_bf16<NB, LS, TNS>(a, lda, n, m0, c0, Lt, Tb + (tj & 1) * (NB * TNS));
                } else {
                    // this thread's 8 x 4 piece of C, loaded now and consumed after the products
                    const int cc = c0 + tx * 4;
                    const bool full = vec && cc + 3 < n;
                    float4 cv[8];
#pragma unroll
                    for (int p = 0; p < 8; p++) {
                        const int r = m0 + ty * 8 + p;
                        const float* src = a + (size_t)r * lda + cc;
                        cv[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                        if (r < n) {
                            if (full) {
                                cv[p] = __ldcg(reinterpret_cast<const float4*>(src));
                            } else {
                                if (cc < n) cv[p].x = src[0];
                                if (cc + 1 < n) cv[p].y = src[1];
                                if (cc + 2 < n) cv[p].z = src[2];
                                if (cc + 3 < n) cv[p].w = src[3];
                            }
                        }
                    }
                    asm volatile("cp.async.wait_group 1;\n" ::: "memory");  // this top tile (earlier group)
                    __syncthreads();
                    const float* T = Tb + (tj & 1) * (NB * TNS);
                    float acc[8][4];
#pragma unroll
                    for (int p = 0; p < 8; p++)
#pragma unroll
                        for (int q = 0; q < 4; q++) acc[p][q] = 0.0f;
#pragma unroll
                    for (int k = 0; k < NB; k++) {  // kb == NB here
                        const float4 l0 = *reinterpret_cast<const float4*>(Lt + k * LS + ty * 8);
                        const float4 l1 = *reinterpret_cast<const float4*>(Lt + k * LS + ty * 8 + 4);
                        const float4 tv = *reinterpret_cast<const float4*>(T + k * TNS + tx * 4);
                        const float l8[8] = {l0.x, l0.y, l0.z, l0.w, l1.x, l1.y, l1.z, l1.w};
                        const float t4[4] = {tv.x, tv.y, tv.z, tv.w};
#pragma unroll
                        for (int p = 0; p < 8; p++)
#pragma unroll
                            for (int q = 0; q < 4; q++) acc[p][q] = fmaf(l8[p], t4[q], acc[p][q]);
                    }
#pragma unroll
                    for (int p = 0; p < 8; p++) {
                        const int r = m0 + ty * 8 + p;
                        if (r >= n) continue;
                        float* dst = a + (size_t)r * lda + cc;
                        if (full) {
                            *reinterpret_cast<float4*>(dst) = make_float4(cv[p].x + acc[p][0], cv[p].y + acc[p][1],
                                                                          cv[p].z + acc[p][2], cv[p].w + acc[p][3]);
                        } else {
                            if (cc < n) dst[0] = cv[p].x + acc[p][0];
                            if (cc + 1 < n) dst[1] = cv[p].y + acc[p][1];
                            if (cc + 2 < n) dst[2] = cv[p].z + acc[p][2];
                            if (cc + 3 < n) dst[3] = cv[p].w + acc[p][3];
                        }
                    }
                }
                __syncthreads();  // this top buffer is refilled next; Lt stays for the row block
            }
        }
    }
}

// Blocked forward/back sweeps, right-hand sides resident in shared memory
// (nrhs <= NR).  Per 64-unknown block: the diagonal block is staged in shared
// memory and one warp per right-hand side walks its 64-step chain (values in
// lanes, pivots by shuffle); then every thread updates up to four later
// (forward) / earlier (backward) unknowns with the block's rows, loading each
// factor element once for all right-hand sides.
constexpr int kSolveBlk = 64;
__shared__ float s_dblk[kSolveBlk * (kSolveBlk + 1)];  // one diagonal block, shared by every instantiation

template <int NR>
__device__ __noinline__ void solve_blocked(const float* a, int lda, int n, float* b, int ldb, int nrhs, float* sm) {
    constexpr int SBK = kSolveBlk, DL = SBK + 1, PT = 4;  // unknowns per thread in the update
    float* Y = sm;                                        // nrhs x n
    float* Dblk = s_dblk;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int idx = tid; idx < nrhs * n; idx += BT) {
        const int q = idx / n, i = idx - q * n;
        Y[idx] = b[(size_t)q * ldb + i];
    }
    __syncthreads();
    // forward: y_i += y_k S[k][i] (i > k)
    for (int k0 = 0; k0 < n; k0 += SBK) {
        const int kb = min(SBK, n - k0);
        for (int idx = tid; idx < kb * kb; idx += BT) {
            const int r = idx / kb, c = idx - r * kb;
            Dblk[r * DL + c] = a[(size_t)(k0 + r) * lda + k0 + c];
        }
        __syncthreads();
        for (int q = warp; q < nrhs; q += BT / 32) {
            float* y = Y + q * n + k0;
            float v0 = lane < kb ? y[lane] : 0.0f, v1 = lane + 32 < kb ? y[lane + 32] : 0.0f;
            for (int k = 0; k < kb; k++) {
                const float yk = __shfl_sync(0xffffffffu, k < 32 ? v0 : v1, k & 31);
                if (lane > k && lane < kb) v0 = fmaf(yk, Dblk[k * DL + lane], v0);
                if (lane + 32 > k && lane + 32 < kb) v1 = fmaf(yk, Dblk[k * DL + lane + 32], v1);
            }
            if (lane < kb) y[lane] = v0;
            if (lane + 32 < kb) y[lane + 32] = v1;
        }
        __syncthreads();
        for (int i0 = k0 + kb + tid; i0 < n; i0 += PT * BT) {
            float acc[PT][NR];
#pragma unroll
            for (int e = 0; e < PT; e++)
#pragma unroll
                for (int q = 0; q < NR; q++) acc[e][q] = 0.0f;
            for (int k = 0; k < kb; k++) {
                const float* row = a + (size_t)(k0 + k) * lda;
                float yk[NR];
#pragma unroll
                for (int q = 0; q < NR; q++) yk[q] = q < nrhs ? Y[q * n + k0 + k] : 0.0f;
#pragma unroll
                for (int e = 0; e < PT; e++) {
                    const int i = i0 + e * BT;
                    const float s = i < n ? row[i] : 0.0f;
#pragma unroll
                    for (int q = 0; q < NR; q++) acc[e][q] = fmaf(yk[q], s, acc[e][q]);
                }
            }
#pragma unroll
            for (int e = 0; e < PT; e++) {
                const int i = i0 + e * BT;
                if (i < n)
#pragma unroll
                    for (int q = 0; q < NR; q++)
                        if (q < nrhs) Y[q * n + i] += acc[e][q];
            }
        }
        __syncthreads();
    }
    // backward: s = y_k S[k][k]; x_k = -s; y_i += s S[k][i] (i < k)
    for (int k0 = ((n - 1) / SBK) * SBK; k0 >= 0; k0 -= SBK) {
        const int kb = min(SBK, n - k0);
        for (int idx = tid; idx < kb * kb; idx += BT) {
            const int r = idx / kb, c = idx - r * kb;
            Dblk[r * DL + c] = a[(size_t)(k0 + r) * lda + k0 + c];
        }
        __syncthreads();
        for (int q = warp; q < nrhs; q += BT / 32) {
            float* y = Y + q * n + k0;
            float v0 = lane < kb ? y[lane] : 0.0f, v1 = lane + 32 < kb ? y[lane + 32] : 0.0f;
            for (int k = kb - 1; k >= 0; k--) {
                const float yk = __shfl_sync(0xffffffffu, k < 32 ? v0 : v1, k & 31);
                const float sk = yk * Dblk[k * DL + k];
                if (lane == (k & 31)) {
                    if (k < 32) v0 = -sk; else v1 = -sk;
                }
                if (lane < k) v0 = fmaf(sk, Dblk[k * DL + lane], v0);
                if (lane + 32 < k) v1 = fmaf(sk, Dblk[k * DL + lane + 32], v1);
            }
            if (lane < kb) y[lane] = v0;
            if (lane + 32 < kb) y[lane + 32] = v1;
        }
        __syncthreads();
        // coefficients s_k = -x_k of this block update the unknowns before it
        for (int i0 = tid; i0 < k0; i0 += PT * BT) {
            float acc[PT][NR];
#pragma unroll
            for (int e = 0; e < PT; e++)
#pragma unroll
                for (int q = 0; q < NR; q++) acc[e][q] = 0.0f;
            for (int k = 0; k < kb; k++) {
                const float* row = a + (size_t)(k0 + k) * lda;
                float sk[NR];
#pragma unroll
                for (int q = 0; q < NR; q++) sk[q] = q < nrhs ? -Y[q * n + k0 + k] : 0.0f;
#pragma unroll
                for (int e = 0; e < PT; e++) {
                    const int i = i0 + e * BT;
                    const float s = i < k0 ? row[i] : 0.0f;
#pragma unroll
                    for (int q = 0; q < NR; q++) acc[e][q] = fmaf(sk[q], s, acc[e][q]);
                }
            }
#pragma unroll
            for (int e = 0; e < PT; e++) {
                const int i = i0 + e * BT;
                if (i < k0)
#pragma unroll
                    for (int q = 0; q < NR; q++)
                        if (q < nrhs) Y[q * n + i] += acc[e][q];
            }
        }
        __syncthreads();
    }
    for (int idx = tid; idx < nrhs * n; idx += BT) {
        const int q = idx / n, i = idx - q * n;
        b[(size_t)q * ldb + i] = Y[idx];
    }
    __syncthreads();
}

__global__ void __launch_bounds__(BT, 2) k_batch_solve(const BatchSys* __restrict__ sys, int count, float* A, float* B,
                                                    int* next, Tune tune) {
    extern __shared__ float sm[];
    __shared__ int s_item;
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(next, 1);
        __syncthreads();
        const int t = s_item;
        __syncthreads();
        if (t >= count) break;
        const BatchSys s = sys[t];
        float* a = tune.absolute ? reinterpret_cast<float*>(s.a_off) : A + s.a_off;
        float* b = tune.absolute ? reinterpret_cast<float*>(s.b_off) : B + s.b_off;
        const bool factor = (s.nrhs & kSolveOnly) == 0;
        const int nrhs = s.nrhs & (kSolveOnly - 1);
        if (s.n <= tune.small_n_max) {
            solve_small(a, s.lda, s.n, b, s.ldb, nrhs, factor, sm);
        } else {
            if (factor) {
                if (tune.nb[bucket_of(s.n)] == 16)
                    factor_blocked<16, false>(a, s.lda, s.n, sm);
                else
                    factor_blocked<32, false>(a, s.lda, s.n, sm);
            }
            if (nrhs == 1)
                solve_blocked<1>(a, s.lda, s.n, b, s.ldb, nrhs, sm);
            else if (nrhs <= 4)
                solve_blocked<4>(a, s.lda, s.n, b, s.ldb, nrhs, sm);
            else
                solve_blocked<16>(a, s.lda, s.n, b, s.ldb, nrhs, sm);
        }
    }
}

// max over the CTA of v[0..3] (non-negative values; NaN marks a non-finite
// input and wins), into out[0..3] for every thread.
__device__ __forceinline__ void block_max4(double (&v)[4], double* red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < 4; q++) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double w = __shfl_xor_sync(0xffffffffu, v[q], o);
            v[q] = (isnan(w) || w > v[q]) ? w : v[q];
        }
    }
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < 4; q++) red[warp * 4 + q] = v[q];
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 4; q++) {
        double m = red[q];
        for (int w = 1; w < BT / 32; w++) {
            const double x = red[w * 4 + q];
            m = (isnan(x) || x > m) ? x : m;
        }
        v[q] = m;
    }
    __syncthreads();
}

// FP64 iterative refinement of one factored system (all threads of the CTA),
// the per-system form of refine_core: x = the FP32 solution in b32, widened;
// repeat r = b - M x (M = S0^T, the original FP32 matrix widened exactly, FP64
// accumulation), HPL scaled residual per right-hand side
// ||r||_inf / ((||M||_inf ||x||_inf + ||b||_inf) n eps), eps = DBL_EPSILON/2
// (LINPACK/src/host/gmres.c:182-193); stop at <= 16 or after max_iters
// refinements, else d = LU \ r (FP32 factors, r rounded to FP32), x += d.
// Returns the refinements made; *resid = the largest scaled residual (NaN if
// any value is not finite).
__device__ int refine_system(const float* __restrict__ lu, const float* __restrict__ a0, int lda, int n,
                             float* b32, const double* __restrict__ b64, double* x64, int ldb, int nrhs,
                             int max_iters, bool small, int nb, float* sm, double* resid) {
    constexpr int PC = 4;  // unknowns per thread (n <= 1024)
    const int tid = threadIdx.x;
    double* xs = reinterpret_cast<double*>(sm);  // 4 right-hand sides x n (FP64)
    double* red = xs + 4 * 1024;                 // 8 warps x 4
    for (int idx = tid; idx < nrhs * n; idx += BT) {
        const int q = idx / n, i = idx - q * n;
        x64[(size_t)q * ldb + i] = (double)b32[(size_t)q * ldb + i];
    }
    __syncthreads();
    double normM = 0.0;
    double worst = 0.0;
    int it = 0;
    for (;; it++) {
        worst = 0.0;
        for (int q0 = 0; q0 < nrhs; q0 += 4) {
            const int nq = min(4, nrhs - q0);
            for (int idx = tid; idx < 4 * n; idx += BT) {
                const int q = idx / n, j = idx - q * n;
                xs[idx] = q < nq ? x64[(size_t)(q0 + q) * ldb + j] : 0.0;
            }
            __syncthreads();
            double acc[PC][4], col[PC];
#pragma unroll
            for (int e = 0; e < PC; e++) {
                col[e] = 0.0;
#pragma unroll
                for (int q = 0; q < 4; q++) acc[e][q] = 0.0;
            }
            // unrolled so that the row loads of several j are in flight at once (the loop is
            // otherwise one L2/HBM round trip per row)
#pragma unroll 8
            for (int j = 0; j < n; j++) {
                const float* row = a0 + (size_t)j * lda;
                double xj[4];
#pragma unroll
                for (int q = 0; q < 4; q++) xj[q] = xs[q * n + j];
#pragma unroll
                for (int e = 0; e < PC; e++) {
                    const int i = tid + e * BT;
                    const double sv = i < n ? (double)row[i] : 0.0;
                    col[e] += fabs(sv);
#pragma unroll
                    for (int q = 0; q < 4; q++) acc[e][q] = fma(sv, xj[q], acc[e][q]);
                }
            }
            // r = b - M x into b32 (FP32, the next correction's right-hand side); norms
            double rm[4] = {0.0, 0.0, 0.0, 0.0}, xm[4] = {0.0, 0.0, 0.0, 0.0}, bm[4] = {0.0, 0.0, 0.0, 0.0};
            double cm[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
            for (int e = 0; e < PC; e++) {
                const int i = tid + e * BT;
                if (i >= n) continue;
                cm[0] = (isnan(col[e]) || col[e] > cm[0]) ? col[e] : cm[0];
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    if (q >= nq) continue;
                    const double bv = b64[(size_t)(q0 + q) * ldb + i];
                    const double r = bv - acc[e][q];
                    b32[(size_t)(q0 + q) * ldb + i] = (float)r;
                    const double ar = fabs(r), ax = fabs(xs[q * n + i]), ab = fabs(bv);
                    rm[q] = (isnan(ar) || ar > rm[q]) ? ar : rm[q];
                    xm[q] = (isnan(ax) || ax > xm[q]) ? ax : xm[q];
                    bm[q] = (isnan(ab) || ab > bm[q]) ? ab : bm[q];
                }
            }
            block_max4(rm, red);
            block_max4(xm, red);
            block_max4(bm, red);
            if (it == 0 && q0 == 0) {
                block_max4(cm, red);
                normM = cm[0];
            }
            for (int q = 0; q < nq; q++) {
                const double h = rm[q] / (normM * xm[q] + bm[q]) / (double)n / (DBL_EPSILON / 2.0);
                worst = (isnan(h) || !(h <= worst)) ? h : worst;
            }
        }
        if (!(worst > 16.0) || isnan(worst) || isinf(worst) || it >= max_iters) break;
        // d = LU \ r, x += d
        if (small)
            solve_small(const_cast<float*>(lu), lda, n, b32, ldb, nrhs, false, sm);
        else if (nrhs == 1)
            solve_blocked<1>(lu, lda, n, b32, ldb, nrhs, sm);
        else if (nrhs <= 4)
            solve_blocked<4>(lu, lda, n, b32, ldb, nrhs, sm);
        else
            solve_blocked<16>(lu, lda, n, b32, ldb, nrhs, sm);
        for (int idx = tid; idx < nrhs * n; idx += BT) {
            const int q = idx / n, i = idx - q * n;
            x64[(size_t)q * ldb + i] += (double)b32[(size_t)q * ldb + i];
        }
        __syncthreads();
    }
    (void)nb;
    *resid = worst;
    return it;
}

// The refined form of k_batch_solve: per system, b32 = (float) b64; factor
// in place (BF16: the blocked path's trailing updates on the tensor cores,
// the diagonal blocks and triangular stages in FP32; systems solved whole in
// shared memory are factored in FP32); FP32 solve into b32; FP64 refinement
// against the original a0 into x64.  iters / resid: per descriptor position.
template <bool BF16>
__global__ void __launch_bounds__(BT, 2)
    k_batch_solve_ir(const BatchSys* __restrict__ sys, int count, float* A, const float* __restrict__ A0, float* B32,
                     const double* __restrict__ B64, double* X64, int* next, Tune tune, int max_iters,
                     int* __restrict__ iters, double* __restrict__ resid) {
    extern __shared__ float sm[];
    __shared__ int s_item;
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(next, 1);
        __syncthreads();
        const int t = s_item;
        __syncthreads();
        if (t >= count) break;
        const BatchSys s = sys[t];
        float* a = A + s.a_off;
        const float* a0 = A0 + s.a_off;
        float* b = B32 + s.b_off;
        const double* b64 = B64 + s.b_off;
        double* x64 = X64 + s.b_off;
        const int nrhs = s.nrhs;
        for (int idx = threadIdx.x; idx < nrhs * s.n; idx += BT) {
            const int q = idx / s.n, i = idx - q * s.n;
            b[(size_t)q * s.ldb + i] = (float)b64[(size_t)q * s.ldb + i];
        }
        __syncthreads();
        const bool small = s.n <= tune.small_n_max;
        const int nb = tune.nb[bucket_of(s.n)];
        if (small) {
            solve_small(a, s.lda, s.n, b, s.ldb, nrhs, true, sm);
        } else {
            if (nb == 16)
                factor_blocked<16, BF16>(a, s.lda, s.n, sm);
            else
                factor_blocked<32, BF16>(a, s.lda, s.n, sm);
            if (nrhs == 1)
                solve_blocked<1>(a, s.lda, s.n, b, s.ldb, nrhs, sm);
            else if (nrhs <= 4)
                solve_blocked<4>(a, s.lda, s.n, b, s.ldb, nrhs, sm);
            else
                solve_blocked<16>(a, s.lda, s.n, b, s.ldb, nrhs, sm);
        }
        double r = 0.0;
        const int k = refine_system(a, a0, s.lda, s.n, b, b64, x64, s.ldb, nrhs, max_iters, small, nb, sm, &r);
        if (threadIdx.x == 0) {
            iters[t] = k;
            resid[t] = r;
        }
    }
}

}  // namespace

int batch_init_attrs() {
    LP_CUDA(cudaFuncSetAttribute(k_batch_solve, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBatchSmem));
    LP_CUDA(cudaFuncSetAttribute(k_batch_solve_ir<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kBatchSmem));
    LP_CUDA(cudaFuncSetAttribute(k_batch_solve_ir<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kBatchSmem));
    return LP_OK;
}

int validate_batch(int count, const lp_system* systems) {
    if (count < 0 || (count > 0 && systems == nullptr)) return fail(LP_E_INVALID, "batch: bad system list");
    for (int i = 0; i < count; i++) {
        const lp_system& s = systems[i];
        if (s.n <= 0 || s.n > 1024 || s.nrhs <= 0 || s.nrhs > RHS_MAX || s.lda < s.n || s.ldb < s.n || s.a_off < 0 ||
            s.b_off < 0)
            return fail(LP_E_INVALID, "batch: system " + std::to_string(i) +
                                          " needs 1 <= n <= 1024, 1 <= nrhs <= 16, lda >= n, ldb >= n");
    }
    return LP_OK;
}

int launch_batch(lp_ctx* c, const lp_system* d_sorted, int count, float* dA, float* dB, const lp_batch_config& cfg,
                 int* d_next, cudaStream_t st, bool absolute) {
    static_assert(kSolveOnly > RHS_MAX, "solve-only flag above the nrhs range");
    Tune tune;
    tune.absolute = absolute ? 1 : 0;
    tune.small_n_max = cfg.small_n_max;
    for (int i = 0; i < NBUCKETS; i++) tune.nb[i] = cfg.nb[i];
    const int per_sm = cfg.ctas_per_sm < 1 ? 1 : (cfg.ctas_per_sm > 3 ? 3 : cfg.ctas_per_sm);
    int grid = c->num_sms * per_sm;
    if (grid > count) grid = count;
    if (grid < 1) return LP_OK;
    LP_CUDA(cudaMemsetAsync(d_next, 0, sizeof(int), st));
    k_batch_solve<<<grid, BT, kBatchSmem, st>>>(reinterpret_cast<const BatchSys*>(d_sorted), count, dA, dB, d_next,
                                                 tune);
    count_launch();
    LP_CUDA(cudaGetLastError());
    return LP_OK;
}

int launch_batch_ir(lp_ctx* c, bool bf16, const lp_system* d_sorted, int count, float* dA, const float* dA0,
                    float* dB32, const double* dB64, double* dX, const lp_batch_config& cfg, int max_iters,
                    int* d_iters, double* d_resid, int* d_next, cudaStream_t st) {
    Tune tune;
    tune.absolute = 0;
    tune.small_n_max = cfg.small_n_max;
    for (int i = 0; i < NBUCKETS; i++) tune.nb[i] = cfg.nb[i];
    const int per_sm = cfg.ctas_per_sm < 1 ? 1 : (cfg.ctas_per_sm > 3 ? 3 : cfg.ctas_per_sm);
    int grid = c->num_sms * per_sm;
    if (grid > count) grid = count;
    if (grid < 1) return LP_OK;
    LP_CUDA(cudaMemsetAsync(d_next, 0, sizeof(int), st));
    const auto* sys = reinterpret_cast<const BatchSys*>(d_sorted);
    if (bf16)
        k_batch_solve_ir<true><<<grid, BT, kBatchSmem, st>>>(sys, count, dA, dA0, dB32, dB64, dX, d_next, tune,
                                                             max_iters, d_iters, d_resid);
    else
        k_batch_solve_ir<false><<<grid, BT, kBatchSmem, st>>>(sys, count, dA, dA0, dB32, dB64, dX, d_next, tune,
                                                              max_iters, d_iters, d_resid);
    count_launch();
    LP_CUDA(cudaGetLastError());
    return LP_OK;
}

}  // namespace lp
