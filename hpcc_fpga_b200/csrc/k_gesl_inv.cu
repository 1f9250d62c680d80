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
// instead of a 128-step sequential chain.
//
// Each sweep is ONE persistent launch over 128-unknown tiles.  A CTA takes
// tiles in ticket order (atomic counter: forward 0, 1, 2, ...; backward from
// the last tile down) and accumulates, for its tile j, the contributions of
// every earlier tile K: acc_j += y_K^T * S[rows of K][columns of j], reading
// each factor element once.  It loads the factor rows of tile K before
// waiting for K's "solved" flag, so the wait overlaps the memory traffic, and
// keeps per-thread partial sums until all K are in; then it reduces them,
// forms y_j with the block operator (prefetched into shared memory when the
// tile started), publishes y_j and raises flag j.  A CTA only waits on tiles
// taken before its own by running CTAs, so progress is guaranteed; every wait
// is bounded nonetheless, and a CTA that gives up records the error, writes
// NaN for its tile (the result then fails every residual check) and still
// raises its flag so no other CTA waits on it.
#include <algorithm>

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

// coef[r][i] = sum_k M[k][i] * acc[r][k] for a 128 x 128 operator M (shared
// memory); all 256 threads: thread (h, i) sums k in [64h, 64h+64).
template <int NR>
__device__ __forceinline__ void block_matvec(const float* M, const float* acc, float* part, float* coef) {
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

constexpr unsigned long long kWaitLimitNs = 250ull * 1000 * 1000;  // a bounded wait gives up after 250 ms

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ int ld_acquire(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(int* p, int v) {
    asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Lane 0 of the calling warp polls flag f (bounded by kWaitLimitNs); the warp
// then proceeds together.  false: the wait gave up or another CTA aborted
// (err set).
__device__ __forceinline__ bool warp_wait_flag(const int* f, int* err) {
    int ok = 1;
    if ((threadIdx.x & 31) == 0) {
        ok = 0;
        const unsigned long long t0 = global_ns();
        for (;;) {
            if (ld_acquire(f) != 0) {
                ok = 1;
                break;
            }
            if (*(volatile int*)err != 0) break;
            if (global_ns() - t0 > kWaitLimitNs) {
                atomicExch(err, 1);
                break;
            }
            __nanosleep(64);
        }
    }
    ok = __shfl_sync(0xffffffffu, ok, 0);
    __syncwarp();
    return ok != 0;
}

// The persistent sweep.  FWD: tiles ascend, acc_j = b_j + sum_{K<j} y_K S[K][j],
// y_j = Y_j^T acc_j -> w (ldw).  Backward: tiles descend,
// acc_j = y_j + sum_{K>j} s_K S[K][j], s_j = X_j^T acc_j -> w (ldw), x_j = -s_j -> out.
// in: b (forward) / y (backward), leading dimension ldi.
template <int NR, bool FWD>
__global__ void __launch_bounds__(GT) k_gesl_sweep(const float* __restrict__ a, int lda, int n,
                                                   const float* __restrict__ inv, const float* __restrict__ in,
                                                   int ldi, const float* __restrict__ wprev, float* __restrict__ w,
                                                   int ldw, float* __restrict__ out, int ldo, int nrhs,
                                                   int* __restrict__ flags, int* __restrict__ ticket,
                                                   int* __restrict__ err, const int* __restrict__ never) {
    extern __shared__ __align__(16) float smem[];
    float* op = smem;                 // 128 x 128 block operator
    float* red = op + BLK2;           // 8 x NR x 128 partial sums
    float* acc = red + 8 * NR * SB;   // NR x 128
    float* part = acc + NR * SB;      // 2 x NR x 128
    float* res = part + 2 * NR * SB;  // NR x 128
    __shared__ int s_tile;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nblk = (n + SB - 1) / SB;
    for (;;) {
        __syncthreads();  // the previous tile's shared data is consumed
        if (tid == 0) s_tile = atomicAdd(ticket, 1);
        __syncthreads();
        const int t = s_tile;
        if (t >= nblk) break;
        const int j = FWD ? t : nblk - 1 - t;
        const int c0 = j * SB, kb = min(SB, n - c0);
        // the tile's block operator (Y for the forward sweep, X backward), 16-byte copies
        {
            const float* src = inv + (size_t)j * 2 * BLK2 + (FWD ? BLK2 : 0);
            for (int idx = tid; idx < BLK2 / 4; idx += GT) {
                const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(op + 4 * idx));
                asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src + 4 * idx) : "memory");
            }
            asm volatile("cp.async.commit_group;\n" ::: "memory");
        }
        // partial sums of this thread: columns c0 + 4 lane .. +3, rows 16 warp .. +15 of every source tile
        float p[NR][4];
#pragma unroll
        for (int q = 0; q < NR; q++)
#pragma unroll
            for (int e = 0; e < 4; e++) p[q][e] = 0.0f;
        const int col = c0 + 4 * lane;
        const bool vec = col + 3 < n;
        bool ok = true;
        const int nsrc = FWD ? j : nblk - 1 - j;
        for (int s = 0; s < nsrc; s++) {
            const int K = FWD ? s : nblk - 1 - s;
            const int k0 = K * SB, kbK = min(SB, n - k0);
            float4 v[16];
#pragma unroll
            for (int r = 0; r < 16; r++) {
                const int row = 16 * warp + r;
                const float* src = a + (size_t)(k0 + row) * lda + col;
                if (row < kbK && vec) {
                    v[r] = *reinterpret_cast<const float4*>(src);
                } else {
                    v[r].x = (row < kbK && col < n) ? src[0] : 0.0f;
                    v[r].y = (row < kbK && col + 1 < n) ? src[1] : 0.0f;
                    v[r].z = (row < kbK && col + 2 < n) ? src[2] : 0.0f;
                    v[r].w = (row < kbK && col + 3 < n) ? src[3] : 0.0f;
                }
            }
            // never (tests only): the second tile waits on a word that nothing sets
            if (!warp_wait_flag((never != nullptr && t == 1 && s == 0) ? never : &flags[K], err)) {
                ok = false;
                break;
            }
#pragma unroll
            for (int r = 0; r < 16; r++) {
                const int row = 16 * warp + r;
#pragma unroll
                for (int q = 0; q < NR; q++) {
                    // written by another CTA after this CTA may have cached the line: read through L2
                    const float yk = (q < nrhs && row < kbK) ? __ldcg(wprev + (size_t)q * ldw + k0 + row) : 0.0f;
                    p[q][0] = fmaf(yk, v[r].x, p[q][0]);
                    p[q][1] = fmaf(yk, v[r].y, p[q][1]);
                    p[q][2] = fmaf(yk, v[r].z, p[q][2]);
                    p[q][3] = fmaf(yk, v[r].w, p[q][3]);
                }
            }
        }
        ok = __syncthreads_and(ok);
#pragma unroll
        for (int q = 0; q < NR; q++)
#pragma unroll
            for (int e = 0; e < 4; e++) red[(warp * NR + q) * SB + 4 * lane + e] = p[q][e];
        asm volatile("cp.async.wait_all;\n" ::: "memory");
        __syncthreads();
        for (int idx = tid; idx < NR * SB; idx += GT) {
            const int q = idx / SB, i = idx - q * SB;
            float v = 0.0f;
            if (q < nrhs && i < kb) {
                v = in[(size_t)q * ldi + c0 + i];
#pragma unroll
                for (int ww = 0; ww < GT / 32; ww++) v += red[(ww * NR + q) * SB + i];
            }
            acc[idx] = v;
        }
        __syncthreads();
        block_matvec<NR>(op, acc, part, res);
        for (int idx = tid; idx < NR * SB; idx += GT) {
            const int q = idx / SB, i = idx - q * SB;
            if (q < nrhs && i < kb) {
                const float v = ok ? res[idx] : __int_as_float(0x7fc00000);  // NaN marks an aborted solve
                w[(size_t)q * ldw + c0 + i] = v;
                if (!FWD) out[(size_t)q * ldo + c0 + i] = -v;
            }
        }
        __threadfence();
        __syncthreads();
        if (tid == 0) st_release(&flags[j], 1);
    }
}

template <int NR>
constexpr size_t sweep_smem() {
    return sizeof(float) * ((size_t)BLK2 + (8 * NR + 4 * NR) * (size_t)SB);
}

template <int NR>
int sweeps(const float* a, int lda, int n, float* b, int ldb, int nrhs, float* w1, float* w2, const float* inv,
           int* sync, int* err, bool stall, int sms, cudaStream_t st) {
    const int nblk = (n + SB - 1) / SB;
    int* flags_f = sync;
    int* flags_b = sync + nblk;
    int* tickets = sync + 2 * nblk;
    const int* never = stall ? tickets + 2 : nullptr;
    LP_CUDA(cudaMemsetAsync(sync, 0, sizeof(int) * gesl_sync_ints(n), st));  // err is the caller's
    const int per_sm = NR >= 16 ? 1 : 2;
    const int grid = std::min(nblk, per_sm * sms);
    // forward: b -> y (w2)
    k_gesl_sweep<NR, true><<<grid, GT, sweep_smem<NR>(), st>>>(a, lda, n, inv, b, ldb, w2, w2, n, nullptr, 0, nrhs,
                                                              flags_f, tickets, err, never);
    // backward: y (w2) -> s (w1), x -> b
    k_gesl_sweep<NR, false><<<grid, GT, sweep_smem<NR>(), st>>>(a, lda, n, inv, w2, n, w1, w1, n, b, ldb, nrhs,
                                                               flags_b, tickets + 1, err, nullptr);
    count_launch(2);
    LP_CUDA(cudaGetLastError());
    return LP_OK;
}

template <int NR>
int inv_attrs() {
    LP_CUDA(cudaFuncSetAttribute(k_gesl_sweep<NR, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)sweep_smem<NR>()));
    LP_CUDA(cudaFuncSetAttribute(k_gesl_sweep<NR, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)sweep_smem<NR>()));
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

// Sync words of the persistent sweeps: flags of both directions, two tickets,
// and one word that nothing sets (the target of the test stall).
size_t gesl_sync_ints(int n) { return 2 * (size_t)((n + SB - 1) / SB) + 3; }

// Forward + back substitution with precomputed block inverses; sync:
// gesl_sync_ints(n) ints (cleared here); err: an error word the caller zeroes
// and reads (set when a bounded wait gave up; that tile is written as NaN).
// stall (tests only): the forward sweep's second tile waits on a word that
// nothing sets, so its bounded wait runs out.
int launch_gesl_inv(const float* a, int lda, int n, float* b, int ldb, int nrhs, float* work, const float* inv,
                    int* sync, int* err, bool stall, cudaStream_t st) {
    if (n <= 0 || nrhs <= 0) return LP_OK;
    if (lda % 4 != 0 || !aligned16(a)) return fail(LP_E_INVALID, "gesl: factors need lda % 4 == 0, 16-byte aligned");
    int dev = 0, sms = 0;
    LP_CUDA(cudaGetDevice(&dev));
    LP_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    for (int r0 = 0; r0 < nrhs; r0 += 16) {
        const int g = (nrhs - r0) < 16 ? (nrhs - r0) : 16;
        float* bb = b + (size_t)r0 * ldb;
        float* w1 = work;
        float* w2 = work + (size_t)n * g;
        if (g == 1)
            LP_CHECK(sweeps<1>(a, lda, n, bb, ldb, g, w1, w2, inv, sync, err, stall && r0 == 0, sms, st));
        else if (g <= 4)
            LP_CHECK(sweeps<4>(a, lda, n, bb, ldb, g, w1, w2, inv, sync, err, stall && r0 == 0, sms, st));
        else
            LP_CHECK(sweeps<16>(a, lda, n, bb, ldb, g, w1, w2, inv, sync, err, stall && r0 == 0, sms, st));
    }
    return LP_OK;
}

}  // namespace lp
