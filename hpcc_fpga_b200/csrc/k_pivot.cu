// LU with partial pivoting (LINPACK dgefa / dgesl convention) — the
// reference's gefa_ref / gesl_ref (LINPACK/src/host/linpack_data.cpp:72-156),
// used by the harness for non-diagonally-dominant ("--uniform") matrices
// (linpack_benchmark.hpp:69, 440-447).
//
// Storage S[r][c] = a[r*lda + c]; the factored matrix is M = S^T, so M's
// column k is storage row k (contiguous) and the pivot search of step k is a
// scan of one storage row.  Encoding on return (reference): diagonal u_kk,
// storage row k right of the diagonal the negated multipliers -l_ik, left of
// it U; ipvt[k] = the pivot row of step k.  In LINPACK's convention the
// interchange of step k touches only M's columns >= k, so the multipliers of
// earlier columns stay in the row order of the step that produced them.
//
// Blocked right-looking form, panel width PB (128, or 64 when a 128-wide
// panel of the tallest column does not fit the SMs' shared memory):
//   k_piv_panel  the PB columns of M (PB storage rows x the trailing length),
//                one cooperative launch: each CTA holds a slice of rows in
//                shared memory; per step a bounded grid barrier publishes
//                every CTA's best candidate and its row, all CTAs agree on
//                the pivot (largest |v|, then smallest index), the two rows
//                are exchanged across CTAs and each CTA scales and updates
//                its rows with the reference's rounding (multiplier in
//                double, product and sum rounded to float separately).
//                Inside the panel whole panel rows are exchanged ("block
//                form"); the earlier multipliers of the same panel are put
//                back into LINPACK order by k_piv_convert at the end.
//   k_piv_rows   every trailing storage row: the panel's interchanges as one
//                composite permutation (gathered, then scattered), the unit
//                lower triangular solve with the panel's diagonal block (U12),
//                and the transposed copy the trailing update reads.
//   inner        k_sgemm_update: C += U12 * L21, the same contraction as the
//                no-pivoting path (hpl_torus_PCIE.cl:711-865).
//   k_piv_gesl   forward (interchanges, then the block's triangular solve and
//                the update of everything below it, per panel) and back
//                substitution, one cooperative launch with one bounded grid
//                barrier per panel and direction.
//
// Every spin-wait is bounded: a barrier that does not complete within the
// iteration limit sets the error word and every CTA returns; the host
// reports LP_E_TIMEOUT.
#include "lp_ctx.cuh"

namespace lp {
namespace {

constexpr int PT = 256;                  // threads per CTA
constexpr int GMAX = 256;                // CTAs of one panel launch, at most
constexpr int PBMAX = 128;               // panel width, at most
constexpr unsigned kSpinLimit = 1u << 21;

// Device scratch of one factorization or solve.
constexpr size_t kKeysOff = 16;                                          // u64 [2][GMAX]
constexpr size_t kRowsOff = kKeysOff + 2 * GMAX * sizeof(unsigned long long);  // float [2][GMAX][PBMAX]
constexpr size_t kKrowOff = kRowsOff + 2 * (size_t)GMAX * PBMAX * sizeof(float);  // float [2][PBMAX]
constexpr size_t kSyncBytes = kKrowOff + 2 * PBMAX * sizeof(float);

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Grid-wide barrier among the co-resident CTAs of a cooperative launch: the
// counter only grows; barrier number b of a launch completes at base + b * G.
// Returns false (and leaves the error word set) if it did not complete
// within the iteration limit or another CTA gave up.
__device__ __forceinline__ bool grid_sync(unsigned* bar, unsigned target, int* err) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(bar, 1u);
        int ok = 1;
        unsigned spins = 0;
        while (ld_acquire_u32(bar) < target) {
            if (*reinterpret_cast<volatile int*>(err) != 0 || ++spins > kSpinLimit) {
                atomicExch(err, 1);
                ok = 0;
                break;
            }
            __nanosleep(32);
        }
        __threadfence();
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

__device__ __forceinline__ unsigned long long warp_max_u64(unsigned long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w > v ? w : v;
    }
    return v;
}

// Candidate key of M row i in the pivot search: |v| in the high word (the
// bit pattern of a non-negative float orders like the value), the index
// complemented in the low word (equal magnitudes: the smaller index wins, as
// the reference's strict "<" scan keeps the first).  NaN never wins, except
// at the diagonal itself, which the reference's scan then never leaves.
__device__ __forceinline__ unsigned long long pivot_key(float v, unsigned i, bool diag) {
    const float a = fabsf(v);
    if (a != a) return diag ? ~0ull : 0ull;
    return (static_cast<unsigned long long>(__float_as_uint(a)) << 32) | (0xFFFFFFFFu - i);
}

__global__ void __launch_bounds__(PT, 1)
    k_piv_panel(float* __restrict__ a, int lda, int n, int k0, int kb, int R, int* __restrict__ ipvt,
                unsigned char* __restrict__ sync, unsigned bar_base) {
    extern __shared__ float slab[];  // kb columns of M x R rows: slab[c * R + r]
    __shared__ float newk[PBMAX];
    __shared__ unsigned long long red[PT / 32];
    __shared__ int s_p, s_wg;
    unsigned* bar = reinterpret_cast<unsigned*>(sync);
    int* err = reinterpret_cast<int*>(sync + 4);
    unsigned long long* keys = reinterpret_cast<unsigned long long*>(sync + kKeysOff);
    float* rows = reinterpret_cast<float*>(sync + kRowsOff);
    float* krow = reinterpret_cast<float*>(sync + kKrowOff);
    const int G = gridDim.x, g = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int row0 = g * R;                       // M rows k0 + row0 ... belong to this CTA
    const int nr = max(0, min(R, n - k0 - row0));
    const size_t cbase = (size_t)k0 + row0;       // their storage column
    for (int c = 0; c < kb; c++) {  // every copy in flight before the first wait
        const float* src = a + (size_t)(k0 + c) * lda + cbase;
        for (int r = tid; r < nr; r += PT) cp_async4(slab + c * R + r, src + r);
    }
    cp_async_wait_all();
    __syncthreads();
    for (int kk = 0; kk < kb; kk++) {
        const int k = k0 + kk, par = kk & 1;
        const int rk = kk - row0;  // local index of M row k (in range only in its owner)
        const bool own_k = rk >= 0 && rk < nr;
        const float* colk = slab + kk * R;
        unsigned long long best = 0;
        for (int r = max(0, rk) + tid; r < nr; r += PT) {
            const unsigned long long key = pivot_key(colk[r], (unsigned)(cbase + r), r == rk);
            best = key > best ? key : best;
        }
        best = warp_max_u64(best);
        if (lane == 0) red[warp] = best;
        __syncthreads();
        if (warp == 0) {
            unsigned long long v = lane < PT / 32 ? red[lane] : 0ull;
            v = warp_max_u64(v);
            if (lane == 0) red[0] = v;
        }
        __syncthreads();
        const unsigned long long mine = red[0];
        // publish this CTA's candidate (its whole panel row) and, from the owner, row k
        if (mine != 0ull) {
            const int rc = mine == ~0ull ? rk : (int)(0xFFFFFFFFu - (unsigned)mine) - (int)cbase;
            float* dst = rows + ((size_t)par * GMAX + g) * PBMAX;
            for (int c = tid; c < kb; c += PT) dst[c] = slab[c * R + rc];
        }
        if (own_k)
            for (int c = tid; c < kb; c += PT) krow[par * PBMAX + c] = slab[c * R + rk];
        if (tid == 0) keys[par * GMAX + g] = mine;
        if (!grid_sync(bar, bar_base + (unsigned)(kk + 1) * (unsigned)G, err)) return;
        if (warp == 0) {
            unsigned long long v = 0;
            int wg = 0;
            for (int q = lane; q < G; q += 32) {
                const unsigned long long x = __ldcg(keys + par * GMAX + q);
                if (x > v) v = x, wg = q;
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const unsigned long long ov = __shfl_xor_sync(0xffffffffu, v, o);
                const int ow = __shfl_xor_sync(0xffffffffu, wg, o);
                if (ov > v || (ov == v && ow < wg)) v = ov, wg = ow;
            }
            if (lane == 0) {
                s_p = v == ~0ull ? k : (int)(0xFFFFFFFFu - (unsigned)v);
                s_wg = wg;
            }
        }
        __syncthreads();
        const int p = s_p, wg = s_wg;
        for (int c = tid; c < kb; c += PT) newk[c] = __ldcg(rows + ((size_t)par * GMAX + wg) * PBMAX + c);
        __syncthreads();
        if (p != k) {  // exchange M rows k and p over the whole panel
            const int rp = p - (int)cbase;
            if (rp >= 0 && rp < nr)
                for (int c = tid; c < kb; c += PT) slab[c * R + rp] = __ldcg(krow + par * PBMAX + c);
            if (own_k)
                for (int c = tid; c < kb; c += PT) slab[c * R + rk] = newk[c];
        }
        if (g == 0 && tid == 0) ipvt[k] = p;
        __syncthreads();
        // multipliers: the reciprocal in double, the product rounded to float
        const double s = -1.0 / (double)newk[kk];
        const int rs = max(0, kk + 1 - row0);  // local rows below the pivot
        float* colm = slab + kk * R;
        for (int r = rs + tid; r < nr; r += PT) colm[r] = (float)((double)colm[r] * s);
        __syncthreads();
        // rank-1 update of the panel's later columns: product and sum rounded separately
        const int nrows = nr - rs;
        if (kk + 1 < kb && nrows > 0) {
            int rw = 32;
            while (rw < nrows && rw < PT) rw <<= 1;
            const int cg = PT / rw, rl = tid & (rw - 1);
            for (int c = kk + 1 + tid / rw; c < kb; c += cg) {
                const float u = newk[c];
                float* colc = slab + c * R;
                for (int r = rs + rl; r < nr; r += rw) colc[r] = __fadd_rn(colc[r], __fmul_rn(colm[r], u));
            }
        }
        __syncthreads();
    }
    for (int c = 0; c < kb; c++) {
        float* dst = a + (size_t)(k0 + c) * lda + cbase;
        for (int r = tid; r < nr; r += PT) dst[r] = slab[c * R + r];
    }
}

// The interchanges of one panel (M rows k0 .. k0+kb-1 with ipvt) as one
// composite permutation, by warp 0: after it, panel position k0+t holds the
// value that was at psrc[t], and outside position odst[e] (>= r0) the value
// that was at osrc[e] (a panel position, or odst[e] itself when the value went
// out and came back).  pv: the panel's ipvt entries in shared memory.
__device__ void build_perm(const int* pv, int k0, int kb, int r0, int* psrc, int* odst, int* osrc, int* s_nout) {
    const int lane = threadIdx.x & 31;
    for (int t = lane; t < kb; t += 32) psrc[t] = k0 + t;
    __syncwarp();
    int nout = 0;
    for (int kk = 0; kk < kb; kk++) {
        const int p = pv[kk];
        if (p == k0 + kk) continue;
        if (p < r0) {
            if (lane == 0) {
                const int t = psrc[kk];
                psrc[kk] = psrc[p - k0];
                psrc[p - k0] = t;
            }
        } else {
            int found = nout;
            for (int e0 = 0; e0 < nout; e0 += 32) {
                const int e = e0 + lane;
                const unsigned hit = __ballot_sync(0xffffffffu, e < nout && odst[e] == p);
                if (hit != 0u) {
                    found = e0 + __ffs(hit) - 1;
                    break;
                }
            }
            if (lane == 0) {
                if (found == nout) odst[found] = p, osrc[found] = p;
                const int t = psrc[kk];
                psrc[kk] = osrc[found];
                osrc[found] = t;
            }
            if (found == nout) nout++;
        }
        __syncwarp();
    }
    if (lane == 0) *s_nout = nout;
}

// Trailing storage rows c >= r0 (M's trailing columns): interchanges, then
// x_t += L[k][t] x_k (t > k) with the panel's unit lower block, written in
// place and transposed into at (at[t * ldat + c - r0]).  One warp per row.
template <int PB>
__global__ void __launch_bounds__(PT)
    k_piv_rows(float* __restrict__ a, int lda, int n, int k0, const int* __restrict__ ipvt, float* __restrict__ at,
               int ldat) {
    constexpr int Q = PB / 32, SS = PB + 4;
    extern __shared__ float sm[];
    float* L = sm;               // L[k * PB + t] = S[k0 + k][k0 + t]
    float* stage = L + PB * PB;  // 8 rows x SS
    __shared__ int pv[PB], psrc[PB], odst[PB], osrc[PB];
    __shared__ int s_nout;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int r0 = k0 + PB, m = n - r0;
    for (int t = tid; t < PB; t += PT) pv[t] = ipvt[k0 + t];
    for (int idx = tid; idx < PB * PB; idx += PT) {
        const int k = idx / PB, t = idx - k * PB;
        cp_async4(L + idx, a + (size_t)(k0 + k) * lda + k0 + t);
    }
    cp_async_wait_all();
    __syncthreads();
    if (warp == 0) build_perm(pv, k0, PB, r0, psrc, odst, osrc, &s_nout);
    __syncthreads();
    const int nout = s_nout;
    for (int base = blockIdx.x * 8; base < m; base += gridDim.x * 8) {
        const int c = r0 + base + warp;
        if (c < n) {
            float* row = a + (size_t)c * lda;
            float x[Q], ov[Q];
#pragma unroll
            for (int q = 0; q < Q; q++) {
                const int e = lane + 32 * q;
                x[q] = row[psrc[e]];
                ov[q] = e < nout ? row[osrc[e]] : 0.0f;
            }
            __syncwarp();
#pragma unroll
            for (int q = 0; q < Q; q++) {
                const int e = lane + 32 * q;
                if (e < nout) row[odst[e]] = ov[q];
            }
#pragma unroll
            for (int k = 0; k < PB; k++) {
                const float xk = __shfl_sync(0xffffffffu, x[k >> 5], k & 31);
#pragma unroll
                for (int q = 0; q < Q; q++) {
                    const int t = lane + 32 * q;
                    if (t > k) x[q] = fmaf(L[k * PB + t], xk, x[q]);
                }
            }
#pragma unroll
            for (int q = 0; q < Q; q++) {
                row[k0 + lane + 32 * q] = x[q];
                stage[warp * SS + lane + 32 * q] = x[q];
            }
        }
        __syncthreads();
        for (int idx = tid; idx < PB * 8; idx += PT) {
            const int t = idx >> 3, j = idx & 7;
            if (base + j < m) at[(size_t)t * ldat + base + j] = stage[j * SS + t];
        }
        __syncthreads();
    }
}

// One composite permutation per panel (layout: psrc[PB], odst[PB], osrc[PB],
// count at [3 PB]), one warp per panel.
template <int PB>
__global__ void k_piv_desc(const int* __restrict__ ipvt, int n, int* __restrict__ desc) {
    __shared__ int pv[PB], psrc[PB], odst[PB], osrc[PB];
    __shared__ int s_nout;
    const int j = blockIdx.x, k0 = j * PB, kb = min(PB, n - k0), lane = threadIdx.x;
    for (int t = lane; t < kb; t += 32) pv[t] = ipvt[k0 + t];
    __syncwarp();
    build_perm(pv, k0, kb, k0 + kb, psrc, odst, osrc, &s_nout);
    __syncwarp();
    int* d = desc + (size_t)j * 4 * PB;
    for (int t = lane; t < PB; t += 32) {
        d[t] = t < kb ? psrc[t] : k0 + t;
        d[PB + t] = odst[t];
        d[2 * PB + t] = osrc[t];
    }
    if (lane == 0) d[3 * PB] = s_nout;
}

// Between block form (whole panel rows exchanged inside a panel) and the
// reference encoding: storage row kp's multipliers take the interchanges of
// the later steps of its own panel (to block form, in step order) or give
// them back (to the reference encoding, in reverse order).  One thread per
// storage row.
__global__ void k_piv_convert(float* __restrict__ a, int lda, int n, int pb, const int* __restrict__ ipvt,
                              int to_reference) {
    const int kp = blockIdx.x * blockDim.x + threadIdx.x;
    if (kp >= n) return;
    const int kend = min((kp / pb + 1) * pb, n);
    float* row = a + (size_t)kp * lda;
    if (to_reference) {
        for (int k = kend - 1; k > kp; k--) {
            const int p = __ldg(ipvt + k);
            if (p != k) {
                const float t = row[k];
                row[k] = row[p];
                row[p] = t;
            }
        }
    } else {
        for (int k = kp + 1; k < kend; k++) {
            const int p = __ldg(ipvt + k);
            if (p != k) {
                const float t = row[k];
                row[k] = row[p];
                row[p] = t;
            }
        }
    }
}

// acc + sgn * sum_{t < kb} ys[t] * S[k0 + t][i] in ascending t, the column
// read 16 rows at a time with all 16 loads in flight before they are used.
__device__ __forceinline__ float panel_dot(const float* __restrict__ a, int lda, int k0, int kb, int i,
                                           const float* ys, float sgn, float acc) {
    const float* col = a + (size_t)k0 * lda + i;
    for (int t0 = 0; t0 < kb; t0 += 16) {
        float v[16];
#pragma unroll
        for (int j = 0; j < 16; j++) v[j] = t0 + j < kb ? __ldg(col + (size_t)(t0 + j) * lda) : 0.0f;
#pragma unroll
        for (int j = 0; j < 16; j++)
            if (t0 + j < kb) acc = fmaf(sgn * ys[t0 + j], v[j], acc);
    }
    return acc;
}

// Forward and back substitution on block-form factors, nrhs right-hand
// sides (rows of b, solutions overwrite them).  w: 3 n floats (the forward
// values y, two alternating trailing vectors).  Per panel every CTA computes
// the block's values itself (warp 0, from the diagonal block staged in
// shared memory), then updates its share of the positions after (forward) or
// before (backward) the block; one grid barrier per panel.
template <int PB>
__global__ void __launch_bounds__(PT, 1)
    k_piv_gesl(const float* __restrict__ a, int lda, int n, const int* __restrict__ desc, float* b, int ldb, int nrhs,
               float* w, unsigned char* __restrict__ sync) {
    constexpr int Q = PB / 32;
    extern __shared__ float sm[];
    float* D = sm;                                      // D[k * PB + t] = S[k0 + k][k0 + t]
    int* ovr = reinterpret_cast<int*>(D + PB * PB);     // this CTA's positions: override source or -1
    __shared__ float ys[PB];
    __shared__ int od[PB], os[PB];
    __shared__ int ps[PB];
    __shared__ int s_nout;
    unsigned* bar = reinterpret_cast<unsigned*>(sync);
    int* err = reinterpret_cast<int*>(sync + 4);
    const int G = gridDim.x, g = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int np = (n + PB - 1) / PB;
    unsigned nbar = 0;
    float* y = w;
    float* buf0 = w + n;
    float* buf1 = w + 2 * (size_t)n;
    for (int q = 0; q < nrhs; q++) {
        float* bq = b + (size_t)q * ldb;
        // forward: phase j reads cur, writes nxt (positions >= r0) and y (the block)
        for (int j = 0; j < np; j++) {
            const int k0 = j * PB, kb = min(PB, n - k0), r0 = k0 + kb;
            const float* cur = j == 0 ? bq : ((j & 1) ? buf0 : buf1);
            float* nxt = (j & 1) ? buf1 : buf0;
            const int* dj = desc + (size_t)j * 4 * PB;
            for (int t = tid; t < PB; t += PT) ps[t] = dj[t], od[t] = dj[PB + t], os[t] = dj[2 * PB + t];
            if (tid == 0) s_nout = dj[3 * PB];
            for (int idx = tid; idx < kb * kb; idx += PT) {
                const int k = idx / kb, t = idx - k * kb;
                cp_async4(D + k * PB + t, a + (size_t)(k0 + k) * lda + k0 + t);
            }
            cp_async_wait_all();
            const int mrest = n - r0, ch = (mrest + G - 1) / G, i0 = r0 + g * ch, i1 = min(n, i0 + ch);
            for (int i = tid; i < ch; i += PT) ovr[i] = -1;
            __syncthreads();
            const int nout = s_nout;
            for (int e = tid; e < nout; e += PT) {
                const int d = od[e];
                if (d >= i0 && d < i1) ovr[d - i0] = os[e];
            }
            if (warp == 0) {
                float x[Q];
#pragma unroll
                for (int qq = 0; qq < Q; qq++) {
                    const int t = lane + 32 * qq;
                    x[qq] = t < kb ? __ldcg(cur + ps[t]) : 0.0f;
                }
#pragma unroll
                for (int k = 0; k < PB; k++) {
                    const float xk = __shfl_sync(0xffffffffu, x[k >> 5], k & 31);
#pragma unroll
                    for (int qq = 0; qq < Q; qq++) {
                        const int t = lane + 32 * qq;
                        if (t > k && t < kb) x[qq] = fmaf(xk, D[k * PB + t], x[qq]);
                    }
                }
#pragma unroll
                for (int qq = 0; qq < Q; qq++) {
                    const int t = lane + 32 * qq;
                    if (t < kb) {
                        ys[t] = x[qq];
                        if (g == 0) y[k0 + t] = x[qq];
                    }
                }
            }
            __syncthreads();
            for (int i = i0 + tid; i < i1; i += PT) {
                const int o = ovr[i - i0];
                nxt[i] = panel_dot(a, lda, k0, kb, i, ys, 1.0f, __ldcg(cur + (o >= 0 ? o : i)));
            }
            if (!grid_sync(bar, (++nbar) * (unsigned)G, err)) return;
        }
        // backward: x_k = y_k / u_kk; y_t -= x_k u_tk (t < k)
        for (int j = np - 1; j >= 0; j--) {
            const int k0 = j * PB, kb = min(PB, n - k0);
            for (int idx = tid; idx < kb * kb; idx += PT) {
                const int k = idx / kb, t = idx - k * kb;
                cp_async4(D + k * PB + t, a + (size_t)(k0 + k) * lda + k0 + t);
            }
            cp_async_wait_all();
            __syncthreads();
            if (warp == 0) {
                float x[Q];
#pragma unroll
                for (int qq = 0; qq < Q; qq++) {
                    const int t = lane + 32 * qq;
                    x[qq] = t < kb ? __ldcg(y + k0 + t) : 0.0f;
                }
#pragma unroll
                for (int k = PB - 1; k >= 0; k--) {
                    if (k < kb) {
                        const float xk = __shfl_sync(0xffffffffu, x[k >> 5], k & 31) / D[k * PB + k];
                        if (lane == (k & 31)) x[k >> 5] = xk;
#pragma unroll
                        for (int qq = 0; qq < Q; qq++) {
                            const int t = lane + 32 * qq;
                            if (t < k) x[qq] = fmaf(-xk, D[k * PB + t], x[qq]);
                        }
                    }
                }
#pragma unroll
                for (int qq = 0; qq < Q; qq++) {
                    const int t = lane + 32 * qq;
                    if (t < kb) {
                        ys[t] = x[qq];
                        if (g == 0) bq[k0 + t] = x[qq];
                    }
                }
            }
            __syncthreads();
            const int ch = (k0 + G - 1) / G, i0 = g * ch, i1 = min(k0, i0 + ch);
            for (int i = i0 + tid; i < i1; i += PT) y[i] = panel_dot(a, lda, k0, kb, i, ys, -1.0f, __ldcg(y + i));
            if (!grid_sync(bar, (++nbar) * (unsigned)G, err)) return;
        }
    }
}

int g_panel_smem_max = 0;  // dynamic shared memory available to k_piv_panel
int g_gesl_smem_max = 0;

template <int PB>
constexpr size_t rows_smem() {
    return sizeof(float) * ((size_t)PB * PB + 8 * (PB + 4));
}

}  // namespace

int piv_init_attrs() {
    int dev = 0, optin = 0;
    LP_CUDA(cudaGetDevice(&dev));
    LP_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    cudaFuncAttributes fa{};
    LP_CUDA(cudaFuncGetAttributes(&fa, k_piv_panel));
    g_panel_smem_max = optin - (int)fa.sharedSizeBytes;
    LP_CUDA(cudaFuncSetAttribute(k_piv_panel, cudaFuncAttributeMaxDynamicSharedMemorySize, g_panel_smem_max));
    LP_CUDA(cudaFuncSetAttribute(k_piv_rows<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rows_smem<128>()));
    LP_CUDA(cudaFuncSetAttribute(k_piv_rows<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rows_smem<64>()));
    LP_CUDA(cudaFuncGetAttributes(&fa, k_piv_gesl<128>));
    g_gesl_smem_max = optin - (int)fa.sharedSizeBytes;
    LP_CUDA(cudaFuncSetAttribute(k_piv_gesl<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, g_gesl_smem_max));
    LP_CUDA(cudaFuncGetAttributes(&fa, k_piv_gesl<64>));
    LP_CUDA(cudaFuncSetAttribute(k_piv_gesl<64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 optin - (int)fa.sharedSizeBytes));
    return LP_OK;
}

size_t piv_sync_bytes() { return kSyncBytes; }

int piv_panel_width(int n, int sms) {
    const long long rows = (n + sms - 1) / sms;
    return rows * 128 * (long long)sizeof(float) <= g_panel_smem_max ? 128 : 64;
}

// CTAs and rows per CTA of the panel launch for m trailing rows: about 128
// rows per CTA, at most one CTA per SM, the slice within shared memory.
static void panel_grid(int m, int kb, int sms, int* G, int* R) {
    int g = std::min(sms, std::max(1, (m + 127) / 128));
    int r = (m + g - 1) / g;
    while ((long long)r * kb * (long long)sizeof(float) > g_panel_smem_max && g < sms) {
        g = std::min(sms, g * 2);
        r = (m + g - 1) / g;
    }
    *G = g;
    *R = r;
}

int launch_piv_panel(float* a, int lda, int n, int k0, int kb, int* ipvt, unsigned char* sync, unsigned* bar_base,
                     int sms, cudaStream_t st) {
    const int m = n - k0;
    int G = 0, R = 0;
    panel_grid(m, kb, sms, &G, &R);
    const size_t smem = (size_t)kb * R * sizeof(float);
    if (kb > PBMAX || G > GMAX || (long long)smem > g_panel_smem_max)
        return fail(LP_E_INVALID, "pivoting panel: matrix too large for the panel width");
    unsigned base = *bar_base;
    void* args[] = {&a, &lda, &n, &k0, &kb, &R, &ipvt, &sync, &base};
    LP_CUDA(cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(k_piv_panel), dim3(G), dim3(PT), args, smem, st));
    count_launch();
    *bar_base = base + (unsigned)G * (unsigned)kb;
    return LP_OK;
}

int launch_piv_rows(float* a, int lda, int n, int k0, int pb, const int* ipvt, float* at, int ldat, int sms,
                    cudaStream_t st) {
    const int m = n - k0 - pb;
    if (m <= 0) return LP_OK;
    const int grid = std::max(1, std::min(2 * sms, (m + 7) / 8));
    if (pb == 128)
        k_piv_rows<128><<<grid, PT, rows_smem<128>(), st>>>(a, lda, n, k0, ipvt, at, ldat);
    else
        k_piv_rows<64><<<grid, PT, rows_smem<64>(), st>>>(a, lda, n, k0, ipvt, at, ldat);
    count_launch();
    LP_CUDA(cudaGetLastError());
    return LP_OK;
}

int launch_piv_desc(const int* ipvt, int n, int pb, int* desc, cudaStream_t st) {
    const int np = (n + pb - 1) / pb;
    if (pb == 128)
        k_piv_desc<128><<<np, 32, 0, st>>>(ipvt, n, desc);
    else
        k_piv_desc<64><<<np, 32, 0, st>>>(ipvt, n, desc);
    count_launch();
    LP_CUDA(cudaGetLastError());
    return LP_OK;
}

int launch_piv_convert(float* a, int lda, int n, int pb, const int* ipvt, bool to_reference, cudaStream_t st) {
    k_piv_convert<<<(n + 127) / 128, 128, 0, st>>>(a, lda, n, pb, ipvt, to_reference ? 1 : 0);
    count_launch();
    LP_CUDA(cudaGetLastError());
    return LP_OK;
}

int launch_piv_gesl(const float* a, int lda, int n, int pb, const int* desc, float* b, int ldb, int nrhs, float* w,
                    unsigned char* sync, int sms, cudaStream_t st) {
    const int G = std::max(1, std::min(sms, (n + 127) / 128));
    const size_t smem = sizeof(float) * (size_t)pb * pb + sizeof(int) * (size_t)((n + G - 1) / G);
    if ((long long)smem > g_gesl_smem_max) return fail(LP_E_INVALID, "pivoting solve: matrix too large");
    void* args[] = {&a, &lda, &n, &desc, &b, &ldb, &nrhs, &w, &sync};
    const void* fn = pb == 128 ? reinterpret_cast<const void*>(k_piv_gesl<128>)
                               : reinterpret_cast<const void*>(k_piv_gesl<64>);
    LP_CUDA(cudaLaunchCooperativeKernel(fn, dim3(G), dim3(PT), args, smem, st));
    count_launch();
    return LP_OK;
}

}  // namespace lp
