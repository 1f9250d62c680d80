// gesl with inverted diagonal blocks — the substitution of every path that
// solves with FP32 factors (the reference's gesl_ref_nopvt,
// LINPACK/src/host/linpack_data.cpp:199-229).
//
// Storage terms (S[r][c] = a[r*lda + c]), blocked by SB = 128 unknowns:
//   forward  acc_j = b_j + sum_{K<j} y_K^T S[K][j],  y_j = Y_j^T acc_j
//   backward acc_j = y_j + sum_{K>j} s_K^T S[K][j],  s_j = X_j^T acc_j,  x_j = -s_j
// with, for the diagonal block D of tile j,
//   Y = (I - U)^-1             U: D's strict upper storage triangle (the
//                              negated multipliers), by the left recurrence
//                              applied to an identity;
//   X = (diag(D_kk)^-1 - L)^-1 L: D's strict lower storage triangle (the U
//                              factor of M), D_kk = -1/d as stored, by the top
//                              recurrence applied to an identity.
// Within a tile the sequential 128-step chain becomes one 128 x 128
// matrix-vector product over all 256 threads.
//
// Each sweep is ONE persistent launch, one CTA per SM.  A CTA takes tiles in
// ticket order (forward 0, 1, 2, ...; backward from the last tile down) and,
// for its tile j:
//   1. starts streaming the factor blocks S[K][j] of every source tile K
//      (forward K < j, backward K > j) through a cp.async ring of 32-row
//      stages (5 to 7 deep), so a whole source tile and more is in flight;
//   2. inverts its own diagonal block into shared memory (Y or X: no
//      separate launch, no global workspace for the operators) when it
//      would otherwise wait for a source that is not published yet;
//   3. for each source tile waits for its published values (one poll loop
//      over the tile's (value, tag) pairs), then adds its contributions;
//   4. forms acc_j, multiplies by the operator, publishes its own values.
// Published values are 64-bit pairs (tag << 32 | float bits), written with
// relaxed stores and read with relaxed loads: a pair is valid on its own, so a
// consumer needs one L2 round trip (no flag, then data).  The forward sweep
// tags with 1, the backward sweep with 2 into the same array (it is cleared
// before the forward sweep), and the backward sweep reads its input y_j
// there.  A CTA only waits on tiles whose tickets were taken before its own
// by running CTAs, so progress is guaranteed even when not every CTA is
// resident; every wait is bounded nonetheless (250 ms by %globaltimer), and a
// CTA that gives up records the error, writes NaN for its tile and still
// publishes it, so no other CTA waits on it.  The summation order is fixed
// (sources in order, rows in order, a fixed two-way reduction), so results
// are deterministic.
#include <algorithm>

#include "gesl_common.cuh"

namespace lp {
namespace {

using namespace gesl;

constexpr int ICH = 32;        // chunk of the inverse recurrences
constexpr int RS = 32;         // factor rows per ring stage
constexpr int SPT = SB / RS;   // stages per source tile
constexpr int STAGE_FLOATS = RS * SB;
constexpr int OPL = SB + 1;              // row stride of the forward operator (its rows are recurrence chains)
constexpr int kOpFloats = SB * OPL;
constexpr int kScratch = 2 * 32 * SB;     // two chunks of the diagonal block (2 x 32 x 128), later the reductions
constexpr unsigned long long kWaitLimitNs = 250ull * 1000 * 1000;  // a bounded wait gives up after 250 ms
constexpr unsigned kTagFwd = 1, kTagBwd = 2, kTagNever = 0x7fff0000u;

__device__ __forceinline__ void cp_async16(float* smem, const float* gmem, int src_bytes) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Rows [r0, r0 + rows) x columns [k0, k0 + cols) of the diagonal block d
// (cols a multiple of 4; entries outside the kb x kb block read as 0) into
// buf (row stride cols) by 16-byte asynchronous copies, committed as one group.
__device__ __forceinline__ void load_block(const float* __restrict__ d, int lda, int kb, int r0, int rows, int k0,
                                           int cols, float* buf) {
    const int q4 = cols / 4;
    for (int idx = threadIdx.x; idx < rows * q4; idx += GT) {
        const int rr = idx / q4, cc = (idx - rr * q4) * 4;
        const int r = r0 + rr, c = k0 + cc, rem = kb - c;
        const int bytes = (r < kb && rem > 0) ? (rem >= 4 ? 16 : 4 * rem) : 0;
        cp_async16(buf + rr * cols + cc, bytes > 0 ? d + (size_t)r * lda + c : d, bytes);
    }
    cp_commit();
}

// X = (diag(D_kk)^-1 - L)^-1 for the diagonal block d (kb valid rows and
// columns; the rest of the 128 x 128 block is the identity) into op (row
// stride SB): the top recurrence applied to the identity, every column at
// once (columns are independent).  Per 32-row chunk of D (double-buffered
// asynchronous copies, the next chunk in flight): one thread per column runs
// the chunk's 32-step recurrence in registers, then all threads apply the
// chunk to the rows below it.  scr: 2 x 128 x 32 floats.  Waiting for its
// copies also completes any copies the calling thread issued before.
__device__ void inv_top_full(const float* __restrict__ d, int lda, int kb, float* scr, float* op) {
    const int tid = threadIdx.x;
    for (int idx = tid; idx < SB * SB; idx += GT) op[idx] = (idx / SB == idx % SB) ? 1.0f : 0.0f;
    load_block(d, lda, kb, 0, SB, 0, ICH, scr);
    for (int r0 = 0, ch = 0; r0 < SB; r0 += ICH, ch++) {
        const int nr = SB - r0;
        float* dch = scr + (ch & 1) * (SB * ICH);  // rows r0.. of columns [r0, r0 + 32), SB x ICH
        if (r0 + ICH < SB) {
            load_block(d, lda, kb, r0 + ICH, nr - ICH, r0 + ICH, ICH, scr + ((ch + 1) & 1) * (SB * ICH));
            cp_wait<1>();
        } else {
            cp_wait<0>();
        }
        __syncthreads();
        if (kb < SB)  // the identity outside the kb x kb block: diagonal entries at and after kb
            for (int rr = tid; rr < min(nr, ICH); rr += GT)
                if (r0 + rr >= kb) dch[rr * ICH + rr] = 1.0f;
        __syncthreads();
        if (tid < SB) {
            float x[ICH];
#pragma unroll
            for (int k = 0; k < ICH; k++) x[k] = op[(r0 + k) * SB + tid];
#pragma unroll
            for (int k = 0; k < ICH; k++) {
                const float xk = x[k] * dch[k * ICH + k];
                x[k] = xk;
#pragma unroll
                for (int j = k + 1; j < ICH; j++) x[j] = fmaf(xk, dch[j * ICH + k], x[j]);
            }
#pragma unroll
            for (int k = 0; k < ICH; k++) op[(r0 + k) * SB + tid] = x[k];
        }
        __syncthreads();
        if (nr > ICH) {
            const int c = tid & (SB - 1), g = tid >> 7;
            float x[ICH];
#pragma unroll
            for (int k = 0; k < ICH; k++) x[k] = op[(r0 + k) * SB + c];
            // four rows at a time: independent FMA chains interleave
#pragma unroll 4
            for (int r = r0 + ICH + g; r < SB; r += GT / SB) {
                float acc = op[r * SB + c];
                const float* drow = dch + (r - r0) * ICH;
#pragma unroll
                for (int k = 0; k < ICH; k++) acc = fmaf(x[k], drow[k], acc);
                op[r * SB + c] = acc;
            }
        }
        __syncthreads();
    }
}

// Y = (I - U)^-1 for the diagonal block d into op (row stride OPL): the left
// recurrence applied to the identity, every row at once (rows are
// independent).  Per 32-column chunk of D (double-buffered asynchronous
// copies): one thread per row runs the chunk's recurrence in registers, then
// all threads apply the chunk to the columns after it, one (row, column)
// element per thread at a time.  scr: 2 x 32 x 128 floats.
__device__ void inv_left_full(const float* __restrict__ d, int lda, int kb, float* scr, float* op) {
    const int tid = threadIdx.x;
    for (int idx = tid; idx < SB * SB; idx += GT) {
        const int rr = idx / SB, c = idx - rr * SB;
        op[rr * OPL + c] = (rr == c) ? 1.0f : 0.0f;
    }
    load_block(d, lda, kb, 0, ICH, 0, SB, scr);
    for (int c0 = 0, ch = 0; c0 < SB; c0 += ICH, ch++) {
        const int nc = SB - c0;
        float* dch = scr + (ch & 1) * (ICH * SB);  // rows [c0, c0 + 32) of columns c0.., ICH x nc
        if (c0 + ICH < SB) {
            load_block(d, lda, kb, c0 + ICH, ICH, c0 + ICH, nc - ICH, scr + ((ch + 1) & 1) * (ICH * SB));
            cp_wait<1>();
        } else {
            cp_wait<0>();
        }
        __syncthreads();
        if (tid < SB) {
            float x[ICH];
            float* row = op + tid * OPL + c0;
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
        const int rest = nc - ICH;
        // four elements at a time: independent FMA chains interleave
#pragma unroll 4
        for (int idx = tid; idx < rest * SB; idx += GT) {
            const int rr = idx / rest, ci = ICH + (idx - rr * rest);
            const float* row = op + rr * OPL + c0;
            float acc = row[ci];
#pragma unroll
            for (int k = 0; k < ICH; k++) acc = fmaf(row[k], dch[k * nc + ci], acc);
            op[rr * OPL + c0 + ci] = acc;
        }
        __syncthreads();
    }
}

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ unsigned long long ld_pair(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_pair(unsigned long long* p, unsigned tag, float v) {
    const unsigned long long w = ((unsigned long long)tag << 32) | (unsigned long long)__float_as_uint(v);
    asm volatile("st.relaxed.gpu.global.b64 [%0], %1;" ::"l"(p), "l"(w) : "memory");
}

// Ring depth per right-hand-side width: as deep as shared memory allows
// (227 KB per CTA) beside the operator, the scratch and the staged values.
template <int NR>
__host__ __device__ constexpr int stages() {
    return NR <= 4 ? 7 : 6;
}

// Published values of one source tile, prefetched into registers: thread t
// owns entries idx = t + m * GT (q = idx / 128, i = idx % 128) of the tile's
// NR x 128 block.
template <int NR>
struct Pending {
    static constexpr int M = (NR * SB + GT - 1) / GT;
    unsigned long long w[M];
};

// Issue the relaxed loads of source tile K's pairs (entries this launch does
// not need read as valid zeros).
template <int NR>
__device__ __forceinline__ void prefetch_tile(Pending<NR>& pd, const unsigned long long* __restrict__ pub, int K,
                                              int g, int kbK, unsigned tag) {
#pragma unroll
    for (int m = 0; m < Pending<NR>::M; m++) {
        const int idx = threadIdx.x + m * GT;
        const int q = idx / SB, i = idx - q * SB;
        pd.w[m] = (idx < NR * SB && q < g && i < kbK) ? ld_pair(pub + ((size_t)K * g + q) * SB + i)
                                                      : ((unsigned long long)tag << 32);
    }
}

// true when every prefetched entry of the calling thread carries `tag`.
template <int NR>
__device__ __forceinline__ bool all_tagged(const Pending<NR>& pd, unsigned tag) {
    bool ok = true;
#pragma unroll
    for (int m = 0; m < Pending<NR>::M; m++) ok = ok && (unsigned)(pd.w[m] >> 32) == tag;
    return ok;
}

// Complete the prefetched values of source tile K: entries not yet carrying
// `tag` are polled (bounded by kWaitLimitNs; another CTA's error ends the
// wait too); the values go to ybuf[i*NR + q].  false (CTA-uniform): a wait
// gave up (here or in another CTA).
template <int NR>
__device__ bool resolve_tile(Pending<NR>& pd, const unsigned long long* __restrict__ pub, int K, int g,
                             unsigned tag, float* ybuf, int* err) {
    bool ok = true;
#pragma unroll
    for (int m = 0; m < Pending<NR>::M; m++) {
        const int idx = threadIdx.x + m * GT;
        if (idx >= NR * SB) continue;
        const int q = idx / SB, i = idx - q * SB;
        unsigned long long w = pd.w[m];
        if ((unsigned)(w >> 32) != tag && ok) {
            const unsigned long long* src = pub + ((size_t)K * g + q) * SB + i;
            const unsigned long long t0 = global_ns();
            for (;;) {
                __nanosleep(32);
                w = ld_pair(src);
                if ((unsigned)(w >> 32) == tag) break;
                if (*(volatile int*)err != 0) {
                    ok = false;
                    break;
                }
                if (global_ns() - t0 > kWaitLimitNs) {
                    atomicExch(err, 1);
                    ok = false;
                    break;
                }
            }
        }
        ybuf[i * NR + q] = __uint_as_float((unsigned)w);
    }
    return __syncthreads_and(ok) != 0;
}

// One sweep (see the file comment).  FWD: in = b (rows of ldb), out: the
// published y.  Backward: in = the forward sweep's published y, out: x = -s
// into xout (rows of ldb) and the published s.  g = right-hand sides of this
// launch (<= NR).  stall (tests only): the forward sweep's second tile waits
// for a tag that is never written, so its bounded wait runs out.
//
// Per source tile the CTA completes the values it prefetched one tile ahead
// (already published sources cost no round trip); the tile's operator is
// computed at the first source that is not yet published (the CTA would wait
// anyway), or at the end; the tile's input is staged into shared memory by
// cp.async with the first ring stage.
template <int NR, bool FWD>
__global__ void __launch_bounds__(GT, 1)
    k_gesl_sweep(const float* __restrict__ a, int lda, int n, const float* __restrict__ bin, float* __restrict__ xout,
                 int ldb, unsigned long long* __restrict__ pub, int g, int* __restrict__ ticket,
                 int* __restrict__ err, int stall) {
    constexpr int STG = stages<NR>();
    extern __shared__ __align__(16) float smem[];
    float* op = smem;                         // 128 x 128 operator of the tile (Y, row stride OPL; or X)
    float* scr = op + kOpFloats;              // a chunk of the diagonal block, later the reductions
    float* ring = scr + kScratch;             // STG x 32 x 128 factor rows
    float* ybuf = ring + STG * STAGE_FLOATS;  // 128 x NR published values of one source tile
    float* inb = ybuf + NR * SB;              // NR x 128 input of the tile (b_j or y_j)
    __shared__ int s_tile;
    const int tid = threadIdx.x;
    const int nblk = (n + SB - 1) / SB;
    const unsigned tag = FWD ? kTagFwd : kTagBwd;
    const int c = tid & (SB - 1), h = tid >> 7;  // compute mapping: column c, rows 16h..16h+15 of a stage
    for (;;) {
        __syncthreads();  // the previous tile's shared data is consumed
        if (tid == 0) s_tile = atomicAdd(ticket, 1);
        __syncthreads();
        const int t = s_tile;
        if (t >= nblk) break;
        const int j = FWD ? t : nblk - 1 - t;
        const int c0 = j * SB, kb = min(SB, n - c0);
        const int nsrc = FWD ? j : nblk - 1 - j;
        const int total = nsrc * SPT;
        // stage s: rows [32 (s % SPT), +32) of source tile K(s / SPT), columns [c0, c0 + 128)
        auto issue = [&](int s) {
            const int si = s / SPT, sr = s - si * SPT;
            const int K = FWD ? si : nblk - 1 - si;
            const int r0 = K * SB + sr * RS;
            float* dst = ring + (s % STG) * STAGE_FLOATS;
#pragma unroll
            for (int it = 0; it < STAGE_FLOATS / 4 / GT; it++) {
                const int idx = tid + it * GT;
                const int r = idx >> 5, cc = (idx & 31) * 4;
                const int rem = n - (c0 + cc);  // columns left in the row: a ragged last float4 is zero-filled
                const int bytes = (r0 + r < n && rem > 0) ? (rem >= 4 ? 16 : 4 * rem) : 0;
                const float* src = bytes > 0 ? a + (size_t)(r0 + r) * lda + c0 + cc : a;
                cp_async16(dst + r * SB + cc, src, bytes);
            }
        };
        // the tile's input: b_j (forward) or the forward sweep's y_j (the low word of its pairs)
        for (int idx = tid; idx < NR * SB; idx += GT) {
            const int q = idx / SB, i = idx - q * SB;
            if (q < g && i < kb) {
                const float* src = FWD ? bin + (size_t)q * ldb + c0 + i
                                       : reinterpret_cast<const float*>(pub + ((size_t)j * g + q) * SB + i);
                cp_async4(inb + idx, src);
            } else {
                inb[idx] = 0.0f;
            }
        }
#pragma unroll
        for (int s = 0; s < STG - 1; s++) {
            if (s < total) issue(s);
            cp_commit();
        }
        const float* d = a + (size_t)c0 * lda + c0;
        auto invert = [&]() {
            if (FWD)
                inv_left_full(d, lda, kb, scr, op);
            else
                inv_top_full(d, lda, kb, scr, op);
        };
        bool inverted = false;
        // PS partial sums per right-hand side (rows round-robin) so that one right-hand side's
        // FMAs form independent chains; combined in a fixed order at the end of the tile
        constexpr int PS = NR == 1 ? 4 : 1;
        float p[NR * PS];
#pragma unroll
        for (int q = 0; q < NR * PS; q++) p[q] = 0.0f;
        bool ok = *(volatile int*)err == 0;
        ok = __syncthreads_and(ok) != 0;
        Pending<NR> pd;
        if (nsrc > 0 && ok) {
            const int K0 = FWD ? 0 : nblk - 1;
            const bool never = FWD && stall != 0 && j == 1;
            prefetch_tile<NR>(pd, pub, K0, g, min(SB, n - K0 * SB), never ? kTagNever : tag);
        }
        // contributions of ring stage s (rows sr*32.. of its source tile) to this thread's sums
        auto consume = [&](int s, int sr) {
            const float* stg = ring + (s % STG) * STAGE_FLOATS;
#pragma unroll
            for (int r = 0; r < RS / 2; r++) {
                const int row = h * (RS / 2) + r;
                const float v = stg[row * SB + c];
                const float* y = ybuf + (sr * RS + row) * NR;
                if constexpr (NR % 4 == 0) {
#pragma unroll
                    for (int q = 0; q < NR; q += 4) {
                        const float4 y4 = *reinterpret_cast<const float4*>(y + q);
                        p[q] = fmaf(y4.x, v, p[q]);
                        p[q + 1] = fmaf(y4.y, v, p[q + 1]);
                        p[q + 2] = fmaf(y4.z, v, p[q + 2]);
                        p[q + 3] = fmaf(y4.w, v, p[q + 3]);
                    }
                } else {
#pragma unroll
                    for (int q = 0; q < NR; q++) p[q * PS + r % PS] = fmaf(y[q], v, p[q * PS + r % PS]);
                }
            }
        };
        for (int s = 0; s < total && ok; s++) {
            const int si = s / SPT, sr = s - si * SPT;
            const int K = FWD ? si : nblk - 1 - si;
            if (sr == 0) {
                const unsigned want = (FWD && stall != 0 && j == 1 && K == 0) ? kTagNever : tag;
                __syncthreads();  // every thread is done with the previous source's values
                if (!inverted && __syncthreads_and(all_tagged<NR>(pd, want)) == 0) {
                    invert();  // this source is not published yet: the CTA would wait anyway
                    inverted = true;
                }
                ok = resolve_tile<NR>(pd, pub, K, g, want, ybuf, err);
                if (!ok) break;
                if (si + 1 < nsrc) {
                    const int K1 = FWD ? si + 1 : nblk - 2 - si;
                    prefetch_tile<NR>(pd, pub, K1, g, min(SB, n - K1 * SB), tag);
                } else {
                    // the last source (on the chain's critical path): all of its stages are in
                    // the ring already (STG > SPT), so one wait and one barrier cover them
                    cp_wait<0>();
                    __syncthreads();
#pragma unroll
                    for (int r4 = 0; r4 < SPT; r4++) consume(s + r4, r4);
                    break;
                }
            }
            cp_wait<STG - 2>();
            __syncthreads();
            if (s + STG - 1 < total) issue(s + STG - 1);
            cp_commit();
            consume(s, sr);
        }
        cp_wait<0>();
        if (!inverted) invert();
        // acc = in + the two half sums; res = operator^T acc; published from the two halves of the product
        float* red = scr;                 // NR x 128: the upper half's sums
        float* acc = red + NR * SB;       // NR x 128
        float* part = acc + NR * SB;      // 2 x NR x 128
        if constexpr (PS > 1) {
#pragma unroll
            for (int q = 0; q < NR; q++) p[q * PS] = (p[q * PS] + p[q * PS + 1]) + (p[q * PS + 2] + p[q * PS + 3]);
        }
        if (h == 1) {
#pragma unroll
            for (int q = 0; q < NR; q++) red[q * SB + c] = p[q * PS];
        }
        ok = __syncthreads_and(ok) != 0;
        if (h == 0) {
#pragma unroll
            for (int q = 0; q < NR; q++)
                acc[q * SB + c] = (q < g && c < kb) ? inb[q * SB + c] + p[q * PS] + red[q * SB + c] : 0.0f;
        }
        __syncthreads();
        {
            const int i = tid & (SB - 1), hh = tid >> 7;
            float pr[NR * PS];
#pragma unroll
            for (int r = 0; r < NR * PS; r++) pr[r] = 0.0f;
#pragma unroll 16
            for (int kk = 0; kk < SB / 2; kk++) {
                const int k = hh * (SB / 2) + kk;
                const float m = op[k * (FWD ? OPL : SB) + i];
#pragma unroll
                for (int r = 0; r < NR; r++) pr[r * PS + kk % PS] = fmaf(m, acc[r * SB + k], pr[r * PS + kk % PS]);
            }
#pragma unroll
            for (int r = 0; r < NR; r++) {
                float v = pr[r * PS];
                if constexpr (PS > 1) v = (pr[r * PS] + pr[r * PS + 1]) + (pr[r * PS + 2] + pr[r * PS + 3]);
                part[(hh * NR + r) * SB + i] = v;
            }
        }
        __syncthreads();
        for (int idx = tid; idx < NR * SB; idx += GT) {
            const int q = idx / SB, i = idx - q * SB;
            if (q < g && i < kb) {
                const float v = ok ? part[q * SB + i] + part[(NR + q) * SB + i]
                                   : __int_as_float(0x7fc00000);  // NaN marks an aborted solve
                if (!FWD) xout[(size_t)q * ldb + c0 + i] = -v;
                st_pair(pub + ((size_t)j * g + q) * SB + i, tag, v);
            }
        }
    }
}

template <int NR>
constexpr size_t sweep_smem() {
    return sizeof(float) *
           ((size_t)kOpFloats + kScratch + (size_t)stages<NR>() * STAGE_FLOATS + 2 * (size_t)NR * SB);
}
// a chunk of the diagonal block and the reductions fit in the scratch
static_assert(2 * SB * ICH <= kScratch && 4 * 16 * SB <= kScratch, "scratch");
static_assert(sweep_smem<1>() <= 227 * 1024 && sweep_smem<4>() <= 227 * 1024 && sweep_smem<16>() <= 227 * 1024,
              "sweep shared memory");

template <int NR>
int sweeps(const float* a, int lda, int n, float* b, int ldb, int g, unsigned long long* pub, int* tickets, int* err,
           bool stall, int sms, cudaStream_t st) {
    const int nblk = (n + SB - 1) / SB;
    const int grid = std::min(nblk, sms);
    LP_CUDA(cudaMemsetAsync(tickets, 0, 2 * sizeof(int), st));
    LP_CUDA(cudaMemsetAsync(pub, 0, sizeof(unsigned long long) * (size_t)nblk * SB * g, st));
    k_gesl_sweep<NR, true><<<grid, GT, sweep_smem<NR>(), st>>>(a, lda, n, b, nullptr, ldb, pub, g, tickets, err,
                                                               stall ? 1 : 0);
    k_gesl_sweep<NR, false><<<grid, GT, sweep_smem<NR>(), st>>>(a, lda, n, nullptr, b, ldb, pub, g, tickets + 1, err,
                                                                0);
    count_launch(2);
    LP_CUDA(cudaGetLastError());
    return LP_OK;
}

template <int NR>
int sweep_attrs() {
    LP_CUDA(cudaFuncSetAttribute(k_gesl_sweep<NR, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)sweep_smem<NR>()));
    LP_CUDA(cudaFuncSetAttribute(k_gesl_sweep<NR, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)sweep_smem<NR>()));
    return LP_OK;
}

}  // namespace

int gesl_inv_init_attrs() {
    LP_CHECK(sweep_attrs<1>());
    LP_CHECK(sweep_attrs<4>());
    LP_CHECK(sweep_attrs<16>());
    return LP_OK;
}

// Published-value pairs of one solve: ceil(n / 128) * 128 * min(nrhs, 16).
size_t gesl_pub_pairs(int n, int nrhs) {
    const size_t g = nrhs < 16 ? nrhs : 16;
    return (size_t)((n + SB - 1) / SB) * SB * g;
}

// Forward + back substitution for nrhs rows of b (overwritten by x), in
// chunks of at most 16 right-hand sides.  pub: gesl_pub_pairs(n, nrhs) pairs;
// tickets: 2 ints; err: an error word the caller zeroes and reads (set when a
// bounded wait gave up; that tile is written as NaN).  pub and tickets are
// cleared here before every chunk.  stall (tests only): see k_gesl_sweep.
int launch_gesl_inv(const float* a, int lda, int n, float* b, int ldb, int nrhs, unsigned long long* pub,
                    int* tickets, int* err, bool stall, cudaStream_t st) {
    if (n <= 0 || nrhs <= 0) return LP_OK;
    if (lda % 4 != 0 || !aligned16(a)) return fail(LP_E_INVALID, "gesl: factors need lda % 4 == 0, 16-byte aligned");
    int dev = 0, sms = 0;
    LP_CUDA(cudaGetDevice(&dev));
    LP_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    for (int r0 = 0; r0 < nrhs; r0 += 16) {
        const int g = (nrhs - r0) < 16 ? (nrhs - r0) : 16;
        float* bb = b + (size_t)r0 * ldb;
        const bool stall_here = stall && r0 == 0;
        if (g == 1)
            LP_CHECK(sweeps<1>(a, lda, n, bb, ldb, g, pub, tickets, err, stall_here, sms, st));
        else if (g <= 4)
            LP_CHECK(sweeps<4>(a, lda, n, bb, ldb, g, pub, tickets, err, stall_here, sms, st));
        else
            LP_CHECK(sweeps<16>(a, lda, n, bb, ldb, g, pub, tickets, err, stall_here, sms, st));
    }
    return LP_OK;
}

}  // namespace lp
