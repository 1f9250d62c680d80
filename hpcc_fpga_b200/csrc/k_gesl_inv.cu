// gesl with inverted diagonal blocks — the substitution of every path that
// solves with FP32 factors (the reference's gesl_ref_nopvt,
// LINPACK/src/host/linpack_data.cpp:199-229).
//
// Storage terms (S[r][c] = a[r*lda + c]), blocked by SB = 128 unknowns:
//   forward  acc_j = b_j + sum_{K<j} y_K^T S[K][j],  y_j = Y_j^T acc_j
//   backward acc_j = y_j + sum_{K>j} s_K^T S[K][j],  s_j = X_j^T acc_j,  x_j = -s_j
// with, for the diagonal block D of tile j,
//   Y = (I - U)^-1             U: D's strict upper storage triangle (the
//                              negated multipliers);
//   X = (diag(D_kk)^-1 - L)^-1 L: D's strict lower storage triangle (the U
//                              factor of M), D_kk = -1/d as stored.
// Within a tile the sequential 128-step chain becomes one 128 x 128
// matrix-vector product.  The operators are built blockwise in shared memory:
// the four 32 x 32 diagonal blocks by one warp each (a lane per column, the
// 32-step recurrence in registers), then the blocks beside the diagonal by
// products, for upper T = [A B; 0 C]: T^-1 = [A^-1, -A^-1 B C^-1; 0, C^-1]
// (lower alike), first for the 32-blocks of each 64 x 64 half, then for the
// 64 x 64 block.
//
// Each sweep is ONE persistent launch, one CTA per SM, taking work items in
// ticket order.  In sweep order (forward: tiles 0, 1, ...; backward: from the
// last tile down) tile t has the sources u = 0 .. t-1.  With a chunk size Q
// (0: no chunks), the sources [0, M Q), M = floor((t - 1) / Q), form M chunk
// items of Q sources that each publish the partial sum of their sources; the
// tile's finisher item takes the remaining sources [M Q, t), adds the chunks'
// sums in chunk order, builds the tile's operator and publishes the tile's
// values.  Long source ranges are thus streamed by several SMs at once
// instead of one.  Items are numbered tile by tile (tile t's chunks, then its
// finisher), and every item waits only on items with lower numbers, whose
// tickets were taken earlier by running CTAs: progress is guaranteed even when
// not every CTA is resident.  Every wait is bounded nonetheless (250 ms by
// %globaltimer); a CTA that gives up records the error, writes NaN for its
// item and still publishes it, so no other CTA waits on it.
//
// Per item the CTA streams the factor blocks S[K][j] of its sources through a
// cp.async ring of nine 32-row stages and, per source, completes the source's
// published values (prefetched one source ahead: already published sources
// cost no round trip) before adding its contributions.  A finisher first
// builds its operator (the diagonal block's pieces use the ring's space
// meanwhile), then streams; the ring holds more than two source tiles, so the
// last source's stages are in flight before the one before it is consumed.
// The finisher keeps its last source's four stages in the ring, forms
// everything else first (the input, the chunks' sums, its other sources), and
// only then waits for the last source, so a step of the tile chain costs one
// 128 x 128 product for the last source and one for the operator.
//
// Published values are 64-bit pairs (tag << 32 | float bits), written with
// relaxed stores and read with relaxed loads: a pair is valid on its own, so a
// consumer needs one L2 round trip (no flag, then data).  The forward sweep
// tags with 1, the backward sweep with 2 into the same array (cleared before
// the forward sweep); the backward sweep reads its input y_j there.  The
// summation order is fixed (sources in order, rows in order, chunks in order,
// fixed two-way reductions), so results are deterministic whichever CTA runs
// an item.
#include <algorithm>

#include "gesl_common.cuh"

namespace lp {
namespace {

using namespace gesl;

constexpr int RS = 32;         // factor rows per ring stage
constexpr int SPT = SB / RS;   // stages per source tile
constexpr int STAGE_FLOATS = RS * SB;
constexpr int LDY = SB + 4;    // row stride of the operator
constexpr int kOpFloats = SB * LDY;
// Pieces of the diagonal block (row strides 36 and 68 keep the products free
// of bank conflicts): the four 32 x 32 diagonal blocks, the two 32 x 32 blocks
// beside the diagonal inside each 64 x 64 half, and the 64 x 64 block joining
// the halves.  The region is reused for the products' temporaries and, once
// the operator is built, for the tile's sums.
constexpr int L32 = 36, L64 = 68;
constexpr int kMidOff = 4 * 32 * L32;
constexpr int kTopOff = kMidOff + 2 * 32 * L32;
constexpr int kScrFloats = kTopOff + 64 * L64;
constexpr int kPieceVecs = (4 * 32 * 32 + 2 * 32 * 32 + 64 * 64) / 4;  // 16-byte vectors of the pieces
constexpr unsigned long long kWaitLimitNs = 250ull * 1000 * 1000;     // a bounded wait gives up after 250 ms
constexpr unsigned kTagFwd = 1, kTagBwd = 2, kTagNever = 0x7fff0000u;
static_assert(kPieceVecs % GT == 0, "piece loads");

__device__ __forceinline__ void cp_async16(float* smem, const float* gmem, int src_bytes) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Work items of one sweep: chunk items of tile t (t >= 1) and the number of
// items before tile t (the finishers of the tiles before it plus their chunks).
__host__ __device__ __forceinline__ int chunks_of(int t, int q) { return (q > 0 && t >= 1) ? (t - 1) / q : 0; }
__host__ __device__ __forceinline__ long long chunks_before(int t, int q) {
    if (q <= 0 || t <= 1) return 0;
    const long long v = t - 1, a = v / q, b = v - a * q;  // sum_{w < v} floor(w / q)
    return q * a * (a - 1) / 2 + a * b;
}
__host__ __device__ __forceinline__ long long items_before(int t, int q) { return t + chunks_before(t, q); }

// D[r][c .. c+3] with the identity outside the kb x kb block.
__device__ __forceinline__ float4 load4_block(const float* __restrict__ d, int lda, int kb, int r, int c) {
    if (r < kb && c + 3 < kb) return *reinterpret_cast<const float4*>(d + (size_t)r * lda + c);
    float v[4];
#pragma unroll
    for (int e = 0; e < 4; e++) {
        const int cc = c + e;
        v[e] = (r < kb && cc < kb) ? d[(size_t)r * lda + cc] : (r == cc ? 1.0f : 0.0f);
    }
    return make_float4(v[0], v[1], v[2], v[3]);
}

// The pieces of the diagonal block d that the operator needs, into scr:
// forward the upper ones (D01, D23 beside the diagonal, D[0:64][64:128]),
// backward the lower ones (D10, D32, D[64:128][0:64]).
template <bool FWD>
__device__ void load_pieces(const float* __restrict__ d, int lda, int kb, float* scr) {
    constexpr int NV = kPieceVecs / GT;
    float4 v[NV];
    int dst[NV];
#pragma unroll
    for (int it = 0; it < NV; it++) {
        const int idx = threadIdx.x + it * GT;
        int r, c, o;
        if (idx < 1024) {  // diagonal blocks
            const int b = idx >> 8, rr = (idx >> 3) & 31, cq = (idx & 7) * 4;
            r = 32 * b + rr;
            c = 32 * b + cq;
            o = b * 32 * L32 + rr * L32 + cq;
        } else if (idx < 1536) {  // beside the diagonal inside each half
            const int i2 = idx - 1024, p = i2 >> 8, rr = (i2 >> 3) & 31, cq = (i2 & 7) * 4;
            r = FWD ? 64 * p + rr : 64 * p + 32 + rr;
            c = FWD ? 64 * p + 32 + cq : 64 * p + cq;
            o = kMidOff + p * 32 * L32 + rr * L32 + cq;
        } else {  // joining the halves
            const int i3 = idx - 1536, rr = i3 >> 4, cq = (i3 & 15) * 4;
            r = FWD ? rr : 64 + rr;
            c = FWD ? 64 + cq : cq;
            o = kTopOff + rr * L64 + cq;
        }
        v[it] = load4_block(d, lda, kb, r, c);
        dst[it] = o;
    }
#pragma unroll
    for (int it = 0; it < NV; it++) *reinterpret_cast<float4*>(scr + dst[it]) = v[it];
}

// C = A B for two independent 32 x 32 products (threads 0-127 and 128-255,
// the caller passes each half its own operands): 2 x 4 outputs per thread.
__device__ __forceinline__ void mm32(const float* A, int lda, const float* B, int ldb, float* C, int ldc) {
    const int t = threadIdx.x & 127, r = (t >> 3) * 2, cb = (t & 7) * 4;
    float acc[2][4];
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = 0.0f;
#pragma unroll
    for (int k = 0; k < 32; k += 4) {
        float4 av[2], bv[4];
#pragma unroll
        for (int i = 0; i < 2; i++) av[i] = *reinterpret_cast<const float4*>(A + (r + i) * lda + k);
#pragma unroll
        for (int kk = 0; kk < 4; kk++) bv[kk] = *reinterpret_cast<const float4*>(B + (k + kk) * ldb + cb);
#pragma unroll
        for (int i = 0; i < 2; i++) {
            const float a4[4] = {av[i].x, av[i].y, av[i].z, av[i].w};
#pragma unroll
            for (int kk = 0; kk < 4; kk++) {
                acc[i][0] = fmaf(a4[kk], bv[kk].x, acc[i][0]);
                acc[i][1] = fmaf(a4[kk], bv[kk].y, acc[i][1]);
                acc[i][2] = fmaf(a4[kk], bv[kk].z, acc[i][2]);
                acc[i][3] = fmaf(a4[kk], bv[kk].w, acc[i][3]);
            }
        }
    }
#pragma unroll
    for (int i = 0; i < 2; i++)
        *reinterpret_cast<float4*>(C + (r + i) * ldc + cb) = make_float4(acc[i][0], acc[i][1], acc[i][2], acc[i][3]);
}

// C = A B, 64 x 64 over all 256 threads: 4 x 4 outputs per thread.
__device__ __forceinline__ void mm64(const float* A, int lda, const float* B, int ldb, float* C, int ldc) {
    const int r = (threadIdx.x >> 4) * 4, cb = (threadIdx.x & 15) * 4;
    float acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = 0.0f;
#pragma unroll 4
    for (int k = 0; k < 64; k += 4) {
        float4 av[4], bv[4];
#pragma unroll
        for (int i = 0; i < 4; i++) av[i] = *reinterpret_cast<const float4*>(A + (r + i) * lda + k);
#pragma unroll
        for (int kk = 0; kk < 4; kk++) bv[kk] = *reinterpret_cast<const float4*>(B + (k + kk) * ldb + cb);
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const float a4[4] = {av[i].x, av[i].y, av[i].z, av[i].w};
#pragma unroll
            for (int kk = 0; kk < 4; kk++) {
                acc[i][0] = fmaf(a4[kk], bv[kk].x, acc[i][0]);
                acc[i][1] = fmaf(a4[kk], bv[kk].y, acc[i][1]);
                acc[i][2] = fmaf(a4[kk], bv[kk].z, acc[i][2]);
                acc[i][3] = fmaf(a4[kk], bv[kk].w, acc[i][3]);
            }
        }
    }
#pragma unroll
    for (int i = 0; i < 4; i++)
        *reinterpret_cast<float4*>(C + (r + i) * ldc + cb) = make_float4(acc[i][0], acc[i][1], acc[i][2], acc[i][3]);
}

// The tile's operator (Y forward, X backward; row stride LDY) from the pieces
// in scr (consumed).  Ends with a barrier.
template <bool FWD>
__device__ void build_operator(float* scr, float* op) {
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    if (w < 4) {  // the diagonal 32 x 32 blocks: warp w inverts block w, lane = column
        const float* db = scr + w * 32 * L32;
        float x[32];
#pragma unroll
        for (int r = 0; r < 32; r++) x[r] = r == lane ? 1.0f : 0.0f;
        if (FWD) {  // (I - U) x = e_lane, from the last row up
#pragma unroll
            for (int k = 31; k > 0; k--) {
                const float xk = x[k];
#pragma unroll
                for (int r = 0; r < k; r++) x[r] = fmaf(db[r * L32 + k], xk, x[r]);
            }
        } else {  // (diag(D_kk)^-1 - L) x = e_lane, from the first row down
#pragma unroll
            for (int k = 0; k < 32; k++) {
                const float xk = db[k * L32 + k] * x[k];
                x[k] = xk;
#pragma unroll
                for (int r = k + 1; r < 32; r++) x[r] = fmaf(db[r * L32 + k], xk, x[r]);
            }
        }
        float* yb = op + (32 * w) * LDY + 32 * w + lane;
#pragma unroll
        for (int r = 0; r < 32; r++) yb[r * LDY] = x[r];
    } else {  // the 32 x 32 blocks that stay zero: below the diagonal (forward) or above it (backward)
        for (int idx = tid - 128; idx < 6 * 1024; idx += 128) {
            const int blk = idx >> 10, e = idx & 1023, rr = e >> 5, cc = e & 31;
            const int hi = blk < 1 ? 1 : (blk < 3 ? 2 : 3);  // (1,0) (2,0) (2,1) (3,0) (3,1) (3,2)
            const int lo = blk - (hi * (hi - 1)) / 2;
            const int rb = FWD ? hi : lo, cb = FWD ? lo : hi;
            op[(32 * rb + rr) * LDY + 32 * cb + cc] = 0.0f;
        }
    }
    __syncthreads();
    {  // the 32 x 32 block beside the diagonal of each 64 x 64 half (threads 0-127: half 0)
        const int o = 64 * (tid >> 7);
        const float* mid = scr + kMidOff + (tid >> 7) * 32 * L32;
        float* wt = scr + (tid >> 7) * 32 * L32;  // over the consumed diagonal pieces
        if (FWD)
            mm32(mid, L32, op + (o + 32) * LDY + o + 32, LDY, wt, L32);  // D01 Y11
        else
            mm32(mid, L32, op + o * LDY + o, LDY, wt, L32);  // D10 X00
        __syncthreads();
        if (FWD)
            mm32(op + o * LDY + o, LDY, wt, L32, op + o * LDY + o + 32, LDY);  // Y01 = Y00 D01 Y11
        else
            mm32(op + (o + 32) * LDY + o + 32, LDY, wt, L32, op + (o + 32) * LDY + o, LDY);  // X10 = X11 D10 X00
        __syncthreads();
    }
    {  // the 64 x 64 block joining the halves
        const float* top = scr + kTopOff;
        float* wt = scr;
        if (FWD)
            mm64(top, L64, op + 64 * LDY + 64, LDY, wt, L64);
        else
            mm64(top, L64, op, LDY, wt, L64);
        __syncthreads();
        if (FWD)
            mm64(op, LDY, wt, L64, op + 64, LDY);
        else
            mm64(op + 64 * LDY + 64, LDY, wt, L64, op + 64 * LDY, LDY);
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

// Ring depth: as deep as shared memory allows (227 KB per CTA) beside the
// operator and the staged values (the diagonal block's pieces use the ring's
// space while the operator is built).  Nine stages hold more than two source
// tiles, so a finisher's last source is in flight before the one before it is
// consumed.
template <int NR>
__host__ __device__ constexpr int stages() {
    return 9;
}

// Published values of one 128-entry block (a source tile's values or a
// chunk's sums), prefetched into registers: thread t owns entries
// idx = t + m * GT (q = idx / 128, i = idx % 128) of the NR x 128 block.
template <int NR>
struct Pending {
    static constexpr int M = (NR * SB + GT - 1) / GT;
    unsigned long long w[M];
};

// Issue the relaxed loads of block K's pairs (entries beyond kbK or g read as
// valid zeros).
template <int NR>
__device__ __forceinline__ void prefetch_tile(Pending<NR>& pd, const unsigned long long* __restrict__ pub, long long K,
                                              int g, int kbK, unsigned tag) {
#pragma unroll
    for (int m = 0; m < Pending<NR>::M; m++) {
        const int idx = threadIdx.x + m * GT;
        const int q = idx / SB, i = idx - q * SB;
        pd.w[m] = (idx < NR * SB && q < g && i < kbK) ? ld_pair(pub + ((size_t)K * g + q) * SB + i)
                                                      : ((unsigned long long)tag << 32);
    }
}

// Complete the prefetched values of block K: entries not yet carrying `tag`
// are polled (bounded by kWaitLimitNs; another CTA's error ends the wait
// too); the values go to ybuf[i*NR + q].  false (CTA-uniform): a wait gave up
// (here or in another CTA).
// The value of the pair at src once it carries `tag`: w is its prefetched
// word, polled again while stale (bounded by kWaitLimitNs; another CTA's error
// ends the wait too, and ok turns false).
__device__ __forceinline__ float complete_pair(unsigned long long w, const unsigned long long* src, unsigned tag,
                                               int* err, bool& ok) {
    if ((unsigned)(w >> 32) != tag && ok) {
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
    return __uint_as_float((unsigned)w);
}

template <int NR>
__device__ bool resolve_tile(Pending<NR>& pd, const unsigned long long* __restrict__ pub, long long K, int g,
                             unsigned tag, float* ybuf, int* err) {
    bool ok = true;
#pragma unroll
    for (int m = 0; m < Pending<NR>::M; m++) {
        const int idx = threadIdx.x + m * GT;
        if (idx >= NR * SB) continue;
        const int q = idx / SB, i = idx - q * SB;
        ybuf[i * NR + q] = complete_pair(pd.w[m], pub + ((size_t)K * g + q) * SB + i, tag, err, ok);
    }
    return __syncthreads_and(ok) != 0;
}

// One sweep (see the file comment).  FWD: in = b (rows of ldb), out: the
// published y.  Backward: in = the forward sweep's published y, out: x = -s
// into xout (rows of ldb) and the published s.  g = right-hand sides of this
// launch (<= NR); q = chunk size (0: none).  pub holds the tiles' values
// (blocks 0 .. nblk-1) and then the chunks' sums (block nblk + slot).  stall
// (tests only): the forward sweep's tile 1 waits for a tag that is never
// written, so its bounded wait runs out.
template <int NR, bool FWD>
__global__ void __launch_bounds__(GT, 1)
    k_gesl_sweep(const float* __restrict__ a, int lda, int n, const float* __restrict__ bin, float* __restrict__ xout,
                 int ldb, unsigned long long* __restrict__ pub, int g, int q, int* __restrict__ ticket,
                 int* __restrict__ err, int stall) {
    constexpr int STG = stages<NR>();
    // PS partial sums per right-hand side (rows round-robin) so that one right-hand side's
    // FMAs form independent chains; combined in a fixed order
    constexpr int PS = NR == 1 ? 4 : 1;
    extern __shared__ __align__(16) float smem[];
    float* op = smem;                         // 128 x 128 operator of the tile (row stride LDY)
    float* ring = op + kOpFloats;             // STG x 32 x 128 factor rows
    float* scr = ring;                        // the diagonal block's pieces while the operator is built
    float* ybuf = ring + STG * STAGE_FLOATS;  // 128 x NR published values of one block
    float* inb = ybuf + NR * SB;              // NR x 128 input of the tile (b_j or y_j)
    __shared__ int s_item[2];
    const int tid = threadIdx.x;
    const int nblk = (n + SB - 1) / SB;
    const long long nitems = items_before(nblk, q);
    const unsigned tag = FWD ? kTagFwd : kTagBwd;
    const int c = tid & (SB - 1), h = tid >> 7;  // compute mapping: column c, rows 16h..16h+15 of a stage
    for (;;) {
        __syncthreads();  // the previous item's shared data is consumed
        if (tid == 0) {
            const long long k = atomicAdd(ticket, 1);
            int t = -1, m = 0;
            if (k < nitems) {  // the tile t with items_before(t) <= k < items_before(t + 1)
                int lo = 0, hi = nblk - 1;
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (items_before(mid, q) <= k)
                        lo = mid;
                    else
                        hi = mid - 1;
                }
                t = lo;
                m = (int)(k - items_before(t, q));
            }
            s_item[0] = t;
            s_item[1] = m;
        }
        __syncthreads();
        const int t = s_item[0], mi = s_item[1];
        if (t < 0) break;
        const int nch = chunks_of(t, q);
        const bool fin = mi == nch;  // the tile's finisher (else chunk mi)
        const int j = FWD ? t : nblk - 1 - t;
        const int c0 = j * SB, kb = min(SB, n - c0);
        const int u0 = mi * q;                     // first source of the item
        const int nsrc = (fin ? t : u0 + q) - u0;  // its sources
        const int total = nsrc * SPT;
        // the finisher's last source stays in the ring and is added after everything else
        const int nloop = fin ? nsrc - 1 : nsrc;
        auto src_tile = [&](int si) { return FWD ? u0 + si : nblk - 1 - (u0 + si); };
        // stage s: rows [32 (s % SPT), +32) of source si = s / SPT, columns [c0, c0 + 128)
        auto issue = [&](int s) {
            const int si = s / SPT, sr = s - si * SPT;
            const int r0 = src_tile(si) * SB + sr * RS;
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
        if (fin) {
            // the tile's input: b_j (forward) or the forward sweep's y_j (the low word of its pairs)
            for (int idx = tid; idx < NR * SB; idx += GT) {
                const int qq = idx / SB, i = idx - qq * SB;
                inb[idx] = (qq < g && i < kb)
                               ? (FWD ? bin[(size_t)qq * ldb + c0 + i]
                                      : __uint_as_float((unsigned)ld_pair(pub + ((size_t)j * g + qq) * SB + i)))
                               : 0.0f;
            }
            // the operator first: its pieces use the ring's space, and the finisher then holds
            // it while the ring streams the sources
            load_pieces<FWD>(a + (size_t)c0 * lda + c0, lda, kb, scr);
            __syncthreads();
            build_operator<FWD>(scr, op);
        }
#pragma unroll
        for (int s = 0; s < STG - 1; s++) {
            if (s < total) issue(s);
            cp_commit();
        }
        float p[NR * PS];
#pragma unroll
        for (int r = 0; r < NR * PS; r++) p[r] = 0.0f;
        bool ok = *(volatile int*)err == 0;
        ok = __syncthreads_and(ok) != 0;
        const bool never = FWD && stall != 0 && t == 1;  // tile 1's only source is tile 0
        Pending<NR> pd;
        if (nsrc > 0 && ok) {
            const int K0 = src_tile(0);
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
                    for (int qq = 0; qq < NR; qq += 4) {
                        const float4 y4 = *reinterpret_cast<const float4*>(y + qq);
                        p[qq] = fmaf(y4.x, v, p[qq]);
                        p[qq + 1] = fmaf(y4.y, v, p[qq + 1]);
                        p[qq + 2] = fmaf(y4.z, v, p[qq + 2]);
                        p[qq + 3] = fmaf(y4.w, v, p[qq + 3]);
                    }
                } else {
#pragma unroll
                    for (int qq = 0; qq < NR; qq++) p[qq * PS + r % PS] = fmaf(y[qq], v, p[qq * PS + r % PS]);
                }
            }
        };
        const unsigned want = never ? kTagNever : tag;
        for (int s = 0; s < total && ok; s++) {
            const int si = s / SPT, sr = s - si * SPT;
            if (sr == 0) {
                __syncthreads();  // every thread is done with the previous source's values
                if (si == nloop) break;  // the finisher's last source: added after the rest
                const int K = src_tile(si);
                ok = resolve_tile<NR>(pd, pub, K, g, want, ybuf, err);
                if (!ok) break;
                if (si + 1 < nsrc) {
                    const int K1 = src_tile(si + 1);
                    prefetch_tile<NR>(pd, pub, K1, g, min(SB, n - K1 * SB), want);
                }
            }
            cp_wait<STG - 2>();
            __syncthreads();
            if (s + STG - 1 < total) issue(s + STG - 1);
            cp_commit();
            consume(s, sr);
        }
        if (!fin) cp_wait<0>();  // (a finisher's last source may still be in flight)
        // this thread's sums of the sources added so far; the upper half's go to red.  The sums
        // use two ring slots whose stages were consumed (the finisher's last source occupies
        // the four slots before them)
        float* red = ring + (total % STG) * STAGE_FLOATS;  // NR x 128
        float* acc = red + NR * SB;                         // 128 x NR (i * NR + q): the tile's accumulated input
        float* part = ring + ((total + 1) % STG) * STAGE_FLOATS;  // 2 x NR x 128
        if constexpr (PS > 1) {
#pragma unroll
            for (int qq = 0; qq < NR; qq++)
                p[qq * PS] = (p[qq * PS] + p[qq * PS + 1]) + (p[qq * PS + 2] + p[qq * PS + 3]);
        }
        if (h == 1) {
#pragma unroll
            for (int qq = 0; qq < NR; qq++) red[qq * SB + c] = p[qq * PS];
        }
        ok = __syncthreads_and(ok) != 0;
        if (!fin) {  // a chunk: publish its sums
            if (h == 0) {
                unsigned long long* dst = pub + (size_t)(nblk + chunks_before(t, q) + mi) * g * SB;
#pragma unroll
                for (int qq = 0; qq < NR; qq++)
                    if (qq < g && c < kb)
                        st_pair(dst + (size_t)qq * SB + c, tag,
                                ok ? p[qq * PS] + red[qq * SB + c] : __int_as_float(0x7fc00000));  // NaN: aborted
            }
            continue;
        }
        // the finisher: acc = (in + the chunks' sums) + its own sources but the last
        float own[NR];
#pragma unroll
        for (int qq = 0; qq < NR; qq++) own[qq] = p[qq * PS] + red[qq * SB + c];
        if (nch > 0 && ok) {
            // the chunks' sums: each thread adds up its entries over the chunks in chunk order
            // (CG chunks' loads in flight at a time), then one barrier
            constexpr int CG = NR == 1 ? 8 : (NR <= 4 ? 4 : 1);
            constexpr int M = Pending<NR>::M;
            const long long base = nblk + chunks_before(t, q);
            float psum[M];
#pragma unroll
            for (int mm = 0; mm < M; mm++) psum[mm] = 0.0f;
            bool okp = true;
            for (int m0 = 0; m0 < nch; m0 += CG) {
                Pending<NR> pc[CG];
#pragma unroll
                for (int e = 0; e < CG; e++)
                    if (m0 + e < nch) prefetch_tile<NR>(pc[e], pub, base + m0 + e, g, kb, tag);
#pragma unroll
                for (int e = 0; e < CG; e++) {
                    if (m0 + e < nch) {
#pragma unroll
                        for (int mm = 0; mm < M; mm++) {
                            const int idx = tid + mm * GT;
                            if (idx < NR * SB) {
                                const int qq = idx / SB, i = idx - qq * SB;
                                psum[mm] += complete_pair(pc[e].w[mm], pub + ((size_t)(base + m0 + e) * g + qq) * SB + i,
                                                          tag, err, okp);
                            }
                        }
                    }
                }
            }
            __syncthreads();  // ybuf is free
#pragma unroll
            for (int mm = 0; mm < M; mm++) {
                const int idx = tid + mm * GT;
                if (idx < NR * SB) ybuf[(idx - (idx / SB) * SB) * NR + idx / SB] = psum[mm];
            }
            ok = __syncthreads_and(ok && okp) != 0;
        }
        if (h == 0) {
#pragma unroll
            for (int qq = 0; qq < NR; qq++)
                acc[c * NR + qq] = (inb[qq * SB + c] + (nch > 0 ? ybuf[c * NR + qq] : 0.0f)) + own[qq];
        }
        // the last source: its values, then its four stages (all in the ring: STG > SPT)
        if (nsrc > 0 && ok) {
            __syncthreads();  // ybuf is free
            ok = resolve_tile<NR>(pd, pub, src_tile(nloop), g, want, ybuf, err);
            cp_wait<0>();
            __syncthreads();
            if (ok) {
#pragma unroll
                for (int r = 0; r < NR * PS; r++) p[r] = 0.0f;
#pragma unroll
                for (int r4 = 0; r4 < SPT; r4++) consume(nloop * SPT + r4, r4);
                if constexpr (PS > 1) {
#pragma unroll
                    for (int qq = 0; qq < NR; qq++)
                        p[qq * PS] = (p[qq * PS] + p[qq * PS + 1]) + (p[qq * PS + 2] + p[qq * PS + 3]);
                }
                if (h == 1) {
#pragma unroll
                    for (int qq = 0; qq < NR; qq++) red[qq * SB + c] = p[qq * PS];
                }
                __syncthreads();
                if (h == 0) {
#pragma unroll
                    for (int qq = 0; qq < NR; qq++) acc[c * NR + qq] += p[qq * PS] + red[qq * SB + c];
                }
            }
        }
        cp_wait<0>();  // nothing of this item stays in flight (also after a wait that gave up)
        ok = __syncthreads_and(ok) != 0;
        {  // res = operator^T acc, from the two halves of the product
            const int i = tid & (SB - 1), hh = tid >> 7;
            float pr[NR * PS];
#pragma unroll
            for (int r = 0; r < NR * PS; r++) pr[r] = 0.0f;
#pragma unroll 16
            for (int kk = 0; kk < SB / 2; kk++) {
                const int k = hh * (SB / 2) + kk;
                const float m = op[k * LDY + i];
#pragma unroll
                for (int r = 0; r < NR; r++) pr[r * PS + kk % PS] = fmaf(m, acc[k * NR + r], pr[r * PS + kk % PS]);
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
            const int qq = idx / SB, i = idx - qq * SB;
            if (qq < g && i < kb) {
                const float v = ok ? part[qq * SB + i] + part[(NR + qq) * SB + i]
                                   : __int_as_float(0x7fc00000);  // NaN marks an aborted solve
                if (!FWD) xout[(size_t)qq * ldb + c0 + i] = -v;
                st_pair(pub + ((size_t)j * g + qq) * SB + i, tag, v);
            }
        }
    }
}

template <int NR>
constexpr size_t sweep_smem() {
    return sizeof(float) * ((size_t)kOpFloats + (size_t)stages<NR>() * STAGE_FLOATS + 2 * (size_t)NR * SB);
}
// the pieces fit in the ring; the tile's sums fit in two slots beside the last source's four
static_assert(kScrFloats <= 9 * STAGE_FLOATS && 64 * L64 <= kMidOff, "scratch");
static_assert(2 * 16 * SB <= STAGE_FLOATS && stages<1>() >= 2 * SPT + 1, "ring");
static_assert(sweep_smem<1>() <= 227 * 1024 && sweep_smem<4>() <= 227 * 1024 && sweep_smem<16>() <= 227 * 1024,
              "sweep shared memory");

template <int NR>
int sweeps(const float* a, int lda, int n, float* b, int ldb, int g, int q, unsigned long long* pub, int* tickets,
           int* err, bool stall, int sms, cudaStream_t st) {
    const int nblk = (n + SB - 1) / SB;
    const long long items = items_before(nblk, q);
    const int grid = (int)std::min<long long>(items, sms);
    LP_CUDA(cudaMemsetAsync(tickets, 0, 2 * sizeof(int), st));
    LP_CUDA(cudaMemsetAsync(pub, 0, sizeof(unsigned long long) * gesl_pub_pairs(n, g, q), st));
    k_gesl_sweep<NR, true><<<grid, GT, sweep_smem<NR>(), st>>>(a, lda, n, b, nullptr, ldb, pub, g, q, tickets, err,
                                                               stall ? 1 : 0);
    k_gesl_sweep<NR, false><<<grid, GT, sweep_smem<NR>(), st>>>(a, lda, n, nullptr, b, ldb, pub, g, q, tickets + 1,
                                                                err, 0);
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

// Published-value pairs of one solve: the tiles' values and, with chunks of
// `chunk` sources, the chunks' sums, each ceil(n / 128) x 128 x min(nrhs, 16).
size_t gesl_pub_pairs(int n, int nrhs, int chunk) {
    const size_t g = nrhs < 16 ? nrhs : 16;
    const int nblk = (n + SB - 1) / SB;
    return (size_t)(nblk + chunks_before(nblk, chunk)) * SB * g;
}

// Forward + back substitution for nrhs rows of b (overwritten by x), in
// chunks of at most 16 right-hand sides.  pub: gesl_pub_pairs(n, nrhs, chunk)
// pairs; tickets: 2 ints; err: an error word the caller zeroes and reads (set
// when a bounded wait gave up; that tile is written as NaN).  pub and tickets
// are cleared here before every group of right-hand sides.  stall (tests
// only): see k_gesl_sweep.
int launch_gesl_inv(const float* a, int lda, int n, float* b, int ldb, int nrhs, unsigned long long* pub,
                    int* tickets, int* err, bool stall, int chunk, cudaStream_t st) {
    if (n <= 0 || nrhs <= 0) return LP_OK;
    if (lda % 4 != 0 || !aligned16(a)) return fail(LP_E_INVALID, "gesl: factors need lda % 4 == 0, 16-byte aligned");
    if (chunk < 0) return fail(LP_E_INVALID, "gesl: negative chunk size");
    int dev = 0, sms = 0;
    LP_CUDA(cudaGetDevice(&dev));
    LP_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    for (int r0 = 0; r0 < nrhs; r0 += 16) {
        const int g = (nrhs - r0) < 16 ? (nrhs - r0) : 16;
        float* bb = b + (size_t)r0 * ldb;
        const bool stall_here = stall && r0 == 0;
        if (g == 1)
            LP_CHECK(sweeps<1>(a, lda, n, bb, ldb, g, chunk, pub, tickets, err, stall_here, sms, st));
        else if (g <= 4)
            LP_CHECK(sweeps<4>(a, lda, n, bb, ldb, g, chunk, pub, tickets, err, stall_here, sms, st));
        else
            LP_CHECK(sweeps<16>(a, lda, n, bb, ldb, g, chunk, pub, tickets, err, stall_here, sms, st));
    }
    return LP_OK;
}

}  // namespace lp
