// inner stage on the 5th-generation tensor cores (mixed-precision form):
//
//     C(m x n, FP32) += sum over 512-wide K segments s of
//                       scale_a[s][m/512] * scale_b[s][n/512] * (Aq_s * Bq_s^T)
//
// Aq: the left panel rounded to BF16 (or FP8 E4M3), m x k, k contiguous;
// Bq: the top panel rounded the same way and stored transposed, n x k.
// Both are K-major operands.  Persistent, warp-specialized: one CTA per SM
// walks 128 x TN C tiles (in groups of 16 tile rows, so that the CTAs in
// flight share their A and B tiles in L2); TN = 256 where the column range allows it (half the operand
// bytes per flop of TN = 128, which matters once K is long), else 128.
// Where both ranges are multiples of 256, k_umma_pair (further down) runs the
// same update with 256 x 256 tiles over CTA pairs (cta_group::2): a third less
// operand traffic per flop than the 128 x 256 tile.
//   warp 0      TMA producer: A and B tiles (128-byte swizzle) into a
//               STAGES-deep shared-memory ring;
//   warp 1      one elected thread issues tcgen05.mma (kind::f16 for BF16,
//               kind::f8f6f4 for E4M3) into one of TWO TN-column FP32
//               accumulators in tensor memory, alternating by tile;
//   warps 2-9   epilogue: while the next tile's MMAs run, read the finished
//               accumulator with tcgen05.ld (warp w reads TMEM lanes
//               32*(w%4).., half (w-2)/4 of the columns), transpose each
//               32 x 32 block through shared memory and add it into C with
//               coalesced loads/stores (the C block is prefetched before the
//               accumulator is ready).  C is read and written once.
// The same kernel runs the mixed schedules' top and left stages as products
// with the inverted triangles of the diagonal block (k_mixed.cu).
//
// Every mbarrier wait is bounded.  On expiry the thread records an error
// code in *err, raises the CTA's abort flag, stops issuing work, lets its own
// copies / MMAs in flight finish (bounded again), and the CTA frees its
// tensor memory and returns; the host reports LP_E_TIMEOUT.
#include <algorithm>

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_fp8.h>

#include "lp_common.cuh"

namespace lp {
namespace {

constexpr int UM = 128;            // tile rows (TMEM lanes)
constexpr int UN = 128;            // narrow tile columns (TMEM columns); the wide tile has 2 UN
constexpr int UKB = 128;           // bytes of k per stage row (one 128-byte swizzle row)
constexpr int UEPI = 8;            // epilogue warps
constexpr int UT = 32 * (2 + UEPI);
constexpr int kTileBytesA = UM * UKB;
constexpr int kScratchFloats = 32 * 33;  // per epilogue warp: one 32 x 32 block, padded
// Ring depth: as deep as 227 KB of shared memory allows beside the epilogue's
// transpose scratch (33 KB): 6 stages of 32 KB for TN = 128, 4 of 48 KB for
// TN = 256.
template <int TN>
__host__ __device__ constexpr int stages() { return TN == 128 ? 6 : 4; }
template <int TN>
__host__ __device__ constexpr int stage_bytes() { return kTileBytesA + TN * UKB; }
template <int TN>
constexpr size_t umma_smem() {
    return (size_t)stages<TN>() * stage_bytes<TN>() + sizeof(float) * UEPI * kScratchFloats + 1024 /*align slack*/ +
           256 /*barriers*/;
}
static_assert(umma_smem<128>() <= 232448 && umma_smem<256>() <= 232448, "umma shared memory");
constexpr uint32_t kSpinLimit = 1u << 26;
constexpr uint64_t kWaitNs = 500ull * 1000 * 1000;

enum : int { kErrFullWait = 1, kErrEmptyWait = 2, kErrDoneWait = 3 };

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Bounded wait: at most kWaitNs of wall time (and kSpinLimit polls); gives
// up early when the CTA's abort flag is raised.  Legitimate waits here last
// microseconds.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* abort_flag) {
    const uint64_t t0 = global_ns();
    for (uint32_t i = 0; i < kSpinLimit; i++) {
        if (mbar_try(bar, parity)) return true;
        if ((i & 63) == 63 && (*abort_flag || global_ns() - t0 > kWaitNs)) return false;
    }
    return false;
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];"
        ::"r"(smem_u32(dst)), "l"(map), "r"(smem_u32(bar)), "r"(x), "r"(y)
        : "memory");
}

// Shared-memory matrix descriptor, K-major with 128-byte swizzle: rows of
// 128 bytes, 8-row core groups 1024 bytes apart (SBO), LBO unused (1),
// descriptor version 1, layout type 2 (SWIZZLE_128B).
__device__ __forceinline__ uint64_t desc_sw128(uint32_t saddr) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
           ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

template <bool FP8>
__device__ __forceinline__ void umma(uint32_t tmem_d, uint64_t ad, uint64_t bd, uint32_t idesc, uint32_t acc) {
    if (FP8) {
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f8f6f4 [%0], %1, %2, %3, p;\n\t}"
            ::"r"(tmem_d), "l"(ad), "l"(bd), "r"(idesc), "r"(acc));
    } else {
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
            ::"r"(tmem_d), "l"(ad), "l"(bd), "r"(idesc), "r"(acc));
    }
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Instruction descriptor: FP32 accumulate (c_format 1), A/B K-major,
// N >> 3 at bits 17-22, M >> 4 at bits 24-28; a/b format 1 = BF16 for
// kind::f16, 0 = E4M3 for kind::f8f6f4.
// Tile t -> its C origin.  Tiles go down groups of kGroupRows tile rows
// column by column, so the ~140 tiles in flight at once span 16 row blocks
// of A and about 9 column blocks of B, which stay in L2; a plain row-major
// order would stream all of B from HBM once per tile row.
constexpr int kGroupRows = 16;
__device__ __forceinline__ void tile_origin(int t, int tiles_n, int tiles, int m_off, int n_off, int tn, int* m0,
                                            int* n0) {
    const int tiles_m = tiles / tiles_n;
    const int group = t / (kGroupRows * tiles_n);
    const int first = group * kGroupRows;
    const int rows = min(kGroupRows, tiles_m - first);
    const int local = t - first * tiles_n;
    *m0 = m_off + (first + local % rows) * UM;
    *n0 = n_off + (local / rows) * tn;
}

template <bool FP8, int TN>
__host__ __device__ constexpr uint32_t idesc_value() {
    return (1u << 4) | ((FP8 ? 0u : 1u) << 7) | ((FP8 ? 0u : 1u) << 10) | ((uint32_t)(TN >> 3) << 17) |
           ((uint32_t)(UM >> 4) << 24);
}

// SEG (E4M3 with K longer than 512): one absmax scale per 512 x 512 block of
// each operand, i.e. per 512-row block and 512-wide K segment of A and per
// 512-column block and K segment of B (scale_x[seg * sstride + block]).  The
// MMA warp accumulates each K segment of a tile into its own accumulator
// (the two TMEM buffers alternate by segment), and the epilogue adds
// s_A(seg) s_B(seg) * acc(seg) into per-thread sums that start from the tile
// of C, then writes the tile back once.
template <bool FP8, int TN, bool SEG = false>
__global__ void __launch_bounds__(UT, 1) k_umma_update(const __grid_constant__ CUtensorMap map_a,
                                                       const __grid_constant__ CUtensorMap map_b,
                                                       float* __restrict__ C, int ldc, int m_off, int n_off,
                                                       int tiles_n, int tiles, int kbytes,
                                                       const float* __restrict__ scale_a,
                                                       const float* __restrict__ scale_b, int nseg, int sstride,
                                                       int* __restrict__ err) {
    constexpr int USTAGES = stages<TN>();
    constexpr int kStageBytes = stage_bytes<TN>();
    constexpr int kBlk = TN / 64;  // 32-column blocks per epilogue warp
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;
    uint8_t* ring = smem_raw + (base - raw);
    float* scratch = reinterpret_cast<float*>(ring + USTAGES * kStageBytes);
    uint64_t* full = reinterpret_cast<uint64_t*>(scratch + UEPI * kScratchFloats);
    uint64_t* empty = full + USTAGES;
    uint64_t* acc_full = empty + USTAGES;   // [2] MMA -> epilogue
    uint64_t* acc_empty = acc_full + 2;     // [2] epilogue -> MMA
    uint64_t* done = acc_empty + 2;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int KT = kbytes / UKB;
    constexpr int kSteps = UKB / 32;  // 32 bytes of k per MMA: 16 BF16 or 32 E4M3

    if (threadIdx.x == 0) {
        for (int s = 0; s < USTAGES; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; b++) {
            mbar_init(&acc_full[b], 1);
            mbar_init(&acc_empty[b], UEPI);
        }
        mbar_init(done, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncwarp();
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"((uint32_t)(2 * TN)));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {  // TMA producer
            int it = 0;
            bool ok = true;
            for (int t = blockIdx.x; t < tiles && ok; t += gridDim.x) {
                int m0, n0;
                tile_origin(t, tiles_n, tiles, m_off, n_off, TN, &m0, &n0);
                for (int kt = 0; kt < KT; kt++, it++) {
                    const int s = it % USTAGES;
                    if (!mbar_wait(&empty[s], ((it / USTAGES) & 1) ^ 1, abort_flag)) {
                        atomicExch(err, kErrEmptyWait);
                        *abort_flag = 1;
                        ok = false;
                        break;
                    }
                    uint8_t* sa = ring + s * kStageBytes;
                    mbar_expect_tx(&full[s], kStageBytes);
                    tma_load_2d(sa, &map_a, &full[s], kt * UKB / (FP8 ? 1 : 2), m0);
                    tma_load_2d(sa + kTileBytesA, &map_b, &full[s], kt * UKB / (FP8 ? 1 : 2), n0);
                }
            }
            // Let this thread's copies still in flight land before the CTA can exit.
            for (int j = it - USTAGES < 0 ? 0 : it - USTAGES; j < it; j++) {
                volatile int no_abort = 0;
                mbar_wait(&full[j % USTAGES], (j / USTAGES) & 1, &no_abort);
            }
        }
    } else if (warp == 1) {
        if (lane == 0 && SEG) {  // MMA issuer, one accumulator per 512-wide K segment
            constexpr uint32_t idesc = idesc_value<FP8, TN>();
            const int ks = KT / nseg;  // ring stages per segment
            int it = 0, u = 0;
            bool ok = true;
            for (int t = blockIdx.x; t < tiles && ok; t += gridDim.x) {
                for (int seg = 0; seg < nseg && ok; seg++, u++) {
                    const int b = u & 1;
                    if (!mbar_wait(&acc_empty[b], ((u >> 1) & 1) ^ 1, abort_flag)) {
                        atomicExch(err, kErrEmptyWait);
                        *abort_flag = 1;
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t acc = tmem + (uint32_t)(b * TN);
                    for (int kk = 0; kk < ks; kk++, it++) {
                        const int s = it % USTAGES;
                        if (!mbar_wait(&full[s], (it / USTAGES) & 1, abort_flag)) {
                            atomicExch(err, kErrFullWait);
                            *abort_flag = 1;
                            ok = false;
                            break;
                        }
                        tc_fence_after();
                        const uint32_t sa = smem_u32(ring + s * kStageBytes);
                        const uint32_t sb = sa + kTileBytesA;
#pragma unroll
                        for (int j = 0; j < kSteps; j++)
                            umma<FP8>(acc, desc_sw128(sa + 32 * j), desc_sw128(sb + 32 * j), idesc,
                                      (kk | j) ? 1u : 0u);
                        umma_commit(&empty[s]);
                    }
                    if (ok) umma_commit(&acc_full[b]);
                }
            }
            umma_commit(done);  // tracks every MMA issued above, also on the abort path
        } else if (lane == 0) {  // MMA issuer
            constexpr uint32_t idesc = idesc_value<FP8, TN>();
            int it = 0, i = 0;
            bool ok = true;
            for (int t = blockIdx.x; t < tiles && ok; t += gridDim.x, i++) {
                const int b = i & 1;
                if (!mbar_wait(&acc_empty[b], ((i >> 1) & 1) ^ 1, abort_flag)) {
                    atomicExch(err, kErrEmptyWait);
                    *abort_flag = 1;
                    break;
                }
                tc_fence_after();
                const uint32_t acc = tmem + (uint32_t)(b * TN);
                for (int kt = 0; kt < KT; kt++, it++) {
                    const int s = it % USTAGES;
                    if (!mbar_wait(&full[s], (it / USTAGES) & 1, abort_flag)) {
                        atomicExch(err, kErrFullWait);
                        *abort_flag = 1;
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t sa = smem_u32(ring + s * kStageBytes);
                    const uint32_t sb = sa + kTileBytesA;
#pragma unroll
                    for (int j = 0; j < kSteps; j++)
                        umma<FP8>(acc, desc_sw128(sa + 32 * j), desc_sw128(sb + 32 * j), idesc, (kt | j) ? 1u : 0u);
                    umma_commit(&empty[s]);
                }
                if (ok) umma_commit(&acc_full[b]);
            }
            umma_commit(done);  // tracks every MMA issued above, also on the abort path
        }
    } else if (SEG) {  // epilogue, per-segment scales
        const int ew = warp - 2;
        const int quarter = warp & 3;      // TMEM lanes this warp may read
        const int half = ew >> 2;          // columns [TN/2 half, TN/2 half + TN/2)
        float* scr = scratch + ew * kScratchFloats;
        int u = 0;
        bool okw = true;
        for (int t = blockIdx.x; t < tiles && okw; t += gridDim.x) {
            int m0, n0;
            tile_origin(t, tiles_n, tiles, m_off, n_off, TN, &m0, &n0);
            const int r0 = m0 + quarter * 32, c0 = n0 + half * (TN / 2);
            // sums in the accumulator layout (lane = tile row, 32 consecutive columns per block),
            // started from this warp's 32 x TN/2 piece of C: coalesced row loads, transposed
            // through shared memory while the first segment's products run
            float sum[kBlk][32];
#pragma unroll
            for (int blk = 0; blk < kBlk; blk++) {
                float cv[32];
#pragma unroll
                for (int r = 0; r < 32; r++) cv[r] = C[(size_t)(r0 + r) * ldc + c0 + 32 * blk + lane];
#pragma unroll
                for (int r = 0; r < 32; r++) scr[r * 33 + lane] = cv[r];
                __syncwarp();
#pragma unroll
                for (int c = 0; c < 32; c++) sum[blk][c] = scr[lane * 33 + c];
                __syncwarp();
            }
            for (int seg = 0; seg < nseg; seg++, u++) {
                const int b = u & 1;
                // one decision per warp: tcgen05.ld below is warp-collective
                const bool got = mbar_wait(&acc_full[b], (u >> 1) & 1, abort_flag);
                if (!__all_sync(0xffffffffu, got)) {
                    if (lane == 0) atomicExch(err, kErrDoneWait);
                    *abort_flag = 1;
                    okw = false;
                    break;
                }
                tc_fence_after();
                const float sc = scale_a[seg * sstride + (m0 >> 9)] * scale_b[seg * sstride + (n0 >> 9)];
                const uint32_t taddr = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(b * TN + half * (TN / 2));
#pragma unroll
                for (int blk = 0; blk < kBlk; blk++) {
                    uint32_t a[32];
                    tmem_ld32(taddr + 32 * blk, a);
                    tmem_wait_ld();
#pragma unroll
                    for (int c = 0; c < 32; c++) sum[blk][c] = fmaf(sc, __uint_as_float(a[c]), sum[blk][c]);
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(&acc_empty[b]);
            }
            if (!okw) break;
#pragma unroll
            for (int blk = 0; blk < kBlk; blk++) {
#pragma unroll
                for (int c = 0; c < 32; c++) scr[lane * 33 + c] = sum[blk][c];
                __syncwarp();
#pragma unroll
                for (int r = 0; r < 32; r++) C[(size_t)(r0 + r) * ldc + c0 + 32 * blk + lane] = scr[r * 33 + lane];
                __syncwarp();
            }
        }
    } else {  // epilogue
        const int ew = warp - 2;
        const int quarter = warp & 3;      // TMEM lanes this warp may read
        const int half = ew >> 2;          // columns [TN/2 half, TN/2 half + TN/2)
        float* scr = scratch + ew * kScratchFloats;
        int i = 0;
        for (int t = blockIdx.x; t < tiles; t += gridDim.x, i++) {
            const int b = i & 1;
            int m0, n0;
            tile_origin(t, tiles_n, tiles, m_off, n_off, TN, &m0, &n0);
            const int r0 = m0 + quarter * 32, c0 = n0 + half * (TN / 2);
            // prefetch the first two 32 x 32 blocks of this warp's 32 x TN/2 piece of C (one
            // coalesced row segment per load); block b + 2 is fetched while block b + 1 is added
            float cv[2][32];
#pragma unroll
            for (int blk = 0; blk < 2; blk++)
#pragma unroll
                for (int r = 0; r < 32; r++) cv[blk][r] = C[(size_t)(r0 + r) * ldc + c0 + 32 * blk + lane];
            // one decision per warp: tcgen05.ld below is warp-collective
            const bool got = mbar_wait(&acc_full[b], (i >> 1) & 1, abort_flag);
            if (!__all_sync(0xffffffffu, got)) {
                if (lane == 0) atomicExch(err, kErrDoneWait);
                *abort_flag = 1;
                break;
            }
            tc_fence_after();
            const float sc = (scale_a != nullptr) ? scale_a[m0 >> 9] * scale_b[n0 >> 9] : 1.0f;
            const uint32_t taddr = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(b * TN + half * (TN / 2));
#pragma unroll
            for (int blk = 0; blk < kBlk; blk++) {
                uint32_t a[32];
                tmem_ld32(taddr + 32 * blk, a);  // lane = tile row, 32 consecutive columns
                tmem_wait_ld();
                if (blk == kBlk - 1) {
                    // both halves of the accumulator are in registers: hand the buffer back
                    tc_fence_before();
                    __syncwarp();
                    if (lane == 0) mbar_arrive(&acc_empty[b]);
                }
#pragma unroll
                for (int c = 0; c < 32; c++) scr[lane * 33 + c] = __uint_as_float(a[c]);
                __syncwarp();
#pragma unroll
                for (int r = 0; r < 32; r++) {
                    const float v = fmaf(sc, scr[r * 33 + lane], cv[blk & 1][r]);
                    C[(size_t)(r0 + r) * ldc + c0 + 32 * blk + lane] = v;
                }
                if (blk + 2 < kBlk) {
#pragma unroll
                    for (int r = 0; r < 32; r++)
                        cv[blk & 1][r] = C[(size_t)(r0 + r) * ldc + c0 + 32 * (blk + 2) + lane];
                }
                __syncwarp();
            }
        }
    }
    __syncwarp();  // the idle lanes of warps 0 and 1 park here instead of polling beside their worker lane
    // Wait for every MMA issued (bounded even when aborting) before tensor memory is freed.
    {
        volatile int no_abort = 0;
        if (!mbar_wait(done, 0, &no_abort)) {
            if (threadIdx.x == 0) atomicExch(err, kErrDoneWait);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)(2 * TN)));
    }
}

// ---- CTA pairs (tcgen05 cta_group::2) ------------------------------------------
// The same update with 256 x 256 tiles over a pair of CTAs (a cluster of two):
// each CTA stages its own 128 rows of A and its own 128 of the tile's 256
// columns of B (32 KB per K step instead of 48 KB for a 128 x 256 tile on one
// SM, so a third less operand traffic from L2 per flop), the even CTA's one
// elected thread issues M = 256 MMAs that read both CTAs' halves, and each
// CTA's tensor memory accumulates its own 128 rows of the tile.  Each CTA's
// TMA loads fill only its own shared memory; they complete on the even CTA's
// stage barrier, whose expected bytes cover both halves.  The even CTA's MMA commits
// arrive on both CTAs' barriers (stage free, accumulator full, done); both
// epilogues arrive on the even CTA's accumulator-free barrier.  Every wait is
// bounded as in the one-CTA kernel.
__device__ __forceinline__ uint32_t cluster_rank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
__device__ __forceinline__ uint32_t cluster_index() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%clusterid.x;" : "=r"(r));
    return r;
}
__device__ __forceinline__ uint32_t cluster_count() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%nclusterid.x;" : "=r"(r));
    return r;
}
// The shared-memory address of the same variable in CTA `rank` of the cluster.
__device__ __forceinline__ uint32_t map_rank(uint32_t saddr, uint32_t rank) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(saddr), "r"(rank));
    return r;
}
__device__ __forceinline__ void cluster_sync() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
__device__ __forceinline__ void tma_load_2d_pair(void* dst, const CUtensorMap* map, uint32_t bar_cluster, int x,
                                                 int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, "
        "%4}], [%2];" ::"r"(smem_u32(dst)),
        "l"(map), "r"(bar_cluster), "r"(x), "r"(y)
        : "memory");
}
template <bool FP8>
__device__ __forceinline__ void umma_pair(uint32_t tmem_d, uint64_t ad, uint64_t bd, uint32_t idesc, uint32_t acc) {
    if (FP8) {
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::2.kind::f8f6f4 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
            "l"(ad), "l"(bd), "r"(idesc), "r"(acc));
    } else {
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
            "l"(ad), "l"(bd), "r"(idesc), "r"(acc));
    }
}
// Arrive on the barrier at this offset in both CTAs of the pair once the MMAs issued so far complete.
__device__ __forceinline__ void umma_commit_pair(uint64_t* bar) {
    asm volatile(
        "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;" ::"r"(
            smem_u32(bar)),
        "h"((uint16_t)3)
        : "memory");
}
__device__ __forceinline__ void mbar_arrive_cluster(uint32_t bar_cluster) {
    asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(bar_cluster) : "memory");
}

template <bool FP8>
__host__ __device__ constexpr uint32_t idesc_pair() {
    return (1u << 4) | ((FP8 ? 0u : 1u) << 7) | ((FP8 ? 0u : 1u) << 10) | ((uint32_t)(256 >> 3) << 17) |
           ((uint32_t)(256 >> 4) << 24);
}

// Pair tile tp -> its C origin (256 x 256), in groups of kGroupRows / 2 pair rows.
__device__ __forceinline__ void pair_origin(int tp, int tiles_n, int tiles, int m_off, int n_off, int* m0, int* n0) {
    const int tiles_m = tiles / tiles_n;
    const int gr = kGroupRows / 2;
    const int group = tp / (gr * tiles_n);
    const int first = group * gr;
    const int rows = min(gr, tiles_m - first);
    const int local = tp - first * tiles_n;
    *m0 = m_off + (first + local % rows) * 256;
    *n0 = n_off + (local / rows) * 256;
}

template <bool FP8>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(UT, 1)
    k_umma_pair(const __grid_constant__ CUtensorMap map_a, const __grid_constant__ CUtensorMap map_b,
                float* __restrict__ C, int ldc, int m_off, int n_off, int tiles_n, int tiles, int kbytes,
                const float* __restrict__ scale_a, const float* __restrict__ scale_b, int* __restrict__ err) {
    constexpr int USTAGES = stages<128>();
    constexpr int kStageBytes = stage_bytes<128>();  // this CTA's A rows and its half of B's columns
    constexpr int TN = 256;                          // columns of the tile, all in each CTA's accumulator
    constexpr int kBlk = TN / 64;
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;
    uint8_t* ring = smem_raw + (base - raw);
    float* scratch = reinterpret_cast<float*>(ring + USTAGES * kStageBytes);
    uint64_t* full = reinterpret_cast<uint64_t*>(scratch + UEPI * kScratchFloats);
    uint64_t* empty = full + USTAGES;
    uint64_t* acc_full = empty + USTAGES;  // [2] MMA -> both epilogues
    uint64_t* acc_empty = acc_full + 2;    // [2] both epilogues -> MMA (the even CTA's)
    uint64_t* done = acc_empty + 2;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t rank = cluster_rank();
    const int cl = (int)cluster_index(), ncl = (int)cluster_count();
    const int KT = kbytes / UKB;
    constexpr int kSteps = UKB / 32;

    if (threadIdx.x == 0) {
        for (int s = 0; s < USTAGES; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; b++) {
            mbar_init(&acc_full[b], 1);
            mbar_init(&acc_empty[b], 2 * UEPI);
        }
        mbar_init(done, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncwarp();
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"((uint32_t)(2 * TN)));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::);
    }
    tc_fence_before();
    __syncthreads();
    cluster_sync();  // both CTAs' barriers exist before either signals the other's
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {  // TMA producer (both CTAs): this CTA's halves, completing on the even CTA's barrier
            int it = 0;
            bool ok = true;
            for (int tp = cl; tp < tiles && ok; tp += ncl) {
                int m0, n0;
                pair_origin(tp, tiles_n, tiles, m_off, n_off, &m0, &n0);
                for (int kt = 0; kt < KT; kt++, it++) {
                    const int s = it % USTAGES;
                    if (!mbar_wait(&empty[s], ((it / USTAGES) & 1) ^ 1, abort_flag)) {
                        atomicExch(err, kErrEmptyWait);
                        *abort_flag = 1;
                        ok = false;
                        break;
                    }
                    uint8_t* sa = ring + s * kStageBytes;
                    if (rank == 0) mbar_expect_tx(&full[s], 2 * kStageBytes);
                    const uint32_t bar = map_rank(smem_u32(&full[s]), 0);
                    const int kx = kt * UKB / (FP8 ? 1 : 2);
                    tma_load_2d_pair(sa, &map_a, bar, kx, m0 + 128 * (int)rank);
                    tma_load_2d_pair(sa + kTileBytesA, &map_b, bar, kx, n0 + 128 * (int)rank);
                }
            }
            // let this CTA's copies still in flight land before either CTA can exit: the even
            // CTA waits for its stage barriers, which count both CTAs' bytes; the odd CTA's
            // copies complete on those barriers, so after an abort it gives them 100 us
            if (rank == 0) {
                for (int j = it - USTAGES < 0 ? 0 : it - USTAGES; j < it; j++) {
                    volatile int no_abort = 0;
                    mbar_wait(&full[j % USTAGES], (j / USTAGES) & 1, &no_abort);
                }
            } else if (!ok) {
                const uint64_t t0 = global_ns();
                while (global_ns() - t0 < 100000ull) __nanosleep(1000);
            }
        }
    } else if (warp == 1) {
        if (lane == 0 && rank == 0) {  // MMA issuer for the pair
            constexpr uint32_t idesc = idesc_pair<FP8>();
            int it = 0, i = 0;
            bool ok = true;
            for (int tp = cl; tp < tiles && ok; tp += ncl, i++) {
                const int b = i & 1;
                if (!mbar_wait(&acc_empty[b], ((i >> 1) & 1) ^ 1, abort_flag)) {
                    atomicExch(err, kErrEmptyWait);
                    *abort_flag = 1;
                    break;
                }
                tc_fence_after();
                const uint32_t acc = tmem + (uint32_t)(b * TN);
                for (int kt = 0; kt < KT; kt++, it++) {
                    const int s = it % USTAGES;
                    if (!mbar_wait(&full[s], (it / USTAGES) & 1, abort_flag)) {
                        atomicExch(err, kErrFullWait);
                        *abort_flag = 1;
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t sa = smem_u32(ring + s * kStageBytes);
                    const uint32_t sb = sa + kTileBytesA;
#pragma unroll
                    for (int j = 0; j < kSteps; j++)
                        umma_pair<FP8>(acc, desc_sw128(sa + 32 * j), desc_sw128(sb + 32 * j), idesc,
                                       (kt | j) ? 1u : 0u);
                    umma_commit_pair(&empty[s]);
                }
                if (ok) umma_commit_pair(&acc_full[b]);
            }
            umma_commit_pair(done);  // tracks every MMA issued above, also on the abort path
        }
    } else {  // epilogue (both CTAs): this CTA's 128 rows of the tile
        const int ew = warp - 2;
        const int quarter = warp & 3;
        const int half = ew >> 2;
        float* scr = scratch + ew * kScratchFloats;
        const uint32_t acc_empty_even[2] = {map_rank(smem_u32(&acc_empty[0]), 0), map_rank(smem_u32(&acc_empty[1]), 0)};
        int i = 0;
        for (int tp = cl; tp < tiles; tp += ncl, i++) {
            const int b = i & 1;
            int m0, n0;
            pair_origin(tp, tiles_n, tiles, m_off, n_off, &m0, &n0);
            const int r0 = m0 + 128 * (int)rank + quarter * 32, c0 = n0 + half * (TN / 2);
            float cv[2][32];
#pragma unroll
            for (int blk = 0; blk < 2; blk++)
#pragma unroll
                for (int r = 0; r < 32; r++) cv[blk][r] = C[(size_t)(r0 + r) * ldc + c0 + 32 * blk + lane];
            const bool got = mbar_wait(&acc_full[b], (i >> 1) & 1, abort_flag);
            if (!__all_sync(0xffffffffu, got)) {
                if (lane == 0) atomicExch(err, kErrDoneWait);
                *abort_flag = 1;
                break;
            }
            tc_fence_after();
            const float sc = (scale_a != nullptr) ? scale_a[(m0 + 128 * (int)rank) >> 9] * scale_b[n0 >> 9] : 1.0f;
            const uint32_t taddr = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(b * TN + half * (TN / 2));
#pragma unroll
            for (int blk = 0; blk < kBlk; blk++) {
                uint32_t a[32];
                tmem_ld32(taddr + 32 * blk, a);
                tmem_wait_ld();
                if (blk == kBlk - 1) {
                    tc_fence_before();
                    __syncwarp();
                    if (lane == 0) mbar_arrive_cluster(acc_empty_even[b]);
                }
#pragma unroll
                for (int c = 0; c < 32; c++) scr[lane * 33 + c] = __uint_as_float(a[c]);
                __syncwarp();
#pragma unroll
                for (int r = 0; r < 32; r++) {
                    const float v = fmaf(sc, scr[r * 33 + lane], cv[blk & 1][r]);
                    C[(size_t)(r0 + r) * ldc + c0 + 32 * blk + lane] = v;
                }
                if (blk + 2 < kBlk) {
#pragma unroll
                    for (int r = 0; r < 32; r++)
                        cv[blk & 1][r] = C[(size_t)(r0 + r) * ldc + c0 + 32 * (blk + 2) + lane];
                }
                __syncwarp();
            }
        }
    }
    __syncwarp();
    {  // every MMA of the pair has completed (the even CTA's commit arrives here too)
        volatile int no_abort = 0;
        if (!mbar_wait(done, 0, &no_abort)) {
            if (threadIdx.x == 0) atomicExch(err, kErrDoneWait);
        }
    }
    tc_fence_before();
    __syncthreads();
    cluster_sync();  // neither CTA leaves while the other may still signal its barriers
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)(2 * TN)));
    }
}

// ---- host side ---------------------------------------------------------------

// The driver's tensor-map encoder, looked up through the runtime so the
// library does not link the driver library (it must load on hosts without
// a GPU driver, where only its host-side entry points are used).
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

int encode_fn(EncodeTiledFn* out) {
    static EncodeTiledFn fn = nullptr;
    if (fn == nullptr) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        LP_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
        if (q != cudaDriverEntryPointSuccess || p == nullptr)
            return fail(LP_E_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
        fn = reinterpret_cast<EncodeTiledFn>(p);
    }
    *out = fn;
    return LP_OK;
}

// 2-D tensor map over a row-major (rows x kbytes-of-k) operand with 128-byte
// swizzled boxes of (128 bytes of k) x box_rows rows.
int make_map(CUtensorMap* map, const void* base, int rows, int kelems, bool fp8, int box_rows) {
    EncodeTiledFn encode = nullptr;
    LP_CHECK(encode_fn(&encode));
    const CUtensorMapDataType dt = fp8 ? CU_TENSOR_MAP_DATA_TYPE_UINT8 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
    const int esz = fp8 ? 1 : 2;
    const cuuint64_t dims[2] = {(cuuint64_t)kelems, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)kelems * esz};
    const cuuint32_t box[2] = {(cuuint32_t)(UKB / esz), (cuuint32_t)box_rows};
    const cuuint32_t estr[2] = {1, 1};
    CUresult r = encode(map, dt, 2, const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                        CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(LP_E_CUDA, "cuTensorMapEncodeTiled failed: CUresult " + std::to_string((int)r));
    return LP_OK;
}

}  // namespace

int umma_init_attrs() {
    LP_CUDA(cudaFuncSetAttribute(k_umma_update<false, 128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)umma_smem<128>()));
    LP_CUDA(cudaFuncSetAttribute(k_umma_update<true, 128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)umma_smem<128>()));
    LP_CUDA(cudaFuncSetAttribute(k_umma_update<false, 256>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)umma_smem<256>()));
    LP_CUDA(cudaFuncSetAttribute(k_umma_update<true, 256>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)umma_smem<256>()));
    LP_CUDA(cudaFuncSetAttribute(k_umma_update<true, 128, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)umma_smem<128>()));
    LP_CUDA(cudaFuncSetAttribute(k_umma_pair<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)umma_smem<128>()));
    LP_CUDA(cudaFuncSetAttribute(k_umma_pair<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)umma_smem<128>()));
    return LP_OK;
}

// C(rows m_off..m_off+m, cols n_off..n_off+n of the matrix at c) += scaled
// product of aq (rows x k, k contiguous) and bq (cols x k).  aq_rows/bq_rows
// are the operands' full row counts (the tensor-map extents); m, n, m_off,
// n_off must be multiples of 128; k a multiple of 64 (BF16) / 128 (E4M3).
// E4M3 scales: scale_a[seg * sstride + m / 512], scale_b[seg * sstride +
// n / 512] for the 512-wide K segments seg (one segment when k <= 512; k a
// multiple of 512 above that).
int launch_umma_update(float* c, int ldc, const void* aq, int aq_rows, const void* bq, int bq_rows, int m_off,
                       int n_off, int m, int n, int k, bool fp8, const float* scale_a, const float* scale_b,
                       int sstride, int* err, cudaStream_t st) {
    if (m <= 0 || n <= 0) return LP_OK;
    const int kbytes = k * (fp8 ? 1 : 2);
    if (m % UM || n % UN || m_off % UM || n_off % UN || kbytes % UKB || ldc % 4 || !aligned16(c) || !aligned16(aq) ||
        !aligned16(bq) || m_off + m > aq_rows || n_off + n > bq_rows)
        return fail(LP_E_INVALID, "umma_update: tile-aligned sizes and 16-byte aligned operands required");
    if (fp8 && (scale_a == nullptr || scale_b == nullptr)) return fail(LP_E_INVALID, "umma_update: fp8 needs scales");
    const bool seg = fp8 && k > 512;
    if (seg && k % 512 != 0) return fail(LP_E_INVALID, "umma_update: E4M3 with k > 512 needs k % 512 == 0");
    const int nseg = seg ? k / 512 : 1;
    // 256 x 256 tiles over CTA pairs where both ranges are multiples of 256 (not the segmented
    // E4M3 form, which keeps its per-segment sums in registers); else the wide one-CTA tile where
    // the column range is a multiple of it, else the narrow one
    const bool pair = !seg && m % 256 == 0 && n % 256 == 0 && m_off % 256 == 0 && n_off % 256 == 0;
    const bool wide = !seg && n % (2 * UN) == 0 && n_off % (2 * UN) == 0;
    const int tn = wide ? 2 * UN : UN;
    CUtensorMap ma, mb;
    LP_CHECK(make_map(&ma, aq, aq_rows, k, fp8, UM));
    LP_CHECK(make_map(&mb, bq, bq_rows, k, fp8, pair ? UN : tn));
    int dev = 0, sms = 0;
    LP_CUDA(cudaGetDevice(&dev));
    LP_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    // Leave a few SMs to the look-ahead panel on the auxiliary stream: one CTA
    // of this kernel fills an SM (shared memory, registers), so a full-width
    // persistent grid would hold the panel off until the update ends.  Measured
    // on B200 (BF16 factorization alone): block 512, n = 32768: 8 free SMs +9 %
    // over none; block 1024, n = 32768: 16 instead of 8 56.7 -> 55.3 ms (E4M3
    // 63.9 -> 59.3 ms), 24 to 48 no further gain; block 2048, n = 65536, and the
    // emulated FP32 form: 8 and 16 alike.
    constexpr int kPanelSMs = 16;
    const int usable = sms - kPanelSMs > 1 ? sms - kPanelSMs : 1;
    if (pair) {
        const int tiles_n = n / 256, tiles = tiles_n * (m / 256);
        const int clusters = std::max(1, std::min(tiles, usable / 2));
        if (fp8)
            k_umma_pair<true><<<2 * clusters, UT, umma_smem<128>(), st>>>(ma, mb, c, ldc, m_off, n_off, tiles_n,
                                                                          tiles, kbytes, scale_a, scale_b, err);
        else
            k_umma_pair<false><<<2 * clusters, UT, umma_smem<128>(), st>>>(ma, mb, c, ldc, m_off, n_off, tiles_n,
                                                                           tiles, kbytes, nullptr, nullptr, err);
        count_launch();
        LP_CUDA(cudaGetLastError());
        return LP_OK;
    }
    const int tiles_n = n / tn, tiles = tiles_n * (m / UM);
    const int grid = tiles < usable ? tiles : usable;
    if (seg)
        k_umma_update<true, 128, true><<<grid, UT, umma_smem<128>(), st>>>(
            ma, mb, c, ldc, m_off, n_off, tiles_n, tiles, kbytes, scale_a, scale_b, nseg, sstride, err);
    else if (fp8 && wide)
        k_umma_update<true, 256><<<grid, UT, umma_smem<256>(), st>>>(ma, mb, c, ldc, m_off, n_off, tiles_n, tiles,
                                                                     kbytes, scale_a, scale_b, 1, sstride, err);
    else if (fp8)
        k_umma_update<true, 128><<<grid, UT, umma_smem<128>(), st>>>(ma, mb, c, ldc, m_off, n_off, tiles_n, tiles,
                                                                     kbytes, scale_a, scale_b, 1, sstride, err);
    else if (wide)
        k_umma_update<false, 256><<<grid, UT, umma_smem<256>(), st>>>(ma, mb, c, ldc, m_off, n_off, tiles_n, tiles,
                                                                      kbytes, nullptr, nullptr, 1, 0, err);
    else
        k_umma_update<false, 128><<<grid, UT, umma_smem<128>(), st>>>(ma, mb, c, ldc, m_off, n_off, tiles_n, tiles,
                                                                      kbytes, nullptr, nullptr, 1, 0, err);
    count_launch();
    LP_CUDA(cudaGetLastError());
    return LP_OK;
}

}  // namespace lp
