// C ABI of liblpcuda.so (declared in include/lpcuda.h): context, workspace,
// the block-step schedule of the factorization, the substitution, and the
// host entry points that stand in for the reference's execution backend.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "lp_common.cuh"
#include "lp_ctx.cuh"

namespace lp {

static thread_local std::string g_last_error;

int fail(int status, const std::string& msg) {
    g_last_error = msg;
    return status;
}

int cuda_fail(cudaError_t e, const char* what, const char* file, int line) {
    char buf[512];
    std::snprintf(buf, sizeof(buf), "%s failed: %s (%s) at %s:%d", what, cudaGetErrorName(e), cudaGetErrorString(e),
                  file, line);
    g_last_error = buf;
    if (e == cudaErrorMemoryAllocation) return LP_E_NOMEM;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return LP_E_NODEVICE;
    return LP_E_CUDA;
}

int Workspace::ensure(size_t bytes) {
    if (bytes <= cap) return LP_OK;
    if (ptr != nullptr) {
        cudaError_t e = cudaFree(ptr);
        ptr = nullptr;
        cap = 0;
        if (e != cudaSuccess) return cuda_fail(e, "cudaFree(workspace)", __FILE__, __LINE__);
    }
    LP_CUDA(cudaMalloc(&ptr, bytes));
    cap = bytes;
    return LP_OK;
}

void Workspace::release() {
    if (ptr != nullptr) cudaFree(ptr);
    ptr = nullptr;
    cap = 0;
}

int wait_stream(lp_ctx* c, cudaStream_t st) {
    LP_CUDA(cudaEventRecord(c->ev_block, st));
    LP_CUDA(cudaEventSynchronize(c->ev_block));
    return LP_OK;
}

int validate_matrix(const void* a, int n, int lda, int bs, const char* who, int max_bs) {
    if (a == nullptr) return fail(LP_E_INVALID, std::string(who) + ": null matrix pointer");
    if (n <= 0) return fail(LP_E_INVALID, std::string(who) + ": n must be positive");
    if (!is_pow2(bs) || bs < 16 || bs > max_bs)
        return fail(LP_E_INVALID,
                    std::string(who) + ": block size must be a power of two in [16, " + std::to_string(max_bs) + "]");
    if (n % bs != 0) return fail(LP_E_INVALID, std::string(who) + ": n must be a multiple of the block size");
    if (lda < n || lda % 4 != 0)
        return fail(LP_E_INVALID, std::string(who) + ": lda must be >= n and a multiple of 4");
    return LP_OK;
}

static std::atomic<long long> g_launches{0};
void count_launch(long long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
long long launch_count() { return g_launches.load(std::memory_order_relaxed); }

int prof_begin(lp_ctx* c, cudaStream_t st) {
    if (!c->prof_on) return -1;
    if (c->prof_used + 2 > c->prof_ev.size()) {
        for (int i = 0; i < 64; i++) {
            cudaEvent_t e;
            LP_CUDA(cudaEventCreate(&e));
            c->prof_ev.push_back(e);
        }
    }
    if (!c->base_recorded) {
        if (c->prof_base == nullptr) LP_CUDA(cudaEventCreate(&c->prof_base));
        LP_CUDA(cudaEventRecord(c->prof_base, st));
        c->base_recorded = true;
    }
    const int e0 = (int)c->prof_used++;
    LP_CUDA(cudaEventRecord(c->prof_ev[e0], st));
    return e0;
}

int prof_end(lp_ctx* c, cudaStream_t st, int kind, int e0, double flops, double bytes) {
    if (e0 < 0) return LP_OK;
    const int e1 = (int)c->prof_used++;
    LP_CUDA(cudaEventRecord(c->prof_ev[e1], st));
    c->marks.push_back(StageMark{kind, st == c->aux ? 1 : (st == c->aux2 ? 2 : 0), e0, e1, flops, bytes});
    return LP_OK;
}

// Folds the recorded marks into the per-stage sums (waits for the stream).
static int prof_collect(lp_ctx* c) {
    if (c->marks.empty()) return LP_OK;
    LP_CUDA(cudaStreamSynchronize(c->stream));
    LP_CUDA(cudaStreamSynchronize(c->aux));
    LP_CUDA(cudaStreamSynchronize(c->aux2));
    for (const auto& m : c->marks) {
        float ms = 0.0f, a = 0.0f, b = 0.0f;
        LP_CUDA(cudaEventElapsedTime(&ms, c->prof_ev[m.e0], c->prof_ev[m.e1]));
        LP_CUDA(cudaEventElapsedTime(&a, c->prof_base, c->prof_ev[m.e0]));
        LP_CUDA(cudaEventElapsedTime(&b, c->prof_base, c->prof_ev[m.e1]));
        c->timeline.push_back(lp_stage_event{m.kind, m.stream, a * 1e-3, b * 1e-3});
        c->prof_s[m.kind] += ms * 1e-3;
        c->prof_flops[m.kind] += m.flops;
        c->prof_bytes[m.kind] += m.bytes;
        c->prof_calls[m.kind] += 1;
    }
    c->marks.clear();
    c->prof_used = 0;
    return LP_OK;
}

// Algorithmic work of the stages (flops; bytes of one pass over the operands).
static double lu_flops(double b) { return 2.0 * b * b * b / 3.0; }
static double trsm_flops(double b, double w) { return b * b * w; }
static double inner_flops(double m, double n, double k) { return 2.0 * m * n * k; }
static double inner_bytes(double m, double n, double k) { return 4.0 * (2.0 * m * n + k * (m + n)); }

// lu stage of one diagonal block.  bs <= 128: one shared-memory kernel.
// Larger blocks are factored as the same blocked algorithm with 128-wide
// inner blocks (lu, top, left, inner on the bs x bs sub-matrix), which keeps
// every piece on the kernels above and spreads the inner work over the GPU.
int lu_stage(lp_ctx* c, float* d, int lda, int bs, cudaStream_t st, const TriInverses* inv) {
    if (bs <= 128) return launch_lu_small(d, lda, bs, st);
    const int ib = 128;
    float* lti = static_cast<float*>(c->lti.ptr);
    for (int kk = 0; kk < bs / ib; kk++) {
        float* dd = d + (size_t)kk * ib * lda + (size_t)kk * ib;
        LP_CHECK(launch_lu_small(dd, lda, ib, st));
        const int r = bs - (kk + 1) * ib;
        if (r > 0) {
            // top on st, left beside it on aux2 (both read only the factored block)
            LP_CUDA(cudaEventRecord(c->ev_side, st));
            LP_CUDA(cudaStreamWaitEvent(c->aux2, c->ev_side, 0));
            LP_CHECK(launch_trsm_top(dd, lda, dd + ib, lda, ib, r, st));
            LP_CHECK(launch_trsm_left(dd, lda, dd + (size_t)ib * lda, lda, ib, r, lti, r, c->aux2));
            LP_CUDA(cudaEventRecord(c->ev_side_done, c->aux2));
            LP_CUDA(cudaStreamWaitEvent(st, c->ev_side_done, 0));
        }
        if (inv != nullptr) {
            // block row and column kk of d are final (the trailing update below
            // touches only rows and columns after them): chunk kk of the two
            // identity recurrences, which read nothing else of d
            LP_CUDA(cudaEventRecord(c->ev_inv[kk], st));
            LP_CUDA(cudaStreamWaitEvent(c->inv_top, c->ev_inv[kk], 0));
            LP_CUDA(cudaStreamWaitEvent(c->inv_left, c->ev_inv[kk], 0));
            LP_CHECK(top_chunk_step(c, d, lda, inv->winv, bs, bs, bs, kk, c->inv_top, true));
            LP_CHECK(left_chunk_step(d, lda, inv->vinv, bs, bs, bs, inv->vlt, bs, kk, c->inv_left, true));
        }
        if (r > 0) LP_CHECK(launch_sgemm_update(dd + (size_t)ib * lda + ib, lda, lti, r, dd + ib, lda, r, r, ib, st));
    }
    if (inv != nullptr) {
        LP_CUDA(cudaEventRecord(c->ev_inv_top, c->inv_top));
        LP_CUDA(cudaEventRecord(c->ev_inv_left, c->inv_left));
        LP_CUDA(cudaStreamWaitEvent(st, c->ev_inv_top, 0));
        LP_CUDA(cudaStreamWaitEvent(st, c->ev_inv_left, 0));
    }
    return LP_OK;
}

// top stage for a whole block row: T (bs x ncols) <- top recurrence with the
// factored diagonal block d.  bs <= 128: one exact-recurrence launch.  Larger
// blocks walk 128-row diagonal chunks: exact recurrence on the chunk's rows
// (full width, every column strip in parallel), then the chunk's
// contribution to the rows below as one GEMM, T[below] += D[below][chunk] *
// T[chunk] (D's sub-block transposed into the k-major operand first).
// unit (T0 = identity): column j stays zero above row j, so chunk kk only
// touches columns below (kk + 1) * 128; the skipped entries are exact zeros.
int top_chunk_step(lp_ctx* c, const float* d, int lda, float* t, int ldt, int bs, int ncols, int kk, cudaStream_t st,
                   bool unit) {
    const int ib = 128;
    float* dt = static_cast<float*>(c->dsub.ptr) + (st == c->aux ? (size_t)ib * bs : 0);
    const float* dkk = d + (size_t)kk * ib * lda + (size_t)kk * ib;
    float* tk = t + (size_t)kk * ib * ldt;
    const int cols = unit ? std::min(ncols, (kk + 1) * ib) : ncols;
    LP_CHECK(launch_trsm_top(dkk, lda, tk, ldt, ib, cols, st));
    const int m2 = bs - (kk + 1) * ib;
    if (m2 <= 0) return LP_OK;
    LP_CHECK(launch_transpose(dkk + (size_t)ib * lda, lda, dt, m2, m2, ib, st));
    return launch_sgemm_update(tk + (size_t)ib * ldt, ldt, dt, m2, tk, ldt, m2, cols, ib, st);
}

int top_blocked(lp_ctx* c, const float* d, int lda, float* t, int ldt, int bs, int ncols, cudaStream_t st,
                bool unit) {
    if (bs <= 128) return launch_trsm_top(d, lda, t, ldt, bs, ncols, st);
    for (int kk = 0; kk < bs / 128; kk++) LP_CHECK(top_chunk_step(c, d, lda, t, ldt, bs, ncols, kk, st, unit));
    return LP_OK;
}

// left stage for a whole block column: L (nrows x bs) <- left recurrence with
// d, and Lt = L^T.  Larger blocks walk 128-column chunks: exact recurrence on
// the chunk's columns (which also writes the chunk's rows of Lt), then
// L[:, after] += L[:, chunk] * D[chunk][after] as one GEMM.
// unit (L0 = identity): row i stays zero left of column i, so chunk kk only
// touches rows above (kk + 1) * 128 (and only those rows of lt are written).
int left_chunk_step(const float* d, int lda, float* l, int ldl, int bs, int nrows, float* lt, int ldlt, int kk,
                    cudaStream_t st, bool unit) {
    const int ib = 128;
    const float* dkk = d + (size_t)kk * ib * lda + (size_t)kk * ib;
    float* lk = l + (size_t)kk * ib;
    float* ltk = lt + (size_t)kk * ib * ldlt;
    const int rows = unit ? std::min(nrows, (kk + 1) * ib) : nrows;
    LP_CHECK(launch_trsm_left(dkk, lda, lk, ldl, ib, rows, ltk, ldlt, st));
    const int m2 = bs - (kk + 1) * ib;
    if (m2 <= 0) return LP_OK;
    return launch_sgemm_update(lk + ib, ldl, ltk, ldlt, dkk + ib, lda, rows, m2, ib, st);
}

int left_blocked(const float* d, int lda, float* l, int ldl, int bs, int nrows, float* lt, int ldlt,
                 cudaStream_t st, bool unit) {
    if (bs <= 128) return launch_trsm_left(d, lda, l, ldl, bs, nrows, lt, ldlt, st);
    for (int kk = 0; kk < bs / 128; kk++) LP_CHECK(left_chunk_step(d, lda, l, ldl, bs, nrows, lt, ldlt, kk, st, unit));
    return LP_OK;
}

// Panel work of block step K: lu on the diagonal block, then the top block
// row and the left block column (Lt written into `lt`, leading dimension the
// number of rows below).  The left stage covers the rows below the diagonal
// block up to row_end (default: all n).
int panel_f32(lp_ctx* c, float* dA, int n, int lda, int bs, int K, float* lt, cudaStream_t st, int row_end) {
    float* d = dA + (size_t)K * bs * lda + (size_t)K * bs;
    const double b = bs;
    int e = prof_begin(c, st);
    LP_CHECK(lu_stage(c, d, lda, bs, st));
    LP_CHECK(prof_end(c, st, LP_STAGE_LU, e, lu_flops(b), 8.0 * b * b));
    const int rest = n - (K + 1) * bs;
    if (rest <= 0) return LP_OK;
    const int below = (row_end < 0 ? n : row_end) - (K + 1) * bs;
    // top on st and left on aux2 run concurrently: both read only the factored
    // diagonal block and write disjoint blocks (top uses st's dsub slot, left Lt)
    if (below > 0) {
        const double r = below;
        LP_CUDA(cudaEventRecord(c->ev_side, st));
        LP_CUDA(cudaStreamWaitEvent(c->aux2, c->ev_side, 0));
        e = prof_begin(c, c->aux2);
        LP_CHECK(left_blocked(d, lda, d + (size_t)bs * lda, lda, bs, below, lt, below, c->aux2));
        LP_CHECK(prof_end(c, c->aux2, LP_STAGE_LEFT, e, trsm_flops(b, r), 12.0 * b * r));
        LP_CUDA(cudaEventRecord(c->ev_side_done, c->aux2));
    }
    const double r = rest;
    e = prof_begin(c, st);
    LP_CHECK(top_blocked(c, d, lda, d + bs, lda, bs, rest, st));
    LP_CHECK(prof_end(c, st, LP_STAGE_TOP, e, trsm_flops(b, r), 8.0 * b * r));
    if (below > 0) LP_CUDA(cudaStreamWaitEvent(st, c->ev_side_done, 0));
    return LP_OK;
}

// Blocked right-looking LU without pivoting (the block-row loop of
// execution_pcie.hpp:177-641, on one GPU) with one step of look-ahead.
// Step K's trailing update C += L_K * T_K is split: first the next block row
// and block column (U_a), then the rest (U_b).  As soon as U_a is done the
// panel of step K+1 (lu, top, left) runs on the high-priority auxiliary
// stream while U_b runs on the main stream; they touch disjoint blocks, and
// Lt is double-buffered so panel K+1 never overwrites the operand U_b reads.
// top and left give the reference recurrences' values up to rounding
// (blocked); the exact recurrences are lp_top_update_dev/lp_left_update_dev.
int gefa_f32(lp_ctx* c, float* dA, int n, int lda, int bs, cudaStream_t st) {
    const size_t pan = sizeof(float) * (size_t)bs * n;
    LP_CHECK(c->lt.ensure(2 * pan));
    if (bs > 128) {
        LP_CHECK(c->lti.ensure(2 * sizeof(float) * (size_t)128 * bs));
        LP_CHECK(c->dsub.ensure(2 * sizeof(float) * (size_t)128 * bs));
    }
    float* ltbuf[2] = {static_cast<float*>(c->lt.ptr), static_cast<float*>(c->lt.ptr) + (size_t)bs * n};
    const int nb = n / bs;
    const double b = bs;
    LP_CHECK(panel_f32(c, dA, n, lda, bs, 0, ltbuf[0], st));
    for (int K = 0; K + 1 < nb; K++) {
        const int rest = n - (K + 1) * bs;
        const double r = rest;
        float* d = dA + (size_t)K * bs * lda + (size_t)K * bs;
        float* top = d + bs;
        float* lt = ltbuf[K & 1];
        float* c11 = d + (size_t)bs * lda + bs;
        int e = prof_begin(c, st);
        LP_CHECK(launch_sgemm_update(c11, lda, lt, rest, top, lda, bs, rest, bs, st));
        if (rest > bs)
            LP_CHECK(launch_sgemm_update(c11 + (size_t)bs * lda, lda, lt + bs, rest, top, lda, rest - bs, bs, bs, st));
        LP_CHECK(prof_end(c, st, LP_STAGE_INNER, e, inner_flops(b, r, b) + inner_flops(r - b, b, b),
                          inner_bytes(b, r, b) + inner_bytes(r - b, b, b)));
        LP_CUDA(cudaEventRecord(c->ev_fork, st));
        LP_CUDA(cudaStreamWaitEvent(c->aux, c->ev_fork, 0));
        LP_CHECK(panel_f32(c, dA, n, lda, bs, K + 1, ltbuf[(K + 1) & 1], c->aux));
        LP_CUDA(cudaEventRecord(c->ev_join, c->aux));
        if (rest > bs) {
            const double r2 = rest - bs;
            e = prof_begin(c, st);
            LP_CHECK(launch_sgemm_update(c11 + (size_t)bs * lda + bs, lda, lt + bs, rest, top + bs, lda, rest - bs,
                                         rest - bs, bs, st));
            LP_CHECK(prof_end(c, st, LP_STAGE_INNER, e, inner_flops(r2, r2, b), inner_bytes(r2, r2, b)));
        }
        LP_CUDA(cudaStreamWaitEvent(st, c->ev_join, 0));
    }
    return LP_OK;
}

// ---- row-slab schedule: the factorization fed from page-locked host memory ----

// One lane of the row-slab schedule: a main and a high-priority side stream,
// their fork / join events, and the double-buffered Lt of the lane's slab.
struct Lane {
    cudaStream_t st, aux;
    cudaEvent_t fork, join;
    float* lt[2];
};

// Block rows [K0, K1) (rows [r0, r1) = [K0 bs, K1 bs)) of the blocked LU, on
// one lane.  First the block steps K < K0 of the rows above, applied to these
// rows only (left with D_K on their block column K, then their update with
// block row K over the full width; one step of look-ahead as in gefa_f32),
// each after panel_done[K]; then the block steps K0..K1-1 restricted to rows
// < r1, recording panel_done[K] (by band(K, stream)) when block row K is
// final.  Every element receives the operations of gefa_f32 in the same order
// (the stages are row- or column-independent, the update adds a k-ordered
// product per element), so the factors equal gefa_f32's.
template <class Band>
static int gefa_rows(lp_ctx* c, float* dA, int n, int lda, int bs, int r0, int r1, const Lane& ln,
                     const cudaEvent_t* panel_done, Band band) {
    const int rows = r1 - r0, k0 = r0 / bs, k1 = r1 / bs;
    const double b = bs, m = rows;
    float* slab = dA + (size_t)r0 * lda;
    cudaStream_t st = ln.st, aux = ln.aux;
    if (k0 > 0) {
        LP_CUDA(cudaStreamWaitEvent(st, panel_done[0], 0));
        int e = prof_begin(c, st);
        LP_CHECK(left_blocked(dA, lda, slab, lda, bs, rows, ln.lt[0], rows, st));
        LP_CHECK(prof_end(c, st, LP_STAGE_LEFT, e, trsm_flops(b, m), 12.0 * b * m));
        for (int K = 0; K < k0; K++) {
            // block row K and D_K are final here: panel_done[K] was waited for
            // before left(K), which precedes this point on st
            const int c1 = (K + 1) * bs, ncols = n - c1;
            const float* tK = dA + (size_t)K * bs * lda + c1;  // block row K right of D_K
            const float* l = ln.lt[K & 1];
            float* cs = slab + c1;
            if (K + 1 < k0) {
                // the slab's block column K+1 first, its left stage beside the rest of the update
                e = prof_begin(c, st);
                LP_CHECK(launch_sgemm_update(cs, lda, l, rows, tK, lda, rows, bs, bs, st));
                LP_CHECK(prof_end(c, st, LP_STAGE_INNER, e, inner_flops(m, b, b), inner_bytes(m, b, b)));
                LP_CUDA(cudaEventRecord(ln.fork, st));
                LP_CUDA(cudaStreamWaitEvent(aux, ln.fork, 0));
                LP_CUDA(cudaStreamWaitEvent(aux, panel_done[K + 1], 0));
                e = prof_begin(c, aux);
                LP_CHECK(left_blocked(dA + (size_t)c1 * lda + c1, lda, cs, lda, bs, rows, ln.lt[(K + 1) & 1], rows,
                                      aux));
                LP_CHECK(prof_end(c, aux, LP_STAGE_LEFT, e, trsm_flops(b, m), 12.0 * b * m));
                LP_CUDA(cudaEventRecord(ln.join, aux));
                const double nc = ncols - bs;  // > 0: the slab's own columns lie beyond c1 + bs
                e = prof_begin(c, st);
                LP_CHECK(launch_sgemm_update(cs + bs, lda, l, rows, tK + bs, lda, rows, ncols - bs, bs, st));
                LP_CHECK(prof_end(c, st, LP_STAGE_INNER, e, inner_flops(m, nc, b), inner_bytes(m, nc, b)));
                LP_CUDA(cudaStreamWaitEvent(st, ln.join, 0));
            } else {
                const double nc = ncols;
                e = prof_begin(c, st);
                LP_CHECK(launch_sgemm_update(cs, lda, l, rows, tK, lda, rows, ncols, bs, st));
                LP_CHECK(prof_end(c, st, LP_STAGE_INNER, e, inner_flops(m, nc, b), inner_bytes(m, nc, b)));
            }
        }
    }
    LP_CHECK(panel_f32(c, dA, n, lda, bs, k0, ln.lt[k0 & 1], st, r1));
    LP_CHECK(band(k0, st));
    for (int K = k0; K + 1 < k1; K++) {
        const int below = r1 - (K + 1) * bs;  // >= bs
        const int rest = n - (K + 1) * bs;    // >= below
        const double rb = below, rc = rest;
        float* d = dA + (size_t)K * bs * lda + (size_t)K * bs;
        float* top = d + bs;
        float* c11 = d + (size_t)bs * lda + bs;
        const float* l = ln.lt[K & 1];
        int e = prof_begin(c, st);
        LP_CHECK(launch_sgemm_update(c11, lda, l, below, top, lda, bs, rest, bs, st));
        if (below > bs)
            LP_CHECK(launch_sgemm_update(c11 + (size_t)bs * lda, lda, l + bs, below, top, lda, below - bs, bs, bs, st));
        LP_CHECK(prof_end(c, st, LP_STAGE_INNER, e, inner_flops(b, rc, b) + inner_flops(rb - b, b, b),
                          inner_bytes(b, rc, b) + inner_bytes(rb - b, b, b)));
        LP_CUDA(cudaEventRecord(ln.fork, st));
        LP_CUDA(cudaStreamWaitEvent(aux, ln.fork, 0));
        LP_CHECK(panel_f32(c, dA, n, lda, bs, K + 1, ln.lt[(K + 1) & 1], aux, r1));
        LP_CHECK(band(K + 1, aux));
        LP_CUDA(cudaEventRecord(ln.join, aux));
        if (below > bs) {
            const double r2 = below - bs, c2 = rest - bs;
            e = prof_begin(c, st);
            LP_CHECK(launch_sgemm_update(c11 + (size_t)bs * lda + bs, lda, l + bs, below, top + bs, lda, below - bs,
                                         rest - bs, bs, st));
            LP_CHECK(prof_end(c, st, LP_STAGE_INNER, e, inner_flops(r2, c2, b), inner_bytes(r2, c2, b)));
        }
        LP_CUDA(cudaStreamWaitEvent(st, ln.join, 0));
    }
    return LP_OK;
}

// Row-slab boundaries of the streamed factorization: heights 1024, 2048, then
// 4096 rows (multiples of bs, at least bs), so the first slab's copy is short.
static std::vector<int> slab_cuts(int n, int bs) {
    std::vector<int> cuts{0};
    const int cap = std::max(bs, 4096 / bs * bs);
    int h = std::max(bs, 1024 / bs * bs);
    while (cuts.back() < n) {
        cuts.push_back(std::min(n, cuts.back() + h));
        h = std::min(cap, 2 * h);
    }
    return cuts;
}

// gefa_f32 on a matrix that is still in page-locked host memory hA: every
// row slab is queued for copying on the copy-in stream at once (after the
// work already queued on st), and each slab is factored as soon as it is
// resident, on two alternating lanes (st with c->aux, and the context's
// second lane), so that slab s+1 catches up on the finished block steps while
// slab s runs its own, whose last steps are short.  Panels never run on both
// lanes at once (a slab's own steps start after the other lane's last panel),
// so the panel's scratch is shared.  With host_out, every block row goes back
// to host_out (leading dimension lda) on the copy stream as soon as it is
// final.  ev: at least 2 n / bs + 2 events.
int gefa_f32_streamed(lp_ctx* c, const float* hA, float* dA, int n, int lda, int bs, cudaStream_t st,
                      float* host_out, const std::vector<cudaEvent_t>& ev) {
    const std::vector<int> cuts = slab_cuts(n, bs);
    const int ns = (int)cuts.size() - 1, nb = n / bs;
    if ((int)ev.size() < nb + ns + 2) return fail(LP_E_INVALID, "streamed factorization: too few events");
    int hmax = 0;
    for (int s = 0; s < ns; s++) hmax = std::max(hmax, cuts[s + 1] - cuts[s]);
    const size_t ltf = (size_t)bs * hmax;
    LP_CHECK(c->lt.ensure(4 * sizeof(float) * ltf));
    if (bs > 128) {
        LP_CHECK(c->lti.ensure(2 * sizeof(float) * (size_t)128 * bs));
        LP_CHECK(c->dsub.ensure(2 * sizeof(float) * (size_t)128 * bs));
    }
    if (c->copy_in == nullptr) LP_CUDA(cudaStreamCreateWithFlags(&c->copy_in, cudaStreamNonBlocking));
    if (host_out != nullptr && c->copy == nullptr) LP_CUDA(cudaStreamCreateWithFlags(&c->copy, cudaStreamNonBlocking));
    float* lt = static_cast<float*>(c->lt.ptr);
    const Lane lanes[2] = {{st, c->aux, c->ev_fork, c->ev_join, {lt, lt + ltf}},
                           {c->lane_st, c->lane_aux, c->lane_fork, c->lane_join, {lt + 2 * ltf, lt + 3 * ltf}}};
    const size_t pitch = sizeof(float) * (size_t)lda;
    // events: block rows' panels ev[0 .. nb), slab arrivals ev[nb .. nb + ns),
    // start ev[nb + ns], the second lane's end ev[nb + ns + 1]
    cudaEvent_t ev_start = ev[nb + ns], ev_lane_end = ev[nb + ns + 1];
    LP_CUDA(cudaEventRecord(ev_start, st));
    LP_CUDA(cudaStreamWaitEvent(c->copy_in, ev_start, 0));
    for (int s = 0; s < ns; s++) {
        const size_t r0 = (size_t)cuts[s];
        LP_CUDA(cudaMemcpy2DAsync(dA + r0 * lda, pitch, hA + r0 * lda, pitch, sizeof(float) * n, cuts[s + 1] - cuts[s],
                                  cudaMemcpyHostToDevice, c->copy_in));
        LP_CUDA(cudaEventRecord(ev[nb + s], c->copy_in));
    }
    auto band = [&](int K, cudaStream_t done_on) -> int {
        LP_CUDA(cudaEventRecord(ev[K], done_on));
        if (host_out == nullptr) return LP_OK;
        LP_CUDA(cudaStreamWaitEvent(c->copy, ev[K], 0));
        const size_t r = (size_t)K * bs;
        LP_CUDA(cudaMemcpy2DAsync(host_out + r * lda, pitch, dA + r * lda, pitch, sizeof(float) * n, bs,
                                  cudaMemcpyDeviceToHost, c->copy));
        return LP_OK;
    };
    // the second lane starts after the work queued on st so far
    LP_CUDA(cudaStreamWaitEvent(c->lane_st, ev_start, 0));
    for (int s = 0; s < ns; s++) {
        const Lane& ln = lanes[s & 1];
        LP_CUDA(cudaStreamWaitEvent(ln.st, ev[nb + s], 0));
        LP_CHECK(gefa_rows(c, dA, n, lda, bs, cuts[s], cuts[s + 1], ln, ev.data(), band));
    }
    LP_CUDA(cudaEventRecord(ev_lane_end, c->lane_st));
    LP_CUDA(cudaStreamWaitEvent(st, ev_lane_end, 0));
    return LP_OK;
}

int gesl_f32(lp_ctx* c, const float* dLU, int n, int lda, float* dB, int nrhs, int ldb, cudaStream_t st) {
    const size_t pairs = gesl_pub_pairs(n, nrhs, kGeslChunk);
    LP_CHECK(c->gw.ensure(sizeof(unsigned long long) * pairs + 4 * sizeof(int)));
    LP_CHECK(c->gerr.ensure(sizeof(int)));
    auto* pub = static_cast<unsigned long long*>(c->gw.ptr);
    int* tickets = reinterpret_cast<int*>(pub + pairs);
    const bool stall = c->stall_site == LP_STALL_GESL;
    c->stall_site = stall ? 0 : c->stall_site;
    const int e = prof_begin(c, st);
    LP_CHECK(launch_gesl_inv(dLU, lda, n, dB, ldb, nrhs, pub, tickets, static_cast<int*>(c->gerr.ptr), stall,
                             kGeslChunk, st));
    const double nn = n;
    return prof_end(c, st, LP_STAGE_GESL, e, 2.0 * nn * nn * nrhs, 4.0 * nn * nn + 16.0 * nn * nrhs);
}

int gesl_clear(lp_ctx* c, cudaStream_t st) {
    LP_CHECK(c->gerr.ensure(sizeof(int)));
    LP_CUDA(cudaMemsetAsync(c->gerr.ptr, 0, sizeof(int), st));
    return LP_OK;
}

int gesl_status(lp_ctx* c, cudaStream_t st, const char* who) {
    if (c->hstat == nullptr) LP_CUDA(cudaMallocHost(&c->hstat, sizeof(int)));
    LP_CHECK(c->gerr.ensure(sizeof(int)));
    *c->hstat = 0;
    LP_CUDA(cudaMemcpyAsync(c->hstat, c->gerr.ptr, sizeof(int), cudaMemcpyDeviceToHost, st));
    LP_CHECK(wait_stream(c, st));
    if (*c->hstat != 0)
        return fail(LP_E_TIMEOUT, std::string(who) + ": a bounded wait of the substitution sweeps expired "
                                                     "(the affected solution entries are NaN)");
    return LP_OK;
}

static float elapsed_s(cudaEvent_t a, cudaEvent_t b) {
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, a, b);
    return ms * 1e-3f;
}

}  // namespace lp

using namespace lp;

extern "C" {

const char* lp_strerror(int status) {
    switch (status) {
        case LP_OK: return "ok";
        case LP_E_INVALID: return "invalid argument";
        case LP_E_CUDA: return "CUDA error";
        case LP_E_NOMEM: return "out of memory";
        case LP_E_TIMEOUT: return "timeout";
        case LP_E_NUMERIC: return "non-finite result";
        case LP_E_STATE: return "invalid state";
        case LP_E_BUDGET: return "device-memory budget exceeded";
        case LP_E_NODEVICE: return "no CUDA device";
        default: return "unknown status";
    }
}

const char* lp_last_error(void) { return g_last_error.c_str(); }

int lp_version(void) { return LPCUDA_VERSION; }

int lp_device_count(int* count) {
    if (count == nullptr) return fail(LP_E_INVALID, "lp_device_count: null output");
    *count = 0;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return cuda_fail(e, "cudaGetDeviceCount", __FILE__, __LINE__) == LP_E_CUDA ? LP_E_NODEVICE : LP_E_NODEVICE;
    }
    *count = n;
    return LP_OK;
}

int lp_ctx_create(int device, lp_ctx** out) {
    if (out == nullptr) return fail(LP_E_INVALID, "lp_ctx_create: null output");
    *out = nullptr;
    int count = 0;
    LP_CHECK(lp_device_count(&count));
    if (device < 0 || device >= count) return fail(LP_E_NODEVICE, "lp_ctx_create: no such CUDA device");
    LP_CUDA(cudaSetDevice(device));
    cudaDeviceProp prop;
    LP_CUDA(cudaGetDeviceProperties(&prop, device));
    if (prop.major < 10)
        return fail(LP_E_NODEVICE, std::string("lp_ctx_create: device '") + prop.name +
                                       "' is not sm_100 (this library is built for sm_100a only)");
    LP_CHECK(lu_init_attrs());
    LP_CHECK(trsm_init_attrs());
    LP_CHECK(sgemm_init_attrs());
    LP_CHECK(gesl_inv_init_attrs());
    LP_CHECK(umma_init_attrs());
    LP_CHECK(batch_init_attrs());
    LP_CHECK(piv_init_attrs());
    LP_CHECK(dgemm_init_attrs());
    lp_ctx* c = new lp_ctx();
    c->device = device;
    c->num_sms = prop.multiProcessorCount;
    std::snprintf(c->name, sizeof(c->name), "%s", prop.name);
    int prio_lo = 0, prio_hi = 0;
    cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi);
    cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&c->aux, cudaStreamNonBlocking, prio_hi);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&c->aux2, cudaStreamNonBlocking, prio_hi);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_side, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_side_done, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_block, cudaEventDisableTiming | cudaEventBlockingSync);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->lane_st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&c->lane_aux, cudaStreamNonBlocking, prio_hi);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->lane_fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->lane_join, cudaEventDisableTiming);
    for (int i = 0; i < 8 && e == cudaSuccess; i++) e = cudaEventCreate(&c->ev[i]);
    if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&c->inv_top, cudaStreamNonBlocking, prio_hi);
    if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&c->inv_left, cudaStreamNonBlocking, prio_hi);
    for (int i = 0; i < kMixedMaxBlock / 128 && e == cudaSuccess; i++)
        e = cudaEventCreateWithFlags(&c->ev_inv[i], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_inv_top, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_inv_left, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        lp_ctx_destroy(c);
        return cuda_fail(e, "lp_ctx_create: stream/event creation", __FILE__, __LINE__);
    }
    *out = c;
    return LP_OK;
}

int lp_ctx_destroy(lp_ctx* c) {
    if (c == nullptr) return LP_OK;
    cudaSetDevice(c->device);
    if (c->stream != nullptr) cudaStreamSynchronize(c->stream);
    if (c->aux != nullptr) cudaStreamSynchronize(c->aux);
    if (c->aux2 != nullptr) cudaStreamSynchronize(c->aux2);
    if (c->copy != nullptr) cudaStreamSynchronize(c->copy);
    if (c->copy_in != nullptr) cudaStreamSynchronize(c->copy_in);
    if (c->lane_st != nullptr) cudaStreamSynchronize(c->lane_st);
    if (c->lane_aux != nullptr) cudaStreamSynchronize(c->lane_aux);
    if (c->inv_top != nullptr) cudaStreamSynchronize(c->inv_top);
    if (c->inv_left != nullptr) cudaStreamSynchronize(c->inv_left);
    c->release_all();
    for (int i = 0; i < kMixedMaxBlock / 128; i++)
        if (c->ev_inv[i] != nullptr) cudaEventDestroy(c->ev_inv[i]);
    if (c->ev_inv_top != nullptr) cudaEventDestroy(c->ev_inv_top);
    if (c->ev_inv_left != nullptr) cudaEventDestroy(c->ev_inv_left);
    if (c->inv_top != nullptr) cudaStreamDestroy(c->inv_top);
    if (c->inv_left != nullptr) cudaStreamDestroy(c->inv_left);
    for (int i = 0; i < 8; i++)
        if (c->ev[i] != nullptr) cudaEventDestroy(c->ev[i]);
    if (c->ev_fork != nullptr) cudaEventDestroy(c->ev_fork);
    if (c->ev_join != nullptr) cudaEventDestroy(c->ev_join);
    if (c->ev_side != nullptr) cudaEventDestroy(c->ev_side);
    if (c->ev_side_done != nullptr) cudaEventDestroy(c->ev_side_done);
    if (c->aux2 != nullptr) cudaStreamDestroy(c->aux2);
    if (c->copy != nullptr) cudaStreamDestroy(c->copy);
    if (c->copy_in != nullptr) cudaStreamDestroy(c->copy_in);
    if (c->lane_fork != nullptr) cudaEventDestroy(c->lane_fork);
    if (c->lane_join != nullptr) cudaEventDestroy(c->lane_join);
    if (c->lane_aux != nullptr) cudaStreamDestroy(c->lane_aux);
    if (c->lane_st != nullptr) cudaStreamDestroy(c->lane_st);
    if (c->ev_block != nullptr) cudaEventDestroy(c->ev_block);
    if (c->aux != nullptr) cudaStreamDestroy(c->aux);
    if (c->stream != nullptr) cudaStreamDestroy(c->stream);
    delete c;
    return LP_OK;
}

int lp_ctx_stream(lp_ctx* c, void** stream) {
    if (c == nullptr || stream == nullptr) return fail(LP_E_INVALID, "lp_ctx_stream: null argument");
    *stream = c->stream;
    return LP_OK;
}

int lp_ctx_sync(lp_ctx* c) {
    if (c == nullptr) return fail(LP_E_INVALID, "lp_ctx_sync: null context");
    LP_CUDA(cudaSetDevice(c->device));
    LP_CUDA(cudaStreamSynchronize(c->stream));
    return LP_OK;
}

int lp_ctx_device_name(lp_ctx* c, char* buf, int buflen) {
    if (c == nullptr || buf == nullptr || buflen <= 0) return fail(LP_E_INVALID, "lp_ctx_device_name: bad argument");
    std::snprintf(buf, (size_t)buflen, "%s", c->name);
    return LP_OK;
}

int lp_ctx_set_profiling(lp_ctx* c, int on) {
    if (c == nullptr) return fail(LP_E_INVALID, "lp_ctx_set_profiling: null context");
    c->prof_on = on != 0;
    return LP_OK;
}

int lp_ctx_read_profile(lp_ctx* c, lp_profile* out, int reset) {
    if (c == nullptr || out == nullptr) return fail(LP_E_INVALID, "lp_ctx_read_profile: null argument");
    LP_CUDA(cudaSetDevice(c->device));
    LP_CHECK(prof_collect(c));
    for (int k = 0; k < LP_NSTAGES; k++) {
        out->stage_s[k] = c->prof_s[k];
        out->stage_flops[k] = c->prof_flops[k];
        out->stage_bytes[k] = c->prof_bytes[k];
        out->stage_calls[k] = c->prof_calls[k];
        if (reset) {
            c->prof_s[k] = c->prof_flops[k] = c->prof_bytes[k] = 0.0;
            c->prof_calls[k] = 0;
        }
    }
    out->kernel_launches = launch_count();
    if (reset) {
        c->timeline.clear();
        c->base_recorded = false;
    }
    return LP_OK;
}

int lp_ctx_read_timeline(lp_ctx* c, lp_stage_event* out, int max, int* count) {
    if (c == nullptr || out == nullptr || count == nullptr || max < 0)
        return fail(LP_E_INVALID, "lp_ctx_read_timeline: bad argument");
    LP_CUDA(cudaSetDevice(c->device));
    LP_CHECK(prof_collect(c));
    const int k = (int)std::min<size_t>((size_t)max, c->timeline.size());
    for (int i = 0; i < k; i++) out[i] = c->timeline[i];
    *count = k;
    return LP_OK;
}

int lp_ctx_test_stall(lp_ctx* c, int site) {
    if (c == nullptr || site < 0 || site > LP_STALL_GESL) return fail(LP_E_INVALID, "lp_ctx_test_stall: bad argument");
    c->stall_site = site;
    return LP_OK;
}

int lp_host_alloc(size_t bytes, void** out) {
    if (out == nullptr || bytes == 0) return fail(LP_E_INVALID, "lp_host_alloc: bad argument");
    *out = nullptr;
    LP_CUDA(cudaHostAlloc(out, bytes, cudaHostAllocPortable));
    return LP_OK;
}

int lp_host_free(void* p) {
    if (p == nullptr) return LP_OK;
    LP_CUDA(cudaFreeHost(p));
    return LP_OK;
}

// ---- block stages -----------------------------------------------------------
int lp_lu_block_dev(lp_ctx* c, float* dA, int lda, int bs) {
    if (c == nullptr || dA == nullptr) return fail(LP_E_INVALID, "lp_lu_block_dev: null argument");
    if (!is_pow2(bs) || bs < 16 || bs > 512 || lda < bs || lda % 4 != 0)
        return fail(LP_E_INVALID, "lp_lu_block_dev: bs must be a power of two in [16, 512], lda >= bs, lda % 4 == 0");
    LP_CUDA(cudaSetDevice(c->device));
    if (bs > 128) LP_CHECK(c->lti.ensure(sizeof(float) * (size_t)128 * bs));
    return lu_stage(c, dA, lda, bs, c->stream);
}

int lp_top_update_dev(lp_ctx* c, const float* dLU, int ldlu, float* dT, int ldt, int bs, int ncols) {
    if (c == nullptr || dLU == nullptr || dT == nullptr) return fail(LP_E_INVALID, "lp_top_update_dev: null argument");
    if (ncols < 0 || ldt < ncols || ldlu < bs) return fail(LP_E_INVALID, "lp_top_update_dev: bad sizes");
    LP_CUDA(cudaSetDevice(c->device));
    return launch_trsm_top(dLU, ldlu, dT, ldt, bs, ncols, c->stream);
}

int lp_left_update_dev(lp_ctx* c, const float* dLU, int ldlu, float* dL, int ldl, int bs, int nrows, float* dLt,
                       int ldlt) {
    if (c == nullptr || dLU == nullptr || dL == nullptr) return fail(LP_E_INVALID, "lp_left_update_dev: null argument");
    if (nrows < 0 || ldl < bs || ldlu < bs || (dLt != nullptr && ldlt < nrows))
        return fail(LP_E_INVALID, "lp_left_update_dev: bad sizes");
    LP_CUDA(cudaSetDevice(c->device));
    return launch_trsm_left(dLU, ldlu, dL, ldl, bs, nrows, dLt, ldlt, c->stream);
}

int lp_inner_update_dev(lp_ctx* c, float* dC, int ldc, const float* dLt, int ldlt, const float* dT, int ldt, int m,
                        int n, int bs) {
    if (c == nullptr || dC == nullptr || dLt == nullptr || dT == nullptr)
        return fail(LP_E_INVALID, "lp_inner_update_dev: null argument");
    if (m < 0 || n < 0 || ldc < n || ldlt < m || ldt < n) return fail(LP_E_INVALID, "lp_inner_update_dev: bad sizes");
    LP_CUDA(cudaSetDevice(c->device));
    return launch_sgemm_update(dC, ldc, dLt, ldlt, dT, ldt, m, n, bs, c->stream);
}

// ---- whole factorization / solve ------------------------------------------------
int lp_gefa_dev(lp_ctx* c, float* dA, int n, int lda, int bs) {
    if (c == nullptr) return fail(LP_E_INVALID, "lp_gefa_dev: null context");
    LP_CHECK(validate_matrix(dA, n, lda, bs, "lp_gefa_dev"));
    if (!aligned16(dA)) return fail(LP_E_INVALID, "lp_gefa_dev: matrix must be 16-byte aligned");
    LP_CUDA(cudaSetDevice(c->device));
    return gefa_f32(c, dA, n, lda, bs, c->stream);
}

int lp_gesl_dev(lp_ctx* c, const float* dLU, int n, int lda, float* dB, int nrhs, int ldb) {
    if (c == nullptr || dLU == nullptr || dB == nullptr) return fail(LP_E_INVALID, "lp_gesl_dev: null argument");
    if (n <= 0 || lda < n || nrhs <= 0 || ldb < n) return fail(LP_E_INVALID, "lp_gesl_dev: bad sizes");
    if (lda % 4 != 0 || !aligned16(dLU))
        return fail(LP_E_INVALID, "lp_gesl_dev: factors must be 16-byte aligned with lda a multiple of 4");
    LP_CUDA(cudaSetDevice(c->device));
    LP_CHECK(gesl_clear(c, c->stream));
    LP_CHECK(gesl_f32(c, dLU, n, lda, dB, nrhs, ldb, c->stream));
    return gesl_status(c, c->stream, "lp_gesl_dev");
}

int lp_gefa_prec_dev(lp_ctx* c, int precision, float* dA, int n, int lda, int bs) {
    if (c == nullptr) return fail(LP_E_INVALID, "lp_gefa_prec_dev: null context");
    LP_CHECK(validate_matrix(dA, n, lda, bs, "lp_gefa_prec_dev", precision == LP_F32 ? 512 : kMixedMaxBlock));
    if (!aligned16(dA)) return fail(LP_E_INVALID, "lp_gefa_prec_dev: matrix must be 16-byte aligned");
    if (precision != LP_F32 && precision != LP_BF16_IR && precision != LP_FP8_IR && precision != LP_F32_BF16X6)
        return fail(LP_E_INVALID, "lp_gefa_prec_dev: unknown precision");
    LP_CUDA(cudaSetDevice(c->device));
    if (precision == LP_F32) return gefa_f32(c, dA, n, lda, bs, c->stream);
    return gefa_mixed(c, precision, dA, n, lda, bs, c->stream);
}

int lp_inner_update_tc_dev(lp_ctx* c, int precision, float* dC, int ldc, const float* dL, int ldl, const float* dT,
                           int ldt, int m, int n, int bs) {
    if (c == nullptr || dC == nullptr || dL == nullptr || dT == nullptr)
        return fail(LP_E_INVALID, "lp_inner_update_tc_dev: null argument");
    if (precision != LP_BF16_IR && precision != LP_FP8_IR)
        return fail(LP_E_INVALID, "lp_inner_update_tc_dev: precision must be LP_BF16_IR or LP_FP8_IR");
    const bool fp8 = precision == LP_FP8_IR;
    if (m <= 0 || n <= 0 || m % 128 || n % 128 || bs <= 0 || bs % 128 || ldc < n || ldl < bs || ldt < n ||
        ldl % 4 || !aligned16(dL))
        return fail(LP_E_INVALID, "lp_inner_update_tc_dev: m, n, bs must be positive multiples of 128");
    LP_CUDA(cudaSetDevice(c->device));
    const size_t esz = fp8 ? 1 : 2;
    const int nblk = ((m > n ? m : n) + 511) / 512;
    LP_CHECK(c->q.ensure(esz * (size_t)bs * ((size_t)m + n)));
    LP_CHECK(c->qs.ensure(6 * sizeof(float) * (size_t)kseg(bs) * nblk));
    LP_CHECK(c->err.ensure(sizeof(int)));
    uint8_t* aq = static_cast<uint8_t*>(c->q.ptr);
    uint8_t* bq = aq + esz * (size_t)bs * m;
    float* sc = static_cast<float*>(c->qs.ptr);
    cudaStream_t st = c->stream;
    LP_CUDA(cudaMemsetAsync(c->err.ptr, 0, sizeof(int), st));
    LP_CHECK(quantize_panel(dL, ldl, dT, ldt, m, n, bs, fp8, aq, bq, sc, nblk, st));
    const size_t ns = (size_t)kseg(bs) * nblk;
    LP_CHECK(launch_umma_update(dC, ldc, aq, m, bq, n, 0, 0, m, n, bs, fp8, fp8 ? sc + ns : nullptr,
                                fp8 ? sc + 4 * ns : nullptr, nblk, static_cast<int*>(c->err.ptr), st));
    int herr = 0;
    LP_CUDA(cudaMemcpyAsync(&herr, c->err.ptr, sizeof(int), cudaMemcpyDeviceToHost, st));
    LP_CUDA(cudaStreamSynchronize(st));
    if (herr != 0) return fail(LP_E_TIMEOUT, "lp_inner_update_tc_dev: a bounded wait expired in the kernel");
    return LP_OK;
}

int lp_refine_dev(lp_ctx* c, const float* dA0, int lda, const float* dLU, int n, const double* dB64, double* dX,
                  int nrhs, int max_iters, lp_timing* t) {
    if (c == nullptr || dA0 == nullptr || dLU == nullptr || dB64 == nullptr || dX == nullptr)
        return fail(LP_E_INVALID, "lp_refine_dev: null argument");
    if (n <= 0 || lda < n || lda % 4 != 0 || nrhs <= 0 || !aligned16(dLU))
        return fail(LP_E_INVALID, "lp_refine_dev: bad sizes");
    LP_CUDA(cudaSetDevice(c->device));
    cudaStream_t st = c->stream;
    LP_CUDA(cudaEventRecord(c->ev[0], st));
    int iters = 0;
    double resid = 0.0;
    const int s = refine_core(c, dA0, lda, dLU, n, dB64, dX, nrhs, max_iters, &iters, &resid, st);
    LP_CUDA(cudaEventRecord(c->ev[1], st));
    LP_CUDA(cudaStreamSynchronize(st));
    if (t != nullptr) {
        std::memset(t, 0, sizeof(*t));
        t->ir_s = elapsed_s(c->ev[0], c->ev[1]);
        t->ir_iters = iters;
        t->hpl_resid = resid;
    }
    return s;
}

// ---- host entry points --------------------------------------------------------------
int lp_calculate(lp_ctx* c, int n, int lda, int bs, int repetitions, float* A, float* b, double* gefa_times,
                 double* gesl_times) {
    if (c == nullptr || b == nullptr || gefa_times == nullptr || gesl_times == nullptr)
        return fail(LP_E_INVALID, "lp_calculate: null argument");
    LP_CHECK(validate_matrix(A, n, lda, bs, "lp_calculate"));
    if (repetitions <= 0) return fail(LP_E_INVALID, "lp_calculate: repetitions must be positive");
    LP_CUDA(cudaSetDevice(c->device));
    const size_t abytes = sizeof(float) * (size_t)n * lda;
    c->fac_n = 0;  // dA is reused: factors of an earlier lp_factor are gone
    LP_CHECK(c->dA.ensure(abytes));
    LP_CHECK(c->dB.ensure(sizeof(float) * (size_t)n));
    float* dA = static_cast<float*>(c->dA.ptr);
    float* dB = static_cast<float*>(c->dB.ptr);
    cudaStream_t st = c->stream;
    // Page-locked A: the factorization reads A in row slabs while it runs
    // (gefa_f32_streamed), and on the last repetition every block row goes back
    // to A as soon as it is final (execution_pcie.hpp copies A to the device
    // before and back after the loop, :695-696).  Pageable A: one copy each way.
    cudaPointerAttributes pa{};
    const bool pinned = cudaPointerGetAttributes(&pa, A) == cudaSuccess && pa.type == cudaMemoryTypeHost;
    cudaGetLastError();  // an unregistered pointer may leave an error behind
    // the slab / band events, destroyed on every way out after the copy streams drained
    struct Events {
        std::vector<cudaEvent_t> v;
        lp_ctx* c = nullptr;
        ~Events() {
            if (c != nullptr && c->copy_in != nullptr) cudaStreamSynchronize(c->copy_in);
            if (c != nullptr) cudaStreamSynchronize(c->lane_st);
            if (c != nullptr && c->copy != nullptr) cudaStreamSynchronize(c->copy);
            for (auto e : v)
                if (e != nullptr) cudaEventDestroy(e);
        }
    } evs;
    if (pinned) {
        evs.c = c;
        evs.v.resize(2 * (size_t)(n / bs) + 2, nullptr);
        for (auto& e : evs.v) LP_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    int status = LP_OK;
    for (int rep = 0; rep < repetitions && status == LP_OK; rep++) {
        const bool last = rep + 1 == repetitions;
        LP_CUDA(cudaMemcpyAsync(dB, b, sizeof(float) * n, cudaMemcpyHostToDevice, st));
        if (pinned) {
            LP_CUDA(cudaEventRecord(c->ev[0], st));
            status = gefa_f32_streamed(c, A, dA, n, lda, bs, st, last ? A : nullptr, evs.v);
        } else {
            LP_CUDA(cudaMemcpyAsync(dA, A, abytes, cudaMemcpyHostToDevice, st));
            LP_CUDA(cudaEventRecord(c->ev[0], st));
            status = gefa_f32(c, dA, n, lda, bs, st);
        }
        if (status != LP_OK) break;
        LP_CUDA(cudaEventRecord(c->ev[1], st));
        status = gesl_clear(c, st);
        if (status == LP_OK) status = gesl_f32(c, dA, n, lda, dB, 1, n, st);
        if (status != LP_OK) break;
        LP_CUDA(cudaEventRecord(c->ev[2], st));
        status = gesl_status(c, st, "lp_calculate");
        if (status != LP_OK) break;
        gefa_times[rep] = elapsed_s(c->ev[0], c->ev[1]);
        gesl_times[rep] = elapsed_s(c->ev[1], c->ev[2]);
    }
    if (status == LP_OK) {
        if (!pinned) LP_CUDA(cudaMemcpyAsync(A, dA, abytes, cudaMemcpyDeviceToHost, st));
        LP_CUDA(cudaMemcpyAsync(b, dB, sizeof(float) * n, cudaMemcpyDeviceToHost, st));
        LP_CUDA(cudaStreamSynchronize(st));
    }
    if (pinned && status == LP_OK) LP_CUDA(cudaStreamSynchronize(c->copy));
    return status;
}

int lp_factor(lp_ctx* c, int precision, int n, int bs, float* A, int lda, lp_timing* t) {
    if (c == nullptr) return fail(LP_E_INVALID, "lp_factor: null context");
    if (precision != LP_F32 && precision != LP_BF16_IR && precision != LP_FP8_IR && precision != LP_F32_BF16X6)
        return fail(LP_E_INVALID, "lp_factor: unknown precision");
    LP_CHECK(validate_matrix(A, n, lda, bs, "lp_factor", precision == LP_F32 ? 512 : kMixedMaxBlock));
    LP_CUDA(cudaSetDevice(c->device));
    return factor_host_impl(c, precision, n, bs, A, lda, t);
}

int lp_solve(lp_ctx* c, int n, int nrhs, const float* B, double* X, lp_timing* t) {
    if (c == nullptr || B == nullptr || X == nullptr) return fail(LP_E_INVALID, "lp_solve: null argument");
    if (c->fac_n <= 0) return fail(LP_E_INVALID, "lp_solve: no resident factors (call lp_factor first)");
    if (n != c->fac_n) return fail(LP_E_INVALID, "lp_solve: n differs from the factored matrix");
    if (nrhs <= 0) return fail(LP_E_INVALID, "lp_solve: nrhs must be positive");
    LP_CUDA(cudaSetDevice(c->device));
    return solve_resident_impl(c, nrhs, B, X, t);
}

int lp_solve_host(lp_ctx* c, int precision, int n, int bs, float* A, int lda, const double* b64, int nrhs,
                  double* x, int max_iters, lp_timing* t) {
    if (c == nullptr || b64 == nullptr || x == nullptr) return fail(LP_E_INVALID, "lp_solve_host: null argument");
    LP_CHECK(validate_matrix(A, n, lda, bs, "lp_solve_host", precision == LP_F32 ? 512 : kMixedMaxBlock));
    if (nrhs <= 0) return fail(LP_E_INVALID, "lp_solve_host: nrhs must be positive");
    if (precision != LP_F32 && precision != LP_BF16_IR && precision != LP_FP8_IR && precision != LP_F32_BF16X6)
        return fail(LP_E_INVALID, "lp_solve_host: unknown precision");
    LP_CUDA(cudaSetDevice(c->device));
    return solve_host_impl(c, precision, n, bs, A, lda, b64, nrhs, x, max_iters, t);
}

}  // extern "C"
