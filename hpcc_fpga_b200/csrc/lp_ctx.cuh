// The lp_ctx object behind the opaque handle of include/lpcuda.h.
#pragma once

#include <vector>

#include "lp_common.cuh"

namespace lp {

// One profiled stage launch: events e0/e1 of the context's pool bracket it.
struct StageMark {
    int kind;
    int stream;  // 0: the context's main stream, 1: its auxiliary stream
    int e0, e1;
    double flops, bytes;
};

// A device allocation that only grows (freed on growth and at destroy).
struct Workspace {
    void* ptr = nullptr;
    size_t cap = 0;
    int ensure(size_t bytes);
    void release();
};

// bs: a power of two in [16, max_bs]; 512 is the reference's largest block
// (the FP32 path), the tensor-core schedules take up to kMixedMaxBlock.
constexpr int kMixedMaxBlock = 2048;
int validate_matrix(const void* a, int n, int lda, int bs, const char* who, int max_bs = 512);
int gefa_f32(lp_ctx* c, float* dA, int n, int lda, int bs, cudaStream_t st);
// gefa_f32 on a matrix still in page-locked host memory hA, copied in row slabs
// while the factorization runs; block rows return to host_out (if not null)
// as they become final.  ev: 2 n / bs + 2 events.
int gefa_f32_streamed(lp_ctx* c, const float* hA, float* dA, int n, int lda, int bs, cudaStream_t st,
                      float* host_out, const std::vector<cudaEvent_t>& ev);
int gefa_mixed(lp_ctx* c, int precision, float* dA, int n, int lda, int bs, cudaStream_t st);
// Panel work of block step K (lu, top, left; Lt into lt), on stream st; the
// left stage covers the rows below the diagonal block up to row_end (-1: n).
int panel_f32(lp_ctx* c, float* dA, int n, int lda, int bs, int K, float* lt, cudaStream_t st, int row_end = -1);
// E4M3: one absmax scale per 512 x 512 block (512 rows of L / columns of T by
// a 512-wide K segment); sc holds 6 arrays of kseg(k) * nblk floats.
int quantize_panel(const float* L, int ldl, const float* T, int ldt, int rows_l, int cols_t, int k, bool fp8,
                   uint8_t* aq, uint8_t* bq, float* sc, int nblk, cudaStream_t st);
inline int kseg(int k) { return (k + 511) / 512; }
// Split-BF16 operands (exact three-term split; 6 or 3 K-segments) of a block step.
int split_panel(const float* L, int ldl, const float* T, int ldt, int rows_l, int cols_t, int k, uint8_t* aq,
                uint8_t* bq, cudaStream_t st, int nseg = 6);
// The stages of panel_f32 (lp_abi.cu): lu of a diagonal block, and the top /
// left recurrences over a block row / column (Lt written into lt).  With
// `unit` the operand is the bs x bs identity: top then yields a lower and left
// an upper triangle, and each 128-wide chunk skips the columns (top) or rows
// (left) that stay exactly zero.
// Inverses of the diagonal block's two triangles for the tensor-core panel:
// top applied to the bs x bs identity (winv) and left applied to it (vinv;
// vlt: scratch for its transposed chunks), both starting from the identity.
struct TriInverses {
    float* winv;
    float* vinv;
    float* vlt;
};
// With inv (bs > 128), chunk kk of both identity recurrences runs on the
// context's inv_top / inv_left streams as soon as step kk of the lu stage has
// made block row and column kk of d final; st waits for both at the end.
int lu_stage(lp_ctx* c, float* d, int lda, int bs, cudaStream_t st, const TriInverses* inv = nullptr);
int top_blocked(lp_ctx* c, const float* d, int lda, float* t, int ldt, int bs, int ncols, cudaStream_t st,
                bool unit = false);
int left_blocked(const float* d, int lda, float* l, int ldl, int bs, int nrows, float* lt, int ldlt, cudaStream_t st,
                 bool unit = false);
// Step kk (128-wide chunk) of top_blocked / left_blocked, for bs > 128.
int top_chunk_step(lp_ctx* c, const float* d, int lda, float* t, int ldt, int bs, int ncols, int kk, cudaStream_t st,
                   bool unit);
int left_chunk_step(const float* d, int lda, float* l, int ldl, int bs, int nrows, float* lt, int ldlt, int kk,
                    cudaStream_t st, bool unit);
// E4M3 scales: scale_x[seg * sstride + block] per 512-wide K segment and
// 512-row (A) / 512-column (B) block (k_umma.cu).
int launch_umma_update(float* c, int ldc, const void* aq, int aq_rows, const void* bq, int bq_rows, int m_off,
                       int n_off, int m, int n, int k, bool fp8, const float* scale_a, const float* scale_b,
                       int sstride, int* err, cudaStream_t st);
int umma_init_attrs();
int batch_init_attrs();
int validate_batch(int count, const lp_system* systems);
// One persistent batched launch over d_sorted (device descriptors, largest n
// first).  absolute: a_off / b_off are device addresses instead of offsets
// into dA / dB; nrhs may then carry the solve-only flag (factors present).
int launch_batch(lp_ctx* c, const lp_system* d_sorted, int count, float* dA, float* dB, const lp_batch_config& cfg,
                 int* d_next, cudaStream_t st, bool absolute = false);
// The refined form: factor (trailing updates in BF16 on the tensor cores if
// bf16), solve and FP64 refinement of every system in one persistent launch.
// dA0: the original matrices (same offsets as dA); dB32: FP32 work vectors,
// dB64 / dX: FP64 right-hand sides / solutions (offsets b_off); d_iters /
// d_resid: per descriptor position.
int launch_batch_ir(lp_ctx* c, bool bf16, const lp_system* d_sorted, int count, float* dA, const float* dA0,
                    float* dB32, const double* dB64, double* dX, const lp_batch_config& cfg, int max_iters,
                    int* d_iters, double* d_resid, int* d_next, cudaStream_t st);
constexpr int kBatchSolveOnly = 1 << 8;
// x = LU \ b, then FP64 refinement against the original matrix a0 until the
// HPL scaled residual is <= 16 or max_iters refinements were made.
int refine_core(lp_ctx* c, const float* a0, int lda, const float* lu, int n, const double* b64, double* x, int nrhs,
                int max_iters, int* iters, double* resid, cudaStream_t st);
int gesl_f32(lp_ctx* c, const float* dLU, int n, int lda, float* dB, int nrhs, int ldb, cudaStream_t st);
// The sweeps of gesl_f32 accumulate their error word in the context: gesl_clear
// zeroes it (stream-ordered), gesl_status copies it back, waits for st and
// returns LP_E_TIMEOUT (naming who) if a bounded wait gave up since the clear.
int gesl_clear(lp_ctx* c, cudaStream_t st);
int gesl_status(lp_ctx* c, cudaStream_t st, const char* who);
// FP64 form (lp_fp64.cu): factorization and substitution in double.
int gefa_f64(lp_ctx* c, double* a, int n, int lda, int bs, cudaStream_t st);
int gesl_f64(lp_ctx* c, const double* a, int n, int lda, double* b, int nrhs, int ldb, cudaStream_t st);
// The same substitution in FP64 arithmetic on FP32 factors (widened exactly).
int gesl_f64_on_f32(lp_ctx* c, const float* a, int n, int lda, double* b, int nrhs, int ldb, cudaStream_t st);
// Partial pivoting (k_pivot.cu): kernels of the blocked LINPACK-convention LU.
int piv_init_attrs();
size_t piv_sync_bytes();
int piv_panel_width(int n, int sms);
int launch_piv_panel(float* a, int lda, int n, int k0, int kb, int* ipvt, unsigned char* sync, unsigned* bar_base,
                     int sms, cudaStream_t st);
int launch_piv_rows(float* a, int lda, int n, int k0, int pb, const int* ipvt, float* at, int ldat, int sms,
                    cudaStream_t st);
int launch_piv_desc(const int* ipvt, int n, int pb, int* desc, cudaStream_t st);
int launch_piv_convert(float* a, int lda, int n, int pb, const int* ipvt, bool to_reference, cudaStream_t st);
int launch_piv_gesl(const float* a, int lda, int n, int pb, const int* desc, float* b, int ldb, int nrhs, float* w,
                    unsigned char* sync, int sms, cudaStream_t st);
// Restarted left-preconditioned GMRES in FP64 (lp_gmres.cu).
int gmres_core(lp_ctx* c, const float* a0, int lda, const float* lu, int n, const double* b, double* x, int restart,
               int max_it, double tol, int* steps_out, double* resid_out, cudaStream_t st);
// Waits for the work queued on st so far without spinning a CPU core.
int wait_stream(lp_ctx* c, cudaStream_t st);
int solve_host_impl(lp_ctx* c, int precision, int n, int bs, float* A, int lda, const double* b64, int nrhs,
                    double* x, int max_iters, lp_timing* t);
// lp_factor / lp_solve: factors of a host matrix kept resident in the context
// (dA, with the original in dA0) between the two calls.
int factor_host_impl(lp_ctx* c, int precision, int n, int bs, float* A, int lda, lp_timing* t);
int solve_resident_impl(lp_ctx* c, int nrhs, const float* B, double* X, lp_timing* t);
// Refinements lp_solve allows the tensor-core precisions.
constexpr int kSolveMaxRefinements = 50;

// Stage profiling: prof_begin returns an event index (or -1 when profiling
// is off); prof_end records the closing event and the stage's work.
int prof_begin(lp_ctx* c, cudaStream_t st);
int prof_end(lp_ctx* c, cudaStream_t st, int kind, int e0, double flops, double bytes);

}  // namespace lp

struct lp_ctx {
    int device = 0;
    int num_sms = 0;
    char name[256] = {0};
    cudaStream_t stream = nullptr;
    cudaStream_t aux = nullptr;               // second (high-priority) stream for concurrent panel work
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    cudaStream_t aux2 = nullptr;              // third stream: the left update runs here beside the top update
    cudaStream_t copy = nullptr;              // device-to-host copies of finished factor bands (lp_calculate)
    cudaStream_t copy_in = nullptr;           // host-to-device copies of the matrix's row slabs (lp_calculate)
    cudaStream_t lane_st = nullptr, lane_aux = nullptr;  // second lane of the row-slab schedule
    cudaEvent_t lane_fork = nullptr, lane_join = nullptr;
    cudaEvent_t ev_side = nullptr, ev_side_done = nullptr;
    cudaEvent_t ev_block = nullptr;           // blocking-sync event: waits yield the CPU instead of spinning
    cudaEvent_t ev[8] = {nullptr};
    // tensor-core panel: the identity recurrences (inverses of the diagonal
    // block's triangles) run on these two streams beside the lu stage, 128
    // rows / columns behind it; ev_inv[kk]: step kk of the lu stage is final
    cudaStream_t inv_top = nullptr, inv_left = nullptr;
    cudaEvent_t ev_inv[lp::kMixedMaxBlock / 128] = {nullptr};
    cudaEvent_t ev_inv_top = nullptr, ev_inv_left = nullptr;
    lp::Workspace lt;    // transposed left panels (2 x bs x n, alternating by block step)
    lp::Workspace dsub;  // transposed diagonal sub-blocks of the blocked top stage (per stream)
    lp::Workspace lti;   // transposed inner left panel of the recursive lu stage (per stream)
    lp::Workspace q;     // tensor-core operands: 2 x (Lq, Tq), BF16 or E4M3, n x bs each
    lp::Workspace qs;    // E4M3 block scales (absmax, scale, 1/scale for L and T), 2 buffers
    lp::Workspace err;   // device error word of the tensor-core update (bounded waits)
    lp::Workspace tri;   // mixed panel: inverses of the diagonal block's triangles (2 x bs x bs) + Lt scratch
    lp::Workspace tq;    // mixed panel: split-BF16 operands of the top and left products
    lp::Workspace gw;    // substitution: published values of the sweeps (64-bit pairs) and their tickets
    lp::Workspace gerr;  // error word of the substitution sweeps (non-zero: a bounded wait gave up)
    int* hstat = nullptr;                     // pinned host copy of an error word
    int stall_site = 0;                       // lp_ctx_test_stall: the next wait of this site never completes
    lp::Workspace dA, dA0, dB;                // host-entry-point matrix, original copy, FP32 rhs
    int fac_n = 0, fac_lda = 0, fac_prec = -1;  // factors resident in dA (lp_factor); fac_n 0: none
    lp::Workspace dB64, dX, dR, dCol;         // FP64 rhs, solution, residual, column sums
    lp::Workspace dnorm;                      // refinement norms (device)
    unsigned long long* hnorm = nullptr;      // their pinned host copy
    size_t hnorm_cap = 0;
    lp::Workspace gmw;                        // GMRES: Krylov basis and work vectors
    double* hgm = nullptr;                    // GMRES: pinned Hessenberg column
    size_t hgm_cap = 0;
    lp::Workspace f64a, f64b, f64lt, f64w;  // FP64: host-entry matrix and rhs, transposed left panel, solve vectors
    lp::Workspace psync, pat, pdesc, pw, pipvt;  // pivoting: barrier + exchange area, transposed U12,
                                                 // interchange permutations, solve vectors, ipvt
    lp::Workspace bsys, bnext;                // batched: sorted system descriptors, work counter
    lp::Workspace bA0, bB32, bout, bsys_ir;   // refined batch: original matrices, FP32 vectors, per-system results,
                                              // sorted descriptors
    lp::Workspace hA, hB, hX;                 // host-buffer batch: device copies of A, B64, X64
    uint64_t bir_hash = 0;                    // descriptors + configuration of the cached refined graph
    cudaGraphExec_t bgraph_ir = nullptr;      // refined batched launch, captured once, replayed
    lp::Workspace tA, tB;                     // batched autotuner: scratch copies of the inputs
    uint64_t bsys_hash = 0;                   // descriptors + configuration of the cached graph
    cudaGraphExec_t bgraph = nullptr;         // batched launch, captured once, replayed
    lp_batch_config bcfg{};                   // autotuned configuration
    bool btuned = false;
    bool prof_on = false;
    std::vector<cudaEvent_t> prof_ev;         // event pool, reused after every read
    size_t prof_used = 0;
    std::vector<lp::StageMark> marks;
    std::vector<lp_stage_event> timeline;     // collected marks, relative to prof_base
    cudaEvent_t prof_base = nullptr;
    bool base_recorded = false;
    double prof_s[LP_NSTAGES] = {0}, prof_flops[LP_NSTAGES] = {0}, prof_bytes[LP_NSTAGES] = {0};
    long long prof_calls[LP_NSTAGES] = {0};
    void release_all() {
        lp::Workspace* all[] = {&lt, &dsub, &lti, &q, &qs, &err, &tri, &tq, &gw, &gerr, &dA, &dA0, &dB, &dB64, &dX, &dR, &dCol,
                                &dnorm, &gmw, &f64a, &f64b, &f64lt, &f64w, &psync, &pat, &pdesc, &pw, &pipvt, &bsys, &bnext, &tA, &tB, &bA0, &bB32, &bout, &bsys_ir, &hA, &hB, &hX};
        for (auto* w : all) w->release();
        if (bgraph != nullptr) cudaGraphExecDestroy(bgraph);
        bgraph = nullptr;
        if (bgraph_ir != nullptr) cudaGraphExecDestroy(bgraph_ir);
        bgraph_ir = nullptr;
        for (auto e : prof_ev) cudaEventDestroy(e);
        prof_ev.clear();
        if (prof_base != nullptr) cudaEventDestroy(prof_base);
        prof_base = nullptr;
        if (hnorm != nullptr) cudaFreeHost(hnorm);
        hnorm = nullptr;
        hnorm_cap = 0;
        if (hgm != nullptr) cudaFreeHost(hgm);
        hgm = nullptr;
        hgm_cap = 0;
        if (hstat != nullptr) cudaFreeHost(hstat);
        hstat = nullptr;
    }
};
