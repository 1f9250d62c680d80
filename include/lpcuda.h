/*
 * lpcuda — B200 (sm_100a) LINPACK LU-without-pivoting + substitution, with the
 * reference's partial-pivoting and double-precision variants.
 *
 * C ABI of liblpcuda.so: plain pointers and sizes, no C++ types, no
 * exceptions.  Every entry point returns an int status (LP_OK = 0, < 0 on
 * error); lp_strerror() names it and lp_last_error() gives the detail of the
 * last failure on the calling thread.
 *
 * Matrix convention (identical to HPCC_FPGA LINPACK): a matrix is a flat
 * array a[] with leading dimension lda; the factored matrix is
 * M(i,j) = a[j*lda + i]; b = M * ones.  After factorization a[] holds the
 * reference's encoding (LINPACK/src/host/linpack_data.cpp:166-196): the
 * diagonal holds -1/u_kk, storage row k right of the diagonal the negated
 * multipliers, storage column k below the diagonal U, unscaled.
 *
 * Functions named *_dev take device pointers and are ordered on the
 * context's CUDA stream (lp_ctx_stream); the others take host pointers and
 * return after the work is done.
 */
#ifndef LPCUDA_H
#define LPCUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LPCUDA_VERSION 100

/* Status codes. */
#define LP_OK 0
#define LP_E_INVALID (-1)   /* bad argument (size, block size, alignment, null) */
#define LP_E_CUDA (-2)      /* a CUDA runtime call failed */
#define LP_E_NOMEM (-3)     /* device or host allocation failed */
#define LP_E_TIMEOUT (-4)   /* a bounded wait expired */
#define LP_E_NUMERIC (-5)   /* non-finite pivot or result */
#define LP_E_STATE (-6)     /* call not valid in the object's current state */
#define LP_E_BUDGET (-7)    /* request exceeds the device-memory budget */
#define LP_E_NODEVICE (-8)  /* no CUDA device / driver */

/* Factorization precision.  LP_F32: every stage in FP32 (the reference's
 * single-precision build).  LP_BF16_IR / LP_FP8_IR: the trailing (inner)
 * update runs on the tensor cores with operands rounded to BF16 or to FP8
 * E4M3 with one absmax scale per 512 x 512 block (512 rows of L or columns
 * of T by a 512-wide K segment), FP32 accumulation; the
 * diagonal-block LU and the triangular updates stay FP32; the solve is
 * refined in FP64 (residual and update) until the HPL scaled residual is
 * at most 16. */
typedef enum { LP_F32 = 0, LP_BF16_IR = 1, LP_FP8_IR = 2, LP_F32_BF16X6 = 3 } lp_precision;
/* LP_F32_BF16X6 (no counterpart in the reference, which computes in FP32):
 * the FP32 trailing update emulated on the BF16 tensor cores.  Every FP32
 * operand is split exactly into three BF16 terms (x = x1 + x2 + x3) and the
 * six cross products whose weight is at least 2^-16 of x1*t1 are accumulated
 * in FP32; the dropped terms are below the FP32 rounding of each product, so
 * the factors have FP32 accuracy and need no refinement (max_iters may be 0). */

typedef struct lp_ctx lp_ctx;

/* Timing and accuracy of one factor/solve, filled by the host entry points. */
typedef struct {
    double gefa_s;     /* factorization, device time (CUDA events) */
    double gesl_s;     /* forward + back substitution, device time */
    double ir_s;       /* refinement loop (residual + solves + update), device time */
    double h2d_s;      /* host->device copies */
    double d2h_s;      /* device->host copies */
    int ir_iters;      /* refinement iterations (0 for LP_F32) */
    int reserved;
    double hpl_resid;  /* HPL scaled residual of the returned x (eps = DBL_EPSILON/2), or -1 */
} lp_timing;

/* ---- errors ------------------------------------------------------------ */
const char* lp_strerror(int status);
/* Detail of the last failure on the calling thread ("" if none). */
const char* lp_last_error(void);
int lp_version(void);

/* ---- context ------------------------------------------------------------
 * Replaces the OpenCL device/context/program setup of the harness
 * (shared/include/hpcc_benchmark.hpp:560-575, shared/setup/fpga_setup.cpp)
 * with one CUDA device, stream and workspace. */
int lp_device_count(int* count);
int lp_ctx_create(int device, lp_ctx** out);
int lp_ctx_destroy(lp_ctx* ctx);
/* The cudaStream_t the *_dev calls are ordered on (as void*). */
int lp_ctx_stream(lp_ctx* ctx, void** stream);
int lp_ctx_sync(lp_ctx* ctx);
/* Name of the device ("NVIDIA B200"), for the JSON "device" key
 * (hpcc_benchmark.hpp:501 getDeviceName). */
int lp_ctx_device_name(lp_ctx* ctx, char* buf, int buflen);
/* Page-locked host memory for matrices and vectors (the reference allocates
 * them 4096-aligned with posix_memalign, linpack_data.hpp:196-198); pinned
 * buffers make the host<->device copies of lp_calculate run at full speed. */
int lp_host_alloc(size_t bytes, void** out);
int lp_host_free(void* p);

/* ---- profiling -------------------------------------------------------------
 * Per-stage device times (CUDA events recorded around every stage launch on
 * the context's stream while profiling is on) and the algorithmic work of
 * those launches; replaces the reference's std::chrono wall clocks around
 * the whole loop (execution_pcie.hpp:158-169,649-669). */
#define LP_STAGE_LU 0
#define LP_STAGE_TOP 1
#define LP_STAGE_LEFT 2
#define LP_STAGE_INNER 3
#define LP_STAGE_GESL 4
#define LP_STAGE_OTHER 5
#define LP_NSTAGES 6
typedef struct {
    double stage_s[LP_NSTAGES];      /* summed device time per stage */
    double stage_flops[LP_NSTAGES];  /* algorithmic flops of those launches */
    double stage_bytes[LP_NSTAGES];  /* algorithmic HBM bytes of those launches */
    long long stage_calls[LP_NSTAGES];
    long long kernel_launches;       /* kernels launched through this library by the process (cumulative) */
} lp_profile;
int lp_ctx_set_profiling(lp_ctx* ctx, int on);
/* Waits for the context's streams, fills out, and clears the stage sums (and
 * the timeline below) if reset. */
int lp_ctx_read_profile(lp_ctx* ctx, lp_profile* out, int reset);
/* One profiled stage launch: when it started and ended on the device, in
 * seconds after the first stage recorded since the last reset, and on which
 * stream (0: the context's main stream, 1: its auxiliary stream, where the
 * look-ahead panel runs). */
typedef struct {
    int stage;                       /* LP_STAGE_* */
    int stream;
    double t0_s, t1_s;
} lp_stage_event;
/* Copies up to max entries of the stage timeline into out (*count of them). */
int lp_ctx_read_timeline(lp_ctx* ctx, lp_stage_event* out, int max, int* count);

/* ---- failure-path test hook (no counterpart in the reference) ------------
 * Every wait inside this library's kernels is bounded: a kernel that gives up
 * records an error word, finishes without touching memory it does not own,
 * and the entry point returns LP_E_TIMEOUT with the context still usable.
 * lp_ctx_test_stall arms that path for tests: the next substitution sweep on
 * this context (LP_STALL_GESL) makes one tile wait on a word that nothing
 * sets, so its bounded wait (250 ms) runs out; the call then returns
 * LP_E_TIMEOUT and the affected solution entries are NaN.  The stall is used
 * once; site 0 disarms it. */
#define LP_STALL_NONE 0
#define LP_STALL_GESL 1
int lp_ctx_test_stall(lp_ctx* ctx, int site);

/* ---- block stages (device pointers) -------------------------------------
 * The four kernels of LINPACK/src/device/hpl_torus_PCIE.cl, as whole-panel
 * launches.  bs is the block size (power of two, 16..512). */

/* lu: factor the bs x bs diagonal block at dA in place
 * (hpl_torus_PCIE.cl:211-446; arithmetic of linpack_data.cpp:166-196). */
int lp_lu_block_dev(lp_ctx* ctx, float* dA, int lda, int bs);
/* top: update the bs x ncols block row right of a factored diagonal block
 * (hpl_torus_PCIE.cl:452-582; host loop test_kernel_communication.cpp:776-789). */
int lp_top_update_dev(lp_ctx* ctx, const float* dLU, int ldlu, float* dT, int ldt, int bs, int ncols);
/* left: update the nrows x bs block column below a factored diagonal block
 * (hpl_torus_PCIE.cl:588-709; host loop test_kernel_communication.cpp:624-631).
 * If dLt is not NULL the result is also written transposed (dLt[k*ldlt + r]),
 * the operand layout of the inner update (the reference's left_block copy,
 * hpl_torus_PCIE.cl:697-708). */
int lp_left_update_dev(lp_ctx* ctx, const float* dLU, int ldlu, float* dL, int ldl, int bs, int nrows,
                       float* dLt, int ldlt);
/* inner: C(m x n) += L(m x bs) * T(bs x n), FP32
 * (inner_update_mm, hpl_torus_PCIE.cl:711-865).  L is given transposed
 * (dLt: bs x m, leading dimension ldlt). */
int lp_inner_update_dev(lp_ctx* ctx, float* dC, int ldc, const float* dLt, int ldlt, const float* dT, int ldt,
                        int m, int n, int bs);

/* inner on the tensor cores: C(m x n) += L(m x bs) * T(bs x n) with L and T
 * rounded to BF16 (LP_BF16_IR) or to E4M3 with one absmax scale per 512 x 512
 * block (LP_FP8_IR: per 512 rows of L, or columns of T, by 512-wide K
 * segment; bs above 512 must be a multiple of 512), FP32 accumulation —
 * the mixed-precision form of inner_update_mm (hpl_torus_PCIE.cl:711-865).
 * L is given row-major (ldl), T row-major (ldt); m, n, bs multiples of 128.
 * Returns LP_E_TIMEOUT if a bounded wait inside the kernel expired. */
int lp_inner_update_tc_dev(lp_ctx* ctx, int precision, float* dC, int ldc, const float* dL, int ldl,
                           const float* dT, int ldt, int m, int n, int bs);

/* ---- whole factorization and solve (device pointers) -------------------- */
/* Blocked right-looking LU without pivoting of the n x n matrix at dA, in
 * place, in the reference encoding.  Replaces the block-row loop of
 * execution::pcie::calculate (execution_types/execution_pcie.hpp:177-641).
 * n must be a multiple of bs. */
int lp_gefa_dev(lp_ctx* ctx, float* dA, int n, int lda, int bs);
/* The same factorization with the trailing updates in the chosen precision
 * (LP_F32: identical to lp_gefa_dev, bs 16..512; LP_BF16_IR / LP_FP8_IR /
 * LP_F32_BF16X6: tensor-core trailing updates and top/left products, bs a
 * power of two in 128..2048 — a wider block cuts the FP32 traffic of the
 * trailing updates; the factors stay FP32). */
int lp_gefa_prec_dev(lp_ctx* ctx, int precision, float* dA, int n, int lda, int bs);
/* x = LU \ b followed by FP64 iterative refinement: r = b - M x with the
 * original FP32 matrix dA0 widened to FP64, d = LU \ r, x += d, until the
 * HPL scaled residual (LINPACK/src/host/gmres.c:182-193, eps = DBL_EPSILON/2)
 * is <= 16 or max_iters refinements were made.  dB64, dX: nrhs rows of n
 * doubles.  t (optional) receives ir_s, ir_iters and hpl_resid. */
int lp_refine_dev(lp_ctx* ctx, const float* dA0, int lda, const float* dLU, int n, const double* dB64, double* dX,
                  int nrhs, int max_iters, lp_timing* t);
/* GMRES-based refinement: the reference's gmres_ref
 * (LINPACK/src/host/gmres.c:53-232) with the factors at dLU (any precision of
 * lp_gefa_prec_dev) as left preconditioner: restarted GMRES in FP64 on
 * LU^-1 A x = LU^-1 b, A the original FP32 matrix dA0 widened to FP64.  dX
 * holds the initial guess on entry (gmres_ref's x) and the solution on return;
 * stops when the preconditioned residual estimate is <= tol * |b| and the HPL
 * scaled residual (eps = DBL_EPSILON/2) is <= 16, or after max_it restart
 * cycles of `restart` steps.  t (optional): ir_s, ir_iters = Arnoldi steps,
 * hpl_resid.  One right-hand side. */
int lp_gmres_dev(lp_ctx* ctx, const float* dA0, int lda, const float* dLU, int n, const double* dB64, double* dX,
                 int restart, int max_it, double tol, lp_timing* t);
/* Forward + back substitution with the encoded factors for nrhs right-hand
 * sides stored as rows of dB (dB[r*ldb + i]); the solutions overwrite dB.
 * Device version of gesl_ref_nopvt (linpack_data.cpp:199-229).  Returns once
 * the solve has finished on the device: it reads back the sweeps' error word
 * and returns LP_E_TIMEOUT if one of their bounded waits expired. */
int lp_gesl_dev(lp_ctx* ctx, const float* dLU, int n, int lda, float* dB, int nrhs, int ldb);

/* The same substitution for callers that cannot allocate device memory: no
 * counterpart in the reference.  Some callers must not call cudaMalloc or
 * cudaFree — code that hands all device memory to its own pool, code that
 * records CUDA graphs or runs inside a latency-bound serving loop (where an
 * allocation can synchronize the device), or a plugin host that forbids it.
 * This entry point allocates nothing and needs no lp_ctx.  It runs the same
 * two persistent sweeps as lp_gesl_dev, whose only global scratch is the
 * array of values the sweeps publish to one another (one 64-bit word per
 * unknown and right-hand side of a 16-wide group, plus the partial sums of
 * the chunk items that stream the late tiles' long source ranges); here that
 * array is one fixed device array of 2^19 words (4 MiB, plus 16 bytes of
 * counters) that every GPU which loads the library holds until the process
 * exits.  Where the chunks' sums fit beside the values the result is
 * bit-identical to lp_gesl_dev's; otherwise the sweeps run without chunk
 * items (slower at large n, summed in another order), which accepts
 * ceil(n / 128) * 128 * min(nrhs, 16) <= 524288 (n <= 32768 with 16 or more
 * right-hand sides, n <= 524288 with one); beyond that it returns
 * LP_E_INVALID.  Unlike lp_gesl_dev it does not wait for the device, so it
 * cannot report a bounded wait of the sweeps that ran out: the affected
 * solution entries are then NaN.
 * The first call on a device (the current device) looks up the array's
 * address and sets kernel attributes for that device; make that first call
 * before any stream capture.  The address is looked up in, and cached for, the
 * device's primary context (the one the CUDA runtime uses): a caller that
 * drives the device through another driver-API context must not use this
 * entry point.  All calls share the array and each call fully rewrites what
 * it reads, but calls whose work overlaps on the GPU (other streams, other
 * threads, same device) race on it: serialize them.
 * stream: a cudaStream_t, or NULL for the default stream.  dLU, dB as for
 * lp_gesl_dev; the solutions overwrite dB. */
int lp_gesl_dev_noalloc(const float* dLU, int n, int lda, float* dB, int nrhs, int ldb, void* stream);

/* ---- FP64 (the reference's _DP build; device pointers) --------------------
 * The same blocked LU without pivoting and the same encoding in double
 * (DATA_TYPE / HOST_DATA_TYPE double, LINPACK/src/host/parameters.h.in):
 * gefa_ref_nopvt / gesl_ref_nopvt of the double build.  bs 64, 128 or 256, n a
 * multiple of bs, lda even, dA 16-byte aligned. */
int lp_gefa_f64_dev(lp_ctx* ctx, double* dA, int n, int lda, int bs);
/* Forward + back substitution, nrhs right-hand sides as rows of dB. */
int lp_gesl_f64_dev(lp_ctx* ctx, const double* dLU, int n, int lda, double* dB, int nrhs, int ldb);

/* ---- LU with partial pivoting (device pointers) ------------------------------
 * The reference's gefa_ref / gesl_ref (LINPACK/src/host/linpack_data.cpp:72-156),
 * which its harness uses for matrices that are not diagonally dominant
 * (the --uniform option, linpack_benchmark.hpp:69, 440-447).  LINPACK
 * convention: ipvt[k] is the row exchanged with row k at step k (the first
 * largest magnitude); the exchange of step k touches only the columns >= k
 * of M = S^T; on return the diagonal holds u_kk, the rest of each storage
 * row right of it the negated multipliers, left of it U — the bytes
 * gefa_ref leaves (up to rounding: the trailing updates are blocked).
 * For n > 128, n and lda must be multiples of 4 and dA 16-byte aligned. */
int lp_gefa_pvt_dev(lp_ctx* ctx, float* dA, int n, int lda, int* dIpvt);
/* Forward (with the interchanges) and back substitution with such factors,
 * nrhs right-hand sides as rows of dB (overwritten by the solutions).  The
 * factors are permuted in place during the call and restored exactly before
 * it returns. */
int lp_gesl_pvt_dev(lp_ctx* ctx, float* dLU, int n, int lda, const int* dIpvt, float* dB, int nrhs, int ldb);

/* ---- host entry points --------------------------------------------------- */
/* The CUDA execution backend: the drop-in for
 *   std::map<std::string, std::vector<double>> execution::pcie::calculate(
 *       const ExecutionSettings<LinpackProgramSettings,...>&, LinpackData&)
 * (LINPACK/src/host/execution_types/execution_pcie.hpp:53-728), selected by
 * LinpackBenchmark::executeKernel (linpack_benchmark.hpp:306-324).
 * For each of `repetitions`: upload A and b (untimed, execution_pcie.hpp:123-127),
 * factor (timed -> gefa_times[rep]), solve on the device (timed ->
 * gesl_times[rep]).  On return A holds the factors (execution_pcie.hpp:695-696)
 * and, unlike the reference (whose GESL runs on the host afterwards,
 * linpack_benchmark.hpp:321-323), b holds the solution x. */
int lp_calculate(lp_ctx* ctx, int n, int lda, int bs, int repetitions, float* A, float* b,
                 double* gefa_times, double* gesl_times);
/* The same backend for the double build: A, b in double, factors in
 * gefa_ref_nopvt<double>'s encoding, b -> x. */
int lp_calculate_f64(lp_ctx* ctx, int n, int lda, int bs, int repetitions, double* A, double* b,
                     double* gefa_times, double* gesl_times);
/* The same backend for matrices that are not diagonally dominant (the
 * harness's --uniform case): partial pivoting, LINPACK convention.  On return
 * A holds the factors in gefa_ref's encoding, ipvt (n entries) the pivots,
 * b the solution x.  gefa_times include putting the factors into that
 * encoding; gesl_times the forward (with interchanges) and back substitution. */
int lp_calculate_pvt(lp_ctx* ctx, int n, int lda, int repetitions, float* A, float* b, int* ipvt,
                     double* gefa_times, double* gesl_times);

/* Factor a host matrix in place and solve for host right-hand sides, with
 * the chosen precision; copies are part of the call and are timed in t.
 * For LP_F32, x = the FP32 solve widened to double; for the mixed
 * precisions, x is refined in FP64 against b64 (FP64 right-hand sides,
 * rows of length n) until the HPL scaled residual is <= 16 or max_iters.
 * bs: as for lp_gefa_prec_dev (16..512 for LP_F32, 128..2048 otherwise). */
int lp_solve_host(lp_ctx* ctx, int precision, int n, int bs, float* A, int lda, const double* b64, int nrhs,
                  double* x, int max_iters, lp_timing* t);

/* The two halves of lp_solve_host, with the factors resident in between, for
 * callers that solve several right-hand sides against one matrix.
 * lp_factor replaces the factorization half of execution::pcie::calculate:
 * the block-row loop (execution_types/execution_pcie.hpp:177-641) and the
 * copy of the factors back into data.A (:695-696).  It factors the host
 * matrix A (n x n, leading dimension lda) in the chosen precision (bs as for
 * lp_gefa_prec_dev), writes the factors back into A in the reference
 * encoding, and keeps them and the original matrix in the context.
 * t (optional): h2d_s, gefa_s, d2h_s. */
int lp_factor(lp_ctx* ctx, int precision, int n, int bs, float* A, int lda, lp_timing* t);
/* lp_solve replaces the host substitution after calculate
 * (gesl_ref_nopvt, LINPACK/src/host/linpack_data.cpp:199-229, called at
 * linpack_benchmark.hpp:321-323).  It solves with the factors of the last
 * lp_factor on this context: B (nrhs rows of n floats, host) -> X (nrhs rows
 * of n doubles, host).  LP_F32 factors: X is the FP32 substitution widened
 * to double.  Tensor-core precisions: FP64 refinement against the original
 * matrix until the HPL scaled residual is <= 16, at most 50 refinements.
 * t (optional): h2d_s, gesl_s, ir_s, d2h_s, ir_iters, hpl_resid.
 * LP_E_INVALID without resident factors or with another n.  lp_calculate,
 * lp_calculate_pvt and lp_solve_host on the same context discard the
 * resident factors. */
int lp_solve(lp_ctx* ctx, int n, int nrhs, const float* B, double* X, lp_timing* t);

/* ---- batched solves (addition: no counterpart in the reference) ------------
 * Many independent diagonally dominant systems (1 <= n <= 1024, 1 <= nrhs
 * <= 16) factored in place (reference encoding) and solved in ONE persistent
 * launch, captured in a CUDA graph and replayed when the same batch comes
 * again.  System i: A_i at dA + a_off (n x n, leading dimension lda), right-
 * hand sides at dB + b_off (nrhs rows of ldb floats), overwritten by X_i. */
typedef struct {
    int n, nrhs, lda, ldb;
    long long a_off, b_off;
} lp_system;
/* Tuning of the batched kernel: systems with n <= small_n_max (<= 128) are
 * solved whole in shared memory; larger ones with panel width nb[bucket]
 * (16 or 32) for the buckets n <= 64, 128, 256, 512, 1024; ctas_per_sm
 * persistent CTAs per SM (1..3). */
typedef struct {
    int small_n_max;
    int nb[5];
    int ctas_per_sm;
    int use_graph;       /* 1: capture the launch in a CUDA graph and replay it for the same batch */
} lp_batch_config;
typedef struct {
    double seconds;      /* device time of the launch (CUDA events) */
    double flops;        /* sum over systems of 2n^3/3 + 2*nrhs*n^2 */
    double gflops;
    double solves_per_s; /* systems per second */
    int systems;
    int graph_replayed;  /* 1 if an instantiated CUDA graph was replayed */
} lp_batch_stats;
int lp_batch_default_config(lp_batch_config* cfg);
/* cfg NULL: the configuration found by the last lp_batch_autotune on this
 * context, else the default. */
int lp_batch_solve_dev(lp_ctx* ctx, int count, const lp_system* systems, float* dA, float* dB,
                       const lp_batch_config* cfg, lp_batch_stats* stats);
/* The refined batch (no counterpart in the reference): every system of the
 * batch factored in `precision` — LP_F32: FP32 throughout; LP_BF16_IR: the
 * trailing updates of systems above small_n_max on the tensor cores with
 * operands rounded to BF16 and FP32 accumulation (warp-level MMA inside each
 * system's CTA), the diagonal blocks, the triangular stages and systems
 * solved whole in shared memory in FP32 — then solved in FP32 and refined in
 * FP64 against its original matrix (r = b - M x with M widened exactly,
 * d = LU \ r, x += d) until its HPL scaled residual (eps = DBL_EPSILON/2,
 * LINPACK/src/host/gmres.c:182-193) is <= 16 or max_iters refinements were
 * made (0: none).  Factorization, solve and refinement of every system run in
 * ONE persistent launch (with a device copy of the originals), captured in a
 * CUDA graph and replayed for the same batch when cfg->use_graph.
 * dA: the matrices as for lp_batch_solve_dev, overwritten by the factors;
 * dB64: FP64 right-hand sides (nrhs rows of ldb doubles at b_off); dX: the
 * FP64 solutions in the same layout.  ir_iters / hpl_resid (optional, host,
 * count entries, in the caller's order): refinements made and the final
 * scaled residual per system.  LP_E_NUMERIC if a solution is not finite. */
int lp_batch_solve_ir_dev(lp_ctx* ctx, int precision, int count, const lp_system* systems, float* dA,
                          const double* dB64, double* dX, int max_iters, const lp_batch_config* cfg,
                          lp_batch_stats* stats, int* ir_iters, double* hpl_resid);
/* The same over host buffers (the batch analogue of lp_solve_host): A (host,
 * packed as for the device call) is copied in, factored and written back with
 * the factors; B (host, FP64 right-hand sides) in, X (host, FP64 solutions)
 * out.  stats->seconds is the device time of the launch alone. */
int lp_batch_solve(lp_ctx* ctx, int precision, int count, const lp_system* systems, float* A, const double* B,
                   double* X, int max_iters, const lp_batch_config* cfg, lp_batch_stats* stats, int* ir_iters,
                   double* hpl_resid);
/* Times candidate configurations per size bucket on copies of the batch
 * (dA, dB are not modified) and returns the fastest in out; the result also
 * becomes the context's default for lp_batch_solve_dev(cfg = NULL). */
int lp_batch_autotune(lp_ctx* ctx, int count, const lp_system* systems, const float* dA, const float* dB,
                      lp_batch_config* out);

/* ---- serving loop (addition: no counterpart in the reference) -------------
 * A request loop on one GPU.  Requests (one diagonally dominant system,
 * 1 <= n <= 16384, 1..16 right-hand sides) are submitted at any time and
 * complete asynchronously (lp_server_poll).  In LP_SERVE_CONTINUOUS mode,
 * requests that arrive while others are on the GPU are admitted as worker
 * slots and device memory free up: systems with n <= batch_max_n gather into
 * waves of the batched kernel (one persistent launch per wave, new
 * factorizations and solves with resident factors side by side), larger ones
 * run on `slots` concurrent streams.  LP_SERVE_PER_REQUEST is the baseline:
 * one request at a time, each with the plain single-system launches.
 * Factors stay resident, keyed by the caller's matrix key, so a later request
 * with the same key and n only solves.  All device memory of the cache and
 * of in-flight requests is charged against hbm_budget_bytes; idle factors
 * are evicted least-recently-used first, a request that can never fit
 * completes with LP_E_BUDGET.  Host buffers should be pinned (lp_host_alloc)
 * so copies overlap; they must stay valid until the request completes. */
#define LP_SERVE_CONTINUOUS 0
#define LP_SERVE_PER_REQUEST 1
typedef struct lp_server lp_server;
typedef struct {
    long long hbm_budget_bytes; /* device memory for resident factors + in-flight work (default 80e9) */
    int mode;                   /* LP_SERVE_CONTINUOUS or LP_SERVE_PER_REQUEST */
    int precision;              /* LP_F32, LP_BF16_IR or LP_FP8_IR */
    int slots;                  /* concurrent large-system streams (1..16; 1 in per-request mode) */
    int batch_workers;          /* concurrent waves of the batched kernel (1..4) */
    int batch_max_n;            /* systems with n <= this (<= 1024) go to the batched kernel; 0: none */
    int batch_max_count;        /* systems per wave */
    int max_refinements;        /* FP64 refinement cap of the mixed precisions */
    int warm_n;                 /* > 0: at start every slot factors and solves an order-warm_n system so its
                                   workspaces are sized, and every wave worker sizes its scratch for the
                                   largest wave; requests up to warm_n then allocate nothing outside the pool */
    long long reserve_bytes;    /* > 0: at start the server's pool maps this much device memory and keeps it;
                                   some headroom above the budget keeps fragmentation from growing the pool
                                   (growing it stalls the device) */
    int large_n;                /* systems with n > large_n run on higher-priority streams ... */
    int large_slots;            /* ... and this many slots (at most slots - 1) take only them */
} lp_server_config;
typedef struct {
    long long key;              /* matrix identity: same key and n reuse resident factors */
    int n, nrhs;
    const float* A;             /* n x n, leading dimension lda; may be NULL if the key is resident */
    int lda;
    const float* B;             /* nrhs right-hand sides as rows of ldb floats */
    int ldb;
    double* X;                  /* solutions, nrhs rows of ldx doubles */
    int ldx;
} lp_request;
typedef struct {
    long long id;               /* from lp_server_submit */
    long long key;
    int status;                 /* LP_OK or LP_E_* of this request */
    int n, nrhs;
    int reused;                 /* 1: resident factors were used */
    int batched;                /* 1: served by a wave of the batched kernel */
    int ir_iters;               /* FP64 refinements made */
    double hpl_resid;           /* max over right-hand sides of ||b-Mx|| / ((||M|| ||x|| + ||b||) n eps), infinity
                                   norms, eps = unit roundoff of the mode: FLT_EPSILON/2 for LP_F32,
                                   DBL_EPSILON/2 for the refined precisions */
    double t_submit, t_start, t_done; /* steady-clock seconds: submitted, work started, result written */
} lp_result;
typedef struct {
    int pending;                /* submitted, not yet started */
    int running;
    int resident;               /* matrices with resident factors */
    long long used_bytes;       /* charged against the budget */
    long long completed, waves, waved_systems, evictions, rejected;
    long long pool_reserved_bytes; /* device memory the server's pool holds (in use or kept for reuse) */
    double slot_busy_s, wave_busy_s; /* summed worker time spent on requests, slot and wave workers */
} lp_server_info;
int lp_server_default_config(lp_server_config* cfg);
/* Starts the worker threads, each with its own context.  cfg NULL: default. */
int lp_server_start(int device, const lp_server_config* cfg, lp_server** out);
/* Waits for the running work, drops pending requests, frees everything. */
int lp_server_stop(lp_server* s);
/* Validates and queues one request (LP_E_INVALID for bad sizes or pointers,
 * LP_E_STATE if A is NULL and the key is not resident). */
int lp_server_submit(lp_server* s, const lp_request* req, long long* id);
/* Copies up to max finished results into out (*count of them).  Waits up to
 * timeout_ms for the first one; LP_E_TIMEOUT if none arrived. */
int lp_server_poll(lp_server* s, lp_result* out, int max, int timeout_ms, int* count);
int lp_server_get_info(lp_server* s, lp_server_info* info);
/* Load replay: submits reqs[i] at arrival_s[i] seconds after the call (the
 * calling thread keeps the schedule), collects every result into out[i], and
 * returns when all completed; LP_E_TIMEOUT if no result arrived for
 * timeout_ms.  Results must not be polled by another thread meanwhile. */
int lp_server_replay(lp_server* s, int count, const lp_request* reqs, const double* arrival_s, lp_result* out,
                     int timeout_ms);

/* ---- input generation (host only, no GPU needed) ------------------------ */
/* LinpackBenchmark::generateInputData for one rank
 * (LINPACK/src/host/linpack_benchmark.hpp:211-297): mt19937(0),
 * uniform_real_distribution<double>(0,1) narrowed to float; diagonal =
 * storage-row sum when diag_dominant; b = storage-column sums. */
int lp_generate_reference(float* A, float* b, int n, int diag_dominant, float* norma, float* normb);
/* The same for the reference's double build (HOST_DATA_TYPE double: the
 * uniform draws kept in double, sums in double). */
int lp_generate_reference_f64(double* A, double* b, int n, int diag_dominant, double* norma, double* normb);
/* Seeded benchmark-workload generator: mt19937(seed), entries
 * (u>>8)*2^-24 - 0.5; diagonal = sum|off-diagonal| + margin; b64 = M*ones in
 * FP64 (exact), b32 = (float)b64.  Either output pointer may be NULL. */
int lp_generate_baseline(float* A, double* b64, float* b32, int n, unsigned seed, double margin);

#ifdef __cplusplus
}
#endif
#endif /* LPCUDA_H */
