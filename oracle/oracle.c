/*
 * ORACLE — test infrastructure only.  Nothing in the product (hpcc_fpga_b200/,
 * include/, the lp_bench harness) links, loads or calls this file; only
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg do, and only
 * as the checker.
 *
 * A plain-C restatement of HPCC_FPGA LINPACK's CPU arithmetic for the
 * LU-without-pivoting path, written from the reference's behaviour:
 *
 *   storage convention: S[r][c] = a[r*lda + c]; the factored matrix is
 *   M = S^T (M(i,j) = a[j*lda + i]), b = M * ones.
 *
 * Pinned bit-for-bit against the reference's own gefa_ref_nopvt /
 * gesl_ref_nopvt compiled from LINPACK/src/host/linpack_data.cpp (see
 * oracle/Makefile, tests/test_oracle.py) and against the committed golden
 * vectors in tests/golden/.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* LINPACK/src/host/linpack_data.cpp:166-196 (gefa_ref_nopvt).
 * Step k: the diagonal becomes -1/d, the rest of storage row k is scaled by
 * it (negated multipliers), and every storage row j>k receives
 * S[j][i] += S[k][i] * S[j][k] for i>k. */
#define GEFA_BODY(T)                                                        \
    for (int k = 0; k < n; k++) {                                           \
        T* rowk = a + (size_t)k * lda;                                      \
        rowk[k] = (T)(-1.0 / rowk[k]);                                      \
        const T inv = rowk[k];                                              \
        for (int i = k + 1; i < n; i++) rowk[i] *= inv;                     \
        for (int j = k + 1; j < n; j++) {                                   \
            T* rowj = a + (size_t)j * lda;                                  \
            const T s = rowj[k];                                            \
            for (int i = k + 1; i < n; i++) rowj[i] += rowk[i] * s;         \
        }                                                                   \
    }

void orc_gefa_nopvt_f32(float* a, int n, int lda) { GEFA_BODY(float) }
void orc_gefa_nopvt_f64(double* a, int n, int lda) { GEFA_BODY(double) }

/* LINPACK/src/host/linpack_data.cpp:199-229 (gesl_ref_nopvt).
 * Forward: y[i] += y[k] * S[k][i] (i>k).  Backward: s = y[k] * S[k][k]
 * (S[k][k] holds -1/d), x[k] = -s, x[i] += s * S[k][i] (i<k). */
#define GESL_BODY(T)                                                        \
    T* y = (T*)malloc(sizeof(T) * (size_t)(n > 0 ? n : 1));                 \
    for (int k = 0; k < n; k++) y[k] = b[k];                                \
    for (int k = 0; k < n - 1; k++) {                                       \
        const T* rowk = a + (size_t)k * lda;                                \
        const T yk = y[k];                                                  \
        for (int i = k + 1; i < n; i++) y[i] += yk * rowk[i];               \
    }                                                                       \
    for (int k = n - 1; k >= 0; k--) {                                      \
        const T* rowk = a + (size_t)k * lda;                                \
        const T s = y[k] * rowk[k];                                         \
        y[k] = -s;                                                          \
        for (int i = 0; i < k; i++) y[i] += s * rowk[i];                    \
    }                                                                       \
    for (int k = 0; k < n; k++) b[k] = y[k];                                \
    free(y);

void orc_gesl_nopvt_f32(const float* a, float* b, int n, int lda) { GESL_BODY(float) }
void orc_gesl_nopvt_f64(const double* a, double* b, int n, int lda) { GESL_BODY(double) }

/* LINPACK/src/host/linpack_data.cpp:72-117 (gefa_ref, partial pivoting,
 * LINPACK dgefa convention).  Step k (k < n-1): the pivot is the first
 * largest |S[k][i]|, i >= k (M's column k, a strict "<" scan, so the first
 * of equal magnitudes wins and a NaN never displaces the running maximum);
 * storage rows i >= k exchange entries k and p (M's rows k and p, columns
 * >= k only: earlier multipliers stay where they were computed); storage
 * row k's entries i > k are scaled by -1/d (the reciprocal taken in double,
 * the product rounded to T); every storage row j > k receives
 * S[j][i] += S[k][i] * S[j][k] for i > k.  The diagonal keeps d. */
#define GEFA_PVT_BODY(T)                                                    \
    for (int i = 0; i < n; i++) ipvt[i] = i;                                \
    for (int k = 0; k + 1 < n; k++) {                                       \
        T* rowk = a + (size_t)k * lda;                                      \
        int p = k;                                                          \
        T best = (T)fabs((double)rowk[k]);                                  \
        for (int i = k + 1; i < n; i++) {                                   \
            const T v = (T)fabs((double)rowk[i]);                           \
            if (best < v) { best = v; p = i; }                              \
        }                                                                   \
        for (int j = k; j < n; j++) {                                       \
            T* rowj = a + (size_t)j * lda;                                  \
            const T t = rowj[k]; rowj[k] = rowj[p]; rowj[p] = t;            \
        }                                                                   \
        ipvt[k] = p;                                                        \
        const double s = -1.0 / (double)rowk[k];                            \
        for (int i = k + 1; i < n; i++) rowk[i] = (T)((double)rowk[i] * s); \
        for (int j = k + 1; j < n; j++) {                                   \
            T* rowj = a + (size_t)j * lda;                                  \
            const T f = rowj[k];                                            \
            for (int i = k + 1; i < n; i++) rowj[i] += rowk[i] * f;         \
        }                                                                   \
    }

void orc_gefa_pvt_f32(float* a, int n, int lda, int* ipvt) { GEFA_PVT_BODY(float) }
void orc_gefa_pvt_f64(double* a, int n, int lda, int* ipvt) { GEFA_PVT_BODY(double) }

/* LINPACK/src/host/linpack_data.cpp:119-156 (gesl_ref).  Forward: for
 * k < n-1, exchange y[k] and y[ipvt[k]], then y[i] += y[k] * S[k][i] (i > k).
 * Backward: y[k] /= S[k][k]; y[i] -= y[k] * S[k][i] (i < k). */
#define GESL_PVT_BODY(T)                                                    \
    T* y = (T*)malloc(sizeof(T) * (size_t)(n > 0 ? n : 1));                 \
    for (int k = 0; k < n; k++) y[k] = b[k];                                \
    for (int k = 0; k + 1 < n; k++) {                                       \
        const int p = ipvt[k];                                              \
        if (p != k) { const T t = y[k]; y[k] = y[p]; y[p] = t; }            \
        const T* rowk = a + (size_t)k * lda;                                \
        for (int i = k + 1; i < n; i++) y[i] += y[k] * rowk[i];             \
    }                                                                       \
    for (int k = n - 1; k >= 0; k--) {                                      \
        const T* rowk = a + (size_t)k * lda;                                \
        y[k] = y[k] / rowk[k];                                              \
        for (int i = 0; i < k; i++) y[i] -= y[k] * rowk[i];                 \
    }                                                                       \
    for (int k = 0; k < n; k++) b[k] = y[k];                                \
    free(y);

void orc_gesl_pvt_f32(const float* a, float* b, const int* ipvt, int n, int lda) { GESL_PVT_BODY(float) }
void orc_gesl_pvt_f64(const double* a, double* b, const int* ipvt, int n, int lda) { GESL_PVT_BODY(double) }

/* Same solve for nrhs right-hand sides stored as rows: B[r*ldb + i]. */
void orc_gesl_nopvt_multi_f64(const double* a, double* B, int n, int lda, int nrhs, int ldb) {
    for (int r = 0; r < nrhs; r++) orc_gesl_nopvt_f64(a, B + (size_t)r * ldb, n, lda);
}

/* "top" stage: LINPACK/tests/test_kernel_communication.cpp:776-789, the host
 * loop that specifies top_update (LINPACK/src/device/hpl_torus_PCIE.cl:452-582).
 * lu is a factored b x b diagonal block; t is the b x ncols block row to its
 * right.  For k: t[k][:] *= lu[k][k]; for j>k: t[j][:] += t[k][:] * lu[j][k]. */
void orc_top_update_f32(const float* lu, int ldlu, float* t, int ldt, int b, int ncols) {
    for (int k = 0; k < b; k++) {
        float* tk = t + (size_t)k * ldt;
        const float dk = lu[(size_t)k * ldlu + k];
        for (int i = 0; i < ncols; i++) tk[i] *= dk;
        for (int j = k + 1; j < b; j++) {
            float* tj = t + (size_t)j * ldt;
            const float s = lu[(size_t)j * ldlu + k];
            for (int i = 0; i < ncols; i++) tj[i] += tk[i] * s;
        }
    }
}

/* "left" stage: LINPACK/tests/test_kernel_communication.cpp:624-631, the host
 * loop that specifies left_update (hpl_torus_PCIE.cl:588-709).  l is the
 * nrows x b block column below the diagonal block.
 * For k, every row j, i>k: l[j][i] += l[j][k] * lu[k][i]. */
void orc_left_update_f32(const float* lu, int ldlu, float* l, int ldl, int b, int nrows) {
    for (int k = 0; k < b; k++) {
        const float* luk = lu + (size_t)k * ldlu;
        for (int j = 0; j < nrows; j++) {
            float* lj = l + (size_t)j * ldl;
            const float s = lj[k];
            for (int i = k + 1; i < b; i++) lj[i] += s * luk[i];
        }
    }
}

/* "inner" stage: hpl_torus_PCIE.cl:711-865 (inner_update_mm).  C += L * T
 * with L an m x b block column (after left) and T a b x n block row (after
 * top).  The FPGA kernel forms partial sums over chunks of GEMM_BLOCK_MM = 8
 * k-values (REGISTER_BLOCK_MM_LOG = 3) and adds each chunk to C
 * (hpl_torus_PCIE.cl:822-843); the same order is kept here. */
void orc_inner_update_f32(float* c, int ldc, const float* l, int ldl, const float* t, int ldt,
                          int m, int n, int b) {
    const int chunk = 8;
    for (int k0 = 0; k0 < b; k0 += chunk) {
        const int k1 = (k0 + chunk < b) ? k0 + chunk : b;
        for (int r = 0; r < m; r++) {
            float* cr = c + (size_t)r * ldc;
            const float* lr = l + (size_t)r * ldl;
            for (int col = 0; col < n; col++) {
                float sum = 0.0f;
                for (int k = k0; k < k1; k++) sum += lr[k] * t[(size_t)k * ldt + col];
                cr[col] += sum;
            }
        }
    }
}

/* The blocked right-looking schedule of the PCIe backend
 * (LINPACK/src/host/execution_types/execution_pcie.hpp:177-641) run on the
 * host with one rank: per block row, lu on the diagonal block, top on every
 * block to its right, left on every block below it, inner on every trailing
 * block.  n must be a multiple of bs. */
void orc_blocked_gefa_f32(float* a, int n, int lda, int bs) {
    const int nb = n / bs;
    for (int kb = 0; kb < nb; kb++) {
        float* d = a + (size_t)kb * bs * lda + (size_t)kb * bs;
        orc_gefa_nopvt_f32(d, bs, lda);
        const int rest = n - (kb + 1) * bs;
        if (rest <= 0) continue;
        float* top = d + bs;
        float* left = d + (size_t)bs * lda;
        orc_top_update_f32(d, lda, top, lda, bs, rest);
        orc_left_update_f32(d, lda, left, lda, bs, rest);
        orc_inner_update_f32(left + bs, lda, left, lda, top, lda, rest, rest, bs);
    }
}

/* Reference validation: LINPACK/src/host/linpack_benchmark.hpp:395-417.
 * resid = max|x_i - 1|, residn = resid / (n * normx * eps), eps the machine
 * epsilon of the working type; normx is normb, the largest entry of the
 * original right-hand side (linpack_benchmark.hpp:294,402). */
double orc_residn_f32(const float* x, int n, double normb, double* resid_out) {
    double resid = 0.0;
    for (int i = 0; i < n; i++) {
        double e = fabs((double)x[i] - 1.0);
        resid = resid > e ? resid : e;
    }
    if (resid_out) *resid_out = resid;
    const double eps = 1.1920928955078125e-07; /* FLT_EPSILON */
    return resid / ((double)n * normb * eps);
}

/* HPL-AI scaled residual of LINPACK/src/host/gmres.c:182-193:
 * ||b - M x||_inf / ((||M||_inf ||x||_inf + ||b||_inf) * n * eps) with
 * M = S^T (storage a[r*lda + c]), so (M x)_i = sum_j a[j*lda + i] x_j and
 * ||M||_inf is the largest storage-column absolute sum.  The FP32 matrix is
 * widened exactly to double.  gmres.c uses eps = DBL_EPSILON/2; a caller
 * checking a single-precision solve passes FLT_EPSILON/2. */
double orc_hpl_resid_f32a(const float* a, int lda, int n, const double* x, const double* b,
                          double eps) {
    double* r = (double*)calloc((size_t)(n > 0 ? n : 1), sizeof(double));
    double* colabs = (double*)calloc((size_t)(n > 0 ? n : 1), sizeof(double));
    for (int j = 0; j < n; j++) {
        const float* row = a + (size_t)j * lda;
        const double xj = x[j];
        for (int i = 0; i < n; i++) {
            r[i] += (double)row[i] * xj;
            colabs[i] += fabs((double)row[i]);
        }
    }
    double rn = 0.0, an = 0.0, xn = 0.0, bn = 0.0;
    for (int i = 0; i < n; i++) {
        double ri = fabs(b[i] - r[i]);
        rn = rn > ri ? rn : ri;
        an = an > colabs[i] ? an : colabs[i];
        xn = xn > fabs(x[i]) ? xn : fabs(x[i]);
        bn = bn > fabs(b[i]) ? bn : fabs(b[i]);
    }
    free(r);
    free(colabs);
    return rn / (an * xn + bn) / (double)n / eps;
}

/* FP64 residual r = b - M x (the iterative-refinement residual, restated
 * as the FP64 GEMV that gmres.c:96-97 performs with dgemv_ref). */
void orc_residual_f64(const float* a, int lda, int n, const double* x, const double* b, double* r) {
    for (int i = 0; i < n; i++) r[i] = b[i];
    for (int j = 0; j < n; j++) {
        const float* row = a + (size_t)j * lda;
        const double xj = x[j];
        for (int i = 0; i < n; i++) r[i] -= (double)row[i] * xj;
    }
}
