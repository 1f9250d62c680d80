// Solve and FP64 iterative refinement:
//   x0 = LU \ b;  repeat  r = b - M x (FP64),  d = LU \ r (FP32 factors),
//   x += d (FP64)
// until the HPL scaled residual (LINPACK/src/host/gmres.c:182-193,
// eps = DBL_EPSILON/2) is <= 16 or max_iters refinements were made.  The
// residual and the update are the only FP64 steps.  lp_solve_host wraps it
// with the factorization and the host copies; lp_factor / lp_solve split the
// two, keeping the factors resident in between.
#include <cfloat>
#include <cmath>
#include <cstring>
#include <vector>

#include "lp_ctx.cuh"

namespace lp {

static float ev_s(cudaEvent_t a, cudaEvent_t b) {
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, a, b);
    return ms * 1e-3f;
}

// Bits of a non-negative double written by launch_rhs_absmax.
static double from_bits(unsigned long long b) {
    double d;
    std::memcpy(&d, &b, sizeof(d));
    return d;
}

int refine_core(lp_ctx* c, const float* a0, int lda, const float* lu, int n, const double* b64, double* x, int nrhs,
                int max_iters, int* iters_out, double* resid_out, cudaStream_t st) {
    const size_t nv = (size_t)n * nrhs;
    LP_CHECK(c->dB.ensure(sizeof(float) * nv));
    LP_CHECK(c->dR.ensure(sizeof(double) * nv));
    LP_CHECK(c->dCol.ensure(sizeof(double) * (size_t)n));
    // norm slots: [0] ||M||, [1] unused, [2, 2+q) ||b_q||, then ||r_q||, then ||x_q||
    const size_t slots = 2 + 3 * (size_t)nrhs;
    LP_CHECK(c->dnorm.ensure(sizeof(unsigned long long) * slots));
    if (c->hnorm_cap < slots) {
        if (c->hnorm != nullptr) cudaFreeHost(c->hnorm);
        c->hnorm = nullptr;
        c->hnorm_cap = 0;
        const size_t cap = slots < 64 ? 64 : slots;  // up to 20 right-hand sides without regrowth
        LP_CUDA(cudaMallocHost(&c->hnorm, sizeof(unsigned long long) * cap));
        c->hnorm_cap = cap;
    }
    float* dB = static_cast<float*>(c->dB.ptr);
    double* dR = static_cast<double*>(c->dR.ptr);
    double* dCol = static_cast<double*>(c->dCol.ptr);
    unsigned long long* dn = static_cast<unsigned long long*>(c->dnorm.ptr);
    unsigned long long* rn = dn + 2 + nrhs;
    unsigned long long* xn = rn + nrhs;

    LP_CHECK(launch_colabs(a0, lda, n, dCol, st));
    LP_CHECK(launch_rhs_absmax(dCol, n, n, 1, dn, st));
    LP_CHECK(launch_rhs_absmax(b64, n, n, nrhs, dn + 2, st));
    LP_CHECK(launch_f64_to_f32(dB, b64, nv, st));
    LP_CHECK(gesl_clear(c, st));
    LP_CHECK(gesl_f32(c, lu, n, lda, dB, nrhs, n, st));
    LP_CHECK(launch_f32_to_f64(x, dB, nv, st));
    LP_CUDA(cudaEventRecord(c->ev[4], st));  // end of the first solve

    const double eps = DBL_EPSILON / 2.0;
    double resid = INFINITY;
    int iters = 0;
    auto measure = [&]() -> int {
        LP_CHECK(launch_residual_f64(a0, lda, n, x, n, b64, n, dR, n, nrhs, st));
        LP_CHECK(launch_rhs_absmax(dR, n, n, nrhs, rn, st));
        LP_CHECK(launch_rhs_absmax(x, n, n, nrhs, xn, st));
        LP_CUDA(cudaMemcpyAsync(c->hnorm, dn, sizeof(unsigned long long) * slots, cudaMemcpyDeviceToHost, st));
        LP_CHECK(gesl_status(c, st, "refinement"));  // waits for st
        const unsigned long long* h = c->hnorm;
        const double normA = from_bits(h[0]);
        resid = 0.0;
        bool finite = std::isfinite(normA);
        for (int q = 0; q < nrhs && finite; q++) {
            const double rq = from_bits(h[2 + nrhs + q]), xq = from_bits(h[2 + 2 * nrhs + q]);
            const double r = rq / (normA * xq + from_bits(h[2 + q])) / (double)n / eps;
            if (!std::isfinite(rq) || !std::isfinite(xq) || !std::isfinite(r)) finite = false;  // fmax drops NaN
            resid = std::fmax(resid, r);
        }
        if (!finite) resid = NAN;
        return LP_OK;
    };
    LP_CHECK(measure());
    const int cap = max_iters < 0 ? 0 : max_iters;
    while (std::isfinite(resid) && resid > 16.0 && iters < cap) {
        LP_CHECK(launch_f64_to_f32(dB, dR, nv, st));
        LP_CHECK(gesl_f32(c, lu, n, lda, dB, nrhs, n, st));
        LP_CHECK(launch_axpy_f64(x, dB, nv, st));
        iters++;
        LP_CHECK(measure());
    }
    *iters_out = iters;
    *resid_out = resid;
    if (!std::isfinite(resid))
        return fail(LP_E_NUMERIC, "non-finite solution (matrix not factorable without pivoting?)");
    return LP_OK;
}

int solve_host_impl(lp_ctx* c, int precision, int n, int bs, float* A, int lda, const double* b64, int nrhs,
                    double* x, int max_iters, lp_timing* t) {
    c->fac_n = 0;  // dA / dA0 are reused below: factors of an earlier lp_factor are gone
    cudaStream_t st = c->stream;
    const size_t abytes = sizeof(float) * (size_t)n * lda;
    const size_t nv = (size_t)n * nrhs;
    LP_CHECK(c->dA.ensure(abytes));
    LP_CHECK(c->dA0.ensure(abytes));
    LP_CHECK(c->dB64.ensure(sizeof(double) * nv));
    LP_CHECK(c->dX.ensure(sizeof(double) * nv));
    float* dA = static_cast<float*>(c->dA.ptr);
    float* dA0 = static_cast<float*>(c->dA0.ptr);
    double* dB64 = static_cast<double*>(c->dB64.ptr);
    double* dX = static_cast<double*>(c->dX.ptr);

    LP_CUDA(cudaEventRecord(c->ev[0], st));
    LP_CUDA(cudaMemcpyAsync(dA0, A, abytes, cudaMemcpyHostToDevice, st));
    LP_CUDA(cudaMemcpyAsync(dB64, b64, sizeof(double) * nv, cudaMemcpyHostToDevice, st));
    LP_CUDA(cudaEventRecord(c->ev[1], st));
    LP_CUDA(cudaMemcpyAsync(dA, dA0, abytes, cudaMemcpyDeviceToDevice, st));
    LP_CUDA(cudaEventRecord(c->ev[2], st));
    if (precision == LP_F32)
        LP_CHECK(gefa_f32(c, dA, n, lda, bs, st));
    else
        LP_CHECK(gefa_mixed(c, precision, dA, n, lda, bs, st));
    LP_CUDA(cudaEventRecord(c->ev[3], st));
    int iters = 0;
    double resid = 0.0;
    const int s = refine_core(c, dA0, lda, dA, n, dB64, dX, nrhs, max_iters, &iters, &resid, st);
    LP_CUDA(cudaEventRecord(c->ev[5], st));
    LP_CUDA(cudaMemcpyAsync(x, dX, sizeof(double) * nv, cudaMemcpyDeviceToHost, st));
    LP_CUDA(cudaEventRecord(c->ev[6], st));
    LP_CUDA(cudaStreamSynchronize(st));
    if (t != nullptr) {
        t->h2d_s = ev_s(c->ev[0], c->ev[1]);
        t->gefa_s = ev_s(c->ev[2], c->ev[3]);
        t->gesl_s = ev_s(c->ev[3], c->ev[4]);
        t->ir_s = ev_s(c->ev[4], c->ev[5]);
        t->d2h_s = ev_s(c->ev[5], c->ev[6]);
        t->ir_iters = iters;
        t->hpl_resid = resid;
    }
    return s;
}

// lp_factor: A (host) -> the context's dA0 (original) and dA (factors, in
// the chosen precision), factors copied back into A.
int factor_host_impl(lp_ctx* c, int precision, int n, int bs, float* A, int lda, lp_timing* t) {
    c->fac_n = 0;
    cudaStream_t st = c->stream;
    const size_t abytes = sizeof(float) * (size_t)n * lda;
    LP_CHECK(c->dA.ensure(abytes));
    LP_CHECK(c->dA0.ensure(abytes));
    float* dA = static_cast<float*>(c->dA.ptr);
    float* dA0 = static_cast<float*>(c->dA0.ptr);
    LP_CUDA(cudaEventRecord(c->ev[0], st));
    LP_CUDA(cudaMemcpyAsync(dA0, A, abytes, cudaMemcpyHostToDevice, st));
    LP_CUDA(cudaEventRecord(c->ev[1], st));
    LP_CUDA(cudaMemcpyAsync(dA, dA0, abytes, cudaMemcpyDeviceToDevice, st));
    LP_CUDA(cudaEventRecord(c->ev[2], st));
    if (precision == LP_F32)
        LP_CHECK(gefa_f32(c, dA, n, lda, bs, st));
    else
        LP_CHECK(gefa_mixed(c, precision, dA, n, lda, bs, st));
    LP_CUDA(cudaEventRecord(c->ev[3], st));
    LP_CUDA(cudaMemcpyAsync(A, dA, abytes, cudaMemcpyDeviceToHost, st));
    LP_CUDA(cudaEventRecord(c->ev[4], st));
    LP_CUDA(cudaStreamSynchronize(st));
    c->fac_n = n;
    c->fac_lda = lda;
    c->fac_prec = precision;
    if (t != nullptr) {
        std::memset(t, 0, sizeof(*t));
        t->h2d_s = ev_s(c->ev[0], c->ev[1]);
        t->gefa_s = ev_s(c->ev[2], c->ev[3]);
        t->d2h_s = ev_s(c->ev[3], c->ev[4]);
    }
    return LP_OK;
}

// lp_solve: B (host, FP32, nrhs rows of n) -> X (host, FP64) with the
// resident factors; FP64 refinement against the original matrix for the
// tensor-core precisions, none for LP_F32 (x = the FP32 solve widened).
int solve_resident_impl(lp_ctx* c, int nrhs, const float* B, double* X, lp_timing* t) {
    cudaStream_t st = c->stream;
    const int n = c->fac_n, lda = c->fac_lda;
    const size_t nv = (size_t)n * nrhs;
    std::vector<double> b64(B, B + nv);  // FP32 right-hand sides widened exactly
    LP_CHECK(c->dB64.ensure(sizeof(double) * nv));
    LP_CHECK(c->dX.ensure(sizeof(double) * nv));
    double* dB64 = static_cast<double*>(c->dB64.ptr);
    double* dX = static_cast<double*>(c->dX.ptr);
    LP_CUDA(cudaEventRecord(c->ev[0], st));
    LP_CUDA(cudaMemcpyAsync(dB64, b64.data(), sizeof(double) * nv, cudaMemcpyHostToDevice, st));
    LP_CUDA(cudaEventRecord(c->ev[1], st));
    int iters = 0;
    double resid = 0.0;
    const int max_iters = c->fac_prec == LP_F32 ? 0 : kSolveMaxRefinements;
    const int s = refine_core(c, static_cast<const float*>(c->dA0.ptr), lda, static_cast<const float*>(c->dA.ptr), n,
                              dB64, dX, nrhs, max_iters, &iters, &resid, st);
    LP_CUDA(cudaEventRecord(c->ev[5], st));
    LP_CUDA(cudaMemcpyAsync(X, dX, sizeof(double) * nv, cudaMemcpyDeviceToHost, st));
    LP_CUDA(cudaEventRecord(c->ev[6], st));
    LP_CUDA(cudaStreamSynchronize(st));
    if (t != nullptr) {
        std::memset(t, 0, sizeof(*t));
        t->h2d_s = ev_s(c->ev[0], c->ev[1]);
        t->gesl_s = ev_s(c->ev[1], c->ev[4]);
        t->ir_s = ev_s(c->ev[4], c->ev[5]);
        t->d2h_s = ev_s(c->ev[5], c->ev[6]);
        t->ir_iters = iters;
        t->hpl_resid = resid;
    }
    return s;
}

}  // namespace lp
