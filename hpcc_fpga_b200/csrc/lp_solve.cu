// Solve and FP64 iterative refinement:
//   x0 = LU \ b;  repeat  r = b - M x (FP64),  d = LU \ r (FP32 factors),
//   x += d (FP64)
// until the HPL scaled residual (LINPACK/src/host/gmres.c:182-193,
// eps = DBL_EPSILON/2) is <= 16 or max_iters refinements were made.  The
// residual and the update are the only FP64 steps.  lp_solve_host wraps it
// with the factorization and the host copies.
#include <cfloat>
#include <cmath>
#include <vector>

#include "lp_ctx.cuh"

namespace lp {

static float ev_s(cudaEvent_t a, cudaEvent_t b) {
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, a, b);
    return ms * 1e-3f;
}

int refine_core(lp_ctx* c, const float* a0, int lda, const float* lu, int n, const double* b64, double* x, int nrhs,
                int max_iters, int* iters_out, double* resid_out, cudaStream_t st) {
    const size_t nv = (size_t)n * nrhs;
    LP_CHECK(c->dB.ensure(sizeof(float) * nv));
    LP_CHECK(c->dR.ensure(sizeof(double) * nv));
    LP_CHECK(c->dCol.ensure(sizeof(double) * (size_t)n));
    float* dB = static_cast<float*>(c->dB.ptr);
    double* dR = static_cast<double*>(c->dR.ptr);
    double* dCol = static_cast<double*>(c->dCol.ptr);

    LP_CHECK(launch_colabs(a0, lda, n, dCol, st));
    LP_CHECK(launch_f64_to_f32(dB, b64, nv, st));
    LP_CHECK(gesl_f32(c, lu, n, lda, dB, nrhs, n, st));
    LP_CHECK(launch_f32_to_f64(x, dB, nv, st));
    LP_CUDA(cudaEventRecord(c->ev[4], st));  // end of the first solve

    std::vector<double> col(n), hx(nv), hr(nv), hb(nv);
    LP_CUDA(cudaMemcpyAsync(col.data(), dCol, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    LP_CUDA(cudaMemcpyAsync(hb.data(), b64, sizeof(double) * nv, cudaMemcpyDeviceToHost, st));
    double normA = -1.0;
    std::vector<double> normb(nrhs, 0.0);

    const double eps = DBL_EPSILON / 2.0;
    double resid = INFINITY;
    int iters = 0;
    auto measure = [&]() -> int {
        LP_CHECK(launch_residual_f64(a0, lda, n, x, n, b64, n, dR, n, nrhs, st));
        LP_CUDA(cudaMemcpyAsync(hx.data(), x, sizeof(double) * nv, cudaMemcpyDeviceToHost, st));
        LP_CUDA(cudaMemcpyAsync(hr.data(), dR, sizeof(double) * nv, cudaMemcpyDeviceToHost, st));
        LP_CUDA(cudaStreamSynchronize(st));
        if (normA < 0.0) {
            normA = 0.0;
            for (int i = 0; i < n; i++) normA = std::fmax(normA, col[i]);
            for (int q = 0; q < nrhs; q++)
                for (int i = 0; i < n; i++) normb[q] = std::fmax(normb[q], std::fabs(hb[(size_t)q * n + i]));
        }
        resid = 0.0;
        bool finite = true;
        for (int q = 0; q < nrhs && finite; q++) {
            double rn = 0.0, xn = 0.0;
            for (int i = 0; i < n; i++) {
                const double ri = hr[(size_t)q * n + i], xi = hx[(size_t)q * n + i];
                if (!std::isfinite(ri) || !std::isfinite(xi)) {
                    finite = false;  // fmax would silently drop a NaN
                    break;
                }
                rn = std::fmax(rn, std::fabs(ri));
                xn = std::fmax(xn, std::fabs(xi));
            }
            const double rq = rn / (normA * xn + normb[q]) / (double)n / eps;
            if (!std::isfinite(rq)) finite = false;
            resid = std::fmax(resid, rq);
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

}  // namespace lp
