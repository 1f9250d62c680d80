// Host side of the partial-pivoting path (kernels in k_pivot.cu): the
// factorization schedule, the solve, the conversion to the reference
// encoding and the C entry points declared in include/lpcuda.h.
#include <string>

#include "lp_ctx.cuh"

namespace lp {
namespace {

int piv_error(lp_ctx* c, cudaStream_t st, const char* who) {
    int herr = 0;
    LP_CUDA(cudaMemcpyAsync(&herr, static_cast<unsigned char*>(c->psync.ptr) + 4, sizeof(int),
                            cudaMemcpyDeviceToHost, st));
    LP_CHECK(wait_stream(c, st));
    if (herr != 0) return fail(LP_E_TIMEOUT, std::string(who) + ": a grid barrier did not complete in time");
    return LP_OK;
}

double event_s(cudaEvent_t a, cudaEvent_t b) {
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, a, b);
    return 1e-3 * ms;
}

int piv_validate(const void* a, int n, int lda, const char* who) {
    if (a == nullptr) return fail(LP_E_INVALID, std::string(who) + ": null matrix pointer");
    if (n <= 0 || lda < n) return fail(LP_E_INVALID, std::string(who) + ": need n > 0 and lda >= n");
    if (n > 128 && (n % 4 != 0 || lda % 4 != 0))
        return fail(LP_E_INVALID, std::string(who) + ": for n > 128, n and lda must be multiples of 4");
    return LP_OK;
}

}  // namespace

// Factorization in block form (interchanges applied to whole panel rows
// inside each panel); ipvt receives the pivots.  pb: the panel width.
int gefa_pvt_block(lp_ctx* c, float* a, int n, int lda, int* ipvt, int pb, cudaStream_t st) {
    if (n > 128 && !aligned16(a)) return fail(LP_E_INVALID, "pivoting LU: matrix must be 16-byte aligned");
    const int ldat = (n + 3) / 4 * 4;
    LP_CHECK(c->psync.ensure(piv_sync_bytes()));
    LP_CHECK(c->pat.ensure(sizeof(float) * (size_t)pb * ldat));
    unsigned char* sync = static_cast<unsigned char*>(c->psync.ptr);
    float* at = static_cast<float*>(c->pat.ptr);
    LP_CUDA(cudaMemsetAsync(sync, 0, 16, st));
    unsigned bar_base = 0;
    for (int k0 = 0; k0 < n; k0 += pb) {
        const int kb = std::min(pb, n - k0), r0 = k0 + kb, m = n - k0, rest = n - r0;
        int e = prof_begin(c, st);
        LP_CHECK(launch_piv_panel(a, lda, n, k0, kb, ipvt, sync, &bar_base, c->num_sms, st));
        LP_CHECK(prof_end(c, st, LP_STAGE_LU, e, (double)m * kb * kb, 8.0 * m * kb));
        if (rest <= 0) break;
        e = prof_begin(c, st);
        LP_CHECK(launch_piv_rows(a, lda, n, k0, pb, ipvt, at, rest, c->num_sms, st));
        LP_CHECK(prof_end(c, st, LP_STAGE_LEFT, e, (double)rest * pb * pb, 12.0 * rest * pb));
        e = prof_begin(c, st);
        LP_CHECK(launch_sgemm_update(a + (size_t)r0 * lda + r0, lda, at, rest, a + (size_t)k0 * lda + r0, lda, rest,
                                     rest, pb, st));
        LP_CHECK(prof_end(c, st, LP_STAGE_INNER, e, 2.0 * rest * rest * pb, 8.0 * rest * rest));
    }
    return piv_error(c, st, "pivoting LU");
}

// Solve with block-form factors: desc must hold the interchange permutations
// of every panel (launch_piv_desc).
int gesl_pvt_block(lp_ctx* c, const float* a, int n, int lda, int pb, const int* desc, float* b, int nrhs, int ldb,
                   cudaStream_t st) {
    LP_CHECK(c->psync.ensure(piv_sync_bytes()));
    LP_CHECK(c->pw.ensure(sizeof(float) * 3 * (size_t)n));
    unsigned char* sync = static_cast<unsigned char*>(c->psync.ptr);
    LP_CUDA(cudaMemsetAsync(sync, 0, 16, st));
    const int e = prof_begin(c, st);
    LP_CHECK(launch_piv_gesl(a, lda, n, pb, desc, b, ldb, nrhs, static_cast<float*>(c->pw.ptr), sync, c->num_sms,
                             st));
    LP_CHECK(prof_end(c, st, LP_STAGE_GESL, e, 2.0 * n * n * nrhs, 4.0 * n * n * nrhs));
    return piv_error(c, st, "pivoting solve");
}

int piv_descriptors(lp_ctx* c, const int* ipvt, int n, int pb, cudaStream_t st, int** desc) {
    const int np = (n + pb - 1) / pb;
    LP_CHECK(c->pdesc.ensure(sizeof(int) * 4 * (size_t)pb * np));
    *desc = static_cast<int*>(c->pdesc.ptr);
    return launch_piv_desc(ipvt, n, pb, *desc, st);
}

}  // namespace lp

using namespace lp;

extern "C" {

int lp_gefa_pvt_dev(lp_ctx* c, float* dA, int n, int lda, int* dIpvt) {
    if (c == nullptr || dIpvt == nullptr) return fail(LP_E_INVALID, "lp_gefa_pvt_dev: null argument");
    LP_CHECK(piv_validate(dA, n, lda, "lp_gefa_pvt_dev"));
    LP_CUDA(cudaSetDevice(c->device));
    const int pb = piv_panel_width(n, c->num_sms);
    LP_CHECK(gefa_pvt_block(c, dA, n, lda, dIpvt, pb, c->stream));
    LP_CHECK(launch_piv_convert(dA, lda, n, pb, dIpvt, true, c->stream));
    return LP_OK;
}

int lp_gesl_pvt_dev(lp_ctx* c, float* dLU, int n, int lda, const int* dIpvt, float* dB, int nrhs, int ldb) {
    if (c == nullptr || dIpvt == nullptr || dB == nullptr) return fail(LP_E_INVALID, "lp_gesl_pvt_dev: null argument");
    LP_CHECK(piv_validate(dLU, n, lda, "lp_gesl_pvt_dev"));
    if (nrhs <= 0 || ldb < n) return fail(LP_E_INVALID, "lp_gesl_pvt_dev: need nrhs > 0 and ldb >= n");
    LP_CUDA(cudaSetDevice(c->device));
    cudaStream_t st = c->stream;
    const int pb = piv_panel_width(n, c->num_sms);
    int* desc = nullptr;
    LP_CHECK(piv_descriptors(c, dIpvt, n, pb, st, &desc));
    LP_CHECK(launch_piv_convert(dLU, lda, n, pb, dIpvt, false, st));
    const int st1 = gesl_pvt_block(c, dLU, n, lda, pb, desc, dB, nrhs, ldb, st);
    // the factors go back to the reference encoding whatever the solve returned
    LP_CHECK(launch_piv_convert(dLU, lda, n, pb, dIpvt, true, st));
    return st1;
}

int lp_calculate_pvt(lp_ctx* c, int n, int lda, int repetitions, float* A, float* b, int* ipvt, double* gefa_times,
                     double* gesl_times) {
    if (c == nullptr || b == nullptr || ipvt == nullptr || gefa_times == nullptr || gesl_times == nullptr)
        return fail(LP_E_INVALID, "lp_calculate_pvt: null argument");
    LP_CHECK(piv_validate(A, n, lda, "lp_calculate_pvt"));
    if (repetitions <= 0) return fail(LP_E_INVALID, "lp_calculate_pvt: repetitions must be positive");
    LP_CUDA(cudaSetDevice(c->device));
    const size_t abytes = sizeof(float) * (size_t)n * lda;
    c->fac_n = 0;  // dA is reused: factors of an earlier lp_factor are gone
    LP_CHECK(c->dA.ensure(abytes));
    LP_CHECK(c->dB.ensure(sizeof(float) * (size_t)n));
    LP_CHECK(c->pipvt.ensure(sizeof(int) * (size_t)n));
    float* dA = static_cast<float*>(c->dA.ptr);
    float* dB = static_cast<float*>(c->dB.ptr);
    int* dP = static_cast<int*>(c->pipvt.ptr);
    cudaStream_t st = c->stream;
    const int pb = piv_panel_width(n, c->num_sms);
    for (int rep = 0; rep < repetitions; rep++) {
        LP_CUDA(cudaMemcpyAsync(dA, A, abytes, cudaMemcpyHostToDevice, st));
        LP_CUDA(cudaMemcpyAsync(dB, b, sizeof(float) * n, cudaMemcpyHostToDevice, st));
        LP_CUDA(cudaEventRecord(c->ev[0], st));
        LP_CHECK(gefa_pvt_block(c, dA, n, lda, dP, pb, st));
        LP_CUDA(cudaEventRecord(c->ev[1], st));
        int* desc = nullptr;
        LP_CHECK(piv_descriptors(c, dP, n, pb, st, &desc));
        LP_CHECK(gesl_pvt_block(c, dA, n, lda, pb, desc, dB, 1, n, st));
        LP_CUDA(cudaEventRecord(c->ev[2], st));
        // the factors in the reference encoding: part of the factorization's time
        LP_CHECK(launch_piv_convert(dA, lda, n, pb, dP, true, st));
        LP_CUDA(cudaEventRecord(c->ev[3], st));
        LP_CUDA(cudaStreamSynchronize(st));
        gefa_times[rep] = event_s(c->ev[0], c->ev[1]) + event_s(c->ev[2], c->ev[3]);
        gesl_times[rep] = event_s(c->ev[1], c->ev[2]);
    }
    LP_CUDA(cudaMemcpyAsync(A, dA, abytes, cudaMemcpyDeviceToHost, st));
    LP_CUDA(cudaMemcpyAsync(b, dB, sizeof(float) * n, cudaMemcpyDeviceToHost, st));
    LP_CUDA(cudaMemcpyAsync(ipvt, dP, sizeof(int) * n, cudaMemcpyDeviceToHost, st));
    LP_CUDA(cudaStreamSynchronize(st));
    return LP_OK;
}

}  // extern "C"
