// GMRES-based refinement: the reference's gmres_ref
// (LINPACK/src/host/gmres.c:53-232) on the device.  Restarted GMRES on the
// left-preconditioned system  M^-1 A x = M^-1 b  in FP64, M = L U the GPU's
// factors (FP32, BF16 or FP8 trailing updates), A the original FP32 matrix
// widened exactly to FP64.  Control flow as in gmres_ref:
//   r = M^-1 (b - A x); stop if |r| / |b| < tol;
//   per restart cycle: V_0 = r / |r|, s_0 = |r|; for i < restart:
//     w = M^-1 (A V_i); orthogonalise against V_0..V_i (H(:, i));
//     H(i+1, i) = |w|; V_{i+1} = w / H(i+1, i);
//     Givens rotations on H and s; |s_{i+1}| / |b| is the residual estimate;
//     when it reaches tol: x += V y (H y = s), accept x if its HPL-AI scaled
//     residual |b - A x|_inf / (|A|_inf |x|_inf + |b|_inf) / n / (eps/2) is
//     at most 16 (gmres.c:182-193), else restore x and keep iterating;
//   at the end of a cycle without acceptance: x += V y with the whole basis.
// B200 form: the basis V (n x (restart+1)) and every n-vector stay on the
// device; A V_i is the FP64 residual kernel, M^-1 the FP64 substitution
// on the FP32 factors;
// the orthogonalisation is classical Gram-Schmidt applied twice (two
// parallel projections instead of i+1 dependent ones, as stable as the
// reference's modified Gram-Schmidt); only the (restart+1)-sized Hessenberg
// column comes back to the host each step for the rotations.
// Differences to gmres_ref, all corrections: H and the restore point x_old
// are reset per restart cycle (the reference keeps both from the first).
#include <cfloat>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "lp_ctx.cuh"

namespace lp {
namespace {

constexpr int GP = 64;    // partial sums per dot product
constexpr int GT = 256;

// partial[k * GP + p] = sum over this block's slice of V_k . w
__global__ void __launch_bounds__(GT) k_dots(const double* __restrict__ V, int n, int count,
                                             const double* __restrict__ w, double* __restrict__ partial) {
    __shared__ double red[GT / 32];
    const int k = blockIdx.x, p = blockIdx.y;
    const double* v = V + (size_t)k * n;
    double s = 0.0;
    for (int j = p * GT + threadIdx.x; j < n; j += GP * GT) s = fma(v[j], w[j], s);
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int q = 0; q < GT / 32; q++) t += red[q];
        partial[k * GP + p] = t;
    }
}

// out[k] = (accumulate ? out[k] : 0) + sum_p partial[k * GP + p], fixed order.
__global__ void k_dots_sum(const double* __restrict__ partial, int count, double* __restrict__ out, int accumulate) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    double t = 0.0;
    for (int p = 0; p < GP; p++) t += partial[k * GP + p];
    out[k] = accumulate ? out[k] + t : t;
}

// w -= sum_k h[k] V_k
__global__ void k_sub_proj(const double* __restrict__ V, int n, int count, const double* __restrict__ h,
                           double* __restrict__ w) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    double s = w[j];
    for (int k = 0; k < count; k++) s = fma(-h[k], V[(size_t)k * n + j], s);
    w[j] = s;
}

// y = x / *d
__global__ void k_scale(double* __restrict__ y, const double* __restrict__ x, const double* __restrict__ d, int n) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < n) y[j] = x[j] / *d;
}

// y = -y
__global__ void k_negate(double* __restrict__ y, int n) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < n) y[j] = -y[j];
}

// x += sum_k y[k] V_k  (y on the device)
__global__ void k_add_comb(const double* __restrict__ V, int n, int count, const double* __restrict__ y,
                           double* __restrict__ x) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    double s = x[j];
    for (int k = 0; k < count; k++) s = fma(y[k], V[(size_t)k * n + j], s);
    x[j] = s;
}

inline double from_bits(unsigned long long b) {
    double d;
    memcpy(&d, &b, sizeof d);
    return d;
}

// gmres.c:31-49 (rotmat): the Givens rotation that zeroes b in (a, b).
void rotmat(double a, double b, double* c, double* s) {
    if (b == 0.0) {
        *c = 1.0;
        *s = 0.0;
    } else if (std::fabs(b) > std::fabs(a)) {
        const double t = a / b;
        *s = 1.0 / std::sqrt(1.0 + t * t);
        *c = t * *s;
    } else {
        const double t = b / a;
        *c = 1.0 / std::sqrt(1.0 + t * t);
        *s = t * *c;
    }
}

}  // namespace

int gmres_core(lp_ctx* c, const float* a0, int lda, const float* lu, int n, const double* b, double* x, int restart,
               int max_it, double tol, int* steps_out, double* resid_out, cudaStream_t st) {
    const int m = restart < n ? restart : n;
    const size_t nn = (size_t)n;
    // device: V (m+1) n, w, t, r, x_old, zero (n each), partial, h, h2, y, norm scalars
    const size_t doubles = (size_t)(m + 1) * nn + 5 * nn + (size_t)(m + 2) * GP + 3 * (size_t)(m + 2) + 8;
    LP_CHECK(c->gmw.ensure(sizeof(double) * doubles));
    double* V = static_cast<double*>(c->gmw.ptr);
    double* w = V + (size_t)(m + 1) * nn;
    double* t = w + nn;
    double* r = t + nn;
    double* x_old = r + nn;
    double* zero = x_old + nn;
    double* partial = zero + nn;
    double* h = partial + (size_t)(m + 2) * GP;   // m + 2
    double* h2 = h + (m + 2);                     // m + 2
    double* y = h2 + (m + 2);                     // m + 2
    double* scal = y + (m + 2);                   // 8 scalars
    const size_t hcap = 2 * (size_t)m + 8;  // two projections of up to m + 1 entries and a norm
    if (c->hgm_cap < hcap) {
        if (c->hgm != nullptr) cudaFreeHost(c->hgm);
        c->hgm = nullptr;
        c->hgm_cap = 0;
        LP_CUDA(cudaMallocHost(&c->hgm, sizeof(double) * hcap));
        c->hgm_cap = hcap;
    }
    double* hh = c->hgm;
    LP_CHECK(c->dCol.ensure(sizeof(double) * nn));
    LP_CHECK(c->dnorm.ensure(sizeof(unsigned long long) * 8));
    double* dCol = static_cast<double*>(c->dCol.ptr);
    unsigned long long* dn = static_cast<unsigned long long*>(c->dnorm.ptr);
    LP_CUDA(cudaMemsetAsync(zero, 0, sizeof(double) * nn, st));
    const int vg = (n + GT - 1) / GT;

    // |v|_2 of a device vector -> host
    auto norm2 = [&](const double* v, double* out) -> int {
        k_dots<<<dim3(1, GP), GT, 0, st>>>(v, n, 1, v, partial);
        k_dots_sum<<<1, 32, 0, st>>>(partial, 1, scal, 0);
        count_launch(2);
        LP_CUDA(cudaMemcpyAsync(hh, scal, sizeof(double), cudaMemcpyDeviceToHost, st));
        LP_CHECK(wait_stream(c, st));
        *out = std::sqrt(hh[0]);
        return LP_OK;
    };
    // out = M^-1 (b - A v)   (v = x, b = rhs)   or   M^-1 (A v)   (b = zero, negated).
    // M^-1 is applied in FP64 arithmetic to the FP32 factors, so that it is one
    // fixed linear operator to FP64 accuracy (a preconditioner rounded to FP32
    // on every application would stall the Krylov iteration at FP32 accuracy).
    auto precond_residual = [&](const double* v, const double* rhs, double* out, bool negate) -> int {
        LP_CHECK(launch_residual_f64(a0, lda, n, v, n, rhs, n, out, n, 1, st));
        LP_CHECK(gesl_f64_on_f32(c, lu, n, lda, out, 1, n, st));
        if (negate) {
            k_negate<<<vg, GT, 0, st>>>(out, n);
            count_launch();
        }
        return LP_OK;
    };
    // HPL-AI scaled residual of x (gmres.c:182-190)
    LP_CHECK(launch_colabs(a0, lda, n, dCol, st));
    LP_CHECK(launch_rhs_absmax(dCol, n, n, 1, dn, st));
    LP_CHECK(launch_rhs_absmax(b, n, n, 1, dn + 1, st));
    auto hpl_resid = [&](double* out) -> int {
        LP_CHECK(launch_residual_f64(a0, lda, n, x, n, b, n, t, n, 1, st));
        LP_CHECK(launch_rhs_absmax(t, n, n, 1, dn + 2, st));
        LP_CHECK(launch_rhs_absmax(x, n, n, 1, dn + 3, st));
        LP_CUDA(cudaMemcpyAsync(hh, dn, sizeof(unsigned long long) * 4, cudaMemcpyDeviceToHost, st));
        LP_CHECK(wait_stream(c, st));
        const unsigned long long* hb = reinterpret_cast<const unsigned long long*>(hh);
        const double nA = from_bits(hb[0]), nb = from_bits(hb[1]), nr = from_bits(hb[2]), nx = from_bits(hb[3]);
        *out = nr / (nA * nx + nb) / (double)n / (DBL_EPSILON / 2.0);
        return LP_OK;
    };

    double norm_b = 0.0;
    LP_CHECK(norm2(b, &norm_b));
    if (norm_b == 0.0) norm_b = 1.0;
    LP_CHECK(precond_residual(x, b, r, false));
    double norm_r = 0.0;
    LP_CHECK(norm2(r, &norm_r));
    int steps = 0;
    double error = norm_r / norm_b;
    if (error < tol) {
        *steps_out = 0;
        return hpl_resid(resid_out);
    }
    std::vector<double> H((size_t)(m + 1) * m), cs(m), sn(m), s(m + 1);
    auto Hat = [&](int i, int j) -> double& { return H[(size_t)j * (m + 1) + i]; };
    // x += V[0..cnt) y, y = upper-triangular solve H(0:cnt, 0:cnt) y = s(0:cnt) on the host
    auto update_x = [&](int cnt) -> int {
        std::vector<double> yy(cnt);
        for (int i = cnt - 1; i >= 0; i--) {
            double acc = s[i];
            for (int k = i + 1; k < cnt; k++) acc -= Hat(i, k) * yy[k];
            yy[i] = acc / Hat(i, i);
        }
        for (int i = 0; i < cnt; i++) hh[i] = yy[i];
        LP_CUDA(cudaMemcpyAsync(y, hh, sizeof(double) * cnt, cudaMemcpyHostToDevice, st));
        k_add_comb<<<vg, GT, 0, st>>>(V, n, cnt, y, x);
        count_launch();
        LP_CHECK(wait_stream(c, st));  // hh is reused right after
        return LP_OK;
    };

    double resid = INFINITY;
    bool accepted = false;
    for (int iter = 0; iter < max_it && !accepted; iter++) {
        if (iter != 0) {
            LP_CHECK(precond_residual(x, b, r, false));
            LP_CHECK(norm2(r, &norm_r));
        }
        LP_CUDA(cudaMemcpyAsync(x_old, x, sizeof(double) * nn, cudaMemcpyDeviceToDevice, st));
        std::fill(H.begin(), H.end(), 0.0);
        std::fill(s.begin(), s.end(), 0.0);
        hh[0] = norm_r;
        LP_CUDA(cudaMemcpyAsync(scal + 1, hh, sizeof(double), cudaMemcpyHostToDevice, st));
        k_scale<<<vg, GT, 0, st>>>(V, r, scal + 1, n);
        count_launch();
        LP_CHECK(wait_stream(c, st));
        s[0] = norm_r;
        bool updated = false;
        for (int i = 0; i < m; i++) {
            steps++;
            LP_CHECK(precond_residual(V + (size_t)i * nn, zero, w, true));
            // classical Gram-Schmidt, twice: h = V^T w; w -= V h; h2 = V^T w; w -= V h2
            k_dots<<<dim3(i + 1, GP), GT, 0, st>>>(V, n, i + 1, w, partial);
            k_dots_sum<<<(i + 64) / 64, 64, 0, st>>>(partial, i + 1, h, 0);
            k_sub_proj<<<vg, GT, 0, st>>>(V, n, i + 1, h, w);
            k_dots<<<dim3(i + 1, GP), GT, 0, st>>>(V, n, i + 1, w, partial);
            k_dots_sum<<<(i + 64) / 64, 64, 0, st>>>(partial, i + 1, h2, 0);
            k_sub_proj<<<vg, GT, 0, st>>>(V, n, i + 1, h2, w);
            k_dots<<<dim3(1, GP), GT, 0, st>>>(w, n, 1, w, partial);
            k_dots_sum<<<1, 32, 0, st>>>(partial, 1, scal + 2, 0);
            count_launch(8);
            LP_CUDA(cudaMemcpyAsync(hh, h, sizeof(double) * (i + 1), cudaMemcpyDeviceToHost, st));
            LP_CUDA(cudaMemcpyAsync(hh + (i + 1), h2, sizeof(double) * (i + 1), cudaMemcpyDeviceToHost, st));
            LP_CUDA(cudaMemcpyAsync(hh + 2 * (i + 1), scal + 2, sizeof(double), cudaMemcpyDeviceToHost, st));
            LP_CHECK(wait_stream(c, st));
            for (int k = 0; k <= i; k++) Hat(k, i) = hh[k] + hh[i + 1 + k];
            const double hn = std::sqrt(hh[2 * (i + 1)]);
            Hat(i + 1, i) = hn;
            hh[0] = hn;
            LP_CUDA(cudaMemcpyAsync(scal + 1, hh, sizeof(double), cudaMemcpyHostToDevice, st));
            k_scale<<<vg, GT, 0, st>>>(V + (size_t)(i + 1) * nn, w, scal + 1, n);
            count_launch();
            // previous rotations, then this step's
            for (int k = 0; k < i; k++) {
                const double tk = cs[k] * Hat(k, i) + sn[k] * Hat(k + 1, i);
                Hat(k + 1, i) = -sn[k] * Hat(k, i) + cs[k] * Hat(k + 1, i);
                Hat(k, i) = tk;
            }
            rotmat(Hat(i, i), Hat(i + 1, i), &cs[i], &sn[i]);
            const double si = cs[i] * s[i];
            s[i + 1] = -sn[i] * s[i];
            s[i] = si;
            Hat(i, i) = cs[i] * Hat(i, i) + sn[i] * Hat(i + 1, i);
            Hat(i + 1, i) = 0.0;
            error = std::fabs(s[i + 1]) / norm_b;
            LP_CHECK(wait_stream(c, st));  // hh was the source of the copy above
            if (!std::isfinite(error)) return fail(LP_E_NUMERIC, "gmres: non-finite residual estimate");
            if (error <= tol) {
                LP_CHECK(update_x(i + 1));
                updated = true;
                LP_CHECK(hpl_resid(&resid));
                if (resid > 16.0) {  // not yet at the HPL threshold: back to x_old, keep going
                    LP_CUDA(cudaMemcpyAsync(x, x_old, sizeof(double) * nn, cudaMemcpyDeviceToDevice, st));
                    updated = false;
                    continue;
                }
                accepted = true;
                break;
            }
        }
        if (!updated && !accepted) LP_CHECK(update_x(m));
        if (accepted) break;
        LP_CHECK(precond_residual(x, b, r, false));
        LP_CHECK(norm2(r, &norm_r));
        if (norm_r / norm_b <= tol) break;
    }
    *steps_out = steps;
    return hpl_resid(resid_out);
}

}  // namespace lp

using namespace lp;

extern "C" int lp_gmres_dev(lp_ctx* c, const float* dA0, int lda, const float* dLU, int n, const double* dB64,
                            double* dX, int restart, int max_it, double tol, lp_timing* t) {
    if (c == nullptr || dA0 == nullptr || dLU == nullptr || dB64 == nullptr || dX == nullptr)
        return fail(LP_E_INVALID, "lp_gmres_dev: null argument");
    if (n <= 0 || lda < n || lda % 4 != 0 || !aligned16(dLU))
        return fail(LP_E_INVALID, "lp_gmres_dev: factors must be 16-byte aligned with lda >= n a multiple of 4");
    if (restart < 1 || max_it < 1 || !(tol > 0.0)) return fail(LP_E_INVALID, "lp_gmres_dev: need restart, max_it >= 1, tol > 0");
    LP_CUDA(cudaSetDevice(c->device));
    cudaStream_t st = c->stream;
    LP_CUDA(cudaEventRecord(c->ev[0], st));
    int steps = 0;
    double resid = -1.0;
    const int s = gmres_core(c, dA0, lda, dLU, n, dB64, dX, restart, max_it, tol, &steps, &resid, st);
    LP_CUDA(cudaEventRecord(c->ev[1], st));
    LP_CUDA(cudaEventSynchronize(c->ev[1]));
    if (t != nullptr) {
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]);
        t->ir_s = 1e-3 * ms;
        t->ir_iters = steps;
        t->hpl_resid = resid;
    }
    return s;
}
