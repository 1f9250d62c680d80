// FP64 pieces of the refinement loop and of the HPL scaled residual
// (LINPACK/src/host/gmres.c:182-193):
//   residual  r = b - M x   with M = S^T, S the FP32 original matrix widened
//             exactly to double, accumulated in double (gmres.c:190-191 does
//             the same GEMV with dgemv_ref);
//   norms     ||M||_inf (largest storage-column absolute sum), max |v| per
//             right-hand side (reduced on the device, a few scalars copied back);
//   update    x += d, and the FP64 -> FP32 narrowing of r for the low-
//             precision solve.
// The residual is a GEMV over storage rows: a CTA covers 256 unknowns
// (coalesced row segments) and a chunk of rows, and adds its partial sums
// with FP64 atomics, so the whole matrix is read once at full width.
#include "lp_common.cuh"

namespace lp {
namespace {

constexpr int RT = 256;

template <int NR>
__global__ void __launch_bounds__(RT) k_residual_f64(const float* __restrict__ a, int lda, int n,
                                                     const double* __restrict__ x, int ldx, double* __restrict__ r,
                                                     int ldr, int nrhs, int rch) {
    const int i = blockIdx.x * RT + threadIdx.x;
    const int j0 = blockIdx.y * rch;
    const int j1 = min(n, j0 + rch);
    if (i >= n) return;
    double acc[NR];
#pragma unroll
    for (int q = 0; q < NR; q++) acc[q] = 0.0;
    const float* col = a + i;
#pragma unroll 4
    for (int j = j0; j < j1; j++) {
        const double v = (double)col[(size_t)j * lda];
#pragma unroll
        for (int q = 0; q < NR; q++)
            if (q < nrhs) acc[q] = fma(v, x[(size_t)q * ldx + j], acc[q]);
    }
#pragma unroll
    for (int q = 0; q < NR; q++)
        if (q < nrhs) atomicAdd(&r[(size_t)q * ldr + i], -acc[q]);
}

__global__ void __launch_bounds__(RT) k_colabs(const float* __restrict__ a, int lda, int n, double* __restrict__ out,
                                               int rch) {
    const int i = blockIdx.x * RT + threadIdx.x;
    const int j0 = blockIdx.y * rch;
    const int j1 = min(n, j0 + rch);
    if (i >= n) return;
    double acc = 0.0;
    const float* col = a + i;
#pragma unroll 4
    for (int j = j0; j < j1; j++) acc += fabs((double)col[(size_t)j * lda]);
    atomicAdd(&out[i], acc);
}

// out[q] = max |v[q*ld + i]| over i < n, for q = blockIdx.y; +infinity if any
// value is not finite (non-negative doubles compare as their bit patterns).
__global__ void __launch_bounds__(RT) k_rhs_absmax(const double* __restrict__ v, int n, int ld,
                                                 unsigned long long* out) {
    const double* vq = v + (size_t)blockIdx.y * ld;
    double m = 0.0;
    for (int i = blockIdx.x * RT + threadIdx.x; i < n; i += gridDim.x * RT) {
        const double a = vq[i];
        m = isfinite(a) ? fmax(m, fabs(a)) : INFINITY;
    }
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out + blockIdx.y, (unsigned long long)__double_as_longlong(m));
}

__global__ void k_axpy_f64(double* __restrict__ x, const float* __restrict__ d, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        x[i] += (double)d[i];
}

__global__ void k_f64_to_f32(float* __restrict__ y, const double* __restrict__ v, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        y[i] = (float)v[i];
}

__global__ void k_f32_to_f64(double* __restrict__ y, const float* __restrict__ v, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        y[i] = (double)v[i];
}

int row_chunk(int n) {
    // Enough row chunks for >= ~8 CTAs per SM on 148 SMs at large n.
    const int cols = (n + RT - 1) / RT;
    int rch = 512;
    while (rch > 64 && (long long)cols * ((n + rch - 1) / rch) < 1184) rch >>= 1;
    return rch;
}

}  // namespace

int launch_residual_f64(const float* a, int lda, int n, const double* x, int ldx, const double* b, int ldb,
                        double* r, int ldr, int nrhs, cudaStream_t st) {
    LP_CUDA(cudaMemcpy2DAsync(r, sizeof(double) * ldr, b, sizeof(double) * ldb, sizeof(double) * n, nrhs,
                              cudaMemcpyDeviceToDevice, st));
    const int rch = row_chunk(n);
    for (int q0 = 0; q0 < nrhs; q0 += 16) {
        const int g = (nrhs - q0) < 16 ? (nrhs - q0) : 16;
        const dim3 grid((n + RT - 1) / RT, (n + rch - 1) / rch);
        const double* xx = x + (size_t)q0 * ldx;
        double* rr = r + (size_t)q0 * ldr;
        if (g == 1)
            k_residual_f64<1><<<grid, RT, 0, st>>>(a, lda, n, xx, ldx, rr, ldr, g, rch);
        else if (g <= 4)
            k_residual_f64<4><<<grid, RT, 0, st>>>(a, lda, n, xx, ldx, rr, ldr, g, rch);
        else
            k_residual_f64<16><<<grid, RT, 0, st>>>(a, lda, n, xx, ldx, rr, ldr, g, rch);
    }
    count_launch();
    LP_CUDA(cudaGetLastError());
    return LP_OK;
}

int launch_colabs(const float* a, int lda, int n, double* out, cudaStream_t st) {
    LP_CUDA(cudaMemsetAsync(out, 0, sizeof(double) * n, st));
    const int rch = row_chunk(n);
    const dim3 grid((n + RT - 1) / RT, (n + rch - 1) / rch);
    k_colabs<<<grid, RT, 0, st>>>(a, lda, n, out, rch);
    count_launch();
    LP_CUDA(cudaGetLastError());
    return LP_OK;
}

int launch_rhs_absmax(const double* v, int n, int ld, int nrhs, unsigned long long* out, cudaStream_t st) {
    LP_CUDA(cudaMemsetAsync(out, 0, sizeof(unsigned long long) * nrhs, st));
    int gx = (n + RT - 1) / RT;
    if (gx > 64) gx = 64;
    if (gx < 1) gx = 1;
    k_rhs_absmax<<<dim3(gx, nrhs), RT, 0, st>>>(v, n, ld, out);
    count_launch();
    LP_CUDA(cudaGetLastError());
    return LP_OK;
}

int launch_axpy_f64(double* x, const float* d, size_t n, cudaStream_t st) {
    k_axpy_f64<<<592, 256, 0, st>>>(x, d, n);
    count_launch();
    LP_CUDA(cudaGetLastError());
    return LP_OK;
}

int launch_f64_to_f32(float* y, const double* v, size_t n, cudaStream_t st) {
    k_f64_to_f32<<<592, 256, 0, st>>>(y, v, n);
    count_launch();
    LP_CUDA(cudaGetLastError());
    return LP_OK;
}

int launch_f32_to_f64(double* y, const float* v, size_t n, cudaStream_t st) {
    k_f32_to_f64<<<592, 256, 0, st>>>(y, v, n);
    count_launch();
    LP_CUDA(cudaGetLastError());
    return LP_OK;
}

}  // namespace lp
