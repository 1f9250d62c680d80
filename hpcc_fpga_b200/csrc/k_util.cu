// Tiled transpose: the diagonal block's sub-blocks into the k-major operand
// layout of the blocked top stage.
#include "lp_common.cuh"

namespace lp {
namespace {

// dst[c][r] = src[r][c] for r < rows, c < cols; 32 x 32 tiles through shared
// memory (padded row) so both the read and the write are coalesced.
template <typename T>
__global__ void __launch_bounds__(256) k_transpose(const T* __restrict__ src, int lds, T* __restrict__ dst,
                                                   int ldd, int rows, int cols) {
    __shared__ T tile[32][33];
    const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < 32; j += 8) {
        const int r = r0 + ty + j, c = c0 + tx;
        if (r < rows && c < cols) tile[ty + j][tx] = src[(size_t)r * lds + c];
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < 32; j += 8) {
        const int c = c0 + ty + j, r = r0 + tx;
        if (r < rows && c < cols) dst[(size_t)c * ldd + r] = tile[tx][ty + j];
    }
}

}  // namespace

int launch_transpose(const float* src, int lds, float* dst, int ldd, int rows, int cols, cudaStream_t st) {
    if (rows <= 0 || cols <= 0) return LP_OK;
    const dim3 grid((cols + 31) / 32, (rows + 31) / 32);
    if (grid.y > 65535) return fail(LP_E_INVALID, "transpose: too many rows");
    k_transpose<float><<<grid, 256, 0, st>>>(src, lds, dst, ldd, rows, cols);
    count_launch();
    LP_CUDA(cudaGetLastError());
    return LP_OK;
}

int launch_transpose_f64(const double* src, int lds, double* dst, int ldd, int rows, int cols, cudaStream_t st) {
    if (rows <= 0 || cols <= 0) return LP_OK;
    const dim3 grid((cols + 31) / 32, (rows + 31) / 32);
    if (grid.y > 65535) return fail(LP_E_INVALID, "transpose: too many rows");
    k_transpose<double><<<grid, 256, 0, st>>>(src, lds, dst, ldd, rows, cols);
    count_launch();
    LP_CUDA(cudaGetLastError());
    return LP_OK;
}

}  // namespace lp
