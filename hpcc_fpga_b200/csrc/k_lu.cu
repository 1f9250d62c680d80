// lu stage: LU without pivoting of one diagonal block (16 <= bs <= 128), the
// block resident in shared memory of one CTA.  Templated on the element type:
// float is the benchmark's type, double the reference's _DP build
// (LINPACK/src/host/parameters.h.in, HOST_DATA_TYPE / DEVICE_DATA_TYPE).
//
// Arithmetic follows gefa_ref_nopvt (LINPACK/src/host/linpack_data.cpp:166-196)
// operation for operation, with no fused multiply-add, so the block result is
// bit-identical to the reference's host routine:
//   d = -1/a_kk   (the reference divides in double and rounds to float; with
//                  53 >= 2*24 + 2 bits that double rounding equals the
//                  correctly rounded float reciprocal, __frcp_rn, negated)
//   a_ki = a_ki * d                       (i > k)
//   a_ji = a_ji + a_ki * a_jk             (j > k, i > k)
//
// Schedule: 32-wide chunks.  For the chunk at k0 the same operations are
// grouped as (1) the 32 x 32 diagonal block, one warp, its columns across the
// lanes; (2) the block row right of it (column-independent: each lane one
// column) and the block column below it (row-independent: each lane one row),
// concurrently on different warps; (3) the trailing update, every element
// receiving its 32 updates in ascending k with a separate multiply and add.
// Every element still sees exactly the reference's sequence of operations;
// only independent operations are reordered.  Three barriers per chunk.
#include "lp_common.cuh"

namespace lp {
namespace {

constexpr int kLuThreads = 512;

// (1) In-place LU of the NB x NB block at D (row stride SL), one warp; lane c
// holds column c (x[j] = D[j][c]).  Kept out of line: inlined into the chunk
// loop, its register array is not fully unrolled and lands in local memory.
template <typename T, int NB, int SL>
__device__ __noinline__ void diag_lu(T* D, int lane) {
    using R = Rn<T>;
    T x[NB];
    const bool act = lane < NB;
#pragma unroll
    for (int j = 0; j < NB; j++) x[j] = act ? D[j * SL + lane] : T(0);
#pragma unroll
    for (int k = 0; k < NB; k++) {
        const T d = R::neg_rcp(__shfl_sync(0xffffffffu, x[k], k));
        if (lane > k)
            x[k] = R::mul(x[k], d);  // scaled row k: the multipliers
        else if (lane == k)
            x[k] = d;
#pragma unroll
        for (int j = k + 1; j < NB; j++) {
            const T sjk = __shfl_sync(0xffffffffu, x[j], k);  // column k, row j
            if (lane > k) x[j] = R::add(x[j], R::mul(x[k], sjk));
        }
    }
    if (act) {
#pragma unroll
        for (int j = 0; j < NB; j++) D[j * SL + lane] = x[j];
    }
}

// (2a) Column `col` of the block row right of the diagonal block at k0:
// for k: t_k *= D_kk; t_j += t_k D_jk (j > k).
template <typename T, int NB, int SL>
__device__ __forceinline__ void top_column(T* S, int k0, int col) {
    using R = Rn<T>;
    T x[NB];
#pragma unroll
    for (int j = 0; j < NB; j++) x[j] = S[(k0 + j) * SL + col];
#pragma unroll
    for (int k = 0; k < NB; k++) {
        x[k] = R::mul(x[k], S[(k0 + k) * SL + k0 + k]);
#pragma unroll
        for (int j = k + 1; j < NB; j++) x[j] = R::add(x[j], R::mul(x[k], S[(k0 + j) * SL + k0 + k]));
    }
#pragma unroll
    for (int j = 0; j < NB; j++) S[(k0 + j) * SL + col] = x[j];
}

// (2b) Row `row` of the block column below the diagonal block at k0:
// for k, i > k: l_i += l_k D_ki.
template <typename T, int NB, int SL>
__device__ __forceinline__ void left_row(T* S, int k0, int row) {
    using R = Rn<T>;
    T x[NB];
#pragma unroll
    for (int i = 0; i < NB; i++) x[i] = S[row * SL + k0 + i];
#pragma unroll
    for (int k = 0; k < NB; k++)
#pragma unroll
        for (int i = k + 1; i < NB; i++) x[i] = R::add(x[i], R::mul(x[k], S[(k0 + k) * SL + k0 + i]));
#pragma unroll
    for (int i = 0; i < NB; i++) S[row * SL + k0 + i] = x[i];
}

template <typename T, int BS>
__global__ void __launch_bounds__(kLuThreads) k_lu_block(T* __restrict__ a, int lda) {
    using R = Rn<T>;
    constexpr int NB = BS < 32 ? BS : 32;
    constexpr int SL = BS + 4;  // 16-byte rows
    extern __shared__ __align__(16) unsigned char lu_raw[];
    T* S = reinterpret_cast<T*>(lu_raw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    for (int idx = tid; idx < BS * BS; idx += kLuThreads) {
        const int r = idx / BS, c = idx - r * BS;
        cp_async_elem(S + r * SL + c, a + (size_t)r * lda + c);
    }
    cp_async_wait_all();
    __syncthreads();

    for (int k0 = 0; k0 < BS; k0 += NB) {
        if (warp == 0) diag_lu<T, NB, SL>(S + k0 * SL + k0, lane);
        __syncthreads();
        const int base = k0 + NB, rest = BS - base;  // a multiple of 32
        if (rest == 0) break;
        if (warp < rest / 32)
            top_column<T, NB, SL>(S, k0, base + 32 * warp + lane);
        else if (warp >= 8 && warp - 8 < rest / 32)
            left_row<T, NB, SL>(S, k0, base + 32 * (warp - 8) + lane);
        __syncthreads();
        // (3) trailing update: rows / columns [base, BS); lane = column, warp = row (two rows per pass)
        for (int g = 0; g < rest / 32; g++) {
            const int i = base + 32 * g + lane;
            T tv[NB];
#pragma unroll
            for (int kk = 0; kk < NB; kk++) tv[kk] = S[(k0 + kk) * SL + i];
            for (int r = base + warp; r < BS; r += 32) {
                const int r2 = r + 16;  // rest / 16 is even
                T acc = S[r * SL + i], acc2 = S[r2 * SL + i];
                const T* l1 = S + r * SL + k0;
                const T* l2 = S + r2 * SL + k0;
#pragma unroll
                for (int kk = 0; kk < NB; kk += 4) {
                    const Quad<T> u = ld_quad(l1 + kk);
                    const Quad<T> v = ld_quad(l2 + kk);
                    acc = R::add(acc, R::mul(tv[kk], u.x));
                    acc2 = R::add(acc2, R::mul(tv[kk], v.x));
                    acc = R::add(acc, R::mul(tv[kk + 1], u.y));
                    acc2 = R::add(acc2, R::mul(tv[kk + 1], v.y));
                    acc = R::add(acc, R::mul(tv[kk + 2], u.z));
                    acc2 = R::add(acc2, R::mul(tv[kk + 2], v.z));
                    acc = R::add(acc, R::mul(tv[kk + 3], u.w));
                    acc2 = R::add(acc2, R::mul(tv[kk + 3], v.w));
                }
                S[r * SL + i] = acc;
                S[r2 * SL + i] = acc2;
            }
        }
        __syncthreads();
    }

    for (int idx = tid; idx < BS * BS; idx += kLuThreads) {
        const int r = idx / BS, c = idx - r * BS;
        a[(size_t)r * lda + c] = S[r * SL + c];
    }
}

template <typename T, int BS>
constexpr size_t lu_smem() {
    return sizeof(T) * (size_t)BS * (BS + 4);
}

}  // namespace

int launch_lu_small(float* a, int lda, int bs, cudaStream_t st) {
    switch (bs) {
        case 16: k_lu_block<float, 16><<<1, kLuThreads, lu_smem<float, 16>(), st>>>(a, lda); break;
        case 32: k_lu_block<float, 32><<<1, kLuThreads, lu_smem<float, 32>(), st>>>(a, lda); break;
        case 64: k_lu_block<float, 64><<<1, kLuThreads, lu_smem<float, 64>(), st>>>(a, lda); break;
        case 128: k_lu_block<float, 128><<<1, kLuThreads, lu_smem<float, 128>(), st>>>(a, lda); break;
        default: return fail(LP_E_INVALID, "lu block: bs must be 16, 32, 64 or 128");
    }
    count_launch();
    LP_CUDA(cudaGetLastError());
    return LP_OK;
}

int launch_lu_small_f64(double* a, int lda, int bs, cudaStream_t st) {
    switch (bs) {
        case 64: k_lu_block<double, 64><<<1, kLuThreads, lu_smem<double, 64>(), st>>>(a, lda); break;
        case 128: k_lu_block<double, 128><<<1, kLuThreads, lu_smem<double, 128>(), st>>>(a, lda); break;
        default: return fail(LP_E_INVALID, "FP64 lu block: bs must be 64 or 128");
    }
    count_launch();
    LP_CUDA(cudaGetLastError());
    return LP_OK;
}

int lu_init_attrs() {
    LP_CUDA(cudaFuncSetAttribute(k_lu_block<float, 128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)lu_smem<float, 128>()));
    LP_CUDA(cudaFuncSetAttribute(k_lu_block<float, 64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)lu_smem<float, 64>()));
    LP_CUDA(cudaFuncSetAttribute(k_lu_block<double, 128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)lu_smem<double, 128>()));
    LP_CUDA(cudaFuncSetAttribute(k_lu_block<double, 64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)lu_smem<double, 64>()));
    return LP_OK;
}

}  // namespace lp
