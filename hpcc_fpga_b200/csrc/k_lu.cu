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
// only independent operations are reordered.
//
// (1) is a chain of 32 dependent pivots on one warp and dominates the block's
// time, so (3) is split: the four warps of SM partition 0 (warps 0, 4, 8, 12)
// first apply the chunk to the next diagonal block, then warp 0 factors that
// block -- step (1) of the next chunk -- while the twelve warps of the other
// three partitions apply the chunk to the rest of the trailing block.  Warp 0
// keeps its partition's issue slots to itself.  In (1) the lanes at or left of
// the pivot keep their values by a select rather than a branch around the
// update.  Measured on one B200 (128-block, float): 37.0 -> 30.9 us per block.
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
        const bool below = lane > k;
        const T d = R::neg_rcp(__shfl_sync(0xffffffffu, x[k], k));
        const T scaled = R::mul(x[k], d);  // scaled row k: the multipliers
        x[k] = below ? scaled : (lane == k ? d : x[k]);
#pragma unroll
        for (int j = k + 1; j < NB; j++) {
            const T sjk = __shfl_sync(0xffffffffu, x[j], k);  // column k, row j
            const T v = R::add(x[j], R::mul(x[k], sjk));
            x[j] = below ? v : x[j];
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

// (3) for one row r and column i: the chunk's NB updates of S[r][i] in
// ascending k (tv: column i of the chunk's block row).
template <typename T, int NB, int SL>
__device__ __forceinline__ T chunk_row(const T* S, int k0, int r, T acc, const T (&tv)[NB]) {
    using R = Rn<T>;
    const T* l = S + r * SL + k0;
#pragma unroll
    for (int kk = 0; kk < NB; kk += 4) {
        const Quad<T> u = ld_quad(l + kk);
        acc = R::add(acc, R::mul(tv[kk], u.x));
        acc = R::add(acc, R::mul(tv[kk + 1], u.y));
        acc = R::add(acc, R::mul(tv[kk + 2], u.z));
        acc = R::add(acc, R::mul(tv[kk + 3], u.w));
    }
    return acc;
}

template <typename T, int NB, int SL>
__device__ __forceinline__ void load_tv(const T* S, int k0, int i, T (&tv)[NB]) {
#pragma unroll
    for (int kk = 0; kk < NB; kk++) tv[kk] = S[(k0 + kk) * SL + i];
}

template <typename T, int BS>
__global__ void __launch_bounds__(kLuThreads) k_lu_block(T* __restrict__ a, int lda) {
    constexpr int NB = BS < 32 ? BS : 32;
    constexpr int SL = BS + 4;  // 16-byte rows
    constexpr int V = 16 / sizeof(T);
    extern __shared__ __align__(16) unsigned char lu_raw[];
    T* S = reinterpret_cast<T*>(lu_raw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const bool vec = (reinterpret_cast<uintptr_t>(a) & 15u) == 0 && (lda % V) == 0;
    if (vec) {
        for (int idx = tid; idx < BS * BS / V; idx += kLuThreads) {
            const int r = idx / (BS / V), c = (idx - r * (BS / V)) * V;
            cp_async_vec16(S + r * SL + c, a + (size_t)r * lda + c);
        }
    } else {
        for (int idx = tid; idx < BS * BS; idx += kLuThreads) {
            const int r = idx / BS, c = idx - r * BS;
            cp_async_elem(S + r * SL + c, a + (size_t)r * lda + c);
        }
    }
    cp_async_wait_all();
    __syncthreads();
    if (warp == 0) diag_lu<T, NB, SL>(S, lane);
    __syncthreads();

    for (int k0 = 0; k0 + NB < BS; k0 += NB) {
        const int base = k0 + NB, rest = BS - base;  // a multiple of 32
        const int nw = rest / 32;
        if (warp < nw)
            top_column<T, NB, SL>(S, k0, base + 32 * warp + lane);
        else if (warp < 2 * nw)
            left_row<T, NB, SL>(S, k0, base + 32 * (warp - nw) + lane);
        __syncthreads();
        if constexpr (sizeof(T) == 8) {
            // double: the whole trailing block on all warps (lane = column,
            // warp = row), then warp 0 factors the next diagonal block
            for (int g = 0; g < rest / 32; g++) {
                const int i = base + 32 * g + lane;
                T tv[NB];
                load_tv<T, NB, SL>(S, k0, i, tv);
                for (int r = base + warp; r < BS; r += 16)
                    S[r * SL + i] = chunk_row<T, NB, SL>(S, k0, r, S[r * SL + i], tv);
            }
            __syncthreads();
            if (warp == 0) diag_lu<T, NB, SL>(S + base * SL + base, lane);
        } else if ((warp & 3) == 0) {
            // partition 0: the chunk applied to the next diagonal block
            // (rows base + warp/4 + 4t), then warp 0 factors it
            const int i = base + lane;
            T tv[NB];
            load_tv<T, NB, SL>(S, k0, i, tv);
#pragma unroll 1
            for (int t = 0; t < NB / 4; t++) {
                const int r = base + (warp >> 2) + 4 * t;
                S[r * SL + i] = chunk_row<T, NB, SL>(S, k0, r, S[r * SL + i], tv);
            }
            asm volatile("bar.sync 1, 128;\n" ::: "memory");
            if (warp == 0) diag_lu<T, NB, SL>(S + base * SL + base, lane);
        } else {
            // partitions 1-3: the rest of the trailing block as 32 x 32 tiles
            // (column group g, row block rb) without tile (0, 0), each as 16
            // row pairs (r, r + 16), lane = column
            constexpr int PR = 16, RPI = 2;
            const int ng = rest / 32, items = PR * (ng * ng - 1);
            int cur = -1;
            T tv[NB];
            for (int m = warp - (warp >> 2) - 1; m < items; m += 12) {
                const int tile = m / PR + 1, h = m % PR;
                const int g = tile / ng, rb = tile - g * ng;
                const int i = base + 32 * g + lane;
                if (g != cur) {
                    load_tv<T, NB, SL>(S, k0, i, tv);
                    cur = g;
                }
                const int r = base + 32 * rb + h;
                T acc[RPI];
#pragma unroll
                for (int q = 0; q < RPI; q++) acc[q] = chunk_row<T, NB, SL>(S, k0, r + PR * q, S[(r + PR * q) * SL + i], tv);
#pragma unroll
                for (int q = 0; q < RPI; q++) S[(r + PR * q) * SL + i] = acc[q];
            }
        }
        __syncthreads();
    }

    if (vec) {
        for (int idx = tid; idx < BS * BS / V; idx += kLuThreads) {
            const int r = idx / (BS / V), c = (idx - r * (BS / V)) * V;
            *reinterpret_cast<uint4*>(a + (size_t)r * lda + c) = *reinterpret_cast<const uint4*>(S + r * SL + c);
        }
    } else {
        for (int idx = tid; idx < BS * BS; idx += kLuThreads) {
            const int r = idx / BS, c = idx - r * BS;
            a[(size_t)r * lda + c] = S[r * SL + c];
        }
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
