// top and left stages: the triangular block updates of the blocked LU.
//
// top (hpl_torus_PCIE.cl:452-582; host loop
// LINPACK/tests/test_kernel_communication.cpp:776-789) acts on the bs x ncols
// block row right of a factored diagonal block D.  Every column is
// independent:   for k: t_k *= D_kk;  for j > k: t_j += t_k * D_jk.
// A CTA owns a strip of 64 columns (all bs rows) in shared memory and walks
// the rows in chunks of CH: (1) two warps solve the CH x CH diagonal chunk,
// one thread per column; (2) all threads apply the solved chunk to the rows
// below it.  Every element receives its updates in ascending k, exactly as
// the host loop does, and with no fused multiply-add, so the result is
// bit-identical to the reference loop.
//
// left (hpl_torus_PCIE.cl:588-709; host loop
// test_kernel_communication.cpp:624-631) acts on the nrows x bs block column
// below D.  Every row is independent:  for k, i > k: l_i += l_k * D_ki.
// A CTA owns 64 rows (all bs columns, row length padded to bs+1 against
// bank conflicts) and walks the columns in chunks of CH the same way.  It
// writes the rows back in place and, optionally, transposed into Lt — the
// k-major operand layout of the trailing update (the reference keeps the
// same transposed copy, left_block, hpl_torus_PCIE.cl:697-708).
#include "lp_common.cuh"

namespace lp {
namespace {

constexpr int kTrsmThreads = 256;
constexpr int kStrip = 64;

template <int CH>
__global__ void __launch_bounds__(kTrsmThreads) k_trsm_top(const float* __restrict__ lu, int ldlu,
                                                         float* __restrict__ t, int ldt, int bs, int ncols) {
    extern __shared__ float sm[];
    float* strip = sm;                // bs x 64
    float* dch = sm + bs * kStrip;    // (bs - r0) x CH
    const int tid = threadIdx.x;
    const int c0 = blockIdx.x * kStrip;

    for (int idx = tid; idx < bs * kStrip; idx += kTrsmThreads) {
        const int r = idx >> 6, c = idx & 63;
        strip[idx] = (c0 + c < ncols) ? t[(size_t)r * ldt + c0 + c] : 0.0f;
    }
    for (int r0 = 0; r0 < bs; r0 += CH) {
        const int nr = bs - r0;
        for (int idx = tid; idx < nr * CH; idx += kTrsmThreads) {
            const int rr = idx / CH, kk = idx - rr * CH;
            dch[idx] = lu[(size_t)(r0 + rr) * ldlu + r0 + kk];
        }
        __syncthreads();
        if (tid < kStrip) {
            float x[CH];
#pragma unroll
            for (int k = 0; k < CH; k++) x[k] = strip[(r0 + k) * kStrip + tid];
#pragma unroll
            for (int k = 0; k < CH; k++) {
                const float xk = __fmul_rn(x[k], dch[k * CH + k]);
                x[k] = xk;
#pragma unroll
                for (int j = k + 1; j < CH; j++) x[j] = __fadd_rn(x[j], __fmul_rn(xk, dch[j * CH + k]));
            }
#pragma unroll
            for (int k = 0; k < CH; k++) strip[(r0 + k) * kStrip + tid] = x[k];
        }
        __syncthreads();
        if (nr > CH) {
            const int c = tid & 63, g = tid >> 6;
            float x[CH];
#pragma unroll
            for (int k = 0; k < CH; k++) x[k] = strip[(r0 + k) * kStrip + c];
            for (int r = r0 + CH + g; r < bs; r += kTrsmThreads / kStrip) {
                float acc = strip[r * kStrip + c];
                const float* drow = dch + (r - r0) * CH;
#pragma unroll
                for (int k = 0; k < CH; k++) acc = __fadd_rn(acc, __fmul_rn(x[k], drow[k]));
                strip[r * kStrip + c] = acc;
            }
        }
        __syncthreads();
    }
    for (int idx = tid; idx < bs * kStrip; idx += kTrsmThreads) {
        const int r = idx >> 6, c = idx & 63;
        if (c0 + c < ncols) t[(size_t)r * ldt + c0 + c] = strip[idx];
    }
}

template <int CH>
__global__ void __launch_bounds__(kTrsmThreads) k_trsm_left(const float* __restrict__ lu, int ldlu,
                                                          float* __restrict__ l, int ldl, int bs, int log2bs,
                                                          int nrows, float* __restrict__ lt, int ldlt) {
    extern __shared__ float sm[];
    const int sl = bs + 1;
    float* strip = sm;               // 64 x (bs+1)
    float* dch = sm + kStrip * sl;   // CH x (bs - c0)
    const int tid = threadIdx.x;
    const int r0 = blockIdx.x * kStrip;

    for (int idx = tid; idx < kStrip * bs; idx += kTrsmThreads) {
        const int rr = idx >> log2bs, c = idx & (bs - 1);
        strip[rr * sl + c] = (r0 + rr < nrows) ? l[(size_t)(r0 + rr) * ldl + c] : 0.0f;
    }
    for (int c0 = 0; c0 < bs; c0 += CH) {
        const int nc = bs - c0;
        for (int idx = tid; idx < CH * nc; idx += kTrsmThreads) {
            const int kk = idx / nc, cc = idx - kk * nc;
            dch[idx] = lu[(size_t)(c0 + kk) * ldlu + c0 + cc];
        }
        __syncthreads();
        if (tid < kStrip) {
            float x[CH];
            float* row = strip + tid * sl + c0;
#pragma unroll
            for (int k = 0; k < CH; k++) x[k] = row[k];
#pragma unroll
            for (int k = 0; k < CH; k++) {
#pragma unroll
                for (int i = k + 1; i < CH; i++) x[i] = __fadd_rn(x[i], __fmul_rn(x[k], dch[k * nc + i]));
            }
#pragma unroll
            for (int k = 0; k < CH; k++) row[k] = x[k];
        }
        __syncthreads();
        for (int ci = CH + tid; ci < nc; ci += kTrsmThreads) {
            float d[CH];
#pragma unroll
            for (int k = 0; k < CH; k++) d[k] = dch[k * nc + ci];
            for (int rr = 0; rr < kStrip; rr++) {
                const float* row = strip + rr * sl + c0;
                float acc = row[ci];
#pragma unroll
                for (int k = 0; k < CH; k++) acc = __fadd_rn(acc, __fmul_rn(row[k], d[k]));
                strip[rr * sl + c0 + ci] = acc;
            }
        }
        __syncthreads();
    }
    for (int idx = tid; idx < kStrip * bs; idx += kTrsmThreads) {
        const int rr = idx >> log2bs, c = idx & (bs - 1);
        if (r0 + rr < nrows) l[(size_t)(r0 + rr) * ldl + c] = strip[rr * sl + c];
    }
    if (lt != nullptr) {
        for (int idx = tid; idx < kStrip * bs; idx += kTrsmThreads) {
            const int c = idx >> 6, rr = idx & 63;
            if (r0 + rr < nrows) lt[(size_t)c * ldlt + r0 + rr] = strip[rr * sl + c];
        }
    }
}

// ---- bs <= 128: 32-wide chunks, each recurrence lane-parallel ----------
// The diagonal block and the CTA's 32 columns (top) or rows (left) sit in
// shared memory.  Per 32-wide chunk: one warp runs the recurrence of the
// chunk with one independent column (top) / row (left) per lane, then all
// warps apply the finished chunk to the remaining rows (top) / columns (left),
// every element receiving its 32 updates in ascending k with a separate
// multiply and add.  Same per-element operation sequence as above.
constexpr int kCW = 32;  // columns (top) / rows (left) per CTA

template <typename E, int BS>
__global__ void __launch_bounds__(kTrsmThreads) k_top_chunk(const E* __restrict__ lu, int ldlu,
                                                          E* __restrict__ t, int ldt, int ncols) {
    using R = Rn<E>;
    constexpr int NB = BS < 32 ? BS : 32;
    constexpr int SL = BS + 4, TL = kCW + 4;
    extern __shared__ __align__(16) unsigned char trsm_raw[];
    E* D = reinterpret_cast<E*>(trsm_raw);  // BS x SL: the factored diagonal block
    E* T = D + BS * SL;                     // BS x TL: the CTA's columns
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int c0 = blockIdx.x * kCW;
    for (int idx = tid; idx < BS * BS; idx += kTrsmThreads) {
        const int j = idx / BS, k = idx - j * BS;
        cp_async_elem(D + j * SL + k, lu + (size_t)j * ldlu + k);
    }
    for (int idx = tid; idx < BS * kCW; idx += kTrsmThreads) {
        const int r = idx / kCW, cc = idx - r * kCW;
        if (c0 + cc < ncols)
            cp_async_elem(T + r * TL + cc, t + (size_t)r * ldt + c0 + cc);
        else
            T[r * TL + cc] = E(0);
    }
    cp_async_wait_all();
    __syncthreads();
    for (int k0 = 0; k0 < BS; k0 += NB) {
        if (warp == 0) {  // rows k0..k0+NB-1 of column `lane`: t_k *= D_kk; t_j += t_k D_jk
            E x[NB];
#pragma unroll
            for (int j = 0; j < NB; j++) x[j] = T[(k0 + j) * TL + lane];
#pragma unroll
            for (int k = 0; k < NB; k++) {
                x[k] = R::mul(x[k], D[(k0 + k) * SL + k0 + k]);
#pragma unroll
                for (int j = k + 1; j < NB; j++)
                    x[j] = R::add(x[j], R::mul(x[k], D[(k0 + j) * SL + k0 + k]));
            }
#pragma unroll
            for (int j = 0; j < NB; j++) T[(k0 + j) * TL + lane] = x[j];
        }
        __syncthreads();
        const int base = k0 + NB;
        if (base == BS) break;
        // rows below the chunk: T[r][c] += sum_kk T[k0+kk][c] D[r][k0+kk]; two rows per pass
        E tv[NB];
#pragma unroll
        for (int kk = 0; kk < NB; kk++) tv[kk] = T[(k0 + kk) * TL + lane];
        for (int r = base + warp; r < BS; r += 16) {
            const int r2 = r + 8;  // (BS - base) / 8 is even
            E acc = T[r * TL + lane], acc2 = T[r2 * TL + lane];
            const E* d1 = D + r * SL + k0;
            const E* d2 = D + r2 * SL + k0;
#pragma unroll
            for (int kk = 0; kk < NB; kk += 4) {
                const Quad<E> u = ld_quad(d1 + kk);
                const Quad<E> v = ld_quad(d2 + kk);
                acc = R::add(acc, R::mul(tv[kk], u.x));
                acc2 = R::add(acc2, R::mul(tv[kk], v.x));
                acc = R::add(acc, R::mul(tv[kk + 1], u.y));
                acc2 = R::add(acc2, R::mul(tv[kk + 1], v.y));
                acc = R::add(acc, R::mul(tv[kk + 2], u.z));
                acc2 = R::add(acc2, R::mul(tv[kk + 2], v.z));
                acc = R::add(acc, R::mul(tv[kk + 3], u.w));
                acc2 = R::add(acc2, R::mul(tv[kk + 3], v.w));
            }
            T[r * TL + lane] = acc;
            T[r2 * TL + lane] = acc2;
        }
        __syncthreads();
    }
    for (int idx = tid; idx < BS * kCW; idx += kTrsmThreads) {
        const int r = idx / kCW, cc = idx - r * kCW;
        if (c0 + cc < ncols) t[(size_t)r * ldt + c0 + cc] = T[r * TL + cc];
    }
}

template <typename E, int BS>
__global__ void __launch_bounds__(kTrsmThreads) k_left_chunk(const E* __restrict__ lu, int ldlu,
                                                           E* __restrict__ l, int ldl, int nrows,
                                                           E* __restrict__ lt, int ldlt) {
    using R = Rn<E>;
    constexpr int NB = BS < 32 ? BS : 32;
    constexpr int SL = BS + 4;
    extern __shared__ __align__(16) unsigned char trsm_raw[];
    E* D = reinterpret_cast<E*>(trsm_raw);  // BS x SL: the factored diagonal block
    E* L = D + BS * SL;                     // kCW x SL: the CTA's rows
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int r0 = blockIdx.x * kCW;
    for (int idx = tid; idx < BS * BS; idx += kTrsmThreads) {
        const int k = idx / BS, i = idx - k * BS;
        cp_async_elem(D + k * SL + i, lu + (size_t)k * ldlu + i);
    }
    for (int idx = tid; idx < kCW * BS; idx += kTrsmThreads) {
        const int r = idx / BS, c = idx - r * BS;
        if (r0 + r < nrows)
            cp_async_elem(L + r * SL + c, l + (size_t)(r0 + r) * ldl + c);
        else
            L[r * SL + c] = E(0);
    }
    cp_async_wait_all();
    __syncthreads();
    for (int k0 = 0; k0 < BS; k0 += NB) {
        if (warp == 0) {  // columns k0..k0+NB-1 of row `lane`: l_i += l_k D_ki (i > k)
            E x[NB];
#pragma unroll
            for (int i = 0; i < NB; i++) x[i] = L[lane * SL + k0 + i];
#pragma unroll
            for (int k = 0; k < NB; k++)
#pragma unroll
                for (int i = k + 1; i < NB; i++)
                    x[i] = R::add(x[i], R::mul(x[k], D[(k0 + k) * SL + k0 + i]));
#pragma unroll
            for (int i = 0; i < NB; i++) L[lane * SL + k0 + i] = x[i];
        }
        __syncthreads();
        const int base = k0 + NB;
        if (base == BS) break;
        // columns after the chunk: L[r][i] += sum_kk L[r][k0+kk] D[k0+kk][i]; lane = column, warp = row
        for (int g = 0; g < (BS - base) / 32; g++) {
            const int i = base + 32 * g + lane;
            E dv[NB];
#pragma unroll
            for (int kk = 0; kk < NB; kk++) dv[kk] = D[(k0 + kk) * SL + i];
            E acc[kCW / 8];
#pragma unroll
            for (int s = 0; s < kCW / 8; s++) acc[s] = L[(warp + 8 * s) * SL + i];
#pragma unroll
            for (int kk = 0; kk < NB; kk += 4) {
#pragma unroll
                for (int s = 0; s < kCW / 8; s++) {
                    const Quad<E> u = ld_quad(L + (warp + 8 * s) * SL + k0 + kk);
                    acc[s] = R::add(acc[s], R::mul(u.x, dv[kk]));
                    acc[s] = R::add(acc[s], R::mul(u.y, dv[kk + 1]));
                    acc[s] = R::add(acc[s], R::mul(u.z, dv[kk + 2]));
                    acc[s] = R::add(acc[s], R::mul(u.w, dv[kk + 3]));
                }
            }
#pragma unroll
            for (int s = 0; s < kCW / 8; s++) L[(warp + 8 * s) * SL + i] = acc[s];
        }
        __syncthreads();
    }
    for (int idx = tid; idx < kCW * BS; idx += kTrsmThreads) {
        const int r = idx / BS, c = idx - r * BS;
        if (r0 + r < nrows) l[(size_t)(r0 + r) * ldl + c] = L[r * SL + c];
    }
    if (lt == nullptr) return;
    for (int idx = tid; idx < kCW * BS; idx += kTrsmThreads) {
        const int c = idx / kCW, r = idx - c * kCW;
        if (r0 + r < nrows) lt[(size_t)c * ldlt + r0 + r] = L[r * SL + c];
    }
}

template <typename E, int BS>
constexpr size_t top_chunk_smem() { return sizeof(E) * ((size_t)BS * (BS + 4) + (size_t)BS * (kCW + 4)); }
template <typename E, int BS>
constexpr size_t left_chunk_smem() { return sizeof(E) * ((size_t)BS * (BS + 4) + (size_t)kCW * (BS + 4)); }

template <int BS, typename E>
void launch_left_chunk(const E* lu, int ldlu, E* l, int ldl, int nrows, E* lt, int ldlt, cudaStream_t st) {
    k_left_chunk<E, BS><<<(nrows + kCW - 1) / kCW, kTrsmThreads, left_chunk_smem<E, BS>(), st>>>(lu, ldlu, l, ldl,
                                                                                                nrows, lt, ldlt);
}
template <int BS, typename E>
void launch_top_chunk(const E* lu, int ldlu, E* t, int ldt, int ncols, cudaStream_t st) {
    k_top_chunk<E, BS><<<(ncols + kCW - 1) / kCW, kTrsmThreads, top_chunk_smem<E, BS>(), st>>>(lu, ldlu, t, ldt,
                                                                                               ncols);
}

int log2i(int x) {
    int r = 0;
    while ((1 << r) < x) r++;
    return r;
}

size_t top_smem(int bs, int ch) { return sizeof(float) * ((size_t)bs * kStrip + (size_t)bs * ch); }
size_t left_smem(int bs, int ch) { return sizeof(float) * ((size_t)kStrip * (bs + 1) + (size_t)ch * bs); }

}  // namespace

int trsm_init_attrs() {
    const int max_smem = (int)left_smem(512, 32);
    LP_CUDA(cudaFuncSetAttribute(k_trsm_top<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)top_smem(512, 32)));
    LP_CUDA(cudaFuncSetAttribute(k_trsm_top<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)top_smem(512, 16)));
    LP_CUDA(cudaFuncSetAttribute(k_trsm_left<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, max_smem));
    LP_CUDA(cudaFuncSetAttribute(k_trsm_left<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)left_smem(512, 16)));
    LP_CUDA(cudaFuncSetAttribute(k_left_chunk<float, 128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)left_chunk_smem<float, 128>()));
    LP_CUDA(cudaFuncSetAttribute(k_top_chunk<float, 128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)top_chunk_smem<float, 128>()));
    LP_CUDA(cudaFuncSetAttribute(k_left_chunk<double, 128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)left_chunk_smem<double, 128>()));
    LP_CUDA(cudaFuncSetAttribute(k_top_chunk<double, 128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)top_chunk_smem<double, 128>()));
    LP_CUDA(cudaFuncSetAttribute(k_left_chunk<double, 64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)left_chunk_smem<double, 64>()));
    LP_CUDA(cudaFuncSetAttribute(k_top_chunk<double, 64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)top_chunk_smem<double, 64>()));
    return LP_OK;
}

int launch_top_chunk_f64(const double* lu, int ldlu, double* t, int ldt, int bs, int ncols, cudaStream_t st) {
    if (ncols <= 0) return LP_OK;
    if (bs == 128)
        launch_top_chunk<128>(lu, ldlu, t, ldt, ncols, st);
    else if (bs == 64)
        launch_top_chunk<64>(lu, ldlu, t, ldt, ncols, st);
    else
        return fail(LP_E_INVALID, "FP64 top update: bs must be 64 or 128");
    count_launch();
    LP_CUDA(cudaGetLastError());
    return LP_OK;
}

int launch_left_chunk_f64(const double* lu, int ldlu, double* l, int ldl, int bs, int nrows, double* lt, int ldlt,
                          cudaStream_t st) {
    if (nrows <= 0) return LP_OK;
    if (bs == 128)
        launch_left_chunk<128>(lu, ldlu, l, ldl, nrows, lt, ldlt, st);
    else if (bs == 64)
        launch_left_chunk<64>(lu, ldlu, l, ldl, nrows, lt, ldlt, st);
    else
        return fail(LP_E_INVALID, "FP64 left update: bs must be 64 or 128");
    count_launch();
    LP_CUDA(cudaGetLastError());
    return LP_OK;
}

int launch_trsm_top(const float* lu, int ldlu, float* t, int ldt, int bs, int ncols, cudaStream_t st) {
    if (!is_pow2(bs) || bs < 16 || bs > 512) return fail(LP_E_INVALID, "top_update: bs must be a power of two in [16, 512]");
    if (ncols <= 0) return LP_OK;
    const dim3 grid((ncols + kStrip - 1) / kStrip);
    if (bs <= 128) {
        if (bs == 128)
            launch_top_chunk<128>(lu, ldlu, t, ldt, ncols, st);
        else if (bs == 64)
            launch_top_chunk<64>(lu, ldlu, t, ldt, ncols, st);
        else if (bs == 32)
            launch_top_chunk<32>(lu, ldlu, t, ldt, ncols, st);
        else
            launch_top_chunk<16>(lu, ldlu, t, ldt, ncols, st);
    } else if (bs >= 32)
        k_trsm_top<32><<<grid, kTrsmThreads, top_smem(bs, 32), st>>>(lu, ldlu, t, ldt, bs, ncols);
    else
        k_trsm_top<16><<<grid, kTrsmThreads, top_smem(bs, 16), st>>>(lu, ldlu, t, ldt, bs, ncols);
    count_launch();
    LP_CUDA(cudaGetLastError());
    return LP_OK;
}

int launch_trsm_left(const float* lu, int ldlu, float* l, int ldl, int bs, int nrows, float* lt, int ldlt,
                     cudaStream_t st) {
    if (!is_pow2(bs) || bs < 16 || bs > 512) return fail(LP_E_INVALID, "left_update: bs must be a power of two in [16, 512]");
    if (nrows <= 0) return LP_OK;
    const dim3 grid((nrows + kStrip - 1) / kStrip);
    const int lg = log2i(bs);
    if (bs <= 128) {
        if (bs == 128)
            launch_left_chunk<128>(lu, ldlu, l, ldl, nrows, lt, ldlt, st);
        else if (bs == 64)
            launch_left_chunk<64>(lu, ldlu, l, ldl, nrows, lt, ldlt, st);
        else if (bs == 32)
            launch_left_chunk<32>(lu, ldlu, l, ldl, nrows, lt, ldlt, st);
        else
            launch_left_chunk<16>(lu, ldlu, l, ldl, nrows, lt, ldlt, st);
    } else if (bs >= 32)
        k_trsm_left<32><<<grid, kTrsmThreads, left_smem(bs, 32), st>>>(lu, ldlu, l, ldl, bs, lg, nrows, lt, ldlt);
    else
        k_trsm_left<16><<<grid, kTrsmThreads, left_smem(bs, 16), st>>>(lu, ldlu, l, ldl, bs, lg, nrows, lt, ldlt);
    count_launch();
    LP_CUDA(cudaGetLastError());
    return LP_OK;
}

}  // namespace lp
