// Serving loop: continuous batching of solve requests on one GPU.
//
// Workers, each a host thread with its own lp_ctx (streams, workspaces):
//   * wave workers: whenever one is free it takes every admissible pending
//     request with n <= batch_max_n (new factorizations and solves with
//     resident factors alike) and runs them as ONE persistent launch of the
//     batched kernel, then a batched FP64 residual kernel (and, for the
//     refined precisions, batched refinement steps);
//   * slot workers: requests with larger n, one at a time each, through the
//     blocked factorization (FP32 SIMT or tensor-core mixed precision) and
//     the FP64 residual / refinement of refine_core.
// Requests that arrive while others are on the GPU are admitted as soon as a
// worker and budget are free; the workers' streams overlap on the device.
// The per-request baseline mode has a single slot worker and no waves.
//
// Device memory.  Every miss gets a slab (factors + original matrix; one slab
// per wave for all its new systems) from a pool owned by the server, so no
// cudaMalloc / cudaFree (which would synchronize the device) runs on the
// request path.  Slabs stay resident as the factor cache (keyed by the
// caller's matrix key); the budget is charged with every slab plus the
// per-request vectors of in-flight work, and idle cache entries are evicted
// least-recently-used first to admit new work.
//
// Large systems are padded to a multiple of the factorization block with an
// identity block: diag(A, I) factors as diag(LU_A, I), and the substitution
// and residual only touch the leading n x n block.
#include <algorithm>
#include <atomic>
#include <cfloat>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <list>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "lp_ctx.cuh"

namespace lp {
namespace {

constexpr int kMaxN = 16384;
constexpr int kMaxRhs = 16;
constexpr int kRT = 256;
constexpr int kWaveMaxN = 1024;
constexpr int kInit = 1, kAccum = 2;

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// ---- device side ----------------------------------------------------------

// Identity in the padding rows / columns [n, npad) of an npad x npad matrix.
__global__ void k_pad_identity(float* a, int ld, int n, int npad) {
    const size_t p = (size_t)(npad - n);
    const size_t rows = p * npad, total = rows + (size_t)n * p;
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total; idx += (size_t)gridDim.x * blockDim.x) {
        size_t r, c;
        if (idx < rows) {
            r = n + idx / npad;
            c = idx % npad;
        } else {
            const size_t k = idx - rows;
            r = k / p;
            c = n + k % p;
        }
        a[r * ld + c] = (r == c) ? 1.0f : 0.0f;
    }
}

// Copies of float4 runs, one CTA per run: the wave's new originals into the
// factor buffers that the batched kernel factors in place.
struct CopyRun {
    const float4* src;
    float4* dst;
    long long n4;
};
__global__ void k_copy_runs(const CopyRun* __restrict__ runs, int count) {
    for (int t = blockIdx.x; t < count; t += gridDim.x) {
        const CopyRun r = runs[t];
        for (long long i = threadIdx.x; i < r.n4; i += blockDim.x) r.dst[i] = r.src[i];
    }
}

struct WaveItem {
    const float* a0;  // original matrix, leading dimension lda
    const float* b0;  // right-hand sides, nrhs rows of ldv floats
    float* x32;       // in: FP32 solve (or correction); out: residual, for the next solve
    double* x64;      // FP64 solution, nrhs rows of ldv doubles
    int n, lda, ldv, nrhs, flags;
};

__device__ double block_max(double v, double* sh) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    __syncthreads();
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    double r = sh[0];
    for (int k = 1; k < kRT / 32; k++) r = fmax(r, sh[k]);
    return r;
}

// Per item (one CTA, grid-stride over items): x64 = x32 (kInit) or
// x64 += x32 (kAccum); r = b - M x64 in FP64 (M = storage transpose, so
// (Mx)_i = sum_j a0[j*lda + i] x_j), r -> x32; the HPL scaled residual
// ||r|| / ((||M|| ||x|| + ||b||) n eps), infinity norms, max over the
// right-hand sides (LINPACK/src/host/gmres.c:182-193); NaN when anything is
// not finite.
__global__ void __launch_bounds__(kRT) k_wave_residual(const WaveItem* __restrict__ items, int count, double eps,
                                                     double* __restrict__ resid) {
    __shared__ double xs[4][kWaveMaxN];
    __shared__ double sh[kRT / 32];
    const int tid = threadIdx.x;
    for (int t = blockIdx.x; t < count; t += gridDim.x) {
        const WaveItem it = items[t];
        const int n = it.n, lda = it.lda, ld = it.ldv;
        for (int idx = tid; idx < it.nrhs * n; idx += kRT) {
            const int q = idx / n, i = idx - q * n;
            const size_t o = (size_t)q * ld + i;
            const double v = (double)it.x32[o];
            it.x64[o] = (it.flags & kAccum) ? it.x64[o] + v : v;
        }
        bool bad = false;
        double cmax = 0.0;
        for (int i = tid; i < n; i += kRT) {
            double s = 0.0;
            for (int j = 0; j < n; j++) s += fabs((double)it.a0[(size_t)j * lda + i]);
            bad |= !isfinite(s);
            cmax = fmax(cmax, s);
        }
        const double normA = block_max(cmax, sh);
        double res = 0.0;
        for (int q0 = 0; q0 < it.nrhs; q0 += 4) {
            const int qn = min(4, it.nrhs - q0);
            __syncthreads();  // xs of the previous chunk / item consumed; x64 writes visible
            for (int idx = tid; idx < qn * n; idx += kRT) {
                const int q = idx / n, i = idx - q * n;
                xs[q][i] = it.x64[(size_t)(q0 + q) * ld + i];
            }
            __syncthreads();
            double rm[4] = {0, 0, 0, 0}, xm[4] = {0, 0, 0, 0}, bm[4] = {0, 0, 0, 0};
            for (int i = tid; i < n; i += kRT) {
                double acc[4], bv[4];
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    bv[q] = q < qn ? (double)it.b0[(size_t)(q0 + q) * ld + i] : 0.0;
                    acc[q] = bv[q];
                }
                for (int j = 0; j < n; j++) {
                    const double a = (double)it.a0[(size_t)j * lda + i];
#pragma unroll
                    for (int q = 0; q < 4; q++) acc[q] = fma(-a, xs[q][j], acc[q]);
                }
#pragma unroll
                for (int q = 0; q < 4; q++)
                    if (q < qn) {
                        it.x32[(size_t)(q0 + q) * ld + i] = (float)acc[q];
                        bad |= !isfinite(acc[q]) || !isfinite(xs[q][i]);
                        rm[q] = fmax(rm[q], fabs(acc[q]));
                        xm[q] = fmax(xm[q], fabs(xs[q][i]));
                        bm[q] = fmax(bm[q], fabs(bv[q]));
                    }
            }
            for (int q = 0; q < qn; q++) {
                const double r = block_max(rm[q], sh), x = block_max(xm[q], sh), b = block_max(bm[q], sh);
                res = fmax(res, r / (normA * x + b) / (double)n / eps);
            }
        }
        bad = __syncthreads_or(bad);
        if (tid == 0) resid[t] = (bad || !isfinite(res)) ? NAN : res;
    }
}

// ---- host side --------------------------------------------------------------

struct Slab {
    void* ptr = nullptr;
    size_t bytes = 0;
    int refs = 0;
};

struct Entry {
    long long key = 0;
    int n = 0, ld = 0;  // ld: padded order (slot systems) or leading dimension (wave systems)
    float* lu = nullptr;
    float* a0 = nullptr;
    Slab* slab = nullptr;
    double last_used = 0.0;
    int users = 0;       // in-flight requests holding it
    bool ready = false;  // factors written
    bool cached = true;  // in the key map (false: private to one request)
    bool in_lru = false;
    std::list<Entry*>::iterator lru_pos;
};

struct Req {
    lp_request q{};
    lp_result res{};
    Entry* entry = nullptr;
    bool hit = false;
    size_t reserve = 0;  // per-request vectors charged to the budget
};

// Factorization block of the slot path: 128 is the fastest for every n the
// server accepts, in FP32 and in the tensor-core precisions (measured on B200
// against 256 and 512 for n = 1024 .. 8192).
int pad_block(int) { return 128; }
int round4(int n) { return (n + 3) / 4 * 4; }
// FP32 / FP64 right-hand-side, solution and residual vectors of one request
size_t vec_bytes(int n, int nrhs) { return (size_t)nrhs * (size_t)(n + 256) * 40 + (size_t)(n + 256) * 8; }
size_t slab_bytes_slot(int n) {
    const size_t bs = pad_block(n), npad = (n + bs - 1) / bs * bs;
    return 2 * sizeof(float) * npad * npad;
}
size_t slab_bytes_wave(int n) { return 2 * sizeof(float) * (size_t)n * round4(n); }

}  // namespace
}  // namespace lp

using namespace lp;

struct lp_worker {
    lp_ctx* c = nullptr;
    bool wave = false;
    bool large_only = false;       // slot reserved for systems with n > large_n
    cudaStream_t base = nullptr;   // the context's own main stream
    cudaStream_t high = nullptr;   // main stream for systems with n > large_n (higher priority)
    Workspace sys, items, next, resid, b0, x32, x64, b32, runs;
    char* stage = nullptr;         // pinned host staging of a wave's descriptors and residuals
    size_t stage_cap = 0;          // systems it holds
};

struct lp_server {
    lp_server_config cfg{};
    int device = 0;
    cudaMemPool_t pool = nullptr;
    cudaStream_t free_stream = nullptr;
    std::vector<lp_worker*> workers;
    std::vector<std::thread> threads;
    std::mutex mu;
    std::condition_variable cv_work, cv_done, cv_ready;
    int ready = 0;                 // workers through their warm-up
    int start_status = LP_OK;
    std::deque<Req*> pending;
    std::deque<lp_result> done;
    std::unordered_map<long long, Entry*> cache;
    std::list<Entry*> lru;  // ready cached entries, least recently used first
    size_t used = 0;
    long long next_id = 1;
    bool stop = false;
    int running = 0;
    long long completed = 0, waves = 0, waved_systems = 0, evictions = 0, rejected = 0;
    double slot_busy = 0.0, wave_busy = 0.0;
};

namespace lp {
namespace {

// ---- cache / budget (caller holds s->mu) ----

void release_slab(lp_server* s, Slab* sl) {
    if (--sl->refs > 0) return;
    if (sl->ptr != nullptr) cudaFreeAsync(sl->ptr, s->free_stream);
    s->used -= sl->bytes;
    delete sl;
}

void drop_entry(lp_server* s, Entry* e) {
    if (e->in_lru) s->lru.erase(e->lru_pos);
    if (e->cached) {
        auto it = s->cache.find(e->key);
        if (it != s->cache.end() && it->second == e) s->cache.erase(it);
    }
    if (e->slab != nullptr) release_slab(s, e->slab);
    delete e;
}

bool make_room(lp_server* s, size_t need) {
    const size_t budget = (size_t)s->cfg.hbm_budget_bytes;
    while (s->used + need > budget) {
        Entry* victim = nullptr;
        for (Entry* e : s->lru)  // in-flight entries are few: the first idle one is close to the front
            if (e->users == 0) {
                victim = e;
                break;
            }
        if (victim == nullptr) return false;
        drop_entry(s, victim);
        s->evictions++;
    }
    return true;
}

void finish_locked(lp_server* s, Req* r, int status) {
    r->res.status = status;
    r->res.t_done = now_s();
    s->used -= r->reserve;
    r->reserve = 0;
    if (Entry* e = r->entry) {
        e->users--;
        e->last_used = r->res.t_done;
        if (status == LP_OK) {
            e->ready = true;
            if (e->cached) {  // most recently used at the back
                if (e->in_lru)
                    s->lru.splice(s->lru.end(), s->lru, e->lru_pos);
                else
                    e->lru_pos = s->lru.insert(s->lru.end(), e);
                e->in_lru = true;
            } else if (e->users == 0) {
                drop_entry(s, e);
            }
        } else if (!e->ready && e->users == 0) {
            drop_entry(s, e);  // its factors were never completed
        }
    }
    s->done.push_back(r->res);
    s->completed++;
    s->running--;
    delete r;
}

// Admission of a pending request: 1 = take it now, 0 = leave it pending,
// -1 = finished with an error (result pushed).  On 1 the request holds its
// budget reservation and its cache entry (resident, or new and not ready).
int admit(lp_server* s, Req* r, bool wave) {
    const lp_request& q = r->q;
    auto it = s->cache.find(q.key);
    Entry* hit = nullptr;
    if (it != s->cache.end() && it->second->n == q.n) {
        if (!it->second->ready) return 0;  // being factored for another request
        hit = it->second;
    }
    if (hit == nullptr && q.A == nullptr) {
        r->res.t_start = now_s();
        fail(LP_E_STATE, "serve: factors no longer resident and no matrix given");
        s->running++;
        finish_locked(s, r, LP_E_STATE);
        return -1;
    }
    const size_t slab = hit != nullptr ? 0 : (wave ? slab_bytes_wave(q.n) : slab_bytes_slot(q.n));
    const size_t need = slab + vec_bytes(q.n, q.nrhs);
    if (need > (size_t)s->cfg.hbm_budget_bytes) {
        r->res.t_start = now_s();
        fail(LP_E_BUDGET, "serve: request larger than the device-memory budget");
        s->rejected++;
        s->running++;
        finish_locked(s, r, LP_E_BUDGET);
        return -1;
    }
    if (hit != nullptr) hit->users++;  // pinned before evicting for room
    if (!make_room(s, need)) {
        if (hit != nullptr) hit->users--;
        return 0;
    }
    s->used += need;
    r->reserve = need - slab;  // the slab part is released with the slab
    r->hit = hit != nullptr;
    if (hit != nullptr) {
        r->entry = hit;
    } else {
        Entry* e = new Entry();
        e->key = q.key;
        e->n = q.n;
        e->users = 1;
        if (it == s->cache.end())
            s->cache[q.key] = e;
        else
            e->cached = false;  // key resident with another n: served without caching
        e->slab = new Slab();   // charged now; memory attached by the worker
        e->slab->bytes = slab;
        e->slab->refs = 1;
        r->entry = e;
    }
    r->res.reused = r->hit ? 1 : 0;
    r->res.batched = wave ? 1 : 0;
    r->res.t_start = now_s();
    s->running++;
    return 1;
}

// ---- slot path: one system through the blocked factorization ----

int run_slot_on(lp_server* s, lp_worker* w, Req* r);

// Systems above large_n define the latency tail: their bulk work runs on the
// worker's higher-priority stream (the panels are on the top-priority
// auxiliary stream either way).
int run_slot(lp_server* s, lp_worker* w, Req* r) {
    const bool large = r->q.n > s->cfg.large_n && w->high != nullptr;
    if (large) w->c->stream = w->high;
    const int st = run_slot_on(s, w, r);
    w->c->stream = w->base;
    return st;
}

int run_slot_on(lp_server* s, lp_worker* w, Req* r) {
    lp_ctx* c = w->c;
    cudaStream_t st = c->stream;
    const lp_request& q = r->q;
    const int n = q.n, nrhs = q.nrhs, prec = s->cfg.precision;
    Entry* e = r->entry;
    if (!r->hit) {
        const int bs = pad_block(n), npad = (n + bs - 1) / bs * bs;
        void* p = nullptr;
        LP_CUDA(cudaMallocFromPoolAsync(&p, e->slab->bytes, s->pool, st));
        e->slab->ptr = p;
        e->ld = npad;
        e->lu = static_cast<float*>(p);
        e->a0 = e->lu + (size_t)npad * npad;
        LP_CUDA(cudaMemcpy2DAsync(e->a0, sizeof(float) * npad, q.A, sizeof(float) * q.lda, sizeof(float) * n, n,
                                  cudaMemcpyHostToDevice, st));
        if (npad > n) {
            k_pad_identity<<<2 * c->num_sms, 256, 0, st>>>(e->a0, npad, n, npad);
            count_launch();
            LP_CUDA(cudaGetLastError());
        }
        LP_CUDA(cudaMemcpyAsync(e->lu, e->a0, sizeof(float) * (size_t)npad * npad, cudaMemcpyDeviceToDevice, st));
        if (prec == LP_F32)
            LP_CHECK(gefa_f32(c, e->lu, npad, npad, bs, st));
        else
            LP_CHECK(gefa_mixed(c, prec, e->lu, npad, npad, bs, st));
    }
    const size_t nv = (size_t)n * nrhs;
    LP_CHECK(w->b32.ensure(sizeof(float) * nv));
    LP_CHECK(c->dB64.ensure(sizeof(double) * nv));
    LP_CHECK(c->dX.ensure(sizeof(double) * nv));
    float* b32 = static_cast<float*>(w->b32.ptr);
    double* b64 = static_cast<double*>(c->dB64.ptr);
    double* x = static_cast<double*>(c->dX.ptr);
    LP_CUDA(cudaMemcpy2DAsync(b32, sizeof(float) * n, q.B, sizeof(float) * q.ldb, sizeof(float) * n, nrhs,
                              cudaMemcpyHostToDevice, st));
    LP_CHECK(launch_f32_to_f64(b64, b32, nv, st));
    int iters = 0;
    double resid = 0.0;
    const int maxit = prec == LP_F32 ? 0 : s->cfg.max_refinements;
    const int rs = refine_core(c, e->a0, e->ld, e->lu, n, b64, x, nrhs, maxit, &iters, &resid, st);
    if (rs != LP_OK && rs != LP_E_NUMERIC) return rs;
    LP_CUDA(cudaMemcpy2DAsync(q.X, sizeof(double) * q.ldx, x, sizeof(double) * n, sizeof(double) * n, nrhs,
                              cudaMemcpyDeviceToHost, st));
    LP_CHECK(wait_stream(c, st));
    // refine_core normalizes with DBL_EPSILON/2; the FP32 mode states its own unit roundoff
    r->res.hpl_resid = prec == LP_F32 ? resid * (DBL_EPSILON / FLT_EPSILON) : resid;
    r->res.ir_iters = iters;
    return rs;
}

// ---- wave path: many systems in one batched launch ----

// Pinned staging per system: lp_system + WaveItem + CopyRun + one residual.
constexpr size_t kStagePer = sizeof(lp_system) + sizeof(WaveItem) + sizeof(CopyRun) + sizeof(double);

int ensure_stage(lp_worker* w, size_t count) {
    if (w->stage_cap >= count) return LP_OK;
    if (w->stage != nullptr) cudaFreeHost(w->stage);
    w->stage = nullptr;
    w->stage_cap = 0;
    LP_CUDA(cudaMallocHost(&w->stage, kStagePer * count));
    w->stage_cap = count;
    return LP_OK;
}

int run_wave(lp_server* s, lp_worker* w, std::vector<Req*>& rs) {
    lp_ctx* c = w->c;
    cudaStream_t st = c->stream;
    const int prec = s->cfg.precision;
    std::stable_sort(rs.begin(), rs.end(), [](const Req* a, const Req* b) { return a->q.n > b->q.n; });
    const int count = (int)rs.size();
    // vectors of all systems; a slab (factors, then the original) per new system
    size_t vtot = 0;
    std::vector<size_t> voff(count);
    for (int i = 0; i < count; i++) {
        voff[i] = vtot;
        vtot += (size_t)rs[i]->q.nrhs * round4(rs[i]->q.n);
    }
    std::vector<CopyRun> dup;
    for (Req* r : rs)
        if (!r->hit) {
            Entry* e = r->entry;
            void* p = nullptr;
            LP_CUDA(cudaMallocFromPoolAsync(&p, e->slab->bytes, s->pool, st));
            e->slab->ptr = p;
            e->ld = round4(e->n);
            e->lu = static_cast<float*>(p);
            e->a0 = e->lu + (size_t)e->n * e->ld;
            dup.push_back(CopyRun{reinterpret_cast<const float4*>(e->a0), reinterpret_cast<float4*>(e->lu),
                                  (long long)e->n * e->ld / 4});
        }
    LP_CHECK(w->b0.ensure(sizeof(float) * vtot));
    LP_CHECK(w->x32.ensure(sizeof(float) * vtot));
    LP_CHECK(w->x64.ensure(sizeof(double) * vtot));
    LP_CHECK(w->sys.ensure(sizeof(lp_system) * count));
    LP_CHECK(w->items.ensure(sizeof(WaveItem) * count));
    LP_CHECK(w->resid.ensure(sizeof(double) * count));
    LP_CHECK(w->next.ensure(sizeof(int)));
    float* b0 = static_cast<float*>(w->b0.ptr);
    float* x32 = static_cast<float*>(w->x32.ptr);
    double* x64 = static_cast<double*>(w->x64.ptr);
    for (int i = 0; i < count; i++) {
        const lp_request& q = rs[i]->q;
        Entry* e = rs[i]->entry;
        if (!rs[i]->hit)
            LP_CUDA(cudaMemcpy2DAsync(e->a0, sizeof(float) * e->ld, q.A, sizeof(float) * q.lda, sizeof(float) * q.n,
                                      q.n, cudaMemcpyHostToDevice, st));
        LP_CUDA(cudaMemcpy2DAsync(b0 + voff[i], sizeof(float) * round4(q.n), q.B, sizeof(float) * q.ldb,
                                  sizeof(float) * q.n, q.nrhs, cudaMemcpyHostToDevice, st));
    }
    LP_CHECK(ensure_stage(w, (size_t)count));
    lp_system* h_sys = reinterpret_cast<lp_system*>(w->stage);
    WaveItem* h_items = reinterpret_cast<WaveItem*>(w->stage + sizeof(lp_system) * w->stage_cap);
    CopyRun* h_runs = reinterpret_cast<CopyRun*>(w->stage + (sizeof(lp_system) + sizeof(WaveItem)) * w->stage_cap);
    double* h_res =
        reinterpret_cast<double*>(w->stage + (sizeof(lp_system) + sizeof(WaveItem) + sizeof(CopyRun)) * w->stage_cap);
    if (!dup.empty()) {
        LP_CHECK(w->runs.ensure(sizeof(CopyRun) * dup.size()));
        std::memcpy(h_runs, dup.data(), sizeof(CopyRun) * dup.size());
        LP_CUDA(cudaMemcpyAsync(w->runs.ptr, h_runs, sizeof(CopyRun) * dup.size(), cudaMemcpyHostToDevice, st));
        k_copy_runs<<<std::min((int)dup.size(), 4 * c->num_sms), 256, 0, st>>>(static_cast<CopyRun*>(w->runs.ptr),
                                                                                (int)dup.size());
        count_launch();
        LP_CUDA(cudaGetLastError());
    }
    LP_CUDA(cudaMemcpyAsync(x32, b0, sizeof(float) * vtot, cudaMemcpyDeviceToDevice, st));

    std::vector<lp_system> sys(count);
    std::vector<WaveItem> items(count);
    for (int i = 0; i < count; i++) {
        const lp_request& q = rs[i]->q;
        Entry* e = rs[i]->entry;
        const int ldv = round4(q.n);
        sys[i] = lp_system{q.n, q.nrhs | (rs[i]->hit ? kBatchSolveOnly : 0), e->ld, ldv,
                           (long long)(uintptr_t)e->lu, (long long)(uintptr_t)(x32 + voff[i])};
        items[i] = WaveItem{e->a0, b0 + voff[i], x32 + voff[i], x64 + voff[i], q.n, e->ld, ldv, q.nrhs, kInit};
    }
    lp_batch_config bc;
    lp_batch_default_config(&bc);
    const double eps = prec == LP_F32 ? FLT_EPSILON / 2.0 : DBL_EPSILON / 2.0;
    // batched kernel on the first m descriptors, then the residual of those systems
    auto step = [&](const std::vector<lp_system>& d, const std::vector<WaveItem>& wi) -> int {
        const int m = (int)d.size();
        std::memcpy(h_sys, d.data(), sizeof(lp_system) * m);
        std::memcpy(h_items, wi.data(), sizeof(WaveItem) * m);
        LP_CUDA(cudaMemcpyAsync(w->sys.ptr, h_sys, sizeof(lp_system) * m, cudaMemcpyHostToDevice, st));
        LP_CUDA(cudaMemcpyAsync(w->items.ptr, h_items, sizeof(WaveItem) * m, cudaMemcpyHostToDevice, st));
        LP_CHECK(launch_batch(c, static_cast<lp_system*>(w->sys.ptr), m, nullptr, nullptr, bc,
                              static_cast<int*>(w->next.ptr), st, true));
        k_wave_residual<<<std::min(m, 4 * c->num_sms), kRT, 0, st>>>(static_cast<WaveItem*>(w->items.ptr), m, eps,
                                                                      static_cast<double*>(w->resid.ptr));
        count_launch();
        LP_CUDA(cudaGetLastError());
        LP_CUDA(cudaMemcpyAsync(h_res, w->resid.ptr, sizeof(double) * m, cudaMemcpyDeviceToHost, st));
        LP_CHECK(wait_stream(c, st));
        return LP_OK;
    };
    LP_CHECK(step(sys, items));
    std::vector<double> final_res(h_res, h_res + count);
    std::vector<int> iters(count, 0);
    if (prec != LP_F32) {
        // batched refinement of the systems above the bound: d = LU \ r (solve only), x += d
        for (int it = 0; it < s->cfg.max_refinements; it++) {
            std::vector<int> idx;
            for (int i = 0; i < count; i++)
                if (std::isfinite(final_res[i]) && final_res[i] > 16.0) idx.push_back(i);
            if (idx.empty()) break;
            std::vector<lp_system> d;
            std::vector<WaveItem> wi;
            for (int i : idx) {
                lp_system x = sys[i];
                x.nrhs = rs[i]->q.nrhs | kBatchSolveOnly;
                d.push_back(x);
                WaveItem y = items[i];
                y.flags = kAccum;
                wi.push_back(y);
            }
            LP_CHECK(step(d, wi));
            for (size_t k = 0; k < idx.size(); k++) {
                final_res[idx[k]] = h_res[k];
                iters[idx[k]]++;
            }
        }
    }
    for (int i = 0; i < count; i++) {
        const lp_request& q = rs[i]->q;
        LP_CUDA(cudaMemcpy2DAsync(q.X, sizeof(double) * q.ldx, x64 + voff[i], sizeof(double) * round4(q.n),
                                  sizeof(double) * q.n, q.nrhs, cudaMemcpyDeviceToHost, st));
    }
    LP_CHECK(wait_stream(c, st));
    for (int i = 0; i < count; i++) {
        rs[i]->res.hpl_resid = final_res[i];
        rs[i]->res.ir_iters = iters[i];
    }
    return LP_OK;
}

// ---- warm-up (lp_server_config::warm_n) ----

// Factor and solve an identity of order warm_n with the maximum number of
// right-hand sides on the slot's stream, so every workspace of the slot path
// reaches its final size before the first request.
int warm_slot(lp_server* s, lp_worker* w) {
    lp_ctx* c = w->c;
    cudaStream_t st = c->stream;
    const int bs = pad_block(s->cfg.warm_n), npad = (s->cfg.warm_n + bs - 1) / bs * bs;
    const size_t nn = (size_t)npad * npad, nv = (size_t)npad * kMaxRhs;
    void* p = nullptr;
    LP_CUDA(cudaMallocFromPoolAsync(&p, 2 * sizeof(float) * nn, s->pool, st));
    float* lu = static_cast<float*>(p);
    float* a0 = lu + nn;
    int rc = LP_OK;
    auto run = [&]() -> int {
        k_pad_identity<<<2 * c->num_sms, 256, 0, st>>>(a0, npad, 0, npad);
        count_launch();
        LP_CUDA(cudaGetLastError());
        LP_CUDA(cudaMemcpyAsync(lu, a0, sizeof(float) * nn, cudaMemcpyDeviceToDevice, st));
        if (s->cfg.precision == LP_F32)
            LP_CHECK(gefa_f32(c, lu, npad, npad, bs, st));
        else
            LP_CHECK(gefa_mixed(c, s->cfg.precision, lu, npad, npad, bs, st));
        LP_CHECK(w->b32.ensure(sizeof(float) * nv));
        LP_CHECK(c->dB64.ensure(sizeof(double) * nv));
        LP_CHECK(c->dX.ensure(sizeof(double) * nv));
        // right-hand sides: the first rows of the identity
        LP_CUDA(cudaMemcpyAsync(w->b32.ptr, a0, sizeof(float) * nv, cudaMemcpyDeviceToDevice, st));
        LP_CHECK(launch_f32_to_f64(static_cast<double*>(c->dB64.ptr), static_cast<float*>(w->b32.ptr), nv, st));
        int iters = 0;
        double resid = 0.0;
        return refine_core(c, a0, npad, lu, npad, static_cast<double*>(c->dB64.ptr),
                           static_cast<double*>(c->dX.ptr), kMaxRhs, 1, &iters, &resid, st);
    };
    rc = run();
    cudaFreeAsync(p, st);
    const int ws = wait_stream(c, st);
    return rc != LP_OK ? rc : ws;
}

// Size a wave worker's scratch for the largest wave the configuration allows.
int warm_wave(lp_server* s, lp_worker* w) {
    const size_t count = (size_t)s->cfg.batch_max_count;
    const size_t vtot = count * kMaxRhs * (size_t)round4(s->cfg.batch_max_n);
    LP_CHECK(w->b0.ensure(sizeof(float) * vtot));
    LP_CHECK(w->x32.ensure(sizeof(float) * vtot));
    LP_CHECK(w->x64.ensure(sizeof(double) * vtot));
    LP_CHECK(w->sys.ensure(sizeof(lp_system) * count));
    LP_CHECK(w->items.ensure(sizeof(WaveItem) * count));
    LP_CHECK(w->resid.ensure(sizeof(double) * count));
    LP_CHECK(w->next.ensure(sizeof(int)));
    LP_CHECK(w->runs.ensure(sizeof(CopyRun) * count));
    return ensure_stage(w, count);
}

// ---- worker threads ----

void worker_loop(lp_server* s, lp_worker* w) {
    cudaSetDevice(s->device);
    const bool per_request = s->cfg.mode == LP_SERVE_PER_REQUEST;
    {
        const int st = s->cfg.warm_n > 0 ? (w->wave ? warm_wave(s, w) : warm_slot(s, w)) : LP_OK;
        std::lock_guard<std::mutex> lock(s->mu);
        if (st != LP_OK && s->start_status == LP_OK) s->start_status = st;
        s->ready++;
        s->cv_ready.notify_all();
    }
    for (;;) {
        std::vector<Req*> take;
        {
            std::unique_lock<std::mutex> lock(s->mu);
            for (;;) {
                if (s->stop) return;
                for (auto it = s->pending.begin(); it != s->pending.end();) {
                    Req* r = *it;
                    const bool small = !per_request && r->q.n <= s->cfg.batch_max_n;
                    if (small != w->wave || (w->large_only && r->q.n <= s->cfg.large_n)) {
                        ++it;
                        continue;
                    }
                    const int a = admit(s, r, w->wave);
                    if (a == 0) {
                        if (per_request) break;  // strict arrival order
                        ++it;
                        continue;
                    }
                    it = s->pending.erase(it);
                    if (a == 1) {
                        take.push_back(r);
                        if (!w->wave || (int)take.size() >= s->cfg.batch_max_count) break;
                    }
                }
                s->cv_done.notify_all();  // rejections may have been pushed
                if (!take.empty()) break;
                s->cv_work.wait(lock);
            }
        }
        const double t0 = now_s();
        const int st = w->wave ? run_wave(s, w, take) : run_slot(s, w, take[0]);
        {
            std::lock_guard<std::mutex> lock(s->mu);
            (w->wave ? s->wave_busy : s->slot_busy) += now_s() - t0;
            if (w->wave) {
                s->waves++;
                s->waved_systems += (long long)take.size();
            }
            for (Req* r : take) {
                int rst = st;
                if (rst == LP_OK && !std::isfinite(r->res.hpl_resid)) rst = LP_E_NUMERIC;
                finish_locked(s, r, rst);
            }
        }
        s->cv_done.notify_all();
        s->cv_work.notify_all();
    }
}

int check_request(const lp_request* q) {
    if (q == nullptr) return fail(LP_E_INVALID, "lp_server_submit: null request");
    if (q->n <= 0 || q->n > kMaxN || q->nrhs <= 0 || q->nrhs > kMaxRhs)
        return fail(LP_E_INVALID, "lp_server_submit: need 1 <= n <= 16384 and 1 <= nrhs <= 16");
    if (q->B == nullptr || q->X == nullptr || q->ldb < q->n || q->ldx < q->n || (q->A != nullptr && q->lda < q->n))
        return fail(LP_E_INVALID, "lp_server_submit: null B / X or leading dimension below n");
    return LP_OK;
}

}  // namespace
}  // namespace lp

extern "C" {

int lp_server_default_config(lp_server_config* cfg) {
    if (cfg == nullptr) return fail(LP_E_INVALID, "lp_server_default_config: null output");
    cfg->hbm_budget_bytes = 80ll * 1000 * 1000 * 1000;
    cfg->mode = LP_SERVE_CONTINUOUS;
    cfg->precision = LP_F32;
    cfg->slots = 6;
    cfg->batch_workers = 2;
    cfg->batch_max_n = 512;
    cfg->batch_max_count = 1024;
    cfg->max_refinements = 50;
    cfg->warm_n = 0;
    cfg->reserve_bytes = 0;
    cfg->large_n = 2048;
    cfg->large_slots = 2;
    return LP_OK;
}

int lp_server_start(int device, const lp_server_config* cfg, lp_server** out) {
    if (out == nullptr) return fail(LP_E_INVALID, "lp_server_start: null output");
    *out = nullptr;
    lp_server_config c;
    if (cfg != nullptr)
        c = *cfg;
    else
        lp_server_default_config(&c);
    if (c.hbm_budget_bytes <= 0 || (c.mode != LP_SERVE_CONTINUOUS && c.mode != LP_SERVE_PER_REQUEST) ||
        (c.precision != LP_F32 && c.precision != LP_BF16_IR && c.precision != LP_FP8_IR) || c.slots < 1 ||
        c.slots > 16 || c.batch_workers < 1 || c.batch_workers > 4 || c.batch_max_n < 0 ||
        c.batch_max_n > kWaveMaxN || c.batch_max_count < 1 || c.max_refinements < 0 || c.warm_n < 0 ||
        c.warm_n > kMaxN || c.reserve_bytes < 0 || c.large_n < 0 ||
        c.large_slots < 0)
        return fail(LP_E_INVALID, "lp_server_start: bad configuration");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(LP_E_NODEVICE, "lp_server_start: no CUDA device");
    }
    if (device < 0 || device >= ndev) return fail(LP_E_INVALID, "lp_server_start: bad device");
    LP_CUDA(cudaSetDevice(device));
    lp_server* s = new lp_server();
    s->cfg = c;
    s->device = device;
    auto undo = [&](int st) {
        for (auto* w : s->workers) {
            if (w->c) lp_ctx_destroy(w->c);
            if (w->high) cudaStreamDestroy(w->high);
            delete w;
        }
        if (s->free_stream) cudaStreamDestroy(s->free_stream);
        if (s->pool) cudaMemPoolDestroy(s->pool);
        delete s;
        return st;
    };
    cudaMemPoolProps props;
    std::memset(&props, 0, sizeof(props));
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    cudaError_t e = cudaMemPoolCreate(&s->pool, &props);
    if (e != cudaSuccess) return undo(cuda_fail(e, "cudaMemPoolCreate", __FILE__, __LINE__));
    uint64_t keep = UINT64_MAX;  // freed slabs stay in the pool for reuse
    e = cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    if (e != cudaSuccess) return undo(cuda_fail(e, "cudaMemPoolSetAttribute", __FILE__, __LINE__));
    e = cudaStreamCreateWithFlags(&s->free_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return undo(cuda_fail(e, "cudaStreamCreate", __FILE__, __LINE__));
    if (c.reserve_bytes > 0) {  // map the memory now; the release threshold keeps it in the pool
        void* p = nullptr;
        e = cudaMallocFromPoolAsync(&p, (size_t)c.reserve_bytes, s->pool, s->free_stream);
        if (e == cudaSuccess) e = cudaFreeAsync(p, s->free_stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s->free_stream);
        if (e != cudaSuccess) return undo(cuda_fail(e, "lp_server_start: pool reservation", __FILE__, __LINE__));
    }
    const bool per_request = c.mode == LP_SERVE_PER_REQUEST;
    const int nslots = per_request ? 1 : c.slots;
    const int nwaves = per_request || c.batch_max_n == 0 ? 0 : c.batch_workers;
    int prio_least = 0, prio_greatest = 0;
    cudaDeviceGetStreamPriorityRange(&prio_least, &prio_greatest);
    const int prio_large = prio_greatest < prio_least ? prio_greatest + 1 : prio_least;
    for (int i = 0; i < nslots + nwaves; i++) {
        lp_worker* w = new lp_worker();
        w->wave = i >= nslots;
        w->large_only = !per_request && i < std::min(c.large_slots, c.slots - 1);
        s->workers.push_back(w);
        const int st = lp_ctx_create(device, &w->c);
        if (st != LP_OK) return undo(st);
        w->base = w->c->stream;
        if (!w->wave && !per_request) {
            e = cudaStreamCreateWithPriority(&w->high, cudaStreamNonBlocking, prio_large);
            if (e != cudaSuccess) return undo(cuda_fail(e, "cudaStreamCreateWithPriority", __FILE__, __LINE__));
        }
    }
    for (auto* w : s->workers) s->threads.emplace_back(worker_loop, s, w);
    int st = LP_OK;
    {
        std::unique_lock<std::mutex> lock(s->mu);
        s->cv_ready.wait(lock, [&] { return s->ready == (int)s->workers.size(); });
        st = s->start_status;
    }
    if (st != LP_OK) {
        lp_server_stop(s);
        return fail(st, "lp_server_start: worker warm-up failed");
    }
    *out = s;
    return LP_OK;
}

int lp_server_stop(lp_server* s) {
    if (s == nullptr) return LP_OK;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    for (auto& t : s->threads) t.join();
    cudaSetDevice(s->device);
    for (auto* r : s->pending) delete r;
    s->pending.clear();
    std::vector<Entry*> all;
    for (auto& kv : s->cache) all.push_back(kv.second);
    for (Entry* e : all) drop_entry(s, e);
    cudaStreamSynchronize(s->free_stream);
    for (auto* w : s->workers) {
        Workspace* ws[] = {&w->sys, &w->items, &w->next, &w->resid, &w->b0, &w->x32, &w->x64, &w->b32, &w->runs};
        for (auto* x : ws) x->release();
        lp_ctx_destroy(w->c);
        if (w->high) cudaStreamDestroy(w->high);
        if (w->stage) cudaFreeHost(w->stage);
        delete w;
    }
    cudaStreamDestroy(s->free_stream);
    cudaMemPoolDestroy(s->pool);
    delete s;
    return LP_OK;
}

int lp_server_submit(lp_server* s, const lp_request* req, long long* id) {
    if (s == nullptr) return fail(LP_E_INVALID, "lp_server_submit: null server");
    LP_CHECK(check_request(req));
    Req* r = new Req();
    r->q = *req;
    r->res.key = req->key;
    r->res.n = req->n;
    r->res.nrhs = req->nrhs;
    r->res.hpl_resid = NAN;
    r->res.t_submit = now_s();
    {
        std::lock_guard<std::mutex> lock(s->mu);
        if (req->A == nullptr) {
            auto it = s->cache.find(req->key);
            if (it == s->cache.end() || it->second->n != req->n) {
                delete r;
                return fail(LP_E_STATE, "lp_server_submit: no matrix given and none resident under this key");
            }
        }
        r->res.id = s->next_id++;
        if (id != nullptr) *id = r->res.id;
        s->pending.push_back(r);
    }
    s->cv_work.notify_all();
    return LP_OK;
}

int lp_server_poll(lp_server* s, lp_result* out, int max, int timeout_ms, int* count) {
    if (s == nullptr || out == nullptr || count == nullptr || max <= 0)
        return fail(LP_E_INVALID, "lp_server_poll: bad argument");
    *count = 0;
    std::unique_lock<std::mutex> lock(s->mu);
    if (s->done.empty() && timeout_ms > 0)
        s->cv_done.wait_for(lock, std::chrono::milliseconds(timeout_ms), [&] { return !s->done.empty(); });
    int k = 0;
    while (!s->done.empty() && k < max) {
        out[k++] = s->done.front();
        s->done.pop_front();
    }
    *count = k;
    if (k == 0) return fail(LP_E_TIMEOUT, "lp_server_poll: no result within the timeout");
    return LP_OK;
}

int lp_server_get_info(lp_server* s, lp_server_info* info) {
    if (s == nullptr || info == nullptr) return fail(LP_E_INVALID, "lp_server_get_info: null argument");
    std::lock_guard<std::mutex> lock(s->mu);
    info->pending = (int)s->pending.size();
    info->running = s->running;
    info->resident = (int)s->cache.size();
    info->used_bytes = (long long)s->used;
    info->completed = s->completed;
    info->waves = s->waves;
    info->waved_systems = s->waved_systems;
    info->evictions = s->evictions;
    info->rejected = s->rejected;
    uint64_t reserved = 0;
    cudaMemPoolGetAttribute(s->pool, cudaMemPoolAttrReservedMemCurrent, &reserved);
    info->pool_reserved_bytes = (long long)reserved;
    info->slot_busy_s = s->slot_busy;
    info->wave_busy_s = s->wave_busy;
    return LP_OK;
}

int lp_server_replay(lp_server* s, int count, const lp_request* reqs, const double* arrival_s, lp_result* out,
                     int timeout_ms) {
    if (s == nullptr || count < 0 || (count > 0 && (reqs == nullptr || arrival_s == nullptr || out == nullptr)) ||
        timeout_ms <= 0)
        return fail(LP_E_INVALID, "lp_server_replay: bad argument");
    std::vector<long long> ids(count, 0);
    std::vector<lp_result> got;
    got.reserve(count);
    std::atomic<int> submitted{0};
    std::atomic<bool> all_submitted{false};
    bool timed_out = false;
    std::thread poller([&] {
        std::vector<lp_result> buf(256);
        double last = now_s();
        for (;;) {
            int k = 0;
            lp_server_poll(s, buf.data(), (int)buf.size(), 20, &k);
            const double t = now_s();
            got.insert(got.end(), buf.begin(), buf.begin() + k);
            const int have = (int)got.size(), sent = submitted.load();
            if (all_submitted.load() && have >= submitted.load()) break;
            if (k > 0 || have >= sent) last = t;  // progress, or nothing outstanding
            if (t - last > timeout_ms * 1e-3) {
                timed_out = true;
                break;
            }
        }
    });
    const double t0 = now_s();
    for (int i = 0; i < count; i++) {
        const double target = t0 + arrival_s[i];
        for (;;) {
            const double d = target - now_s();
            if (d <= 0) break;
            if (d > 3e-4) std::this_thread::sleep_for(std::chrono::duration<double>(d - 2e-4));
        }
        long long id = 0;
        const int st = lp_server_submit(s, &reqs[i], &id);
        if (st == LP_OK) {
            ids[i] = id;
            submitted.fetch_add(1);
        } else {
            ids[i] = -1;
            out[i] = lp_result{};
            out[i].id = -1;
            out[i].key = reqs[i].key;
            out[i].status = st;
            out[i].n = reqs[i].n;
            out[i].nrhs = reqs[i].nrhs;
            out[i].hpl_resid = NAN;
            out[i].t_submit = out[i].t_start = out[i].t_done = now_s();
        }
    }
    all_submitted.store(true);
    poller.join();
    std::unordered_map<long long, int> where;
    for (int i = 0; i < count; i++)
        if (ids[i] > 0) where[ids[i]] = i;
    for (const auto& r : got) {
        auto it = where.find(r.id);
        if (it != where.end()) out[it->second] = r;
    }
    if (timed_out) return fail(LP_E_TIMEOUT, "lp_server_replay: no result within the timeout");
    return LP_OK;
}

}  // extern "C"
