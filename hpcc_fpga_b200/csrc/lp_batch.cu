// Host side of the batched solver: the system list sorted by decreasing n
// (largest first, so one persistent launch balances any size mix), the
// launch captured once in a CUDA graph and replayed for the same batch, the
// per-bucket autotuner.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "lp_ctx.cuh"

namespace lp {

namespace {

uint64_t fnv(const void* p, size_t bytes, uint64_t h = 1469598103934665603ull) {
    const unsigned char* s = static_cast<const unsigned char*>(p);
    for (size_t i = 0; i < bytes; i++) h = (h ^ s[i]) * 1099511628211ull;
    return h;
}

double batch_flops(const std::vector<lp_system>& v) {
    double f = 0.0;
    for (const auto& s : v) {
        const double n = s.n;
        f += 2.0 * n * n * n / 3.0 + 2.0 * s.nrhs * n * n;
    }
    return f;
}

int bucket_of_host(int n) { return n <= 64 ? 0 : n <= 128 ? 1 : n <= 256 ? 2 : n <= 512 ? 3 : 4; }

// Upload the sorted descriptors (if they changed) and launch through the
// cached graph (captured on first use for this batch and configuration).
int run_batch(lp_ctx* c, const std::vector<lp_system>& sorted, float* dA, float* dB, const lp_batch_config& cfg,
              bool use_graph, int* replayed) {
    cudaStream_t st = c->stream;
    const int count = (int)sorted.size();
    LP_CHECK(c->bsys.ensure(sizeof(lp_system) * (size_t)(count > 0 ? count : 1)));
    LP_CHECK(c->bnext.ensure(sizeof(int)));
    uint64_t h = fnv(sorted.data(), sizeof(lp_system) * sorted.size());
    h = fnv(&cfg, sizeof(cfg), h);
    h = fnv(&dA, sizeof(dA), h);
    h = fnv(&dB, sizeof(dB), h);
    if (h != c->bsys_hash) {
        LP_CUDA(cudaMemcpyAsync(c->bsys.ptr, sorted.data(), sizeof(lp_system) * sorted.size(), cudaMemcpyHostToDevice,
                                st));
        if (c->bgraph != nullptr) {
            cudaGraphExecDestroy(c->bgraph);
            c->bgraph = nullptr;
        }
        c->bsys_hash = h;
    }
    *replayed = 0;
    if (!use_graph)
        return launch_batch(c, static_cast<lp_system*>(c->bsys.ptr), count, dA, dB, cfg,
                            static_cast<int*>(c->bnext.ptr), st);
    if (c->bgraph == nullptr) {
        cudaGraph_t g = nullptr;
        LP_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        const int s = launch_batch(c, static_cast<lp_system*>(c->bsys.ptr), count, dA, dB, cfg,
                                   static_cast<int*>(c->bnext.ptr), st);
        const cudaError_t e = cudaStreamEndCapture(st, &g);
        if (s != LP_OK) {
            if (g != nullptr) cudaGraphDestroy(g);
            return s;
        }
        if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture(batch)", __FILE__, __LINE__);
        const cudaError_t ie = cudaGraphInstantiate(&c->bgraph, g, 0);
        cudaGraphDestroy(g);
        if (ie != cudaSuccess) return cuda_fail(ie, "cudaGraphInstantiate(batch)", __FILE__, __LINE__);
    } else {
        *replayed = 1;
    }
    LP_CUDA(cudaGraphLaunch(c->bgraph, st));
    return LP_OK;
}

std::vector<lp_system> sorted_by_n(int count, const lp_system* systems) {
    std::vector<lp_system> v(systems, systems + count);
    std::stable_sort(v.begin(), v.end(), [](const lp_system& x, const lp_system& y) { return x.n > y.n; });
    return v;
}

// The same order as positions: order[k] = index (in the caller's list) of the k-th system run.
std::vector<int> order_by_n(int count, const lp_system* systems) {
    std::vector<int> o(count);
    for (int i = 0; i < count; i++) o[i] = i;
    std::stable_sort(o.begin(), o.end(), [&](int x, int y) { return systems[x].n > systems[y].n; });
    return o;
}

// Extents (in elements) of the matrix and vector regions a batch touches.
void batch_extents(int count, const lp_system* systems, size_t* na, size_t* nb) {
    *na = 0;
    *nb = 0;
    for (int i = 0; i < count; i++) {
        const lp_system& s = systems[i];
        *na = std::max(*na, (size_t)(s.a_off + (long long)(s.n - 1) * s.lda + s.n));
        *nb = std::max(*nb, (size_t)(s.b_off + (long long)(s.nrhs - 1) * s.ldb + s.n));
    }
}

// The refined batched solve on device buffers (see lp_batch_solve_ir_dev):
// the originals are copied into the context, then one persistent launch
// (through a cached CUDA graph when use_graph) factors, solves and refines.
int run_batch_ir(lp_ctx* c, int precision, int count, const lp_system* systems, float* dA, const double* dB64,
                 double* dX, int max_iters, const lp_batch_config& cfg, lp_batch_stats* stats, int* iters_out,
                 double* resid_out) {
    cudaStream_t st = c->stream;
    size_t na = 0, nb = 0;
    batch_extents(count, systems, &na, &nb);
    const std::vector<int> order = order_by_n(count, systems);
    std::vector<lp_system> sorted(count);
    for (int k = 0; k < count; k++) sorted[k] = systems[order[k]];
    LP_CHECK(c->bA0.ensure(sizeof(float) * (na > 0 ? na : 1)));
    LP_CHECK(c->bB32.ensure(sizeof(float) * (nb > 0 ? nb : 1)));
    LP_CHECK(c->bout.ensure((sizeof(int) + sizeof(double)) * (size_t)(count > 0 ? count : 1)));
    LP_CHECK(c->bsys_ir.ensure(sizeof(lp_system) * (size_t)(count > 0 ? count : 1)));
    LP_CHECK(c->bnext.ensure(sizeof(int)));
    double* d_resid = static_cast<double*>(c->bout.ptr);
    int* d_iters = reinterpret_cast<int*>(d_resid + count);
    const bool bf16 = precision == LP_BF16_IR;
    uint64_t h = fnv(sorted.data(), sizeof(lp_system) * sorted.size());
    h = fnv(&cfg, sizeof(cfg), h);
    const void* ptrs[3] = {dA, dB64, dX};
    h = fnv(ptrs, sizeof(ptrs), h);
    const int key[2] = {precision, max_iters};
    h = fnv(key, sizeof(key), h);
    if (h != c->bir_hash) {
        LP_CUDA(cudaMemcpyAsync(c->bsys_ir.ptr, sorted.data(), sizeof(lp_system) * sorted.size(),
                                cudaMemcpyHostToDevice, st));
        if (c->bgraph_ir != nullptr) {
            cudaGraphExecDestroy(c->bgraph_ir);
            c->bgraph_ir = nullptr;
        }
        c->bir_hash = h;
    }
    auto enqueue = [&]() -> int {
        LP_CUDA(cudaMemcpyAsync(c->bA0.ptr, dA, sizeof(float) * na, cudaMemcpyDeviceToDevice, st));
        return launch_batch_ir(c, bf16, static_cast<lp_system*>(c->bsys_ir.ptr), count, dA,
                               static_cast<float*>(c->bA0.ptr), static_cast<float*>(c->bB32.ptr), dB64, dX, cfg,
                               max_iters, d_iters, d_resid, static_cast<int*>(c->bnext.ptr), st);
    };
    int replayed = 0;
    LP_CUDA(cudaEventRecord(c->ev[0], st));
    if (cfg.use_graph == 0) {
        LP_CHECK(enqueue());
    } else {
        if (c->bgraph_ir == nullptr) {
            cudaGraph_t g = nullptr;
            LP_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            const int s = enqueue();
            const cudaError_t e = cudaStreamEndCapture(st, &g);
            if (s != LP_OK) {
                if (g != nullptr) cudaGraphDestroy(g);
                return s;
            }
            if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture(refined batch)", __FILE__, __LINE__);
            const cudaError_t ie = cudaGraphInstantiate(&c->bgraph_ir, g, 0);
            cudaGraphDestroy(g);
            if (ie != cudaSuccess) return cuda_fail(ie, "cudaGraphInstantiate(refined batch)", __FILE__, __LINE__);
        } else {
            replayed = 1;
        }
        LP_CUDA(cudaGraphLaunch(c->bgraph_ir, st));
    }
    LP_CUDA(cudaEventRecord(c->ev[1], st));
    std::vector<double> res(count);
    std::vector<int> its(count);
    if (count > 0) {
        LP_CUDA(cudaMemcpyAsync(res.data(), d_resid, sizeof(double) * count, cudaMemcpyDeviceToHost, st));
        LP_CUDA(cudaMemcpyAsync(its.data(), d_iters, sizeof(int) * count, cudaMemcpyDeviceToHost, st));
    }
    LP_CUDA(cudaStreamSynchronize(st));
    bool finite = true;
    for (int k = 0; k < count; k++) {
        if (iters_out != nullptr) iters_out[order[k]] = its[k];
        if (resid_out != nullptr) resid_out[order[k]] = res[k];
        finite = finite && std::isfinite(res[k]);
    }
    if (stats != nullptr) {
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]);
        stats->seconds = ms * 1e-3;
        stats->flops = batch_flops(sorted);
        stats->gflops = stats->seconds > 0 ? stats->flops / stats->seconds / 1e9 : 0.0;
        stats->solves_per_s = stats->seconds > 0 ? count / stats->seconds : 0.0;
        stats->systems = count;
        stats->graph_replayed = replayed;
    }
    if (!finite) return fail(LP_E_NUMERIC, "refined batch: a system's solution is not finite");
    return LP_OK;
}

int resolve_config(lp_ctx* c, const lp_batch_config* cfg, lp_batch_config* use) {
    if (cfg != nullptr)
        *use = *cfg;
    else if (c->btuned)
        *use = c->bcfg;
    else
        lp_batch_default_config(use);
    if (use->small_n_max > 128 || use->small_n_max < 0) return fail(LP_E_INVALID, "batch: small_n_max must be <= 128");
    for (int i = 0; i < 5; i++)
        if (use->nb[i] != 16 && use->nb[i] != 32) return fail(LP_E_INVALID, "batch: nb must be 16 or 32");
    return LP_OK;
}

}  // namespace

}  // namespace lp

using namespace lp;

extern "C" {

int lp_batch_default_config(lp_batch_config* cfg) {
    if (cfg == nullptr) return fail(LP_E_INVALID, "lp_batch_default_config: null output");
    cfg->small_n_max = 128;
    for (int i = 0; i < 5; i++) cfg->nb[i] = 32;
    cfg->ctas_per_sm = 2;
    cfg->use_graph = 1;
    return LP_OK;
}

int lp_batch_solve_dev(lp_ctx* c, int count, const lp_system* systems, float* dA, float* dB,
                       const lp_batch_config* cfg, lp_batch_stats* stats) {
    if (c == nullptr || dA == nullptr || dB == nullptr) return fail(LP_E_INVALID, "lp_batch_solve_dev: null argument");
    LP_CHECK(validate_batch(count, systems));
    lp_batch_config use;
    if (cfg != nullptr)
        use = *cfg;
    else if (c->btuned)
        use = c->bcfg;
    else
        lp_batch_default_config(&use);
    if (use.small_n_max > 128 || use.small_n_max < 0) return fail(LP_E_INVALID, "batch: small_n_max must be <= 128");
    for (int i = 0; i < 5; i++)
        if (use.nb[i] != 16 && use.nb[i] != 32) return fail(LP_E_INVALID, "batch: nb must be 16 or 32");
    LP_CUDA(cudaSetDevice(c->device));
    std::vector<lp_system> sorted = sorted_by_n(count, systems);
    cudaStream_t st = c->stream;
    LP_CUDA(cudaEventRecord(c->ev[0], st));
    int replayed = 0;
    LP_CHECK(run_batch(c, sorted, dA, dB, use, use.use_graph != 0, &replayed));
    LP_CUDA(cudaEventRecord(c->ev[1], st));
    LP_CUDA(cudaStreamSynchronize(st));
    if (stats != nullptr) {
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]);
        stats->seconds = ms * 1e-3;
        stats->flops = batch_flops(sorted);
        stats->gflops = stats->seconds > 0 ? stats->flops / stats->seconds / 1e9 : 0.0;
        stats->solves_per_s = stats->seconds > 0 ? count / stats->seconds : 0.0;
        stats->systems = count;
        stats->graph_replayed = replayed;
    }
    return LP_OK;
}

int lp_batch_autotune(lp_ctx* c, int count, const lp_system* systems, const float* dA, const float* dB,
                      lp_batch_config* out) {
    if (c == nullptr || dA == nullptr || dB == nullptr || out == nullptr)
        return fail(LP_E_INVALID, "lp_batch_autotune: null argument");
    LP_CHECK(validate_batch(count, systems));
    LP_CUDA(cudaSetDevice(c->device));
    size_t na = 0, nbf = 0;
    for (int i = 0; i < count; i++) {
        const lp_system& s = systems[i];
        na = std::max(na, (size_t)(s.a_off + (long long)(s.n - 1) * s.lda + s.n));
        nbf = std::max(nbf, (size_t)(s.b_off + (long long)(s.nrhs - 1) * s.ldb + s.n));
    }
    LP_CHECK(c->tA.ensure(sizeof(float) * (na > 0 ? na : 1)));
    LP_CHECK(c->tB.ensure(sizeof(float) * (nbf > 0 ? nbf : 1)));
    float* tA = static_cast<float*>(c->tA.ptr);
    float* tB = static_cast<float*>(c->tB.ptr);
    cudaStream_t st = c->stream;
    lp_batch_config best;
    lp_batch_default_config(&best);

    // Time one configuration on one subset (fresh copies of the inputs each run).
    auto time_cfg = [&](const std::vector<lp_system>& sub, const lp_batch_config& cfg, double* sec) -> int {
        double t_best = 1e30;
        for (int rep = 0; rep < 2; rep++) {
            LP_CUDA(cudaMemcpyAsync(tA, dA, sizeof(float) * na, cudaMemcpyDeviceToDevice, st));
            LP_CUDA(cudaMemcpyAsync(tB, dB, sizeof(float) * nbf, cudaMemcpyDeviceToDevice, st));
            LP_CUDA(cudaEventRecord(c->ev[0], st));
            int replayed = 0;
            LP_CHECK(run_batch(c, sub, tA, tB, cfg, false, &replayed));
            LP_CUDA(cudaEventRecord(c->ev[1], st));
            LP_CUDA(cudaStreamSynchronize(st));
            float ms = 0.0f;
            LP_CUDA(cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]));
            t_best = std::min(t_best, (double)ms);
        }
        *sec = t_best * 1e-3;
        return LP_OK;
    };

    std::vector<lp_system> all = sorted_by_n(count, systems);
    // small-path threshold: on the systems with n <= 128
    {
        std::vector<lp_system> sub;
        for (const auto& s : all)
            if (s.n <= 128) sub.push_back(s);
        if (!sub.empty()) {
            double tbest = 1e30;
            for (int thr : {64, 128}) {
                lp_batch_config cfg = best;
                cfg.small_n_max = thr;
                double t = 0;
                LP_CHECK(time_cfg(sub, cfg, &t));
                if (t < tbest) {
                    tbest = t;
                    best.small_n_max = thr;
                }
            }
        }
    }
    // panel width per bucket
    for (int b = 0; b < 5; b++) {
        std::vector<lp_system> sub;
        for (const auto& s : all)
            if (bucket_of_host(s.n) == b && s.n > best.small_n_max) sub.push_back(s);
        if (sub.empty()) continue;
        double tbest = 1e30;
        for (int nbw : {16, 32}) {
            lp_batch_config cfg = best;
            cfg.nb[b] = nbw;
            double t = 0;
            LP_CHECK(time_cfg(sub, cfg, &t));
            if (t < tbest) {
                tbest = t;
                best.nb[b] = nbw;
            }
        }
    }
    // residency
    {
        double tbest = 1e30;
        const int pick = best.ctas_per_sm;
        best.ctas_per_sm = pick;
        for (int per : {1, 2}) {
            lp_batch_config cfg = best;
            cfg.ctas_per_sm = per;
            double t = 0;
            LP_CHECK(time_cfg(all, cfg, &t));
            if (t < tbest) {
                tbest = t;
                best.ctas_per_sm = per;
            }
        }
    }
    // drop the graph built for the scratch buffers
    if (c->bgraph != nullptr) {
        cudaGraphExecDestroy(c->bgraph);
        c->bgraph = nullptr;
    }
    c->bsys_hash = 0;
    c->bcfg = best;
    c->btuned = true;
    *out = best;
    return LP_OK;
}

int lp_batch_solve_ir_dev(lp_ctx* c, int precision, int count, const lp_system* systems, float* dA,
                          const double* dB64, double* dX, int max_iters, const lp_batch_config* cfg,
                          lp_batch_stats* stats, int* ir_iters, double* hpl_resid) {
    if (c == nullptr || dA == nullptr || dB64 == nullptr || dX == nullptr)
        return fail(LP_E_INVALID, "lp_batch_solve_ir_dev: null argument");
    if (precision != LP_F32 && precision != LP_BF16_IR)
        return fail(LP_E_INVALID, "lp_batch_solve_ir_dev: precision must be LP_F32 or LP_BF16_IR");
    if (max_iters < 0) return fail(LP_E_INVALID, "lp_batch_solve_ir_dev: max_iters must be >= 0");
    LP_CHECK(validate_batch(count, systems));
    lp_batch_config use;
    LP_CHECK(resolve_config(c, cfg, &use));
    LP_CUDA(cudaSetDevice(c->device));
    return run_batch_ir(c, precision, count, systems, dA, dB64, dX, max_iters, use, stats, ir_iters, hpl_resid);
}

int lp_batch_solve(lp_ctx* c, int precision, int count, const lp_system* systems, float* A, const double* B,
                   double* X, int max_iters, const lp_batch_config* cfg, lp_batch_stats* stats, int* ir_iters,
                   double* hpl_resid) {
    if (c == nullptr || A == nullptr || B == nullptr || X == nullptr)
        return fail(LP_E_INVALID, "lp_batch_solve: null argument");
    if (precision != LP_F32 && precision != LP_BF16_IR)
        return fail(LP_E_INVALID, "lp_batch_solve: precision must be LP_F32 or LP_BF16_IR");
    if (max_iters < 0) return fail(LP_E_INVALID, "lp_batch_solve: max_iters must be >= 0");
    LP_CHECK(validate_batch(count, systems));
    lp_batch_config use;
    LP_CHECK(resolve_config(c, cfg, &use));
    LP_CUDA(cudaSetDevice(c->device));
    size_t na = 0, nb = 0;
    batch_extents(count, systems, &na, &nb);
    if (count == 0) return LP_OK;
    LP_CHECK(c->hA.ensure(sizeof(float) * na));
    LP_CHECK(c->hB.ensure(sizeof(double) * nb));
    LP_CHECK(c->hX.ensure(sizeof(double) * nb));
    cudaStream_t st = c->stream;
    float* dA = static_cast<float*>(c->hA.ptr);
    double* dB = static_cast<double*>(c->hB.ptr);
    double* dX = static_cast<double*>(c->hX.ptr);
    LP_CUDA(cudaMemcpyAsync(dA, A, sizeof(float) * na, cudaMemcpyHostToDevice, st));
    LP_CUDA(cudaMemcpyAsync(dB, B, sizeof(double) * nb, cudaMemcpyHostToDevice, st));
    const int s = run_batch_ir(c, precision, count, systems, dA, dB, dX, max_iters, use, stats, ir_iters, hpl_resid);
    if (s != LP_OK && s != LP_E_NUMERIC) return s;
    LP_CUDA(cudaMemcpyAsync(A, dA, sizeof(float) * na, cudaMemcpyDeviceToHost, st));
    LP_CUDA(cudaMemcpyAsync(X, dX, sizeof(double) * nb, cudaMemcpyDeviceToHost, st));
    LP_CUDA(cudaStreamSynchronize(st));
    return s;
}

}  // extern "C"
