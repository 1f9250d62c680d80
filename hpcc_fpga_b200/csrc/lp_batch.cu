// Host side of the batched solver: the system list sorted by decreasing n
// (largest first, so one persistent launch balances any size mix), the
// launch captured once in a CUDA graph and replayed for the same batch, the
// per-bucket autotuner.
#include <algorithm>
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

}  // extern "C"
