// lp_gesl_dev_noalloc: the substitution for callers that cannot allocate
// device memory (the reference runs gesl_ref_nopvt on the host,
// linpack_data.cpp:199-229; this entry point has no counterpart there).
//
// It runs the same two persistent sweeps as lp_gesl_dev (k_gesl_inv.cu), whose
// only global scratch is the array of published values (64-bit pairs, one per
// unknown and right-hand side of a 16-wide group, and the chunk items' partial
// sums) plus two tickets and an error word.  Here that scratch is one fixed
// device array instead of a context workspace, so the call allocates nothing:
// 2^19 pairs (4 MiB) and 16 bytes of counters.  With chunk items where their
// sums fit (then bit-identical to lp_gesl_dev), else without, which needs
// ceil(n / 128) * 128 * min(nrhs, 16) <= 2^19.
// Every GPU that loads the library holds the array until the process exits.
// Host code only sees a host-side stand-in for the array's name; the device
// address is looked up once per device with cudaGetSymbolAddress.
#include <mutex>

#include "gesl_common.cuh"

namespace lp {

constexpr size_t kNoAllocPairs = size_t(1) << 19;
static __device__ __align__(256) unsigned long long g_gesl_scratch[kNoAllocPairs + 2];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
unsigned long long* g_noalloc_ptr[kMaxDevices] = {nullptr};

// Once per device, with that device current: attributes of the sweep kernels
// and the scratch array's device address.
int noalloc_setup(int dev, unsigned long long** out) {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (g_noalloc_ptr[dev] == nullptr) {
        LP_CHECK(gesl_inv_init_attrs());
        void* p = nullptr;
        LP_CUDA(cudaGetSymbolAddress(&p, g_gesl_scratch));
        g_noalloc_ptr[dev] = static_cast<unsigned long long*>(p);
    }
    *out = g_noalloc_ptr[dev];
    return LP_OK;
}
}  // namespace

}  // namespace lp

extern "C" int lp_gesl_dev_noalloc(const float* dLU, int n, int lda, float* dB, int nrhs, int ldb, void* stream) {
    using namespace lp;
    if (dLU == nullptr || dB == nullptr) return fail(LP_E_INVALID, "lp_gesl_dev_noalloc: null argument");
    if (n <= 0 || lda < n || nrhs <= 0 || ldb < n) return fail(LP_E_INVALID, "lp_gesl_dev_noalloc: bad sizes");
    if (lda % 4 != 0 || !aligned16(dLU))
        return fail(LP_E_INVALID, "lp_gesl_dev_noalloc: factors must be 16-byte aligned with lda a multiple of 4");
    if (gesl_pub_pairs(n, nrhs, 0) > kNoAllocPairs)
        return fail(LP_E_INVALID, "lp_gesl_dev_noalloc: ceil(n / 128) * 128 * min(nrhs, 16) exceeds the fixed scratch "
                                  "of 524288 values (4 MiB); use lp_gesl_dev for larger systems");
    int dev = 0;
    LP_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return fail(LP_E_INVALID, "lp_gesl_dev_noalloc: device index out of range");
    unsigned long long* scratch = nullptr;
    LP_CHECK(noalloc_setup(dev, &scratch));
    int* words = reinterpret_cast<int*>(scratch + kNoAllocPairs);  // tickets[2], error word
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    LP_CUDA(cudaMemsetAsync(words + 2, 0, sizeof(int), st));
    const int chunk = gesl_pub_pairs(n, nrhs, kGeslChunk) <= kNoAllocPairs ? kGeslChunk : 0;
    return launch_gesl_inv(dLU, lda, n, dB, ldb, nrhs, scratch, words, words + 2, false, chunk, st);
}
