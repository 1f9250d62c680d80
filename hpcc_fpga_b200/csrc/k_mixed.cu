// Mixed-precision factorization (tensor-core trailing update): see gefa_mixed.
#include "lp_ctx.cuh"

namespace lp {

int gefa_mixed(lp_ctx* c, int precision, float* dA, int n, int lda, int bs, cudaStream_t st) {
    (void)c; (void)precision; (void)dA; (void)n; (void)lda; (void)bs; (void)st;
    return fail(LP_E_INVALID, "mixed-precision factorization is not available in this build");
}

}  // namespace lp
