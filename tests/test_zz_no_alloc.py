"""lp_gesl_dev_noalloc: the substitution for callers that cannot allocate
device memory (their memory belongs to a pool, they are recording CUDA graphs,
or they sit in a serving loop where an allocation may stall the device).  Its
work vectors live in one fixed 4 MiB device array instead of a context
workspace.  Checked through the C ABI against lp_gesl_dev, the allocating
entry point, on two calls in a row (the second call reuses the array with the
first call's contents still in it).  This file is collected last on purpose."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu
FLT_EPS = float(np.finfo(np.float32).eps)


def _solve_noalloc(lp, dev, dLU, n, B):
    dB = dev.put(B)
    st = lp.lib().lp_gesl_dev_noalloc(dLU.data_ptr(), n, n, dB.data_ptr(), B.shape[0], n, None)
    lp.check(st, "lp_gesl_dev_noalloc")
    dev.torch.cuda.synchronize()
    return dB.cpu().numpy()


def _solve_alloc(ctx, dev, dLU, n, B):
    dB = dev.put(B)
    ctx.gesl(dLU.data_ptr(), n, n, dB.data_ptr(), B.shape[0], n)
    return dev.get(dB)


@pytest.mark.parametrize("n,nrhs", [(1024, 1), (768, 5)])
def test_noalloc_matches_allocating_entry_point_twice(ctx, dev, lp, n, nrhs):
    A, _, _, _ = oracle.gen_reference(n)
    LU = oracle.gefa_nopvt(A)
    dLU = dev.put(LU)
    rng = np.random.default_rng(n + nrhs)
    LU64 = LU.astype(np.float64)
    for call in range(2):
        B = rng.uniform(-1, 1, (nrhs, n)).astype(np.float32)
        want = _solve_alloc(ctx, dev, dLU, n, B)
        got = _solve_noalloc(lp, dev, dLU, n, B)
        # Same kernels as lp_gesl_dev, so the tolerance of the substitution
        # tests (test_gpu_solve.py::test_gesl_multi_rhs) holds a fortiori.
        for r in range(nrhs):
            x64 = oracle.gesl_nopvt(LU64, B[r].astype(np.float64))
            x32 = oracle.gesl_nopvt(LU, B[r])
            tol = 8 * np.abs(x32 - x64).max() + 64 * FLT_EPS * np.abs(x64).max()
            assert np.abs(got[r] - x64).max() <= tol, f"call {call}, rhs {r}"
        assert np.allclose(got, want, rtol=0, atol=64 * FLT_EPS * np.abs(want).max()), f"call {call}"


def test_noalloc_rejects_sizes_beyond_the_fixed_scratch(lp, dev):
    n = 1 << 16
    dLU = dev.empty((16,))
    dB = dev.empty((16,))
    # 2 * 65536 * 16 floats > 2^20: rejected before any device work.
    st = lp.lib().lp_gesl_dev_noalloc(dLU.data_ptr(), n, n, dB.data_ptr(), 16, n, None)
    assert st == lp.LP_E_INVALID
    assert "fixed scratch" in lp.last_error()
