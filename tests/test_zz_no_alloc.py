"""lp_gesl_dev_noalloc: the substitution for callers that cannot allocate
device memory (their memory belongs to a pool, they are recording CUDA graphs,
or they sit in a serving loop where an allocation may stall the device).  Its
sweeps' published values live in one fixed 4 MiB device array instead of a
context workspace.  Checked through the C ABI against lp_gesl_dev, the allocating
entry point, on two calls in a row (the second call reuses the array with the
first call's contents still in it).  This file is collected last on purpose.

Both entry points run the same two persistent sweeps (k_gesl_sweep, each
finisher CTA inverting its own diagonal block, chunk items streaming the late
tiles' long source ranges).  Where the chunks' partial sums fit in the fixed
array the results must be bit-identical; where they do not (the scratch limit
case) the allocation-free sweeps run without chunk items and sum in another
order.  Both are held to the FP64 solution of the same factors with a bound
scaled by the FP32 oracle's own error (the sweeps sum in another order than
the oracle)."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu
FLT_EPS = float(np.finfo(np.float32).eps)


def _solve_noalloc(lp, torch, dLU, n, B):
    dB = torch.from_numpy(np.ascontiguousarray(B)).cuda()
    torch.cuda.synchronize()
    st = lp.lib().lp_gesl_dev_noalloc(dLU.data_ptr(), n, n, dB.data_ptr(), B.shape[0], n, None)
    lp.check(st, "lp_gesl_dev_noalloc")
    torch.cuda.synchronize()
    return dB.cpu().numpy()


def _solve_alloc(ctx, dev, dLU, n, B):
    dB = dev.put(B)
    ctx.gesl(dLU.data_ptr(), n, n, dB.data_ptr(), B.shape[0], n)
    return dev.get(dB)


@pytest.mark.parametrize("n,nrhs", [(1024, 1), (768, 5), (512, 20)])
def test_noalloc_matches_allocating_entry_point_twice(ctx, dev, lp, n, nrhs):
    """nrhs = 20 runs two chunks (16 + 4 right-hand sides) through the shared
    array within one call."""
    A, _, _, _ = oracle.gen_reference(n)
    LU = oracle.gefa_nopvt(A)
    dLU = dev.put(LU)
    rng = np.random.default_rng(n + nrhs)
    LU64 = LU.astype(np.float64)
    for call in range(2):
        B = rng.uniform(-1, 1, (nrhs, n)).astype(np.float32)
        want = _solve_alloc(ctx, dev, dLU, n, B)
        got = _solve_noalloc(lp, dev.torch, dLU, n, B)
        for r in range(nrhs):
            x64 = oracle.gesl_nopvt(LU64, B[r].astype(np.float64))
            x32 = oracle.gesl_nopvt(LU, B[r])
            tol = 8 * np.abs(x32 - x64).max() + 64 * FLT_EPS * np.abs(x64).max()
            assert np.abs(got[r] - x64).max() <= tol, f"call {call}, rhs {r}"
            assert np.abs(want[r] - x64).max() <= tol, f"call {call}, rhs {r} (lp_gesl_dev)"
        assert np.array_equal(got, want), f"call {call}"


def test_noalloc_at_the_scratch_limit(ctx, dev, lp):
    """ceil(n / 128) * 128 * min(nrhs, 16) == 2^19 exactly (n = 32768, 16
    right-hand sides) is accepted.  The factors come from lp_gefa_dev on a seeded diagonally
    dominant matrix made on the device; the FP64 substitution of the same
    factors (lp_gesl_f64_dev on the factors widened exactly) is the reference
    solution for both entry points."""
    torch = dev.torch
    n, nrhs = 32768, 16
    g = torch.Generator(device="cuda")
    g.manual_seed(5)
    dA = torch.rand((n, n), generator=g, device="cuda", dtype=torch.float32) - 0.5
    dA.diagonal().copy_(dA.abs().sum(1) + 1.0)
    torch.cuda.synchronize()  # torch's stream and the library's stream are not ordered
    ctx.gefa(dA.data_ptr(), n, n, 512)
    ctx.sync()
    B = np.random.default_rng(11).uniform(-1, 1, (nrhs, n)).astype(np.float32)
    dLU64 = dA.double()
    dX64 = torch.from_numpy(B.astype(np.float64)).cuda()
    torch.cuda.synchronize()
    ctx.gesl_f64(dLU64.data_ptr(), n, n, dX64.data_ptr(), nrhs, n)
    x64 = dev.get(dX64)
    del dLU64
    # At this size the allocation-free array has no room for the chunk items' sums, so the
    # two entry points sum in different orders: both are checked against the FP64
    # solution, and each must repeat itself bit for bit.
    first = None
    for call in range(2):
        want = _solve_alloc(ctx, dev, dA, n, B)
        got = _solve_noalloc(lp, torch, dA, n, B)
        tol = 64 * n ** 0.5 * FLT_EPS * np.abs(x64).max()
        assert np.abs(got - x64).max() <= tol, f"call {call}"
        assert np.abs(want - x64).max() <= tol, f"call {call} (lp_gesl_dev)"
        if first is None:
            first = (got, want)
        else:
            assert np.array_equal(got, first[0]) and np.array_equal(want, first[1])


def test_noalloc_rejects_sizes_beyond_the_fixed_scratch(lp, dev):
    n = 1 << 16
    dLU = dev.empty((16,))
    dB = dev.empty((16,))
    # 65536 * 16 values > 2^19: rejected before any device work.
    st = lp.lib().lp_gesl_dev_noalloc(dLU.data_ptr(), n, n, dB.data_ptr(), 16, n, None)
    assert st == lp.LP_E_INVALID
    assert "fixed scratch" in lp.last_error()
    # one row more than the limit allows, with 16 right-hand sides
    st = lp.lib().lp_gesl_dev_noalloc(dLU.data_ptr(), 32769, 32772, dB.data_ptr(), 16, 32772, None)
    assert st == lp.LP_E_INVALID
