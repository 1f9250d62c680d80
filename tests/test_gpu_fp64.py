"""The FP64 form (the reference's double build, DATA_TYPE double) through the C
ABI, against the oracle's double restatement (pinned to the compiled
reference's gefa_ref_nopvt / gesl_ref_nopvt in double, tests/test_oracle.py).

One block (n = bs) is the lu kernel alone, with the reference's operation
order: bit-identical.  At n = 2 bs the top block row and the left block column
are still the reference's order (bit-identical); the trailing block goes
through the FP64 GEMM (another summation order).  Larger systems: factors and
solutions within FP64 rounding bounds, and the reference's validation with
the double machine epsilon (linpack_benchmark.hpp:395-417).
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu
DBL_EPS = float(np.finfo(np.float64).eps)


def bits(a):
    return np.ascontiguousarray(a).view(np.uint64)


def dominant(n, seed):
    """The reference generator's shape in double: U(0,1) entries, each storage
    row's diagonal the row sum, b = column sums (x = ones)."""
    rng = np.random.default_rng(seed)
    A = rng.random((n, n))
    np.fill_diagonal(A, 0.0)
    np.fill_diagonal(A, A.sum(axis=1))
    b = A.sum(axis=0)
    return A, b


def gpu_gefa(ctx, dev, A, bs):
    d = dev.put(A)
    ctx.gefa_f64(d.data_ptr(), A.shape[0], A.shape[1], bs)
    return dev.get(d)


@pytest.mark.parametrize("bs", [64, 128])
def test_one_block_bitexact(ctx, dev, bs):
    A, _ = dominant(bs, bs)
    got = gpu_gefa(ctx, dev, A, bs)
    want = oracle.gefa_nopvt(A)
    assert np.array_equal(bits(got), bits(want))
    ref = oracle.ref("f64")
    if ref is not None:
        theirs = A.copy()
        ref.ref_gefa_nopvt_f64(theirs, bs, bs)
        assert np.array_equal(bits(got), bits(theirs))


@pytest.mark.parametrize("bs", [64, 128])
def test_two_blocks_stages_bitexact(ctx, dev, bs):
    n = 2 * bs
    A, _ = dominant(n, 5)
    got = gpu_gefa(ctx, dev, A, bs)
    want = oracle.gefa_nopvt(A)
    assert np.array_equal(bits(got[:bs, :]), bits(want[:bs, :]))      # lu + top
    assert np.array_equal(bits(got[bs:, :bs]), bits(want[bs:, :bs]))  # left
    tail = np.abs(got[bs:, bs:] - want[bs:, bs:]) / np.maximum(1.0, np.abs(want[bs:, bs:]))
    assert tail.max() < 64 * n * DBL_EPS


@pytest.mark.parametrize("n,bs", [(256, 64), (1024, 128), (2048, 128), (1024, 256), (2048, 256)])
def test_factor_and_solve(ctx, dev, n, bs):
    A, b = dominant(n, n)
    got = gpu_gefa(ctx, dev, A, bs)
    want = oracle.gefa_nopvt(A)
    assert np.abs(got - want).max() <= 8 * n * DBL_EPS * np.abs(want).max()
    dLU = dev.put(got)
    dB = dev.put(b)
    ctx.gesl_f64(dLU.data_ptr(), n, n, dB.data_ptr(), 1, n)
    x = dev.get(dB)
    xr = oracle.gesl_nopvt(want, b)
    assert np.abs(x - xr).max() <= 1e3 * n * DBL_EPS
    resid = np.abs(x - 1.0).max()
    assert resid / (n * np.abs(b).max() * DBL_EPS) < 1.0


def test_multi_rhs(ctx, dev):
    n, nrhs = 512, 5
    A, _ = dominant(n, 9)
    lu = oracle.gefa_nopvt(A)
    B = np.random.default_rng(3).random((nrhs, n))
    dLU = dev.put(lu)
    dB = dev.put(B)
    ctx.gesl_f64(dLU.data_ptr(), n, n, dB.data_ptr(), nrhs, n)
    X = dev.get(dB)
    for q in range(nrhs):
        want = oracle.gesl_nopvt(lu, B[q])
        assert np.abs(X[q] - want).max() <= 1e3 * n * DBL_EPS * max(1.0, np.abs(want).max())


def test_calculate_f64_host_api(ctx):
    n = 1024
    A, b = dominant(n, 4)
    A0, normb = A.copy(), np.abs(b).max()
    times = ctx.calculate_f64(A, b, bs=128, repetitions=2)
    assert len(times["gefa"]) == 2 and min(times["gefa"]) > 0 and min(times["gesl"]) > 0
    assert np.abs(b - 1.0).max() / (n * normb * DBL_EPS) < 1.0
    want = oracle.gefa_nopvt(A0)
    assert np.abs(A - want).max() <= 8 * n * DBL_EPS * np.abs(want).max()


def test_f64_invalid_arguments(ctx, lp):
    with pytest.raises(lp.LpError):
        ctx.gefa_f64(0, 128, 128, 128)
    with pytest.raises(lp.LpError):
        ctx.calculate_f64(np.zeros((96, 96)), np.zeros(96), bs=64)  # n not a multiple of bs
