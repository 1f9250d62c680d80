"""Partial pivoting (gefa_ref / gesl_ref, LINPACK/src/host/linpack_data.cpp:72-156)
on the GPU through the C ABI, against the oracle.

A matrix that fits one panel (n <= 128) is factored by the panel kernel alone
with the reference's operation order (multiplier in double, product and sum
rounded separately), so factors and pivots must be bit-identical.  Larger
matrices use the blocked trailing update (another summation order): pivots
equal to the oracle's on these well-separated inputs, factors within the
normwise FP32 bound 8 n eps max|factors| of each other (both are FP32
factorizations of the same matrix), and the solution within the HPL
scaled-residual threshold and the reference's own validation (residn < 1,
linpack_benchmark.hpp:395-417).
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu
FLT_EPS = float(np.finfo(np.float32).eps)


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def uniform(n, seed):
    return np.random.default_rng(seed).random((n, n)).astype(np.float32)


def close_factors(got, want):
    n = want.shape[0]
    diff = np.abs(got.astype(np.float64) - want.astype(np.float64)).max()
    return diff <= 8 * n * FLT_EPS * np.abs(want).max()


def gpu_gefa_pvt(ctx, dev, torch, A):
    n = A.shape[0]
    d = dev.put(A)
    p = torch.zeros(n, dtype=torch.int32, device="cuda")
    ctx.gefa_pvt(d.data_ptr(), n, A.shape[1], p.data_ptr())
    return dev.get(d), dev.get(p)


@pytest.mark.parametrize("n", [1, 2, 3, 17, 64, 100, 128])
def test_single_panel_bitexact(ctx, dev, torch_cuda, n):
    A, _, _, _ = oracle.gen_reference(n, diag_dominant=False)
    got, p = gpu_gefa_pvt(ctx, dev, torch_cuda, A)
    want, pw = oracle.gefa_pvt(A)
    assert np.array_equal(p, pw)
    assert np.array_equal(bits(got), bits(want))
    ref = oracle.ref("f32")
    if ref is not None:  # the reference's own gefa_ref, compiled
        theirs = A.copy()
        pr = np.zeros(n, np.int32)
        ref.ref_gefa_pvt_f32(theirs, n, n, pr)
        assert np.array_equal(bits(got), bits(theirs)) and np.array_equal(p, pr)


def test_pivot_edge_cases_bitexact(ctx, dev, torch_cuda):
    """Zero diagonal (an exchange is forced), equal magnitudes of opposite sign
    (the first wins), NaN below the diagonal (never chosen) and on it (kept)."""
    n = 96
    A = uniform(n, 11)
    A[0, 0] = 0.0
    A[1, 1:] = 0.5
    A[1, 3] = -0.5
    A[1, 1] = 0.25
    A[5, 40] = np.nan     # M's column 5, row 40
    got, p = gpu_gefa_pvt(ctx, dev, torch_cuda, A)
    want, pw = oracle.gefa_pvt(A)
    assert np.array_equal(p, pw)
    fin = np.isfinite(want)
    assert np.array_equal(fin, np.isfinite(got))
    assert np.array_equal(bits(got[fin]), bits(want[fin]))
    B = uniform(8, 3)
    B[0, 0] = np.nan
    got, p = gpu_gefa_pvt(ctx, dev, torch_cuda, B)
    _, pw = oracle.gefa_pvt(B)
    assert p[0] == 0 and np.array_equal(p, pw)


@pytest.mark.parametrize("n", [256, 384, 1000, 2048])
def test_blocked_factors_and_pivots(ctx, dev, torch_cuda, n):
    A, b, _, normb = oracle.gen_reference(n, diag_dominant=False)
    got, p = gpu_gefa_pvt(ctx, dev, torch_cuda, A)
    want, pw = oracle.gefa_pvt(A)
    assert np.array_equal(p, pw)
    assert close_factors(got, want)
    # the reference's own solve on the GPU's factors validates
    x = oracle.gesl_pvt(got, p, b)
    rn, _ = oracle.residn(x, normb)
    assert rn < 1.0


@pytest.mark.parametrize("n,nrhs", [(100, 1), (512, 1), (1000, 3), (2048, 2)])
def test_gesl_pvt_vs_oracle(ctx, dev, torch_cuda, n, nrhs):
    """The GPU solve on the oracle's factors (reference encoding); the factors
    come back bit-identical."""
    A = uniform(n, n)
    lu, p = oracle.gefa_pvt(A)
    rng = np.random.default_rng(2)
    B = rng.random((nrhs, n)).astype(np.float32)
    dlu = dev.put(lu)
    dp = dev.put(p)
    dB = dev.put(B)
    ctx.gesl_pvt(dlu.data_ptr(), n, n, dp.data_ptr(), dB.data_ptr(), nrhs, n)
    X = dev.get(dB)
    assert np.array_equal(bits(dev.get(dlu)), bits(lu))
    for q in range(nrhs):
        want = oracle.gesl_pvt(lu, p, B[q])
        scale = np.abs(want).max()
        assert np.abs(X[q] - want).max() <= 1e-4 * max(1.0, scale)
        hpl = oracle.hpl_resid(A, X[q].astype(np.float64), B[q].astype(np.float64), eps=FLT_EPS / 2)
        assert hpl < 16.0, hpl


@pytest.mark.parametrize("n", [128, 1024, 4096])
def test_calculate_pvt_host_api(ctx, n):
    """The --uniform backend: A -> factors in gefa_ref's encoding, b -> x,
    validation as the reference does it."""
    A, b, _, normb = oracle.gen_reference(n, diag_dominant=False)
    A0 = A.copy()
    times, p = ctx.calculate_pvt(A, b, repetitions=2)
    assert len(times["gefa"]) == 2 and min(times["gefa"]) > 0 and min(times["gesl"]) > 0
    rn, _ = oracle.residn(b, normb)
    assert rn < 1.0
    if n <= 1024:
        want, pw = oracle.gefa_pvt(A0)
        assert np.array_equal(p, pw)
        assert close_factors(A, want)


def test_dominant_input_needs_no_exchange(ctx, dev, torch_cuda):
    A, _, _, _ = oracle.gen_reference(512, diag_dominant=True)
    _, p = gpu_gefa_pvt(ctx, dev, torch_cuda, A)
    assert np.array_equal(p, np.arange(512))


def test_pivot_invalid_arguments(ctx, lp):
    with pytest.raises(lp.LpError):
        ctx.gefa_pvt(0, 16, 16, 0)
    A = np.zeros((130, 130), np.float32)   # n > 128 must be a multiple of 4
    with pytest.raises(lp.LpError):
        ctx.calculate_pvt(A, np.zeros(130, np.float32))
