"""Whole factorization + substitution on the GPU against the oracle.

Mirrors LINPACK/tests/test_kernel_functionality_and_host_integration.cpp:
executeKernel on 1, 2 and 3 blocks (:128-131) must give |x_i - 1| < 1e-3 for
every i (:43-48) and pass validateOutput (residn < 1,
linpack_benchmark.hpp:416-417,465); the factors must agree with
gefa_ref_nopvt (the disabled GEFA test, :53-74, tolerance 1e-3).  Tighter
bounds are stated per test."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu
FLT_EPS = float(np.finfo(np.float32).eps)
DBL_EPS = float(np.finfo(np.float64).eps)


@pytest.mark.parametrize("bs", [16, 32, 128, 512])
@pytest.mark.parametrize("blocks", [1, 2, 3])
def test_calculate_reference_inputs(ctx, bs, blocks):
    n = bs * blocks
    A, b, _, normb = oracle.gen_reference(n)
    A_dev, b_dev = A.copy(), b.copy()
    t = ctx.calculate(A_dev, b_dev, bs, repetitions=1)
    assert len(t["gefa"]) == 1 and t["gefa"][0] > 0 and t["gesl"][0] > 0
    assert np.all(np.abs(b_dev - 1.0) < 1e-3)
    residn, _ = oracle.residn(b_dev, normb)
    assert residn < 1.0
    want = oracle.gefa_nopvt(A)
    assert np.abs(A_dev - want).max() < 1e-3
    rel = np.abs(A_dev.astype(np.float64) - want) / np.maximum(1.0, np.abs(want))
    assert rel.max() < 256 * FLT_EPS
    # The FP32 solution is as accurate as the reference's own FP32 solution.
    x_ref = oracle.gesl_nopvt(want, b)
    assert np.abs(b_dev - 1.0).max() <= 4 * max(np.abs(x_ref - 1.0).max(), n * FLT_EPS)


@pytest.mark.parametrize("n,bs,reps,pad", [(1024, 128, 1, 0), (2048, 512, 2, 0), (1024, 256, 1, 8),
                                           (4096, 128, 1, 0), (3328, 256, 1, 4), (8192, 512, 2, 16)])
def test_calculate_pinned_overlapped_copy(ctx, lp, n, bs, reps, pad):
    """Page-locked A: the matrix is copied in row slabs (1024, 2048, then 4096
    rows) while the factorization runs, each slab catching up on the block
    steps of the rows above on one of two alternating lanes, and every block
    row returns as soon as it is final; the result equals the pageable path's
    (gefa_f32) exactly, also with lda > n (the padding columns stay as they
    were) and a ragged last slab."""
    A0, b, _, _ = oracle.gen_reference(n)
    A = np.full((n, n + pad), 7.0, np.float32)
    A[:, :n] = A0
    A1, b1 = A.copy(), b.copy()
    ctx.calculate(A1, b1, bs, repetitions=reps)
    assert np.all(A1[:, n:] == 7.0)
    pa, pb = lp.Pinned((n, n + pad)), lp.Pinned((n,))
    try:
        pa.array[:] = A
        pb.array[:] = b
        ctx.calculate(pa.array, pb.array, bs, repetitions=reps)
        assert np.array_equal(pa.array, A1) and np.array_equal(pb.array, b1)
    finally:
        pa.free()
        pb.free()


def test_calculate_repetitions_restart_from_original(ctx):
    n, bs = 256, 64
    A, b, _, _ = oracle.gen_reference(n)
    A1, b1 = A.copy(), b.copy()
    t = ctx.calculate(A1, b1, bs, repetitions=3)
    assert len(t["gefa"]) == 3 and len(t["gesl"]) == 3
    A2, b2 = A.copy(), b.copy()
    ctx.calculate(A2, b2, bs, repetitions=1)
    assert np.array_equal(A1, A2) and np.array_equal(b1, b2)


@pytest.mark.parametrize("n,bs", [(1024, 128), (2048, 512)])
def test_baseline_inputs_hpl_residual(ctx, n, bs):
    """Benchmark generator (seed 42, margin 1): HPL scaled residual with the
    FP32 unit roundoff <= 16, and FP64-oracle error (x_true = ones exactly)."""
    A, b64, b32 = oracle.gen_baseline(n, seed=42, margin=1.0)
    A_dev, x = A.copy(), b32.copy()
    ctx.calculate(A_dev, x, bs)
    r = oracle.hpl_resid(A, x.astype(np.float64), b32.astype(np.float64), eps=FLT_EPS / 2)
    assert r <= 16.0
    x_cpu = oracle.gesl_nopvt(oracle.gefa_nopvt(A), b32)
    assert np.abs(x - 1.0).max() <= 4 * np.abs(x_cpu - 1.0).max() + 1e-6


@pytest.mark.parametrize("n,nrhs", [(384, 1), (384, 3), (384, 16), (384, 17), (300, 2), (4, 1), (1000, 5)])
def test_gesl_multi_rhs(ctx, dev, n, nrhs):
    """Ragged n (not a multiple of the 128-wide substitution blocks) included."""
    A, _, _, _ = oracle.gen_reference(n)
    LU = oracle.gefa_nopvt(A)
    rng = np.random.default_rng(nrhs)
    B = rng.uniform(-1, 1, (nrhs, n)).astype(np.float32)
    dLU, dB = dev.put(LU), dev.put(B)
    ctx.gesl(dLU.data_ptr(), n, n, dB.data_ptr(), nrhs, n)
    X = dev.get(dB)
    LU64 = LU.astype(np.float64)
    for r in range(nrhs):
        x64 = oracle.gesl_nopvt(LU64, B[r].astype(np.float64))
        x32 = oracle.gesl_nopvt(LU, B[r])
        tol = 8 * np.abs(x32 - x64).max() + 64 * FLT_EPS * np.abs(x64).max()
        assert np.abs(X[r] - x64).max() <= tol


@pytest.mark.parametrize("n,nrhs", [(9000, 1), (9000, 3), (9000, 16), (8324, 17), (4480, 2)])
def test_gesl_chunked_sources(ctx, dev, n, nrhs):
    """Sizes where the substitution splits the long source ranges of the late
    tiles into chunk items (tiles past the 33rd; two chunks past the 65th),
    ragged n included.  Encoded factors made directly (multipliers up to
    1e-3, stored diagonal -1/d with d in [1, 2]) keep the oracle fast at these
    sizes.  Two runs must agree bit for bit: whichever CTA runs a chunk, the
    summation order is fixed."""
    rng = np.random.default_rng(n + nrhs)
    LU = ((rng.random((n, n), dtype=np.float32) - 0.5) * 2e-3).astype(np.float32)
    LU[np.arange(n), np.arange(n)] = (-1.0 / (1.0 + rng.random(n))).astype(np.float32)
    B = rng.uniform(-1, 1, (nrhs, n)).astype(np.float32)
    dLU = dev.put(LU)
    outs = []
    for _ in range(2):
        dB = dev.put(B)
        ctx.gesl(dLU.data_ptr(), n, n, dB.data_ptr(), nrhs, n)
        outs.append(dev.get(dB))
    assert np.array_equal(outs[0].view(np.uint32), outs[1].view(np.uint32))
    X = outs[0]
    LU64 = LU.astype(np.float64)
    for r in range(nrhs):
        x64 = oracle.gesl_nopvt(LU64, B[r].astype(np.float64))
        x32 = oracle.gesl_nopvt(LU, B[r])
        tol = 8 * np.abs(x32 - x64).max() + 64 * FLT_EPS * np.abs(x64).max()
        assert np.abs(X[r] - x64).max() <= tol


def test_gefa_dev_deterministic(ctx, dev):
    n, bs = 1024, 256
    A, _, _, _ = oracle.gen_reference(n)
    d1, d2 = dev.put(A), dev.put(A)
    ctx.gefa(d1.data_ptr(), n, n, bs)
    ctx.gefa(d2.data_ptr(), n, n, bs)
    assert np.array_equal(dev.get(d1), dev.get(d2))


def test_solve_host_f32_and_refined(ctx):
    n, bs = 1024, 128
    A, b64, _ = oracle.gen_baseline(n, seed=42, margin=1.0)
    x, t = ctx.solve_host(A, b64, bs, "f32", max_iters=0)
    assert t["ir_iters"] == 0
    r32 = oracle.hpl_resid(A, x, b64, eps=FLT_EPS / 2)
    assert r32 <= 16.0
    assert np.isclose(t["hpl_resid"], oracle.hpl_resid(A, x, b64), rtol=1e-6)
    x2, t2 = ctx.solve_host(A, b64, bs, "f32", max_iters=10)
    assert t2["hpl_resid"] <= 16.0 and t2["ir_iters"] >= 1
    assert oracle.hpl_resid(A, x2, b64) <= 16.0
    # Refinement stops at the HPL threshold, not at full FP64 accuracy.
    assert np.abs(x2 - 1.0).max() < 1e-10


@pytest.mark.parametrize("prec", ["f32", "bf16", "fp8", "f32_bf16x6"])
def test_factor_then_solve_matches_solve_host(ctx, dev, lp, prec):
    """lp_factor + lp_solve (factors resident between the calls) give what
    lp_solve_host gives in one call, on two solves against one factorization;
    the factors written back equal the device factorization's."""
    n, bs = 1024, 256
    A, _, _ = oracle.gen_baseline(n, seed=42, margin=1.0)
    Af = A.copy()
    t = ctx.factor(Af, bs, prec)
    assert t["gefa_s"] > 0
    d = dev.put(A)
    if prec == "f32":
        ctx.gefa(d.data_ptr(), n, n, bs)
    else:
        ctx.gefa_prec(prec, d.data_ptr(), n, n, bs)
    assert np.array_equal(Af, dev.get(d))
    rng = np.random.default_rng(3)
    refine = 0 if prec == "f32" else 50
    with lp.Context(0) as other:
        for rep in range(2):
            B = rng.uniform(-1, 1, (2, n)).astype(np.float32)
            x, ts = ctx.solve(B)
            x_ref, _ = other.solve_host(A, B.astype(np.float64), bs, prec, max_iters=refine)
            # the same arithmetic; refined solves may stop one refinement apart at the threshold
            assert np.abs(x - x_ref).max() <= (1e-9 if refine else 1e-13) * np.abs(x_ref).max()
            eps = DBL_EPS / 2 if refine else FLT_EPS / 2
            for q in range(2):
                assert oracle.hpl_resid(A, x[q], B[q].astype(np.float64), eps=eps) <= 16.0
            if refine:
                assert ts["hpl_resid"] <= 16.0


def test_solve_needs_resident_factors(lp):
    """lp_solve without factors, with another n, or after an entry point
    that reuses the context's matrix workspace is rejected."""
    n, bs = 256, 64
    A, _, b32 = oracle.gen_baseline(n, seed=1, margin=1.0)
    with lp.Context(0) as c:
        with pytest.raises(lp.LpError) as e:
            c.solve(b32)
        assert e.value.status == lp.LP_E_INVALID
        c.factor(A.copy(), bs)
        x, _ = c.solve(b32)
        assert np.abs(x - 1.0).max() < 1e-3
        with pytest.raises(lp.LpError) as e:
            c.solve(np.ones(n - 64, np.float32))
        assert e.value.status == lp.LP_E_INVALID
        c.solve_host(A, b32.astype(np.float64), bs, "f32")
        with pytest.raises(lp.LpError) as e:
            c.solve(b32)
        assert e.value.status == lp.LP_E_INVALID


def test_non_dominant_matrix_reports_numeric_error(ctx, lp):
    """A zero pivot (not factorable without pivoting) must surface as
    LP_E_NUMERIC, not as a silent result."""
    n, bs = 128, 64
    A = np.zeros((n, n), np.float32)
    A[0, 1] = 1.0
    with pytest.raises(lp.LpError) as e:
        ctx.solve_host(A, np.ones(n), bs, "f32")
    assert e.value.status == lp.LP_E_NUMERIC


def test_bad_sizes_rejected(ctx, lp):
    A = np.zeros((100, 100), np.float32)
    with pytest.raises(lp.LpError) as e:
        ctx.calculate(A, np.zeros(100, np.float32), 64)
    assert e.value.status == lp.LP_E_INVALID


@pytest.mark.parametrize("api", ["gesl_dev", "calculate", "solve_host"])
def test_substitution_wait_that_runs_out_reports_timeout(ctx, dev, lp, api):
    """A bounded wait of the substitution sweeps that runs out (armed by
    lp_ctx_test_stall: one tile waits on a word that nothing sets) must come
    back as LP_E_TIMEOUT through every entry point that runs the sweeps, with
    no GPU fault, and leave the context usable: the next identical call
    succeeds and validates."""
    n, bs = 1024, 128
    A, b, _, normb = oracle.gen_reference(n)

    def run():
        if api == "gesl_dev":
            LU = oracle.gefa_nopvt(A)
            dLU, dB = dev.put(LU), dev.put(b)
            ctx.gesl(dLU.data_ptr(), n, n, dB.data_ptr(), 1, n)
            return dev.get(dB)
        if api == "calculate":
            Ac, bc = A.copy(), b.copy()
            ctx.calculate(Ac, bc, bs, repetitions=1)
            return bc
        x, _ = ctx.solve_host(A.copy(), b.astype(np.float64), bs, "bf16", max_iters=10)
        return x

    ctx.test_stall(lp.LP_STALL_GESL)
    with pytest.raises(lp.LpError) as e:
        run()
    assert e.value.status == lp.LP_E_TIMEOUT
    assert "bounded wait" in str(e.value)
    x = run()  # the stall was used once; the context still works
    residn, _ = oracle.residn(np.asarray(x, np.float32), normb)
    assert np.all(np.isfinite(x)) and residn < 1.0
