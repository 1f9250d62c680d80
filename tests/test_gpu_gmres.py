"""GMRES-based refinement (gmres_ref, LINPACK/src/host/gmres.c:53-232) on the
device through the C ABI: restarted left-preconditioned GMRES in FP64 with the
GPU's factors as preconditioner.  Checked against the compiled reference's
own gmres_ref on the same factors and right-hand side, and against the
classical refinement: every solution reaches the HPL threshold (scaled
residual <= 16 with eps = DBL_EPSILON/2, gmres.c:182-193)."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def lapack_lu(S):
    """The reference encoding (negated multipliers, -1/u_kk on the diagonal) as
    the unit-lower / upper LU that gmres_ref's triangular solves read (same
    column-major layout: M = S^T)."""
    LU = S.astype(np.float64).copy()
    iu = np.triu_indices(S.shape[0], 1)
    LU[iu] = -LU[iu]
    d = np.arange(S.shape[0])
    LU[d, d] = -1.0 / LU[d, d]
    return LU


def setup(ctx, dev, torch, n, bs, precision, margin=1.0, seed=42):
    A, b64, _ = oracle.gen_baseline(n, seed=seed, margin=margin)
    dA0 = dev.put(A)
    dLU = dev.put(A)
    if precision == "f32":
        ctx.gefa(dLU.data_ptr(), n, n, bs)
    else:
        ctx.gefa_prec(precision, dLU.data_ptr(), n, n, bs)
    return A, b64, dA0, dLU


@pytest.mark.parametrize("n,bs,prec", [(1024, 128, "f32"), (2048, 512, "bf16"), (2048, 512, "fp8")])
def test_gmres_reaches_hpl_threshold(ctx, dev, torch_cuda, n, bs, prec):
    A, b64, dA0, dLU = setup(ctx, dev, torch_cuda, n, bs, prec)
    dB = dev.put(b64)
    dX = torch_cuda.zeros(n, dtype=torch_cuda.float64, device="cuda")
    t = ctx.gmres(dA0.data_ptr(), n, dLU.data_ptr(), n, dB.data_ptr(), dX.data_ptr(), 50, 3, 1e-12)
    x = dev.get(dX)
    assert t["hpl_resid"] <= 16.0 and 1 <= t["ir_iters"] <= 150
    assert oracle.hpl_resid(A, x, b64) <= 16.0
    assert np.abs(x - 1.0).max() < 1e-9


def test_gmres_matches_reference_gmres(ctx, dev, torch_cuda):
    """Same factors (the GPU's, in the reference's LU layout), same b, same
    start x = b, restart 50, one cycle, tol 1e-8 (the reference test's
    arguments, test_host_reference_implementations.cpp:55-80)."""
    ref = oracle.ref("f32")
    if ref is None:
        pytest.skip("reference library not built (oracle/_ref)")
    n, bs = 256, 64
    A, b64, dA0, dLU = setup(ctx, dev, torch_cuda, n, bs, "f32", seed=3)
    LU = lapack_lu(dev.get(dLU))
    A64 = A.astype(np.float64)
    x_ref = b64.copy()
    ref.gmres_ref(n, A64, n, x_ref, b64.copy(), LU, n, 50, 1, 1e-8)
    dB = dev.put(b64)
    dX = dev.put(b64.copy())
    t = ctx.gmres(dA0.data_ptr(), n, dLU.data_ptr(), n, dB.data_ptr(), dX.data_ptr(), 50, 1, 1e-8)
    x = dev.get(dX)
    assert oracle.hpl_resid(A, x_ref, b64) <= 16.0
    assert oracle.hpl_resid(A, x, b64) <= 16.0 and t["hpl_resid"] <= 16.0
    assert np.abs(x - x_ref).max() <= 1e-9


def test_gmres_no_more_work_than_classical_refinement(ctx, dev, torch_cuda):
    """FP8 factors: GMRES reaches the threshold in no more preconditioner
    applications than classical refinement (one per iteration plus the first
    solve)."""
    n, bs = 2048, 512
    A, b64, dA0, dLU = setup(ctx, dev, torch_cuda, n, bs, "fp8", margin=1.0, seed=5)
    dB = dev.put(b64)
    dX = torch_cuda.zeros(n, dtype=torch_cuda.float64, device="cuda")
    ir = ctx.refine(dA0.data_ptr(), n, dLU.data_ptr(), n, dB.data_ptr(), dX.data_ptr(), 1, 50)
    dX2 = torch_cuda.zeros(n, dtype=torch_cuda.float64, device="cuda")
    gm = ctx.gmres(dA0.data_ptr(), n, dLU.data_ptr(), n, dB.data_ptr(), dX2.data_ptr(), 50, 3, 1e-12)
    assert ir["hpl_resid"] <= 16.0 and gm["hpl_resid"] <= 16.0
    assert gm["ir_iters"] + 1 <= ir["ir_iters"] + 2


def test_gmres_invalid_arguments(ctx, lp):
    with pytest.raises(lp.LpError):
        ctx.gmres(0, 64, 0, 64, 0, 0)
