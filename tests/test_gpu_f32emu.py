"""FP32 emulated on the BF16 tensor cores (LP_F32_BF16X6) through the C ABI.

The trailing update splits every FP32 operand exactly into three BF16 terms
and keeps the six products that carry FP32's 24 bits, so the factorization
must be as accurate as the FP32 SIMT one: factors within the same normwise
bound of the oracle's unblocked FP32 factors, the plain FP32 solve (no
refinement) within the HPL threshold with the FP32 unit roundoff, and the
reference's own validation (residn < 1, linpack_benchmark.hpp:395-417).
"""
import functools

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu
FLT_EPS = float(np.finfo(np.float32).eps)


def factor(ctx, dev, A, bs, precision):
    d = dev.put(A)
    if precision == "f32":
        ctx.gefa(d.data_ptr(), A.shape[0], A.shape[1], bs)
    else:
        ctx.gefa_prec(precision, d.data_ptr(), A.shape[0], A.shape[1], bs)
    return d


@functools.lru_cache(maxsize=None)
def _oracle_factors(n):
    A, _, _, _ = oracle.gen_reference(n)
    return A, oracle.gefa_nopvt(A).astype(np.float64)


@pytest.mark.parametrize("n,bs", [(1024, 128), (2048, 512), (4096, 512), (4096, 1024)])
def test_factors_as_accurate_as_fp32(ctx, dev, n, bs):
    """Block 1024 is the emulated schedule's own (the FP32 path stops at 512,
    so its factors for comparison use block 512)."""
    A, want = _oracle_factors(n)
    emu = dev.get(factor(ctx, dev, A, bs, "f32_bf16x6")).astype(np.float64)
    simt = dev.get(factor(ctx, dev, A, min(bs, 512), "f32")).astype(np.float64)
    scale = np.abs(want).max()
    err_emu = np.abs(emu - want).max()
    err_simt = np.abs(simt - want).max()
    assert err_emu <= 8 * n * FLT_EPS * scale
    assert err_emu <= 4 * err_simt + 16 * FLT_EPS * scale


@pytest.mark.parametrize("n,bs", [(2048, 512), (4096, 512)])
def test_plain_solve_validates(ctx, dev, n, bs):
    A, b, _, normb = oracle.gen_reference(n)
    d = factor(ctx, dev, A, bs, "f32_bf16x6")
    dB = dev.put(b)
    ctx.gesl(d.data_ptr(), n, n, dB.data_ptr(), 1, n)
    x = dev.get(dB)
    rn, _ = oracle.residn(x, normb)
    assert rn < 1.0
    assert oracle.hpl_resid(A, x.astype(np.float64), b.astype(np.float64), eps=FLT_EPS / 2) < 16.0


def test_solve_host_without_refinement(ctx):
    n, bs = 2048, 512
    A, b64, _ = oracle.gen_baseline(n, seed=7, margin=1.0)
    x, t = ctx.solve_host(A, b64, bs, "f32_bf16x6", max_iters=0)
    assert t["ir_iters"] == 0
    assert oracle.hpl_resid(A, x, b64, eps=FLT_EPS / 2) <= 16.0
