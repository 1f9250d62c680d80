"""Per-stage parity of the CUDA kernels against the oracle, through the C ABI.

Mirrors LINPACK/tests/test_kernel_communication.cpp: the LU block against
gefa_ref_nopvt (:906-918), the left block against the host loop (:614-641),
the top block against the host loop (:748-799).  The reference allows a max
absolute error of FLT_EPSILON; the lu (bs <= 128), top and left kernels here
use the reference's operation order without fused multiply-add and must be
bit-identical.  The inner update (a GEMM, summation order free) is checked
against an FP64 product with the FP32 rounding bound k*eps*sum|L||T|.
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu
FLT_EPS = float(np.finfo(np.float32).eps)


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


@pytest.mark.parametrize("bs", [16, 32, 64, 128])
def test_lu_block_bitexact(ctx, dev, bs):
    A, _, _, _ = oracle.gen_reference(bs)
    d = dev.put(A)
    ctx.lu_block(d.data_ptr(), bs, bs)
    got = dev.get(d)
    want = oracle.gefa_nopvt(A)
    assert np.array_equal(bits(got), bits(want))


@pytest.mark.parametrize("bs", [256, 512])
def test_lu_block_recursive(ctx, dev, bs):
    """bs > 128: factored as 128-wide inner blocks whose trailing step is a
    GEMM (different summation order), so the bound is relative:
    |got - want| <= 64 eps max(1, |want|); the reference's own GEFA check
    allows 1e-3 absolute
    (test_kernel_functionality_and_host_integration.cpp:65-67)."""
    A, _, _, _ = oracle.gen_reference(bs)
    d = dev.put(A)
    ctx.lu_block(d.data_ptr(), bs, bs)
    got = dev.get(d)
    want = oracle.gefa_nopvt(A)
    err = np.abs(got.astype(np.float64) - want) / np.maximum(1.0, np.abs(want))
    assert err.max() < 64 * FLT_EPS
    assert np.abs(got - want).max() < 1e-3


def test_lu_block_in_larger_matrix(ctx, dev):
    """The block is addressed inside a matrix with lda > bs."""
    n, bs = 256, 64
    A, _, _, _ = oracle.gen_reference(n)
    d = dev.put(A)
    off = (64 * n + 64) * 4
    ctx.lu_block(d.data_ptr() + off, n, bs)
    got = dev.get(d)
    want = A.copy()
    want[64:128, 64:128] = oracle.gefa_nopvt(A[64:128, 64:128].copy())
    assert np.array_equal(bits(got), bits(want))


@pytest.mark.parametrize("bs,ncols", [(16, 16), (32, 100), (128, 128), (128, 1000), (512, 512), (512, 130)])
def test_top_update_bitexact(ctx, dev, bs, ncols):
    """test_kernel_communication.cpp:748-799: a uniform block right of a
    factored diagonal block."""
    D = oracle.gefa_nopvt(oracle.gen_reference(bs)[0])
    rng = np.random.default_rng(bs + ncols)
    T = rng.uniform(0.0, 1.0, (bs, ncols)).astype(np.float32)
    dD, dT = dev.put(D), dev.put(T)
    ctx.top_update(dD.data_ptr(), bs, dT.data_ptr(), ncols, bs, ncols)
    got = dev.get(dT)
    want = oracle.top_update(D, T)
    assert np.array_equal(bits(got), bits(want))


@pytest.mark.parametrize("bs,nrows", [(16, 16), (32, 70), (128, 128), (128, 1000), (512, 512), (512, 200)])
def test_left_update_bitexact(ctx, dev, bs, nrows):
    """test_kernel_communication.cpp:614-641; also the transposed copy."""
    D = oracle.gefa_nopvt(oracle.gen_reference(bs)[0])
    rng = np.random.default_rng(7 * bs + nrows)
    L = rng.uniform(0.0, 1.0, (nrows, bs)).astype(np.float32)
    ldlt = (nrows + 3) // 4 * 4
    dD, dL, dLt = dev.put(D), dev.put(L), dev.empty((bs, ldlt))
    ctx.left_update(dD.data_ptr(), bs, dL.data_ptr(), bs, bs, nrows, dLt.data_ptr(), ldlt)
    got = dev.get(dL)
    want = oracle.left_update(D, L)
    assert np.array_equal(bits(got), bits(want))
    assert np.array_equal(bits(dev.get(dLt)[:, :nrows]), bits(np.ascontiguousarray(want.T)))


@pytest.mark.parametrize("m,n,bs", [(16, 16, 16), (128, 128, 128), (48, 80, 32), (300, 260, 64), (512, 1024, 512),
                                    (1024, 1536, 512), (1100, 1300, 128), (2048, 520, 16)])
def test_inner_update(ctx, dev, m, n, bs):
    rng = np.random.default_rng(m * n + bs)
    C = rng.uniform(-1, 1, (m, n)).astype(np.float32)
    L = rng.uniform(-1, 1, (m, bs)).astype(np.float32)
    T = rng.uniform(-1, 1, (bs, n)).astype(np.float32)
    ldlt = (m + 3) // 4 * 4
    Lt = np.zeros((bs, ldlt), np.float32)
    Lt[:, :m] = L.T
    dC, dLt, dT = dev.put(C), dev.put(Lt), dev.put(T)
    ctx.inner_update(dC.data_ptr(), n, dLt.data_ptr(), ldlt, dT.data_ptr(), n, m, n, bs)
    got = dev.get(dC).astype(np.float64)
    exact = C.astype(np.float64) + L.astype(np.float64) @ T.astype(np.float64)
    bound = (bs + 1) * FLT_EPS * (np.abs(C) + np.abs(L).astype(np.float64) @ np.abs(T).astype(np.float64))
    assert np.all(np.abs(got - exact) <= bound)
    orc = oracle.inner_update(C, L, T).astype(np.float64)
    assert np.all(np.abs(orc - exact) <= bound)


def test_stage_argument_errors(ctx, lp):
    with pytest.raises(lp.LpError) as e:
        ctx.lu_block(1 << 20, 48, 48)
    assert e.value.status == lp.LP_E_INVALID
    with pytest.raises(lp.LpError):
        ctx.top_update(1 << 20, 64, 1 << 20, 64, 24, 64)
    with pytest.raises(lp.LpError):
        ctx.inner_update(1 << 20, 64, 1 << 20, 64, 1 << 20, 64, 64, 64, 20)
