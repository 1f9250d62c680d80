"""The oracle pinned: the C restatement (oracle/oracle.c, gen.cpp) against the
reference's own compiled routines (oracle/_ref, built from
LINPACK/src/host/linpack_data.cpp) and against the committed golden vectors,
plus the reference's host tests (LINPACK/tests/test_host_reference_implementations.cpp)."""
import os

import numpy as np
import pytest

import oracle

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "linpack_golden.npz")


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32 if a.dtype == np.float32 else np.uint64)


def need_ref(precision="f32"):
    lib = oracle.ref(precision)
    if lib is None:
        pytest.skip("reference library not built (oracle/_ref)")
    return lib


@pytest.mark.parametrize("n", [1, 2, 16, 33, 128, 200])
def test_restatement_bitexact_vs_reference_f32(n):
    ref = need_ref("f32")
    A, b, _, _ = oracle.gen_reference(n)
    mine = oracle.gefa_nopvt(A)
    theirs = A.copy()
    ref.ref_gefa_nopvt_f32(theirs, n, n)
    assert np.array_equal(bits(mine), bits(theirs))
    x_mine = oracle.gesl_nopvt(mine, b)
    x_ref = b.copy()
    ref.ref_gesl_nopvt_f32(theirs, x_ref, n, n)
    assert np.array_equal(bits(x_mine), bits(x_ref))


@pytest.mark.parametrize("n", [16, 100])
def test_restatement_bitexact_vs_reference_f64(n):
    ref = need_ref("f64")
    A, b64, _ = oracle.gen_baseline(n, seed=3)
    a = A.astype(np.float64)
    mine = oracle.gefa_nopvt(a)
    theirs = a.copy()
    ref.ref_gefa_nopvt_f64(theirs, n, n)
    assert np.array_equal(bits(mine), bits(theirs))
    x_mine = oracle.gesl_nopvt(mine, b64)
    x_ref = b64.copy()
    ref.ref_gesl_nopvt_f64(theirs, x_ref, n, n)
    assert np.array_equal(bits(x_mine), bits(x_ref))


def test_golden_vectors():
    """Vectors produced by the reference's own gefa/gesl (tests/golden/make_golden.py)."""
    g = np.load(GOLDEN)
    for n in g["sizes"]:
        A, b, _, normb = oracle.gen_reference(int(n))
        assert np.array_equal(bits(A), bits(g[f"A_{n}"])), "reference generator drifted"
        assert np.array_equal(bits(b), bits(g[f"b_{n}"]))
        lu = oracle.gefa_nopvt(A)
        assert np.array_equal(bits(lu), bits(g[f"lu_{n}"]))
        x = oracle.gesl_nopvt(lu, b)
        assert np.array_equal(bits(x), bits(g[f"x_{n}"]))
    for n in g["bsizes"]:
        A, b64, b32 = oracle.gen_baseline(int(n), seed=42, margin=1.0)
        assert np.array_equal(bits(A), bits(g[f"BA_{n}"]))
        assert np.array_equal(bits(b64), bits(g[f"Bb64_{n}"]))
        lu = oracle.gefa_nopvt(A)
        assert np.array_equal(bits(lu), bits(g[f"Blu_{n}"]))


def test_generate_uniform_matrix():
    """test_host_reference_implementations.cpp:30-38: entries in (0,1)."""
    A, _, _, _ = oracle.gen_reference(64, diag_dominant=False)
    assert np.all(A > 0.0) and np.all(A < 1.0)


def test_generate_diagonally_dominant_matrix():
    """test_host_reference_implementations.cpp:40-53: diagonal = sum of the
    storage row's off-diagonal entries (float accumulation)."""
    n = 64
    A, _, _, _ = oracle.gen_reference(n)
    for i in range(n):
        off = np.delete(A[i], i)
        assert np.all(off > 0.0) and np.all(off < 1.0)
        s = np.float32(0.0)
        for v in off:
            s = np.float32(s + v)
        assert np.isclose(A[i, i], s, rtol=4 * np.finfo(np.float32).eps, atol=0)


def test_b_is_column_sum():
    """b = M * ones with M = S^T: b[j] = sum of storage column j."""
    A, b, _, normb = oracle.gen_reference(50)
    assert np.allclose(b, A.astype(np.float64).sum(axis=0), rtol=1e-5)
    assert normb == b.max()


@pytest.mark.parametrize("n", [16, 128, 256])
def test_reference_solve_without_pivoting(n):
    """test_host_reference_implementations.cpp:92-98: gefa_ref_nopvt +
    gesl_ref_nopvt passes validateOutput (residn < 1)."""
    A, b, _, normb = oracle.gen_reference(n)
    x = oracle.gesl_nopvt(oracle.gefa_nopvt(A), b)
    residn, resid = oracle.residn(x, normb)
    assert residn < 1.0
    assert resid < 1e-3


def test_baseline_generator_exact_rhs():
    """b64 = M * ones exactly: the FP64 solve of (M, b64) returns ones."""
    A, b64, b32 = oracle.gen_baseline(96, seed=42, margin=1.0)
    assert np.array_equal(b64, A.astype(np.float64).T @ np.ones(96))
    assert np.array_equal(b32, b64.astype(np.float32))
    x = oracle.gesl_nopvt(oracle.gefa_nopvt(A.astype(np.float64)), b64)
    assert np.max(np.abs(x - 1.0)) < 1e-12
    off = np.abs(A.astype(np.float64)).sum(axis=1) - np.abs(np.diag(A))
    assert np.all(np.diag(A) >= off + 1.0 - 1e-3)


@pytest.mark.parametrize("n,bs", [(64, 16), (256, 64), (384, 128)])
def test_blocked_schedule_matches_unblocked(n, bs):
    """The per-stage loops composed in the PCIe schedule give the unblocked
    factors up to rounding."""
    A, _, _, _ = oracle.gen_reference(n)
    blk = oracle.blocked_gefa(A, bs)
    unb = oracle.gefa_nopvt(A)
    scale = np.maximum(1.0, np.abs(unb))
    assert np.max(np.abs(blk - unb) / scale) < 1e-5


def test_stage_loops_compose():
    """lu on the first block, then top/left/inner, equal the unblocked
    factorization's first block row/column exactly (top and left are exact
    restatements of the same recurrences)."""
    n, bs = 96, 32
    A, _, _, _ = oracle.gen_reference(n)
    unb = oracle.gefa_nopvt(A)
    d = oracle.gefa_nopvt(A[:bs, :bs].copy())
    assert np.array_equal(bits(d), bits(unb[:bs, :bs]))
    top = oracle.top_update(d, A[:bs, bs:])
    left = oracle.left_update(d, A[bs:, :bs])
    assert np.array_equal(bits(top), bits(unb[:bs, bs:]))
    assert np.array_equal(bits(left), bits(unb[bs:, :bs]))


def test_hpl_residual_definition():
    """gmres.c:182-193 restated: check against numpy on M = S^T."""
    n = 40
    A, b64, _ = oracle.gen_baseline(n, seed=1)
    x = np.ones(n) + 1e-9 * np.arange(n)
    M = A.astype(np.float64).T
    r = b64 - M @ x
    want = np.abs(r).max() / (np.abs(M).sum(axis=1).max() * np.abs(x).max() + np.abs(b64).max()) / n / (oracle.DBL_EPS / 2)
    assert np.isclose(oracle.hpl_resid(A, x, b64), want, rtol=1e-6)  # r is a cancelling difference
    assert np.allclose(oracle.residual_f64(A, x, b64), r, rtol=0, atol=1e-9)


# ---- partial pivoting: gefa_ref / gesl_ref (linpack_data.cpp:72-156) ------------

def _pivot_cases(n, rng):
    """A uniform (non-dominant) matrix plus edge cases of the pivot search:
    a zero diagonal, equal magnitudes of opposite sign (the first wins)."""
    A = rng.random((n, n)).astype(np.float32)
    if n >= 4:
        A[0, 0] = 0.0                       # step 0 must exchange
        A[1, 1:] = 0.5
        A[1, 3] = -0.5                      # |.| tie in M's column 1
        A[1, 1] = 0.25
    return A


@pytest.mark.parametrize("n", [1, 2, 5, 33, 128, 257])
def test_pivot_restatement_bitexact_vs_reference_f32(n):
    ref = need_ref("f32")
    A = _pivot_cases(n, np.random.default_rng(n))
    mine, p_mine = oracle.gefa_pvt(A)
    theirs = A.copy()
    p_ref = np.zeros(n, np.int32)
    ref.ref_gefa_pvt_f32(theirs, n, n, p_ref)
    assert np.array_equal(p_mine, p_ref)
    assert np.array_equal(bits(mine), bits(theirs))
    b = np.random.default_rng(1).random(n).astype(np.float32)
    x_mine = oracle.gesl_pvt(mine, p_mine, b)
    x_ref = b.copy()
    ref.ref_gesl_pvt_f32(theirs, x_ref, p_ref, n, n)
    assert np.array_equal(bits(x_mine), bits(x_ref))


@pytest.mark.parametrize("n", [16, 100])
def test_pivot_restatement_bitexact_vs_reference_f64(n):
    ref = need_ref("f64")
    A = _pivot_cases(n, np.random.default_rng(7)).astype(np.float64)
    mine, p_mine = oracle.gefa_pvt(A)
    theirs = A.copy()
    p_ref = np.zeros(n, np.int32)
    ref.ref_gefa_pvt_f64(theirs, n, n, p_ref)
    assert np.array_equal(p_mine, p_ref)
    assert np.array_equal(bits(mine), bits(theirs))


def test_pivot_search_semantics():
    """First of equal magnitudes; NaN below the diagonal never chosen; a NaN
    diagonal is kept (the reference's strict '<' scan)."""
    S = np.eye(4, dtype=np.float32)
    S[0] = [0.5, -2.0, 2.0, 1.0]            # M's column 0: tie between rows 1 and 2
    _, p = oracle.gefa_pvt(S)
    assert p[0] == 1
    S = np.eye(4, dtype=np.float32) * 3
    S[0] = [1.0, np.nan, 2.0, 0.0]
    _, p = oracle.gefa_pvt(S)
    assert p[0] == 2
    S[0] = [np.nan, 5.0, 2.0, 0.0]
    _, p = oracle.gefa_pvt(S)
    assert p[0] == 0


def test_pivot_solution_uniform_reference_input():
    """The harness's --uniform input (no diagonal dominance) solves to
    x = ones with the reference's residn < 1."""
    n = 200
    A, b, _, normb = oracle.gen_reference(n, diag_dominant=False)
    lu, p = oracle.gefa_pvt(A)
    x = oracle.gesl_pvt(lu, p, b)
    rn, _ = oracle.residn(x, normb)
    assert rn < 1.0
