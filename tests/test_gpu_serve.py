"""Serving loop on the GPU: every result is the same alone and in the mix
(FP32: bit for bit; refined precisions: within 1e-12 of max|x|, the FP64
refinement's atomics may round differently), passes the HPL scaled-residual
bound checked by the oracle (FP32: eps = FLT_EPSILON/2; refined:
DBL_EPSILON/2), and the server's reported residual agrees with the oracle's.
Also: reuse of resident factors, eviction and rejection under a small
budget, malformed requests, non-finite results, and the per-request mode."""
import numpy as np
import pytest

import oracle
from hpcc_fpga_b200 import serve

FLT_EPS = float(np.finfo(np.float32).eps)
DBL_EPS = float(np.finfo(np.float64).eps)

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def wl(lp):
    w = serve.Workload(master_n=3072, seed=42)
    yield w
    w.close()


def _copy_results(res, views):
    return [(r, v.copy()) for r, v in zip(res, views)]


def _check_against_oracle(wl, specs, results, views, eps, bound=16.0):
    """Oracle residual of every returned solution within the bound.  For FP32
    solutions the residual is far above FP64 rounding, so the server's own
    figure must agree with the oracle's; after FP64 refinement both sit at
    FP64 rounding level and only the bound is compared."""
    for spec, r, X in zip(specs, results, views):
        assert r["status"] == 0, r
        A = wl.matrix(spec)
        B = wl.rhs(spec)
        worst = max(oracle.hpl_resid(A, X[q], B[q].astype(np.float64), eps=eps / 2) for q in range(spec[2]))
        assert worst <= bound, (spec, worst)
        assert 0.0 <= r["hpl_resid"] <= bound, (spec, r["hpl_resid"])
        if eps == FLT_EPS:
            assert r["hpl_resid"] == pytest.approx(worst, rel=1e-3, abs=1e-4), (spec, r["hpl_resid"], worst)


def _alone(lp, wl, specs, **cfg):
    """Each request on an idle server, with a fresh key (so it factors itself)."""
    out = []
    with lp.Server(0, **cfg) as srv:
        for i, spec in enumerate(specs):
            reqs, views = wl.requests([(10 ** 6 + i,) + tuple(spec[1:])])
            srv.submit(reqs[0])
            got = srv.wait(1, timeout_ms=60000)
            out.append((got[0], views[0].copy()))
    return out


def _mix(lp, wl, specs, rate=20000.0, **cfg):
    arrival = np.arange(len(specs)) / rate
    with lp.Server(0, **cfg) as srv:
        reqs, views = wl.requests(specs)
        res = srv.replay(reqs, arrival, timeout_ms=60000)
        info = srv.info()
    return res, [v.copy() for v in views], info


def test_alone_equals_mix_f32(lp, wl):
    _, specs = serve.schedule(64, 1000.0, wl.master_n, lo=16, hi=3072, seed=11)
    mix, mix_x, info = _mix(lp, wl, specs)
    alone = _alone(lp, wl, specs)
    assert info["completed"] == len(specs) and info["waves"] >= 1
    assert info["waved_systems"] > info["waves"], "no wave held more than one system"
    assert sum(r["reused"] for r in mix) > 0
    for spec, r, x, (ra, xa) in zip(specs, mix, mix_x, alone):
        assert r["status"] == 0 and ra["status"] == 0
        assert np.array_equal(x, xa), f"request {spec} differs alone vs in the mix"
        assert r["batched"] == (spec[1] <= lp.server_config().batch_max_n)
    _check_against_oracle(wl, specs, mix, mix_x, FLT_EPS)
    # the work overlapped: some requests ran at the same time
    iv = sorted((r["t_start"], r["t_done"]) for r in mix)
    assert any(iv[i + 1][0] < iv[i][1] for i in range(len(iv) - 1))


@pytest.mark.parametrize("precision", ["bf16", "fp8"])
def test_alone_equals_mix_refined(lp, wl, precision):
    _, specs = serve.schedule(24, 1000.0, wl.master_n, lo=48, hi=3072, rhs_max=4, seed=5)
    mix, mix_x, _ = _mix(lp, wl, specs, precision=precision)
    alone = _alone(lp, wl, specs, precision=precision)
    for spec, r, x, (ra, xa) in zip(specs, mix, mix_x, alone):
        assert r["status"] == 0 and ra["status"] == 0
        assert np.abs(x - xa).max() <= 1e-12 * np.abs(xa).max(), spec
        if r["batched"]:
            assert np.array_equal(x, xa)       # batched refinement has no atomics
    _check_against_oracle(wl, specs, mix, mix_x, DBL_EPS)


def test_small_systems_match_fp64_oracle(lp, wl):
    _, specs = serve.schedule(12, 500.0, wl.master_n, lo=8, hi=400, seed=2)
    res, xs, _ = _mix(lp, wl, specs)
    for spec, r, X in zip(specs, res, xs):
        A = wl.matrix(spec).astype(np.float64)
        lu = oracle.gefa_nopvt(A)
        for q in range(spec[2]):
            x64 = oracle.gesl_nopvt(lu, wl.rhs(spec)[q].astype(np.float64))
            assert np.abs(X[q] - x64).max() <= 64 * FLT_EPS * np.abs(x64).max() * np.log2(spec[1] + 1)


def test_reuse_resident_factors(lp, wl):
    spec = (7, 1500, 3, 100, 200)
    with lp.Server(0) as srv:
        reqs, views = wl.requests([spec])
        srv.submit(reqs[0])
        r1 = srv.wait(1)[0]
        x1 = views[0].copy()
        assert r1["reused"] == 0
        # same key without the matrix, another right-hand-side block
        spec2 = (7, 1500, 3, 100, 900)
        reqs2, views2 = wl.requests([spec2])
        reqs2[0].A = None
        srv.submit(reqs2[0])
        r2 = srv.wait(1)[0]
        assert r2["status"] == 0 and r2["reused"] == 1
        _check_against_oracle(wl, [spec2], [r2], views2, FLT_EPS)
        assert not np.array_equal(views2[0], x1)
        # unknown key without a matrix
        reqs3, _ = wl.requests([(99, 64, 1, 0, 0)])
        reqs3[0].A = None
        with pytest.raises(lp.LpError) as e:
            srv.submit(reqs3[0])
        assert e.value.status == lp.LP_E_STATE


def test_budget_eviction_and_rejection(lp, wl):
    budget = 40 * 2 ** 20
    specs = [(k, 900, 2, 37 * k, 11 * k) for k in range(1, 13)]    # 6.5 MB of factors + originals each
    with lp.Server(0, hbm_budget_bytes=budget) as srv:
        reqs, views = wl.requests(specs)
        res = srv.replay(reqs, np.arange(len(specs)) * 1e-3)
        info = srv.info()
        assert all(r["status"] == 0 for r in res)
        assert info["evictions"] > 0 and info["used_bytes"] <= budget
        _check_against_oracle(wl, specs, res, views, FLT_EPS)
        # the first key was evicted: it is factored again from its matrix
        reqs2, views2 = wl.requests([specs[0]])
        srv.submit(reqs2[0])
        r = srv.wait(1)[0]
        assert r["status"] == 0 and r["reused"] == 0
        assert np.array_equal(views2[0], views[0])
        # larger than the whole budget
        big, _ = wl.requests([(500, 2500, 1, 0, 0)])
        srv.submit(big[0])
        r = srv.wait(1)[0]
        assert r["status"] == lp.LP_E_BUDGET and srv.info()["rejected"] == 1


def test_malformed_requests_and_timeouts(lp, wl):
    with lp.Server(0) as srv:
        reqs, _ = wl.requests([(1, 100, 1, 0, 0)])
        r = reqs[0]
        for field, value in [("n", 0), ("n", 20000), ("nrhs", 0), ("nrhs", 17), ("ldb", 50), ("ldx", 99),
                             ("lda", 10), ("B", None), ("X", None)]:
            old = getattr(r, field)
            setattr(r, field, value)
            with pytest.raises(lp.LpError) as e:
                srv.submit(r)
            assert e.value.status == lp.LP_E_INVALID, field
            setattr(r, field, old)
        assert srv.poll(timeout_ms=20) == []
        with pytest.raises(lp.LpError) as e:
            srv.wait(1, timeout_ms=50)
        assert e.value.status == lp.LP_E_TIMEOUT
        assert srv.info()["completed"] == 0


def test_non_finite_result_reported(lp, wl):
    zeros = lp.Pinned((1200, 1200), np.float32)
    zeros.array[:] = 0.0
    with lp.Server(0) as srv:
        for n in (200, 1100):                                      # wave path and slot path
            reqs, _ = wl.requests([(n, n, 1, 0, 0)])
            reqs[0].A, reqs[0].lda = zeros.ptr, 1200
            srv.submit(reqs[0])
            r = srv.wait(1)[0]
            assert r["status"] == lp.LP_E_NUMERIC, r
        # the server keeps serving, and the failed key was not kept
        specs = [(200, 200, 1, 5, 5)]
        reqs, views = wl.requests(specs)
        srv.submit(reqs[0])
        r = srv.wait(1)[0]
        assert r["status"] == 0 and r["reused"] == 0
        _check_against_oracle(wl, specs, [r], views, FLT_EPS)
    zeros.free()


def test_per_request_mode(lp, wl):
    _, specs = serve.schedule(20, 2000.0, wl.master_n, lo=16, hi=3072, seed=4)
    res, xs, info = _mix(lp, wl, specs, mode="per_request")
    assert info["waves"] == 0
    assert all(r["batched"] == 0 for r in res)
    iv = sorted((r["t_start"], r["t_done"]) for r in res)
    assert all(iv[i + 1][0] >= iv[i][1] for i in range(len(iv) - 1))   # strictly one at a time
    _check_against_oracle(wl, specs, res, xs, FLT_EPS)
