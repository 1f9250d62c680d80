"""Serving loop, host side (no GPU): configuration and argument checks of the
C ABI, the Poisson workload schedule and the latency / throughput summaries."""
import ctypes
import math

import numpy as np
import pytest

from hpcc_fpga_b200 import serve


def test_default_config(lp):
    cfg = lp.server_config()
    assert cfg.hbm_budget_bytes == 80 * 10 ** 9
    assert cfg.mode == lp.LP_SERVE_CONTINUOUS and cfg.precision == lp.LP_F32
    assert cfg.batch_max_n == 512 and cfg.slots == 6 and cfg.large_slots == 2 and cfg.batch_workers >= 1
    assert cfg.warm_n == 0 and cfg.reserve_bytes == 0
    c2 = lp.server_config(precision="bf16", mode="per_request", slots=2)
    assert c2.precision == lp.LP_BF16_IR and c2.mode == lp.LP_SERVE_PER_REQUEST and c2.slots == 2


@pytest.mark.parametrize("field,value", [("slots", 0), ("slots", 17), ("batch_max_n", 2048), ("precision", 7),
                                         ("mode", 3), ("hbm_budget_bytes", 0), ("batch_workers", 0),
                                         ("max_refinements", -1), ("batch_max_count", 0)])
def test_bad_config_rejected_before_device(lp, field, value):
    cfg = lp.server_config()
    setattr(cfg, field, value)
    h = ctypes.c_void_p()
    assert lp.lib().lp_server_start(0, ctypes.byref(cfg), ctypes.byref(h)) == lp.LP_E_INVALID
    assert not h.value


def test_null_arguments(lp):
    L = lp.lib()
    r = lp.LpRequest()
    rid = ctypes.c_longlong()
    assert L.lp_server_submit(None, ctypes.byref(r), ctypes.byref(rid)) == lp.LP_E_INVALID
    out = (lp.LpResult * 4)()
    k = ctypes.c_int()
    assert L.lp_server_poll(None, out, 4, 10, ctypes.byref(k)) == lp.LP_E_INVALID
    assert L.lp_server_get_info(None, None) == lp.LP_E_INVALID
    assert L.lp_server_stop(None) == lp.LP_OK
    assert L.lp_server_start(0, None, None) == lp.LP_E_INVALID


def test_start_without_device(lp):
    if lp.device_count() > 0:
        pytest.skip("a GPU is present")
    with pytest.raises(lp.LpError) as e:
        lp.Server(0)
    assert e.value.status == lp.LP_E_NODEVICE


def test_schedule_distribution():
    arr, specs = serve.schedule(20000, 1000.0, 8192, seed=3)
    assert arr[0] == 0.0 and np.all(np.diff(arr) >= 0)
    gaps = np.diff(arr)
    assert abs(gaps.mean() - 1e-3) < 0.05e-3                      # mean inter-arrival 1/rate
    assert abs(gaps.std() / gaps.mean() - 1.0) < 0.05             # exponential: cv = 1
    n = np.array([s[1] for s in specs])
    assert n.min() >= 64 and n.max() <= 8192
    assert abs(np.median(np.log(n)) - 0.5 * (math.log(64) + math.log(8192))) < 0.1   # log-uniform
    nrhs = np.array([s[2] for s in specs])
    assert nrhs.min() == 1 and nrhs.max() == 16
    keys = [s[0] for s in specs]
    reuse = 1.0 - len(set(keys)) / len(keys)
    assert abs(reuse - 0.3) < 0.02
    first = {}
    for key, n_, _, off, boff in specs:                           # a key always names the same matrix
        assert first.setdefault(key, (n_, off)) == (n_, off)
        assert 0 <= off <= 8192 - n_ and 0 <= boff <= 8192 - n_
    arr2, specs2 = serve.schedule(20000, 1000.0, 8192, seed=3)
    assert np.array_equal(arr, arr2) and specs == specs2


def test_schedule_key_base_and_bounds():
    _, specs = serve.schedule(500, 100.0, 2048, lo=16, hi=4096, seed=1, key_base=5000)
    assert min(s[0] for s in specs) == 5001
    assert max(s[1] for s in specs) <= 2048


def _res(t_submit, t_done, n=1000, nrhs=1, reused=0, status=0, resid=1.0):
    return {"status": status, "t_submit": t_submit, "t_start": t_submit, "t_done": t_done, "n": n, "nrhs": nrhs,
            "reused": reused, "batched": 1, "ir_iters": 0, "hpl_resid": resid}


def test_summarize():
    res = [_res(i * 0.01, i * 0.01 + 0.002 * (1 + i % 10)) for i in range(100)]
    res.append(_res(1.0, 1.5, status=-7))
    arr = np.array([r["t_submit"] for r in res])
    s = serve.summarize(res, arr, None)
    assert s["ok"] == 100 and s["errors"] == 1
    assert s["p50_ms"] == pytest.approx(11.0, abs=1.0)
    assert s["p99_ms"] == pytest.approx(20.0, abs=0.5)
    assert s["solves_per_s"] == pytest.approx(100 / 1.5, rel=1e-3)
    assert s["gflops"] == pytest.approx(100 * (2e9 / 3 + 2e6) / 1.5 / 1e9, rel=1e-2)


def test_equal_p99():
    base = [{"rate": 100, "offered_per_s": 100, "solves_per_s": 99, "p99_ms": 20},
            {"rate": 500, "offered_per_s": 500, "solves_per_s": 480, "p99_ms": 60},
            {"rate": 1000, "offered_per_s": 1000, "solves_per_s": 520, "p99_ms": 900}]
    cont = [{"rate": 100, "offered_per_s": 100, "solves_per_s": 100, "p99_ms": 10},
            {"rate": 1000, "offered_per_s": 1000, "solves_per_s": 990, "p99_ms": 40},
            {"rate": 2000, "offered_per_s": 2000, "solves_per_s": 1500, "p99_ms": 300}]
    e = serve.equal_p99(base, cont)
    assert e["p99_bound_ms"] == 60 and e["baseline_solves_per_s"] == 480
    assert e["continuous_solves_per_s"] == 990 and e["ratio"] == pytest.approx(990 / 480, abs=0.01)
