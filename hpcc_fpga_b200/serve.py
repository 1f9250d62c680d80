"""Serving workload and load runs for the request loop (lp_server_*).

A stream of solve requests with Poisson arrivals: n log-uniform in [lo, hi],
1..rhs_max right-hand sides uniform in [-1, 1), and a fraction `reuse` of the
requests naming a matrix submitted before (drawn from the last `window` new
matrices), so their factors may still be resident.

Host data are pinned (lp_host_alloc), so the server's copies overlap:
  * one master matrix of order master_n from the seeded workload generator
    (lp_generate_baseline: off-diagonal entries in [-0.5, 0.5), diagonal =
    sum of |off-diagonal| + 1).  Request matrices are its principal
    submatrices M[o:o+n, o:o+n] at seeded offsets o, passed with
    lda = master_n; a principal submatrix of a strictly diagonally dominant
    matrix is strictly diagonally dominant, and no two offsets give the
    same matrix;
  * a pool of 16 right-hand-side rows; a request's B starts at a seeded
    column offset of the pool (ldb = master_n);
  * an arena for the FP64 solutions.
The schedule is replayed by lp_server_replay (submissions timed by a C++
thread), and the results are summarized as latency percentiles, solves/s
and the residual distribution.
"""
from __future__ import annotations

import math

import numpy as np

from . import lpcuda as lp


def flops(n: int, nrhs: int, factored: bool) -> float:
    """2n^3/3 (when factored) + 2 nrhs n^2 (LINPACK/src/host/linpack_benchmark.hpp:509-510)."""
    return (2.0 * n ** 3 / 3.0 if factored else 0.0) + 2.0 * nrhs * n * n


def schedule(count: int, rate: float, master_n: int, lo: int = 64, hi: int = 8192, rhs_max: int = 16,
             reuse: float = 0.3, window: int = 64, seed: int = 7, key_base: int = 0):
    """Arrival times (s, first at 0; exponential gaps of mean 1/rate) and
    request specs (key, n, nrhs, offset, b_offset)."""
    hi = min(hi, master_n)
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, count)
    arrival = np.concatenate([[0.0], np.cumsum(gaps[:-1])]) if count else np.zeros(0)
    specs = []
    recent: list[tuple[int, int, int]] = []
    next_key = key_base + 1
    for _ in range(count):
        nrhs = int(rng.integers(1, rhs_max + 1))
        if recent and rng.random() < reuse:
            key, n, off = recent[int(rng.integers(len(recent)))]
        else:
            n = int(min(hi, max(lo, math.floor(math.exp(rng.uniform(math.log(lo), math.log(hi + 1)))))))
            off = int(rng.integers(0, master_n - n + 1))
            key = next_key
            next_key += 1
            recent.append((key, n, off))
            if len(recent) > window:
                recent.pop(0)
        boff = int(rng.integers(0, master_n - n + 1))
        specs.append((key, n, nrhs, off, boff))
    return arrival, specs


class Workload:
    def __init__(self, master_n: int = 8192, seed: int = 42):
        self.master_n = master_n
        self.master = lp.Pinned((master_n, master_n), np.float32)
        lp.check(lp.lib().lp_generate_baseline(self.master.array, None, None, master_n, seed, 1.0),
                 "lp_generate_baseline")
        rng = np.random.default_rng(seed + 1)
        self.bpool = lp.Pinned((16, master_n), np.float32)
        self.bpool.array[:] = rng.uniform(-1.0, 1.0, (16, master_n)).astype(np.float32)
        self.xarena: lp.Pinned | None = None

    def close(self) -> None:
        for p in (self.master, self.bpool, self.xarena):
            if p is not None:
                p.free()

    def schedule(self, count: int, rate: float, **kw):
        return schedule(count, rate, self.master_n, **kw)

    def requests(self, specs):
        """lp_request array for the specs and the numpy views of their solutions."""
        total = sum(nrhs * n for _, n, nrhs, _, _ in specs)
        if self.xarena is None or self.xarena.array.size < total:
            if self.xarena is not None:
                self.xarena.free()
            self.xarena = lp.Pinned((max(total, 1 << 20),), np.float64)
        reqs, views = [], []
        m = self.master_n
        xo = 0
        for key, n, nrhs, off, boff in specs:
            r = lp.LpRequest()
            r.key, r.n, r.nrhs = key, n, nrhs
            r.A, r.lda = self.master.ptr + 4 * (off * m + off), m
            r.B, r.ldb = self.bpool.ptr + 4 * boff, m
            r.X, r.ldx = self.xarena.ptr + 8 * xo, n
            reqs.append(r)
            views.append(self.xarena.array[xo:xo + nrhs * n].reshape(nrhs, n))
            xo += nrhs * n
        return reqs, views

    def matrix(self, spec) -> np.ndarray:
        _, n, _, off, _ = spec
        return self.master.array[off:off + n, off:off + n]

    def rhs(self, spec) -> np.ndarray:
        _, n, nrhs, _, boff = spec
        return self.bpool.array[:nrhs, boff:boff + n]


def summarize(results: list[dict], arrival: np.ndarray, specs) -> dict:
    ok = [r for r in results if r["status"] == lp.LP_OK]
    lat = np.array([(r["t_done"] - r["t_submit"]) * 1e3 for r in ok]) if ok else np.zeros(1)
    t0 = min(r["t_submit"] for r in results) if results else 0.0
    t1 = max(r["t_done"] for r in results) if results else 1.0
    span = max(t1 - t0, 1e-9)
    fl = sum(flops(r["n"], r["nrhs"], not r["reused"]) for r in ok)
    resid = np.array([r["hpl_resid"] for r in ok]) if ok else np.zeros(1)
    offered = len(results) / max(float(arrival[-1]), 1e-9) if len(arrival) > 1 else 0.0
    return {
        "requests": len(results),
        "ok": len(ok),
        "errors": len(results) - len(ok),
        "offered_per_s": round(offered, 1),
        "solves_per_s": round(len(ok) / span, 1),
        "rhs_per_s": round(sum(r["nrhs"] for r in ok) / span, 1),
        "gflops": round(fl / span / 1e9, 1),
        "p50_ms": round(float(np.percentile(lat, 50)), 3),
        "p99_ms": round(float(np.percentile(lat, 99)), 3),
        "max_ms": round(float(lat.max()), 3),
        "reused_frac": round(sum(r["reused"] for r in ok) / max(len(ok), 1), 3),
        "batched_frac": round(sum(r["batched"] for r in ok) / max(len(ok), 1), 3),
        "ir_iters_mean": round(float(np.mean([r["ir_iters"] for r in ok])) if ok else 0.0, 3),
        "resid_p50": float(np.percentile(resid, 50)),
        "resid_p99": float(np.percentile(resid, 99)),
        "resid_max": float(resid.max()),
    }


def run(server: lp.Server, wl: Workload, rate: float, count: int, seed: int = 7, timeout_ms: int = 120000,
        **sched) -> tuple[dict, list[dict], list]:
    """One replay at `rate` req/s; returns (summary, results, specs)."""
    arrival, specs = wl.schedule(count, rate, seed=seed, **sched)
    reqs, _ = wl.requests(specs)
    res = server.replay(reqs, arrival, timeout_ms=timeout_ms)
    return summarize(res, arrival, specs), res, specs


def count_for_rate(rate: float) -> int:
    """Requests per replay: about 4 s of arrivals, at least 400, at most 2400."""
    return int(min(2400, max(400, 4.0 * rate)))


def ladder(server_factory, wl: Workload, rates, count=count_for_rate, seed: int = 7, warm: int = 300,
           overload: int = 600, **sched) -> list:
    """Replays at increasing rates on one server, after a warm-up burst.  The
    first rate the server does not sustain (solves/s below 0.85 x offered)
    ends the sweep; the highest rate of `rates` is then replayed once with
    `overload` requests (marked "overload") to show the saturated behaviour."""
    out = []
    rates = sorted(rates)
    with server_factory() as srv:
        run(srv, wl, 1e6, warm, seed=seed + 1000, key_base=10_000_000, **sched)
        for i, rate in enumerate(rates):
            s, _, _ = run(srv, wl, rate, count(rate), seed=seed + i, key_base=(i + 1) * 1_000_000, **sched)
            s["rate"] = rate
            out.append(s)
            if s["solves_per_s"] < 0.85 * s["offered_per_s"]:
                if rate < rates[-1] and overload > 0:
                    o, _, _ = run(srv, wl, rates[-1], overload, seed=seed + 500, key_base=50_000_000, **sched)
                    o["rate"] = rates[-1]
                    o["overload"] = True
                    out.append(o)
                break
    return out


def equal_p99(baseline: list, continuous: list) -> dict:
    """Throughput of both modes at the same p99 latency.  The bound is the
    baseline's p99 at its highest sustained rate (solves/s >= 0.9 x offered);
    each mode's best solves/s among its sustained runs within that bound."""
    def sustained(runs):
        return [r for r in runs if not r.get("overload") and r["solves_per_s"] >= 0.9 * r["offered_per_s"]]

    base = sustained(baseline) or [min(baseline, key=lambda r: r["p99_ms"])]
    ref = max(base, key=lambda r: r["solves_per_s"])
    bound = ref["p99_ms"]
    cont_ok = [r for r in sustained(continuous) if r["p99_ms"] <= bound]
    c = max(cont_ok, key=lambda r: r["solves_per_s"]) if cont_ok else None
    return {
        "p99_bound_ms": bound,
        "baseline_solves_per_s": ref["solves_per_s"],
        "baseline_rate": ref.get("rate"),
        "continuous_solves_per_s": c["solves_per_s"] if c else None,
        "continuous_rate": c.get("rate") if c else None,
        "continuous_p99_ms": c["p99_ms"] if c else None,
        "ratio": round(c["solves_per_s"] / ref["solves_per_s"], 2) if c else None,
    }
