#!/usr/bin/env python
"""LINPACK LU + solve on B200 — prints ONE compact JSON line.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl lpcuda|reference]
                    [--n 32768] [--bs 512] [--details PATH]

A step is one factorization (blocked LU without pivoting, the reference's
lu/top/left/inner stages) plus forward/back substitution of one n x n system
(default n = 32768, block 512, FP32: the plain FP32 workload), with the
system's matrix restored from a pristine device copy at the start of every
step.  ``value`` is GFLOP/s by the reference's formula 2n^3/3 + 2n^2
(LINPACK/src/host/linpack_benchmark.hpp:509-535) over device time of K steps
(CUDA events on the library's stream), inputs resident in HBM; ``e2e`` is the
same metric through the C ABI host call lp_calculate (the drop-in for
execution::pcie::calculate) with pinned host buffers: host->device copy of A
and b, factor, solve, device->host copy of the factors and x, all inside the
wall-clock timed call.

Beside the headline the run measures the mixed-precision forms (BF16 / FP8
E4M3 trailing updates + FP64 refinement) with the diagonal-dominance margin
swept over {1, 0.1 sqrt(n), n} at n = 32768 and n = 65536, the emulated-FP32,
pivoting and FP64 paths, the batched solver and the serving loop.  The last
stdout line is a compact summary of a few KB; every table in full goes to the
JSON file named by --details.

Multi-GPU: the path does not shard (one system per GPU); under torchrun each
rank runs an independent replica, time = max over ranks, value = total work
of all ranks / that time.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "LU+solve GFLOP/s FP32 vs BF16/FP8+IR at equal residual; batched solves/s, p99 ms"
UNIT = "GFLOP/s"
NUM_SMS = 148
FP32_LANES_PER_SM = 128
FLT_EPS_HALF = float(np.finfo(np.float32).eps) / 2
LINE_LIMIT = 2600  # bytes: the summary line must survive a few-KB stdout tail whole


def flops(n: int) -> float:
    return 2.0 * n ** 3 / 3.0 + 2.0 * n ** 2


def margins_for(n: int) -> list:
    """The diagonal-dominance margins of the mixed-precision sweep: 1, 0.1 sqrt(n), n."""
    return [1.0, 0.1 * math.sqrt(n), float(n)]


def peaks() -> dict:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        d["source"] = "measured"
        return d
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0, "sm_max_mhz": 1965.0,
            "source": "fallback"}


def host_cpu() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9 and parts[1].isdigit():
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "samples": 0}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
        sm = [int(r[1]) for r in rows]
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": int(rows[0][2]), "reasons": reasons,
                "samples": len(rows), "power_w_max": max(float(r[3]) for r in rows if r[3].replace(".", "").isdigit())}


class CpuBaseline:
    """The reference's own gefa_ref_nopvt + gesl_ref_nopvt (compiled from
    LINPACK/src/host/linpack_data.cpp into oracle/_ref/ref_bench), timed on
    one host core on the configured sample (same seeded generator).  The
    reference code is serial, so it runs as a background process on one core
    while the GPU legs run, and is collected before the serving leg (whose
    worker threads want the host cores)."""

    def __init__(self, n: int, reps: int):
        self.n, self.reps = n, reps
        self.exe = os.path.join(ROOT, "oracle", "_ref", "ref_bench")
        self.proc = None
        self.t0 = time.perf_counter()
        if os.path.exists(self.exe):
            self.proc = subprocess.Popen([self.exe, "--n", str(n), "--reps", str(reps), "--mode", "baseline",
                                          "--seed", "42", "--margin", "1"], stdout=subprocess.PIPE,
                                         stderr=subprocess.PIPE, text=True)

    def result(self) -> dict:
        if self.proc is None:
            return {"value": None, "unit": UNIT, "cores": 1, "kind": "reference",
                    "sample": "unavailable: oracle/_ref/ref_bench not built"}
        out, err = self.proc.communicate()
        if self.proc.returncode != 0:
            return {"value": None, "unit": UNIT, "cores": 1, "kind": "reference",
                    "sample": f"ref_bench failed ({self.proc.returncode}): {err.strip()[:200]}"}
        r = json.loads(out.strip().splitlines()[-1])
        return {"value": r["gflops"], "unit": UNIT, "cores": 1, "kind": "reference",
                "sample": f"one n={self.n} system (seed 42, margin 1), best of {self.reps}: gefa_ref_nopvt + "
                          "gesl_ref_nopvt compiled from the reference sources (g++ -O3 -march=x86-64-v3), "
                          "serial code on one core",
                "n": self.n, "t_min_s": r["t_min"], "gflops_lu": r["gflops_lu"], "residual_norm": r["residual_norm"],
                "host_nproc": os.cpu_count(), "host_cpu": host_cpu(),
                "wall_s": round(time.perf_counter() - self.t0, 1)}


def mixed_block(n: int, bs: int) -> int:
    """Block size of the tensor-core schedules: the largest power of two that
    leaves at least 32 block steps, at most 2048 and not below the FP32 block.
    Their update reads and writes FP32 C once per block step, so a wider block
    cuts that traffic; the panel chain grows with it.  Measured on one B200
    (BF16+IR): n=65536 block 512 / 1024 / 2048 -> 423 / 536 / 570 TFLOP/s;
    n=32768 -> 300 / 328 / 313."""
    b = 1
    while b * 2 <= min(2048, n // 32):
        b *= 2
    return max(bs, b)


def timed_steps(torch, ctx, stream, step, steps: int, warmup: int):
    """warmup untimed steps, then `steps` steps between two CUDA events on the
    library's stream, with the stage profile of the timed steps."""
    for _ in range(warmup):
        step()
    ctx.sync()
    ctx.set_profiling(True)
    ctx.read_profile(reset=True)
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    out = [step() for _ in range(steps)]
    ev1.record(stream)
    torch.cuda.synchronize()
    prof = ctx.read_profile(reset=True)
    ctx.set_profiling(False)
    return ev0.elapsed_time(ev1) * 1e-3, prof, out


def run_f32(ctx, lp, torch, stream, dA0, dA, dB0, dB, n, bs, steps, warmup) -> dict:
    """The plain FP32 step on one system: restore A and b, factor, solve."""
    def step():
        with torch.cuda.stream(stream):
            dA.copy_(dA0)
            dB.copy_(dB0)
        ctx.gefa(dA.data_ptr(), n, n, bs)
        ctx.gesl(dA.data_ptr(), n, n, dB.data_ptr(), 1, n)

    t, prof, _ = timed_steps(torch, ctx, stream, step, steps, warmup)
    inner = prof["inner"]
    return {"n": n, "block": bs, "value": steps * flops(n) / t / 1e9, "ms_per_step": 1e3 * t / steps,
            "inner_tflops": inner["flops"] / inner["s"] / 1e12 if inner["s"] > 0 else None,
            "max_abs_err_x": float((dB.double() - 1.0).abs().max()),
            "stages": {k: {"s": prof[k]["s"], "calls": prof[k]["calls"]} for k in lp.STAGES if prof[k]["calls"]}}


def run_mixed(ctx, lp, torch, stream, dA0, dA, dB64, n, bs, prec, steps, warmup, f32_value, pk,
              with_gmres: bool = True) -> dict:
    """BF16 / FP8 trailing updates + FP64 refinement to the HPL threshold on
    the system in dA0 (right-hand side dB64, exact solution all ones): GFLOP/s
    by the same formula over factor + all solves + refinement (the
    refinement's own 2n^2 flop per iteration not credited)."""
    with torch.cuda.stream(stream):
        dX = torch.empty(n, dtype=torch.float64, device="cuda")
    info = {}

    def step():
        with torch.cuda.stream(stream):
            dA.copy_(dA0)
        ctx.gefa_prec(prec, dA.data_ptr(), n, n, bs)
        info.update(ctx.refine(dA0.data_ptr(), n, dA.data_ptr(), n, dB64.data_ptr(), dX.data_ptr(), 1, 50))
        return info["ir_iters"], info["hpl_resid"]

    t, prof, res = timed_steps(torch, ctx, stream, step, steps, warmup)
    err = float((dX - 1.0).abs().max())
    inner = prof["inner"]
    gbs = inner["bytes"] / inner["s"] / 1e9 if inner["s"] > 0 else None
    tfs = inner["flops"] / inner["s"] / 1e12 if inner["s"] > 0 else None
    value = steps * flops(n) / t / 1e9
    # The update reads and writes FP32 C once (8 B per element) for 2*bs flop per element:
    # intensity bs/4 flop/B.  Below the ridge (tensor peak / HBM peak) the launch is
    # HBM-bound, above it tensor-bound.  No FP8 peak is measured: FP8 counts as twice
    # the measured BF16 rate (the part's nominal ratio).
    tpk = pk["bf16_tflops"] * (2.0 if prec == "fp8" else 1.0)
    ridge = tpk * 1e12 / (pk["hbm_gbs"] * 1e9)
    tensor_bound = bs / 4.0 > ridge
    out = {
        "n": n, "block": bs, "precision": prec,
        "value": value, "unit": UNIT, "ms_per_step": 1e3 * t / steps,
        "speedup_vs_f32": value / f32_value if f32_value else None,
        "ir_iters": max(r[0] for r in res), "hpl_resid": max(r[1] for r in res), "hpl_eps": "DBL_EPSILON/2",
        "max_abs_err_vs_fp64_oracle": err,
        "roofline": {"bound": "tensor" if tensor_bound else "hbm",
                     "kernel": (f"k_umma_pair<{prec}> (inner stage, tcgen05 256 x 256 tiles on CTA pairs)"
                                if prec == "bf16" or bs <= 512 else
                                "k_umma_update<fp8, SEG> (inner stage, tcgen05, per-512 K segments)"),
                     "achieved": tfs if tensor_bound else gbs,
                     "peak": tpk if tensor_bound else pk["hbm_gbs"],
                     "unit": "TFLOP/s" if tensor_bound else "GB/s",
                     "frac": (tfs / tpk if tensor_bound else gbs / pk["hbm_gbs"]) if gbs else None,
                     "hbm_frac": gbs / pk["hbm_gbs"] if gbs else None,
                     "tensor_frac": tfs / tpk if tfs else None,
                     "per_unit": f"8*m*n bytes (FP32 C read+write) and 2*m*n*{bs} flop per m x n trailing "
                                 f"update: intensity {bs / 4:.0f} flop/B against the {prec} ridge {ridge:.0f} flop/B",
                     "peak_source": pk["source"] + ("; FP8 peak = 2 x the measured BF16 rate" if prec == "fp8"
                                                    else "")},
        "stages": {k: {"s": prof[k]["s"], "calls": prof[k]["calls"]} for k in lp.STAGES if prof[k]["calls"]},
    }
    if with_gmres:
        # GMRES-based refinement (gmres_ref on the device) on the same factors, from x = 0
        with torch.cuda.stream(stream):
            dXg = torch.zeros(n, dtype=torch.float64, device="cuda")
        g = ctx.gmres(dA0.data_ptr(), n, dA.data_ptr(), n, dB64.data_ptr(), dXg.data_ptr(), 50, 3, 1e-12)
        out["gmres"] = {"seconds": g["ir_s"], "arnoldi_steps": g["ir_iters"], "hpl_resid": g["hpl_resid"],
                        "max_abs_err_vs_fp64_oracle": float((dXg - 1.0).abs().max()),
                        "note": "restart 50, 3 cycles, tol 1e-12, preconditioner = these factors applied in FP64"}
    return out


def run_margin_sweep(ctx, lp, torch, stream, dA0, dA, n, bs, precs, steps, warmup, f32_value, pk,
                     skip_margin_one: dict | None = None) -> list:
    """The mixed-precision forms over the margins {1, 0.1 sqrt(n), n} of the
    seeded generator: the diagonal (and b64) of dA0 are rewritten on the
    device per margin — bit-identical to drawing the matrix again with that
    margin — and restored to margin 1 afterwards.  Per case: IR iterations,
    HPL scaled residual and max |x - 1| (the FP64 oracle's solution is exactly
    all ones)."""
    from hpcc_fpga_b200.workload import set_margin

    rows = []
    diag1 = dA0.diagonal().clone()
    try:
        for m in margins_for(n):
            if m == 1.0 and skip_margin_one:
                for prec in precs:
                    r = skip_margin_one.get(prec)
                    if r is not None:
                        rows.append({"n": n, "precision": prec, "block": bs, "margin": m, "value": r["value"],
                                     "ir_iters": r["ir_iters"], "hpl_resid": r["hpl_resid"],
                                     "max_abs_err": r["max_abs_err_vs_fp64_oracle"]})
                continue
            with torch.cuda.stream(stream):
                dB64 = set_margin(torch, dA0, n, m)
            torch.cuda.synchronize()
            for prec in precs:
                r = run_mixed(ctx, lp, torch, stream, dA0, dA, dB64, n, bs, prec, steps, warmup, f32_value, pk,
                              with_gmres=False)
                rows.append({"n": n, "precision": prec, "block": bs, "margin": m, "value": r["value"],
                             "ir_iters": r["ir_iters"], "hpl_resid": r["hpl_resid"],
                             "max_abs_err": r["max_abs_err_vs_fp64_oracle"]})
            del dB64
    finally:
        with torch.cuda.stream(stream):
            dA0.diagonal().copy_(diag1)
        torch.cuda.synchronize()
    return rows


def run_f32emu(ctx, lp, torch, stream, dA0, dA, dB0, dB, dB64, n, bs, steps, warmup, f32_value, pk) -> dict:
    """FP32 emulated on the BF16 tensor cores (LP_F32_BF16X6: exact three-term
    BF16 split of every operand, six products, FP32 accumulation) on the same
    system and the same step as the FP32 headline: restore A and b, factor,
    plain FP32 solve — no refinement."""
    def step():
        with torch.cuda.stream(stream):
            dA.copy_(dA0)
            dB.copy_(dB0)
        ctx.gefa_prec("f32_bf16x6", dA.data_ptr(), n, n, bs)
        ctx.gesl(dA.data_ptr(), n, n, dB.data_ptr(), 1, n)

    t, prof, _ = timed_steps(torch, ctx, stream, step, steps, warmup)
    err = float((dB.double() - 1.0).abs().max())
    with torch.cuda.stream(stream):
        dXr = torch.empty(n, dtype=torch.float64, device="cuda")
    r32 = ctx.refine(dA0.data_ptr(), n, dA.data_ptr(), n, dB64.data_ptr(), dXr.data_ptr(), 1, 0)["hpl_resid"]
    inner = prof["inner"]
    tf32eq = inner["flops"] / inner["s"] / 1e12 if inner["s"] > 0 else None
    value = steps * flops(n) / t / 1e9
    spk = pk.get("bf16_tflops_sustained", pk["bf16_tflops"])
    return {
        "workload": f"the FP32 workload's system and step (n={n}) in blocks of {bs}, with the trailing update "
                    "and the panel's top/left products emulated on the BF16 tensor cores: exact 3-term BF16 split, "
                    "6 products, FP32 accumulation; plain FP32 solve, no refinement",
        "block": bs,
        "value": value, "unit": UNIT, "ms_per_step": 1e3 * t / steps, "speedup_vs_f32_simt": value / f32_value,
        "max_abs_err_x": err,
        "hpl_resid": {"eps_flt_half": r32 * 2.0 ** -29, "eps_dbl_half": r32},
        # timed inside a seconds-long factorization: the sustained BF16 figure is the denominator
        "roofline": {"bound": "tensor", "kernel": "k_umma_pair (inner stage, K = 6 bs)",
                     "achieved": 6 * tf32eq if tf32eq else None, "peak": spk, "unit": "TFLOP/s",
                     "frac": 6 * tf32eq / spk if tf32eq else None,
                     "fp32_equivalent_tflops": tf32eq,
                     "peak_source": pk["source"] + " (bf16_tflops_sustained; burst " + str(pk["bf16_tflops"]) + ")",
                     "per_unit": "6 x 2*m*n*bs BF16 flop per m x n trailing update (2*m*n*bs FP32-equivalent)"},
        "stages": {k: {"s": prof[k]["s"], "calls": prof[k]["calls"]} for k in lp.STAGES if prof[k]["calls"]},
    }


def run_batched(ctx, lp, torch, stream, steps, warmup, peak_tf, count=4096) -> dict:
    """The batched workload: `count` systems, n log-uniform in [32, 1024]
    (seed 7), 1..8 right-hand sides, seeded diagonally dominant matrices.
    FP32: one persistent graph-replayed launch with the autotuned
    configuration; BF16+IR: the refined batch (BF16 trailing updates on the
    tensor cores, FP32 solve, FP64 refinement to the HPL threshold, all in one
    launch).  Inputs are restored from pristine device copies before every
    step (not timed).  Baselines: every system through the single-system
    device path on the whole GPU (identity-padded to a multiple of 64,
    lp_gefa_dev + lp_gesl_dev per system, wall clock), and the batched
    kernel launched once per system."""
    from hpcc_fpga_b200 import batch as hb

    b = hb.make_batch(count, 32, 1024, 7, rhs_max=8)
    B64 = b.B.astype(np.float64)
    with torch.cuda.stream(stream):
        dA0 = torch.from_numpy(b.A).to("cuda")
        dB0 = torch.from_numpy(b.B).to("cuda")
        dB64 = torch.from_numpy(B64).to("cuda")
        dA = torch.empty_like(dA0)
        dB = torch.empty_like(dB0)
        dX = torch.empty_like(dB64)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    cfg = ctx.batch_autotune(b.systems, dA0.data_ptr(), dB0.data_ptr())
    tune_s = time.perf_counter() - t0

    def restore():
        with torch.cuda.stream(stream):
            dA.copy_(dA0)
            dB.copy_(dB0)

    secs = []
    replayed = 0
    for i in range(warmup + steps):
        restore()
        st = ctx.batch_solve(b.systems, dA.data_ptr(), dB.data_ptr())
        if i >= warmup:
            secs.append(st["seconds"])
            replayed += st["graph_replayed"]
    t = sum(secs) / len(secs)
    X = dB.cpu().numpy()
    # accuracy of a sample of systems: scaled residual in FP64 on the host
    worst = 0.0
    for i in range(0, count, max(1, count // 64)):
        s = b.systems[i]
        M = b.mat(i).astype(np.float64).T
        xq = X[s.b_off:s.b_off + s.nrhs * s.ldb].reshape(s.nrhs, s.ldb)[:, :s.n].astype(np.float64)
        for q in range(s.nrhs):
            rhs = b.rhs(i)[q].astype(np.float64)
            r = rhs - M @ xq[q]
            den = (np.abs(M).sum(axis=1).max() * np.abs(xq[q]).max() + np.abs(rhs).max()) * s.n * FLT_EPS_HALF
            worst = max(worst, float(np.abs(r).max() / den))
    flops_b = b.flops()

    # BF16 + FP64 refinement, the same systems and configuration
    secs_ir, its_max, res_max, replayed_ir = [], 0, 0.0, 0
    for i in range(warmup + steps):
        restore()
        st, its, res = ctx.batch_solve_ir(b.systems, dA.data_ptr(), dB64.data_ptr(), dX.data_ptr(), "bf16",
                                          max_iters=10)
        if i >= warmup:
            secs_ir.append(st["seconds"])
            replayed_ir += st["graph_replayed"]
            its_max = max(its_max, int(its.max()))
            res_max = max(res_max, float(res.max()))
    t_ir = sum(secs_ir) / len(secs_ir)
    X64 = dX.cpu().numpy()
    # the solutions against the FP64 oracle on a sample (np.linalg.solve of M x = b in FP64)
    err_ir = 0.0
    for i in range(0, count, max(1, count // 64)):
        s = b.systems[i]
        M = b.mat(i).astype(np.float64).T
        xq = X64[s.b_off:s.b_off + s.nrhs * s.ldb].reshape(s.nrhs, s.ldb)[:, :s.n]
        want = np.linalg.solve(M, b.rhs(i).astype(np.float64).T).T
        err_ir = max(err_ir, float(np.abs(xq - want).max() / max(1e-300, np.abs(want).max())))

    # every system through the single-system device path on the whole GPU (what a caller
    # without the batched kernel runs): identity-padded to a multiple of 64, factor + solve
    def padded(i):
        s = b.systems[i]
        npad = (s.n + 63) // 64 * 64
        P = np.eye(npad, dtype=np.float32)
        P[:s.n, :s.n] = b.mat(i)
        R = np.zeros((s.nrhs, npad), np.float32)
        R[:, :s.n] = b.rhs(i)
        return npad, P, R

    pads = [padded(i) for i in range(count)]
    with torch.cuda.stream(stream):
        dP = [torch.from_numpy(P).to("cuda") for _, P, _ in pads]
        dR = [torch.from_numpy(R).to("cuda") for _, _, R in pads]
    torch.cuda.synchronize()
    w0 = time.perf_counter()
    for (npad, _, _), p, r, s in zip(pads, dP, dR, b.systems):
        bsp = 128 if npad % 128 == 0 else 64
        ctx.gefa(p.data_ptr(), npad, npad, bsp)
        ctx.gesl(p.data_ptr(), npad, npad, r.data_ptr(), s.nrhs, npad)  # returns after the solve finished
    full_wall = time.perf_counter() - w0
    del dP, dR, pads

    # the batched kernel launched once per system, no graph
    cfg1 = lp.LpBatchConfig.from_buffer_copy(cfg)
    cfg1.use_graph = 0
    restore()
    torch.cuda.synchronize()
    loop_dev = 0.0
    w0 = time.perf_counter()
    for s in b.systems:
        loop_dev += ctx.batch_solve([s], dA.data_ptr(), dB.data_ptr(), cfg1)["seconds"]
    loop_wall = time.perf_counter() - w0
    value = flops_b / t / 1e9
    return {
        "workload": f"{count} systems, n log-uniform in [32,1024] (seed 7), 1-8 RHS uniform in [-1,1)",
        "value": value, "unit": UNIT, "solves_per_s": count / t, "ms_per_batch": 1e3 * t,
        "graph_replays": replayed, "config": cfg.as_dict(), "autotune_s": tune_s,
        "hpl_resid_flt_eps_max_sample": worst,
        "frac": value / 1e3 / peak_tf,
        "roofline": {"bound": "fp32_simt", "achieved": value / 1e3, "peak": peak_tf, "unit": "TFLOP/s",
                     "frac": value / 1e3 / peak_tf,
                     "note": "whole launch (every system's factor + solve) against the derived FP32 SIMT peak; "
                             "each CTA owns one system, so small systems are latency-bound"},
        "bf16": {"value": flops_b / t_ir / 1e9, "unit": UNIT, "solves_per_s": count / t_ir, "ms_per_batch": 1e3 * t_ir,
                 "ir_iters_max": its_max, "hpl_resid_max": res_max, "hpl_eps": "DBL_EPSILON/2",
                 "max_rel_err_vs_fp64_sample": err_ir, "graph_replays": replayed_ir,
                 "note": "trailing updates of systems above small_n_max in BF16 on the tensor cores (warp-level "
                         "MMA), FP32 solve, FP64 refinement in the same launch; refinement flops not credited"},
        "full_gpu_loop": {"solves_per_s": count / full_wall, "gflops": flops_b / full_wall / 1e9,
                          "s_wall": full_wall,
                          "how": "per system: identity-padded to a multiple of 64, lp_gefa_dev + lp_gesl_dev "
                                 "(block 128 or 64) on the whole GPU, wall clock"},
        "speedup_vs_full_gpu_loop": full_wall / t,
        "per_system_loop": {"solves_per_s_wall": count / loop_wall, "solves_per_s_device": count / loop_dev,
                            "gflops_wall": flops_b / loop_wall / 1e9, "ms_wall": 1e3 * loop_wall,
                            "how": "the batched kernel launched once per system (one CTA), no graph"},
        "speedup_vs_per_system_loop_wall": loop_wall / t,
    }


def run_fp64(ctx, lp, torch, stream, dA32, db64, n, steps, warmup, peak_fp64) -> dict:
    """The double build (DATA_TYPE double): the same system's FP32 entries
    widened to double, b in double (x = ones exactly); a step = restore A,
    lp_gefa_f64_dev (bs 256) + lp_gesl_f64_dev, on device time."""
    bs = 256
    with torch.cuda.stream(stream):
        dA0 = dA32.double()
        dA = torch.empty_like(dA0)
        dB = torch.empty_like(db64)
    torch.cuda.synchronize()

    def step():
        with torch.cuda.stream(stream):
            dA.copy_(dA0)
            dB.copy_(db64)
        ctx.gefa_f64(dA.data_ptr(), n, n, bs)
        ctx.gesl_f64(dA.data_ptr(), n, n, dB.data_ptr(), 1, n)

    t, prof, _ = timed_steps(torch, ctx, stream, step, steps, warmup)
    resid = float((dB - 1.0).abs().max())
    normb = float(db64.abs().max())
    inner = prof["inner"]
    tfs = inner["flops"] / inner["s"] / 1e12 if inner["s"] > 0 else None
    stage_s = {k: prof[k]["s"] for k in lp.STAGES if prof[k]["calls"]}
    tot = sum(stage_s.values())
    del dA0, dA
    return {
        "workload": f"FP64 LU without pivoting + substitution (the double build), n={n}, block {bs}, the FP32 "
                    "workload's entries widened to double, b = A*ones in double",
        "value": steps * flops(n) / t / 1e9, "unit": UNIT, "ms_per_step": 1e3 * t / steps,
        "max_abs_err_x": resid, "residn_dbl": resid / (n * normb * float(np.finfo(np.float64).eps)),
        "roofline": {"bound": "fp64_simt", "kernel": "k_dgemm_update (inner stage)", "achieved": tfs,
                     "peak": peak_fp64, "unit": "TFLOP/s", "frac": tfs / peak_fp64 if tfs else None,
                     "peak_source": "derived: 148 SMs x 64 FP64 lanes x 2 flop x median SM clock under load"},
        "stages": {k: {"s": v, "share": v / tot if tot > 0 else None, "calls": prof[k]["calls"]}
                   for k, v in stage_s.items()},
    }


def run_pivot(ctx, lp, torch, stream, n, steps, warmup, peak_tf) -> dict:
    """LU with partial pivoting (the harness's --uniform case, gefa_ref /
    gesl_ref convention) on a non-dominant matrix: U(0,1) entries (seed 42,
    torch's device generator), b = column sums of the storage (x = ones).
    A step = restore A, lp_gefa_pvt_dev + lp_gesl_pvt_dev, on device time."""
    with torch.cuda.stream(stream):
        g = torch.Generator(device="cuda")
        g.manual_seed(42)
        dA0 = torch.rand((n, n), generator=g, device="cuda", dtype=torch.float32)
        db0 = torch.zeros(n, dtype=torch.float64, device="cuda")
        for r in range(0, n, 4096):
            db0 += dA0[r:r + 4096].double().sum(0)
        db0 = db0.float()
        dA = torch.empty_like(dA0)
        dB = torch.empty_like(db0)
        dP = torch.zeros(n, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()

    def step():
        with torch.cuda.stream(stream):
            dA.copy_(dA0)
            dB.copy_(db0)
        ctx.gefa_pvt(dA.data_ptr(), n, n, dP.data_ptr())
        ctx.gesl_pvt(dA.data_ptr(), n, n, dP.data_ptr(), dB.data_ptr(), 1, n)

    t, prof, _ = timed_steps(torch, ctx, stream, step, steps, warmup)
    x = dB.double()
    resid = float((x - 1.0).abs().max())
    normb = float(db0.max())
    swaps = int((dP.cpu().numpy() != np.arange(n)).sum())
    inner = prof["inner"]
    tfs = inner["flops"] / inner["s"] / 1e12 if inner["s"] > 0 else None
    stage_s = {k: prof[k]["s"] for k in lp.STAGES if prof[k]["calls"]}
    tot = sum(stage_s.values())
    return {
        "workload": f"FP32 LU with partial pivoting + substitution, n={n}, U(0,1) entries (no diagonal dominance), "
                    "b = A*ones, seed 42",
        "value": steps * flops(n) / t / 1e9, "unit": UNIT, "ms_per_step": 1e3 * t / steps,
        "row_exchanges": swaps, "max_abs_err_x": resid,
        "residn": resid / (n * normb * float(np.finfo(np.float32).eps)),
        "roofline": {"bound": "fp32_simt", "kernel": "k_sgemm_update (inner stage)", "achieved": tfs,
                     "peak": peak_tf, "unit": "TFLOP/s", "frac": tfs / peak_tf if tfs else None},
        "stages": {k: {"s": v, "share": v / tot if tot > 0 else None, "calls": prof[k]["calls"]}
                   for k, v in stage_s.items()},
        "stage_names": {"lu": "k_piv_panel (pivot search, exchange, panel update)",
                        "left": "k_piv_rows (interchanges + triangular solve of the block row)",
                        "inner": "k_sgemm_update", "gesl": "k_piv_gesl"},
    }


def run_gesl_noalloc(lp, torch, stream, dLU, dB0, n, steps) -> dict:
    """lp_gesl_dev_noalloc (the allocation-free substitution: the same two
    persistent sweeps as lp_gesl_dev, their published values in the library's
    fixed device array) on the factors of the FP32 run, one right-hand side;
    device time per solve."""
    dB = torch.empty_like(dB0)
    L = lp.lib()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    secs = 0.0
    for i in range(1 + steps):
        with torch.cuda.stream(stream):
            dB.copy_(dB0)
            ev0.record(stream)
        lp.check(L.lp_gesl_dev_noalloc(dLU.data_ptr(), n, n, dB.data_ptr(), 1, n, ctypes.c_void_p(stream.cuda_stream)),
                 "lp_gesl_dev_noalloc")
        with torch.cuda.stream(stream):
            ev1.record(stream)
        torch.cuda.synchronize()
        if i > 0:
            secs += ev0.elapsed_time(ev1) * 1e-3
    s = secs / steps
    return {"kernels": "k_gesl_sweep forward + backward (as lp_gesl_dev), scratch in the library's static array",
            "s_per_solve": s, "GBps": 4.0 * n * n / s / 1e9,
            "max_abs_err_x": float((dB.double() - 1.0).abs().max())}


RESERVE = 110 * 10 ** 9  # pool mapped at start: the 80 GB budget plus headroom against fragmentation


def run_serving(lp, rates, precisions, master_n=8192) -> dict:
    """The serving workload: Poisson arrivals at each rate of the ladder, n
    log-uniform in [64, 8192], 1..16 right-hand sides, 30% of the requests
    naming a matrix submitted before, 80 GB budget; continuous batching
    against the per-request baseline (one request at a time, plain
    launches), per precision.  Latency = completion - submission, measured
    by the server's steady clock; solves/s over the first submission to the
    last completion of each replay."""
    from hpcc_fpga_b200 import serve

    wl = serve.Workload(master_n=master_n, seed=42)
    out = {"workload": f"Poisson arrivals, n log-uniform in [64,{master_n}], 1-16 RHS, 30% reuse of one of the "
                       f"last 64 matrices, principal submatrices of a seed-42 diagonally dominant {master_n}^2 "
                       "matrix, 80 GB budget",
           "rates": list(rates)}
    try:
        for prec in precisions:
            res = {}
            for mode in ("per_request", "continuous"):
                t0 = time.perf_counter()
                res[mode] = serve.ladder(
                    lambda: lp.Server(0, precision=prec, mode=mode, warm_n=master_n, reserve_bytes=RESERVE), wl,
                    rates, seed=7)
                res[mode + "_wall_s"] = round(time.perf_counter() - t0, 1)
            res["equal_p99"] = serve.equal_p99(res["per_request"], res["continuous"])
            out[prec] = res
    finally:
        wl.close()
    return out


# ---------------------------------------------------------------- the summary line
def sig(x, d: int = 4):
    """x rounded to d significant digits; None for missing or non-finite values."""
    if x is None:
        return None
    if isinstance(x, bool):
        return x
    if isinstance(x, int):
        return x
    try:
        xf = float(x)
    except (TypeError, ValueError):
        return x
    if not math.isfinite(xf):
        return None
    if xf == 0.0:
        return 0.0
    return float(f"{xf:.{d}g}")


def _mixed_summary(r: dict | None) -> dict | None:
    if not r:
        return None
    return {"value": sig(r.get("value")), "x_f32": sig(r.get("speedup_vs_f32"), 3), "iters": r.get("ir_iters"),
            "hpl": sig(r.get("hpl_resid"), 3), "err": sig(r.get("max_abs_err_vs_fp64_oracle"), 2),
            "frac": sig((r.get("roofline") or {}).get("frac"), 3)}


def compact_line(full: dict) -> dict:
    """The stdout summary: the contract's keys, the headline roofline, e2e,
    CPU baseline and clocks, and one flat summary per extension.  Strict JSON
    (no NaN / infinity) and at most LINE_LIMIT bytes; the full tables stay in
    the details file."""
    line = {k: full.get(k) for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                                     "higher_is_better", "scaling", "vs_baseline", "dtype", "data")}
    for k in ("value", "ms_per_step"):
        line[k] = sig(line[k], 6)
    line["config"] = full.get("config")
    rl = full.get("roofline") or {}
    line["roofline"] = {"bound": rl.get("bound"), "achieved": sig(rl.get("achieved")), "peak": sig(rl.get("peak")),
                        "unit": rl.get("unit"), "frac": sig(rl.get("frac"), 3), "traffic": sig(rl.get("traffic")),
                        "kernel": "k_sgemm_update", "peak_src": rl.get("peak_short")}
    e = full.get("e2e")
    if e:
        line["e2e"] = {"value": sig(e.get("value"), 6), "unit": e.get("unit"),
                       "h2d_bytes_per_step": e.get("h2d_bytes_per_step"),
                       "d2h_bytes_per_step": e.get("d2h_bytes_per_step"), "ms_per_step": sig(e.get("ms_per_step"))}
    c = full.get("cpu_baseline")
    if c:
        line["cpu_baseline"] = {"value": sig(c.get("value")), "unit": c.get("unit"), "cores": c.get("cores"),
                                "kind": c.get("kind"),
                                "sample": f"n={c.get('n')} gefa_ref_nopvt+gesl_ref_nopvt, serial, 1 of "
                                          f"{c.get('host_nproc')} cores"
                                if c.get("value") else c.get("sample")}
    ck = full.get("clocks") or {}
    line["clocks"] = {"sm_mhz": ck.get("sm_mhz"), "sm_max_mhz": ck.get("sm_max_mhz"), "reasons": ck.get("reasons")}
    line["gpu_launches"] = full.get("gpu_launches")
    line["accuracy"] = {"max_abs_err_x": sig(full.get("max_abs_err_x"), 3),
                        "hpl_resid_flt": sig((full.get("hpl_resid") or {}).get("eps_flt_half"), 3)}
    g = full.get("gesl") or {}
    line["gesl"] = {"GBps": sig(g.get("GBps")), "frac": sig(g.get("frac_hbm"), 3)}
    if full.get("gesl_noalloc"):
        line["gesl"]["noalloc_GBps"] = sig(full["gesl_noalloc"].get("GBps"))
    mx = full.get("mixed") or {}
    if mx:
        first = next(iter(mx.values()))
        line["mixed"] = {"n": first.get("n"), "block": first.get("block")}
        line["mixed"].update({p: _mixed_summary(mx.get(p)) for p in ("bf16", "fp8") if mx.get(p)})
    lg = full.get("large")
    if lg:
        f = lg.get("f32") or {}
        line["large"] = {"n": lg.get("n"), "block": (lg.get("bf16") or lg.get("fp8") or {}).get("block"),
                         "f32": sig(f.get("value")), "f32_frac": sig(f.get("frac"), 3)}
        for p in ("bf16", "fp8"):
            if lg.get(p):
                line["large"][p] = _mixed_summary(lg[p])
    ms = full.get("margins")
    if ms:
        # the margins once per n, then per n and precision one [iters, hpl, err] row per margin
        rows, mlist = {}, {}
        for r in ms:
            mlist.setdefault(str(r["n"]), [])
            if sig(r["margin"], 3) not in mlist[str(r["n"])]:
                mlist[str(r["n"])].append(sig(r["margin"], 3))
            rows.setdefault(f"{r['n']} {r['precision']}", []).append(
                [r["ir_iters"], sig(r["hpl_resid"], 3), sig(r["max_abs_err"], 2)])
        line["margins"] = {"cols": ["iters", "hpl", "err"], "margin": mlist, **rows}
    em = full.get("f32_bf16x6")
    if em:
        line["f32_bf16x6"] = {"value": sig(em.get("value")), "x_f32": sig(em.get("speedup_vs_f32_simt"), 3),
                              "frac": sig((em.get("roofline") or {}).get("frac"), 3),
                              "err": sig(em.get("max_abs_err_x"), 2)}
    for key in ("pivot", "fp64"):
        v = full.get(key)
        if v:
            line[key] = {"value": sig(v.get("value")), "frac": sig((v.get("roofline") or {}).get("frac"), 3)}
    bt = full.get("batched")
    if bt:
        line["batched"] = {"solves_per_s": sig(bt.get("solves_per_s")), "value": sig(bt.get("value")),
                           "frac": sig(bt.get("frac"), 3), "x_full_gpu_loop": sig(bt.get("speedup_vs_full_gpu_loop"), 3)}
        if bt.get("bf16"):
            b16 = bt["bf16"]
            line["batched"]["bf16"] = {"solves_per_s": sig(b16.get("solves_per_s")),
                                       "iters": b16.get("ir_iters_max"), "hpl": sig(b16.get("hpl_resid_max"), 3),
                                       "err": sig(b16.get("max_rel_err_vs_fp64_sample"), 2)}
    sv = full.get("serving")
    if sv:
        line["serving"] = {}
        for p in ("f32", "bf16", "fp8"):
            eq = (sv.get(p) or {}).get("equal_p99")
            if eq:
                line["serving"][p] = {"x_equal_p99": eq.get("ratio"), "p99_ms": sig(eq.get("p99_bound_ms"), 3)}
    if full.get("details"):
        line["details"] = full["details"]
    # the line must survive a stdout tail whole: drop the least central sections if it is long
    for key in ("serving", "pivot", "fp64", "f32_bf16x6", "accuracy", "batched", "margins"):
        if len(dumps_line(line)) <= LINE_LIMIT:
            break
        if line.pop(key, None) is not None:
            line.setdefault("trimmed", []).append(key)
    return line


def dumps_line(line: dict) -> str:
    return json.dumps(line, allow_nan=False, separators=(",", ":"))


def run_reference(args, rank: int) -> None:
    if rank != 0:
        return
    n = args.ref_n
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_bench")
    if not os.path.exists(exe):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/ref_bench not built"}))
        return
    times = []
    for i in range(args.warmup + args.steps):
        out = subprocess.run([exe, "--n", str(n), "--reps", "1", "--mode", "baseline", "--seed", "42", "--margin",
                              "1"], capture_output=True, text=True, check=True).stdout
        r = json.loads(out.strip().splitlines()[-1])
        if i >= args.warmup:
            times.append(r["t_min"])
    total = sum(times)
    value = args.steps * flops(n) / total / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"plain FP32 LU without pivoting + solve, bounded CPU sample n={n} "
                               f"(of the n={args.n} block-{args.bs} workload), seed 42, margin 1",
                   "n": n, "sample_of_n": args.n, "block": args.bs},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "reference",
                         "sample": f"{args.steps} x one n={n} system; the reference's gefa_ref_nopvt/gesl_ref_nopvt "
                                   "are single-threaded (no OpenMP in linpack_data.cpp), so one core is all they use; "
                                   f"host {host_cpu()}, {os.cpu_count()} cores"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="lpcuda", choices=["lpcuda", "reference"])
    ap.add_argument("--n", type=int, default=32768)
    ap.add_argument("--bs", type=int, default=512)
    ap.add_argument("--large-n", type=int, default=65536,
                    help="order of the second system (FP32 and the mixed forms with their margin sweep); 0: skip")
    ap.add_argument("--cpu-n", type=int, default=8192, help="order of the CPU-baseline sample (reference code)")
    ap.add_argument("--cpu-reps", type=int, default=1)
    ap.add_argument("--ref-n", type=int, default=2048, help="order of each step of the --impl reference arm")
    ap.add_argument("--ext-steps", type=int, default=3,
                    help="timed steps of the margin sweep and the large-n legs (the headline uses --steps)")
    ap.add_argument("--details", default=os.path.join(ROOT, "bench_details.json"),
                    help="where the full result tables are written")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--no-margins", action="store_true")
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--batch-count", type=int, default=4096)
    ap.add_argument("--no-serve", action="store_true")
    ap.add_argument("--no-pivot", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-f32emu", action="store_true")
    ap.add_argument("--mixed-bs", type=int, default=None,
                    help="block size of the tensor-core schedules (BF16/FP8 + IR, emulated FP32); "
                         "default: the largest power of two leaving >= 32 block steps, at most 2048")
    ap.add_argument("--serve-rates", default="100,200,300,400,500,600,700,800,900,1000,1250,1500,2000,5000,20000")
    ap.add_argument("--serve-precisions", default="f32,bf16")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return

    import torch
    import torch.distributed as dist
    from datetime import timedelta
    from hpcc_fpga_b200 import lpcuda as lp
    from hpcc_fpga_b200.replicas import job_rate

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))
    cpu = CpuBaseline(args.cpu_n, args.cpu_reps) if (world == 1 and not args.no_cpu) else None
    n, bs = args.n, args.bs
    ctx = lp.Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream)
    pk = peaks()
    ext_steps = max(1, min(args.steps, args.ext_steps))
    ext_warm = max(1, min(args.warmup, 2))

    A, b64, b32 = lp.generate_baseline(n, 42, 1.0)
    with torch.cuda.stream(stream):
        dA0 = torch.from_numpy(A).to("cuda")
        dB0 = torch.from_numpy(b32).to("cuda")
        dB64 = torch.from_numpy(b64).to("cuda")
        dA = torch.empty_like(dA0)
        dB = torch.empty_like(dB0)
    torch.cuda.synchronize()

    def step():
        with torch.cuda.stream(stream):
            dA.copy_(dA0)
            dB.copy_(dB0)
        ctx.gefa(dA.data_ptr(), n, n, bs)
        ctx.gesl(dA.data_ptr(), n, n, dB.data_ptr(), 1, n)

    for _ in range(args.warmup):
        step()
    ctx.sync()
    ctx.set_profiling(True)
    ctx.read_profile(reset=True)
    launches0 = ctx.read_profile(reset=False)["kernel_launches"]
    clocks = ClockSampler(local).start()
    time.sleep(0.3)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        step()
    ev1.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    elapsed = ev0.elapsed_time(ev1) * 1e-3
    prof = ctx.read_profile(reset=True)
    launches = prof["kernel_launches"] - launches0
    ctx.set_profiling(False)
    max_err = float((dB.double() - 1.0).abs().max())
    # HPL scaled residual of the plain FP32 solution (no refinement), in both
    # unit roundoffs, for the equal-residual comparison with the mixed forms.
    with torch.cuda.stream(stream):
        dXr = torch.empty(n, dtype=torch.float64, device="cuda")
    r32 = ctx.refine(dA0.data_ptr(), n, dA.data_ptr(), n, dB64.data_ptr(), dXr.data_ptr(), 1, 0)["hpl_resid"]
    del dXr
    value, t_max = job_rate(args.steps * flops(n) / 1e9, elapsed, device="cuda")
    f32_value = value / world

    # ---- roofline of the dominant kernel (the FP32 trailing update) ----
    inner = prof["inner"]
    achieved_tf = inner["flops"] / inner["s"] / 1e12 if inner["s"] > 0 else None
    sm_mhz = clk.get("sm_mhz") or 1965.0
    peak_tf = NUM_SMS * FP32_LANES_PER_SM * 2 * sm_mhz * 1e6 / 1e12
    stage_share = {k: prof[k]["s"] / max(1e-12, sum(prof[s]["s"] for s in lp.STAGES)) for k in lp.STAGES}
    gesl = prof["gesl"]

    full = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * t_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"FP32 LU without pivoting + solve, n={n}, block {bs}, 1 RHS, seeded diagonally "
                               "dominant (seed 42, margin 1), b = A*ones",
                   "n": n, "block": bs, "rhs": 1,
                   "l2": f"inputs larger than L2 ({4 * n * n / 2**30:.0f} GiB matrix restored every step)",
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
        "max_abs_err_x": max_err,
        "hpl_resid": {"eps_dbl_half": r32, "eps_flt_half": r32 * 2.0 ** -29,
                      "note": "plain FP32 solution, HPL scaled residual (gmres.c:182-193) with eps = 2^-53 and "
                              "with the FP32 unit roundoff 2^-24"},
        "roofline": {"bound": "fp32_simt", "kernel": "k_sgemm_update (inner stage)",
                     "achieved": achieved_tf, "peak": peak_tf, "unit": "TFLOP/s",
                     "frac": (achieved_tf / peak_tf) if achieved_tf else None,
                     "peak_source": f"derived: {NUM_SMS} SMs x {FP32_LANES_PER_SM} FP32 lanes x 2 flop x median SM "
                                    f"clock under load ({sm_mhz} MHz); MEASURED_PEAKS.json has no FP32 figure",
                     "peak_short": f"derived FP32: {NUM_SMS}x{FP32_LANES_PER_SM}x2x{sm_mhz:.0f}MHz",
                     "per_unit": "2*m*m*bs flop per trailing update of an m x m trailing matrix",
                     "launches": inner["calls"],
                     # DRAM bytes per trailing update: the n=8192 ncu capture of this kernel
                     # (profiles/k_sgemm_update_n8192_b512.md) read+wrote 388.6 MB for 440.4 MB of
                     # algorithmic bytes (a 7168^2 x 512 update); scaled by the algorithmic bytes of
                     # this run's updates.
                     "traffic": (inner["bytes"] / inner["calls"] * 388.6 / 440.4) if inner["calls"] else None,
                     "traffic_unit": "bytes per trailing update (scaled from the n=8192 capture)"},
        "stages": {k: {"s": prof[k]["s"], "share": stage_share[k], "calls": prof[k]["calls"]} for k in lp.STAGES
                   if prof[k]["calls"]},
        "gesl": {"s_per_step": gesl["s"] / max(1, args.steps),
                 "GBps": gesl["bytes"] / gesl["s"] / 1e9 if gesl["s"] > 0 else None,
                 "frac_hbm": (gesl["bytes"] / gesl["s"] / 1e9 / pk["hbm_gbs"]) if gesl["s"] > 0 else None},
        "gpu_launches": launches,
        "clocks": clk,
        "peaks": pk,
    }
    # the allocation-free substitution on the same factors
    full["gesl_noalloc"] = run_gesl_noalloc(lp, torch, stream, dA, dB0, n, ext_steps)

    mbs = args.mixed_bs or mixed_block(n, bs)
    if not args.no_mixed and mbs % 128 == 0:
        full["mixed"] = {}
        for prec in ("bf16", "fp8"):
            full["mixed"][prec] = run_mixed(ctx, lp, torch, stream, dA0, dA, dB64, n, mbs, prec, args.steps,
                                            ext_warm, f32_value, pk)
        if not args.no_margins:
            full["margins"] = run_margin_sweep(ctx, lp, torch, stream, dA0, dA, n, mbs, ("bf16", "fp8"), ext_steps,
                                               ext_warm, f32_value, pk, skip_margin_one=full["mixed"])

    if not args.no_f32emu and mbs % 128 == 0:
        full["f32_bf16x6"] = run_f32emu(ctx, lp, torch, stream, dA0, dA, dB0, dB, dB64, n, mbs, ext_steps, ext_warm,
                                        f32_value, pk)

    if not args.no_pivot:
        full["pivot"] = run_pivot(ctx, lp, torch, stream, n, ext_steps, ext_warm, peak_tf)

    if not args.no_fp64 and n % 256 == 0:
        full["fp64"] = run_fp64(ctx, lp, torch, stream, dA0, dB64, n, ext_steps, ext_warm,
                                NUM_SMS * 64 * 2 * sm_mhz * 1e6 / 1e12)

    if not args.no_batch:
        full["batched"] = run_batched(ctx, lp, torch, stream, ext_steps, ext_warm, peak_tf, args.batch_count)

    # ---- end to end through the C ABI with pinned host buffers ----
    if not args.no_e2e:
        L = lp.lib()
        pa, pb = ctypes.c_void_p(), ctypes.c_void_p()
        lp.check(L.lp_host_alloc(ctypes.c_size_t(4 * n * n), ctypes.byref(pa)), "lp_host_alloc")
        lp.check(L.lp_host_alloc(ctypes.c_size_t(4 * n), ctypes.byref(pb)), "lp_host_alloc")
        hA = np.ctypeslib.as_array((ctypes.c_float * (n * n)).from_address(pa.value)).reshape(n, n)
        hb = np.ctypeslib.as_array((ctypes.c_float * n).from_address(pb.value))
        walls = []
        for _ in range(1 + args.steps):
            np.copyto(hA, A)
            np.copyto(hb, b32)
            if world > 1:
                dist.barrier()
            t0 = time.perf_counter()
            ctx.calculate(hA, hb, bs, repetitions=1)
            walls.append(time.perf_counter() - t0)
        walls = walls[1:]
        e2e_err = float(np.abs(hb.astype(np.float64) - 1.0).max())
        e2e_value, wt = job_rate(args.steps * flops(n) / 1e9, sum(walls), device="cuda")
        full["e2e"] = {"value": e2e_value, "unit": UNIT,
                       "h2d_bytes_per_step": 4 * n * n + 4 * n, "d2h_bytes_per_step": 4 * n * n + 4 * n,
                       "ms_per_step": 1e3 * wt / args.steps, "max_abs_err_x": e2e_err,
                       "api": "lp_calculate (C ABI, pinned host A and b)"}
        del hA, hb
        L.lp_host_free(pa)
        L.lp_host_free(pb)

    # ---- the second, larger system: FP32 against the mixed forms and their margin sweep ----
    del dA0, dA, dB0, dB, dB64, A
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    nl = args.large_n
    if nl and not args.no_mixed:
        lbs = args.mixed_bs or mixed_block(nl, bs)
        Al, bl64, _ = lp.generate_baseline(nl, 42, 1.0)
        with torch.cuda.stream(stream):
            dA0 = torch.from_numpy(Al).to("cuda")
            dB64 = torch.from_numpy(bl64).to("cuda")
            dA = torch.empty_like(dA0)
            dB0 = dB64.float()
            dB = torch.empty_like(dB0)
        torch.cuda.synchronize()
        del Al
        f = run_f32(ctx, lp, torch, stream, dA0, dA, dB0, dB, nl, bs, ext_steps, 1)
        f["frac"] = f["inner_tflops"] / peak_tf if f["inner_tflops"] else None
        large = {"n": nl, "f32": f}
        for prec in ("bf16", "fp8"):
            large[prec] = run_mixed(ctx, lp, torch, stream, dA0, dA, dB64, nl, lbs, prec, ext_steps, 1, f["value"],
                                    pk, with_gmres=False)
        full["large"] = large
        if not args.no_margins:
            full["margins"] = full.get("margins", []) + run_margin_sweep(
                ctx, lp, torch, stream, dA0, dA, nl, lbs, ("bf16", "fp8"), ext_steps, 1, f["value"], pk,
                skip_margin_one=large)
        del dA0, dA, dB0, dB, dB64
        torch.cuda.synchronize()
        torch.cuda.empty_cache()

    if cpu is not None:
        full["cpu_baseline"] = cpu.result()

    if not args.no_serve and world == 1:
        full["serving"] = run_serving(lp, [float(r) for r in args.serve_rates.split(",")],
                                      args.serve_precisions.split(","))

    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return
    full["details"] = os.path.relpath(args.details, ROOT) if args.details.startswith(ROOT) else args.details
    try:
        with open(args.details, "w") as fh:
            json.dump(full, fh, indent=1, default=str)
    except OSError as exc:
        full["details"] = f"not written: {exc}"
    print(dumps_line(compact_line(full)), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
