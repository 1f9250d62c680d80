"""bench.py's stdout summary: built from a canned full result with every
section present (including NaN and infinity where a leg measured nothing),
it must be strict JSON, one line, small enough to survive a few-KB stdout
tail whole, and carry the contract's keys."""
import json
import math

import bench

REQUIRED = ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
            "vs_baseline", "dtype", "data", "config", "roofline", "e2e", "cpu_baseline", "clocks", "gpu_launches")


def _mixed(prec, n, bs, v):
    return {"n": n, "block": bs, "precision": prec, "value": v, "speedup_vs_f32": v / 49385.123,
            "ir_iters": 1, "hpl_resid": 11.7612345, "max_abs_err_vs_fp64_oracle": 2.6123e-10,
            "roofline": {"bound": "tensor", "frac": 0.5912345, "achieved": 975.123, "peak": 1649.8}}


def canned_full() -> dict:
    margins = []
    for n in (32768, 65536):
        for prec in ("bf16", "fp8"):
            for m in bench.margins_for(n):
                margins.append({"n": n, "precision": prec, "block": 1024, "margin": m, "value": 333216.12345,
                                "ir_iters": 2, "hpl_resid": 0.41234567, "max_abs_err": 4.5123e-12})
    ladder = [{"rate": r, "p99_ms": 40.0, "solves_per_s": r * 0.99, "offered_per_s": r} for r in range(100, 2100, 100)]
    return {
        "metric": bench.METRIC, "value": 49385.123456789, "unit": "GFLOP/s", "n_gpus": 1, "steps": 20, "warmup": 5,
        "ms_per_step": 475.123456789, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": "FP32 LU without pivoting + solve, n=32768, block 512, 1 RHS, seeded diagonally "
                               "dominant (seed 42, margin 1), b = A*ones",
                   "n": 32768, "block": 512, "rhs": 1, "l2": "inputs larger than L2 (4 GiB matrix restored every step)",
                   "parallelism": "single GPU"},
        "max_abs_err_x": 1.0728836059570312e-06, "hpl_resid": {"eps_flt_half": 0.0123456, "eps_dbl_half": 6.6e6},
        "roofline": {"bound": "fp32_simt", "achieved": 49.2123, "peak": 74.4512, "unit": "TFLOP/s", "frac": 0.6612345,
                     "traffic": 2.8123456e9, "peak_short": "derived FP32: 148x128x2x1965MHz",
                     "peak_source": "derived " * 20},
        "stages": {"inner": {"s": 1.0}}, "gesl": {"GBps": 1792.123, "frac_hbm": 0.274123},
        "gesl_noalloc": {"GBps": 1101.5},
        "gpu_launches": 123456, "clocks": {"sm_mhz": 1965.0, "sm_max_mhz": 1965, "reasons": ["sw_power_cap"],
                                           "samples": 120, "power_w_max": 990.1},
        "mixed": {"bf16": _mixed("bf16", 32768, 1024, 333216.1), "fp8": _mixed("fp8", 32768, 1024, 338303.1)},
        "large": {"n": 65536, "f32": {"value": 51391.1234, "frac": 0.6912345},
                  "bf16": _mixed("bf16", 65536, 2048, 638010.1), "fp8": _mixed("fp8", 65536, 2048, 792812.1)},
        "margins": margins,
        "f32_bf16x6": {"value": 143626.1, "speedup_vs_f32_simt": 2.91234, "max_abs_err_x": 1.07e-6,
                       "roofline": {"frac": 0.771234}},
        "pivot": {"value": 27859.1, "roofline": {"frac": float("nan")}},
        "fp64": {"value": 19195.1, "roofline": {"frac": 0.551234}},
        "batched": {"solves_per_s": 237925.1, "value": 16641.1, "speedup_vs_per_system_loop_wall": 192.1,
                    "hpl_resid_flt_eps_max_sample": 3.21, "frac": 0.22345, "speedup_vs_full_gpu_loop": 12.345,
                    "bf16": {"solves_per_s": 200000.1, "value": 14000.1, "ir_iters_max": 2, "hpl_resid_max": 9.1}},
        "serving": {p: {"per_request": ladder, "continuous": ladder,
                        "equal_p99": {"ratio": 2.69, "p99_bound_ms": 77.078123, "continuous_solves_per_s": 788.4,
                                      "baseline_solves_per_s": 293.3}} for p in ("f32", "bf16")},
        "e2e": {"value": 47866.552387657386, "unit": "GFLOP/s", "h2d_bytes_per_step": 4295098368,
                "d2h_bytes_per_step": 4295098368, "ms_per_step": 490.0790713500015},
        "cpu_baseline": {"value": 1.95123, "unit": "GFLOP/s", "cores": 1, "kind": "reference", "n": 8192,
                         "host_nproc": 224, "host_cpu": "Intel(R) Xeon(R) Platinum 8570 with a long model name"},
        "details": "bench_details.json",
    }


def test_compact_line_is_strict_small_and_complete():
    full = canned_full()
    line = bench.compact_line(full)
    text = bench.dumps_line(line)
    assert "\n" not in text
    assert len(text.encode()) <= bench.LINE_LIMIT, len(text)
    back = json.loads(text)
    for k in REQUIRED:
        assert k in back, k
    assert back["value"] > 0 and back["e2e"]["value"] > 0
    assert back["e2e"]["h2d_bytes_per_step"] > 0 and back["e2e"]["d2h_bytes_per_step"] > 0
    for k in ("bound", "achieved", "peak", "unit", "frac", "traffic"):
        assert k in back["roofline"], k
    for k in ("value", "unit", "cores", "kind", "sample"):
        assert k in back["cpu_baseline"], k
    # every margin case carries its iteration count, HPL residual and oracle error
    rows = {k: v for k, v in back["margins"].items() if k not in ("cols", "margin")}
    assert sum(len(v) for v in rows.values()) == 12
    assert all(len(r) == len(back["margins"]["cols"]) for v in rows.values() for r in v)
    assert all(len(back["margins"]["margin"][k.split()[0]]) == len(v) for k, v in rows.items())
    assert back["pivot"]["frac"] is None  # NaN became null, not an invalid token
    assert back["serving"]["bf16"]["x_equal_p99"] == 2.69
    assert "trimmed" not in back  # nothing had to be dropped to fit


def test_compact_line_with_legs_skipped():
    full = canned_full()
    for k in ("mixed", "large", "margins", "f32_bf16x6", "pivot", "fp64", "batched", "serving", "gesl_noalloc"):
        full.pop(k)
    full["cpu_baseline"] = {"value": None, "unit": "GFLOP/s", "cores": 1, "kind": "reference",
                            "sample": "unavailable: oracle/_ref/ref_bench not built"}
    text = bench.dumps_line(bench.compact_line(full))
    back = json.loads(text)
    assert back["cpu_baseline"]["value"] is None
    assert len(text.encode()) <= bench.LINE_LIMIT


def test_sig_rounding():
    assert bench.sig(49385.123456, 4) == 49390.0
    assert bench.sig(float("inf")) is None
    assert bench.sig(math.nan) is None
    assert bench.sig(3) == 3
    assert bench.sig(None) is None


def test_compact_line_trims_least_central_sections_when_long():
    full = canned_full()
    full["config"] = dict(full["config"], workload=full["config"]["workload"] + " " + "x" * 500)
    line = bench.compact_line(full)
    text = bench.dumps_line(line)
    back = json.loads(text)
    assert len(text.encode()) <= bench.LINE_LIMIT, len(text)
    assert back["trimmed"][0] == "serving" and "serving" not in back
    for k in REQUIRED:
        assert k in back, k
