"""The C++ harness (lp_bench): the reference's HpccFpgaBenchmark /
LinpackBenchmark host API over liblpcuda.so.

CPU: flow tests with mock benchmarks (after
shared/tests/hpcc_base_benchmark_test.cpp), CLI behaviour in --test mode.
GPU: end-to-end runs — exit code, "Validation: SUCCESS!", the console tables
that the reference's evaluation regex reads
(scripts/evaluation/parse_raw_to_csv.py:61-70), and the JSON keys checked by
LINPACK/tests/test_kernel_functionality_and_host_integration.cpp:200-226."""
import json
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "hpcc_fpga_b200", "_lib")
EXE = os.path.join(LIB, "lp_bench")


def run(args, **kw):
    return subprocess.run([EXE] + args, capture_output=True, text=True, timeout=600, **kw)


def test_harness_flow_with_mocks(tmp_path, lp):
    exe = tmp_path / "harness_flow_test"
    subprocess.run(["g++", "-O1", "-std=c++17", "-I", os.path.join(ROOT, "include"),
                    "-I", os.path.join(ROOT, "hpcc_fpga_b200", "csrc", "host"),
                    os.path.join(ROOT, "tests", "cpp", "harness_flow_test.cpp"), "-o", str(exe),
                    "-L", LIB, "-llpcuda", f"-Wl,-rpath,{LIB}"], check=True)
    r = subprocess.run([str(exe), str(tmp_path)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "ALL PASSED" in r.stdout


def test_help_lists_reference_options(lp):
    r = run(["-h"])
    assert r.returncode == 0
    for opt in ["-f, --file", "-n", "--skip-validation", "--device", "--platform", "--platform_str", "-r",
                "--comm-type", "--dump-json", "--test", "-h, --help", "-m", "-b", "-p", "--uniform", "--emulation",
                "--precision"]:
        assert opt in r.stdout, opt


def test_test_mode_prints_configuration(lp):
    r = run(["-f", "hpl_CUDA", "-m", "64", "-b", "9", "--test"])
    assert r.returncode == 0
    assert re.search(r"Matrix Size\s+32768", r.stdout)
    assert re.search(r"Block Size\s+512", r.stdout)
    assert "SUCCESSFULLY parsed input parameters!" in r.stdout


def test_missing_kernel_file_fails(lp):
    r = run(["-m", "2"])
    assert r.returncode == 1
    assert "Kernel file must be given with option -f!" in r.stderr


def test_bad_option_values_fail(lp):
    assert run(["-f", "k", "--test", "-m", "x"]).returncode == 1
    assert run(["-f", "k", "--test", "--precision", "fp4"]).returncode == 1
    assert run(["-f", "k", "--test", "-p", "2"]).returncode == 1   # one rank: P must divide 1


RESULT_RE = re.compile(
    r"\s+norm\. residual\s+res\. error\s+mach\. eps\n"
    r"\s+(?P<error>\S+)\s+(?P<resid>\S+)\s+(?P<eps>\S+)\n"
    r"(.*\n)+\sMethod\s+best\s+mean\s+GFLOPS\s*\n"
    r"\stotal\s+(?P<t_best>\S+)\s+s\s+(?P<t_mean>\S+)\s+s\s+(?P<gflops>\S+)\s+GFLOP/s\s*\n"
    r"\sGEFA\s+(?P<lu_best>\S+)\s+s\s+(?P<lu_mean>\S+)\s+s\s+(?P<lu_gflops>\S+)\s+GFLOP/s\s*\n"
    r"\sGESL\s+(?P<sl_best>\S+)\s+s\s+(?P<sl_mean>\S+)\s+s\s+(?P<sl_gflops>\S+)\s+GFLOP/s\s*\n")


@pytest.mark.gpu
@pytest.mark.parametrize("m,b", [(1, 7), (2, 7), (3, 7), (4, 9)])
def test_lp_bench_end_to_end(tmp_path, lp, m, b):
    out = tmp_path / "linpack.json"
    r = run(["-f", "hpl_torus_CUDA", "-m", str(m), "-b", str(b), "-n", "2", "--dump-json", str(out)])
    assert r.returncode == 0, r.stdout + r.stderr
    assert "Validation: SUCCESS!" in r.stdout
    mo = RESULT_RE.search(r.stdout)
    assert mo, r.stdout
    assert float(mo["error"]) < 1.0 and float(mo["gflops"]) > 0
    j = json.loads(out.read_text())
    assert set(j["timings"]) >= {"gefa", "gesl"} and len(j["timings"]["gefa"]) == 2
    assert set(j["results"]) >= {"gflops", "gflops_lu", "gflops_sl", "t_mean", "t_min", "tlu_mean", "tlu_min",
                                 "tsl_mean", "tsl_min"}
    assert set(j["errors"]) >= {"epsilon", "residual", "residual_norm"}
    assert j["validated"] is True and j["name"] == "LINPACK"
    assert j["settings"]["Matrix Size"] == m * (1 << b) and j["settings"]["Block Size"] == 1 << b
    assert j["settings"]["FPGA Torus"] == {"P": 1, "Q": 1}
    assert "B200" in j["device"]


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["bf16", "fp8"])
def test_lp_bench_mixed_precision(tmp_path, lp, prec):
    out = tmp_path / "mixed.json"
    r = run(["-f", "hpl_CUDA", "-m", "8", "-b", "8", "-n", "1", "--precision", prec, "--generator", "baseline",
             "--dump-json", str(out)])
    assert r.returncode == 0, r.stdout + r.stderr
    j = json.loads(out.read_text())
    assert j["errors"]["hpl_resid_norm"] <= 16.0
    assert j["results"]["ir_iterations"]["value"] >= 1


@pytest.mark.gpu
def test_lp_bench_fp32_emulated(tmp_path, lp):
    """FP32 emulated on the tensor cores validates like FP32, with no refinement."""
    out = tmp_path / "emu.json"
    r = run(["-f", "hpl_CUDA", "-m", "8", "-b", "9", "-n", "1", "--precision", "f32_bf16x6", "--max-refinements", "0",
             "--dump-json", str(out)])
    assert r.returncode == 0, r.stdout + r.stderr
    assert "Validation: SUCCESS!" in r.stdout
    j = json.loads(out.read_text())
    assert j["errors"]["residual_norm"] < 1.0


@pytest.mark.gpu
@pytest.mark.parametrize("generator", ["reference", "baseline"])
def test_lp_bench_double_build(tmp_path, lp, generator):
    """--precision f64: the reference's DATA_TYPE double variant end to end,
    validated with the double machine epsilon."""
    out = tmp_path / "dp.json"
    r = run(["-f", "hpl_CUDA", "-m", "8", "-b", "7", "-n", "2", "--precision", "f64", "--generator", generator,
             "--dump-json", str(out)])
    assert r.returncode == 0, r.stdout + r.stderr
    assert "Validation: SUCCESS!" in r.stdout
    j = json.loads(out.read_text())
    # the settings table names the data type (the JSON writes non-integer settings as booleans,
    # as the reference's jsonifySettingsMap does)
    assert any("Data Type" in line and "double" in line for line in r.stdout.splitlines())
    assert j["errors"]["residual_norm"] < 1.0
    assert abs(j["errors"]["epsilon"] - 2.220446049250313e-16) < 1e-20


@pytest.mark.gpu
def test_lp_bench_unsupported_comm_type(lp):
    r = run(["-f", "hpl_torus_PCIE.aocx", "-m", "2", "-b", "5", "--comm-type", "PCIE"])
    assert r.returncode == 1
    assert "No calculate method implemented for communication type PCIE" in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("m,b", [(2, 5), (8, 7)])
def test_lp_bench_uniform_matrix_pivoting(tmp_path, lp, m, b):
    """--uniform: no diagonal dominance, solved with partial pivoting
    (gefa_ref / gesl_ref convention) and validated as the reference does."""
    out = tmp_path / "uniform.json"
    r = run(["-f", "hpl_CUDA", "-m", str(m), "-b", str(b), "-n", "2", "--uniform", "--dump-json", str(out)])
    assert r.returncode == 0, r.stdout + r.stderr
    assert "Validation: SUCCESS!" in r.stdout
    j = json.loads(out.read_text())
    assert j["settings"]["Diagonally Dominant"] in (False, "No")
    assert j["errors"]["residual_norm"] < 1.0


@pytest.mark.gpu
def test_lp_bench_uniform_mixed_rejected(lp):
    r = run(["-f", "hpl_CUDA", "-m", "2", "-b", "5", "--uniform", "--precision", "bf16"])
    assert r.returncode == 1
    assert "pivoting" in r.stderr
