"""Build liblpcuda.so (and the lp_bench harness) in-tree for sm_100a.

    python -m hpcc_fpga_b200.build [--force] [-j N]

Outputs go to hpcc_fpga_b200/_lib/ (git-ignored; they travel with the tree).
Every .cu under csrc/ is compiled by nvcc with
``-gencode arch=compute_100a,code=sm_100a -O3 -lineinfo``; host-only .cpp
files by g++.  Rebuilds only what changed (by modification time, including
the headers under csrc/ and include/).
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
HOST = os.path.join(CSRC, "host")
LIB = os.path.join(PKG, "_lib")
OBJ = os.path.join(LIB, "obj")
INCLUDE = os.path.join(ROOT, "include")
SONAME = "liblpcuda.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _headers() -> list[str]:
    return (glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h"))
            + glob.glob(os.path.join(INCLUDE, "*.h")))


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {os.path.basename(cmd[-1])}")


def compile_cu(src: str, force: bool, extra: list[str] | None = None) -> str:
    obj = os.path.join(OBJ, os.path.basename(src) + ".o")
    if force or _stale(obj, [src] + _headers()):
        cmd = [nvcc_path(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
               "--expt-relaxed-constexpr", "-I", INCLUDE, "-c", src, "-o", obj]
        if extra:
            cmd[1:1] = extra
        _run(cmd)
    return obj


def compile_cpp(src: str, force: bool) -> str:
    obj = os.path.join(OBJ, os.path.basename(src) + ".o")
    if force or _stale(obj, [src] + _headers()):
        _run(["g++", "-O2", "-std=c++17", "-fPIC", "-I", INCLUDE, "-c", src, "-o", obj])
    return obj


def build(force: bool = False, jobs: int = 8, verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    cus = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    cpps = sorted(glob.glob(os.path.join(CSRC, "*.cpp")))
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        futs = [ex.submit(compile_cu, s, force) for s in cus] + [ex.submit(compile_cpp, s, force) for s in cpps]
        objs = [f.result() for f in futs]
    so = os.path.join(LIB, SONAME)
    if force or _stale(so, objs):
        _run([nvcc_path(), *ARCH, "-shared", "-o", so, *objs])
        if verbose:
            print("linked", so)
    harness = build_harness(force)
    if verbose and harness:
        print("harness", harness)
    return so


def build_harness(force: bool = False) -> str | None:
    """The C++ HpccFpgaBenchmark-style driver (lp_bench), linked against
    liblpcuda.so with an $ORIGIN rpath."""
    mains = glob.glob(os.path.join(HOST, "*.cpp"))
    if not mains:
        return None
    exe = os.path.join(LIB, "lp_bench")
    hdrs = glob.glob(os.path.join(HOST, "*.hpp")) + _headers()
    so = os.path.join(LIB, SONAME)
    if force or _stale(exe, mains + hdrs + [so]):
        _run(["g++", "-O2", "-std=c++17", "-I", INCLUDE, "-I", HOST, *sorted(mains), "-o", exe,
              "-L", LIB, "-llpcuda", "-Wl,-rpath,$ORIGIN", "-lpthread"])
    return exe


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=8)
    a = ap.parse_args()
    print(build(force=a.force, jobs=a.j, verbose=True))


if __name__ == "__main__":
    main()
