"""ORACLE — test infrastructure only.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg import this package, and only as the checker.  The product
(``hpcc_fpga_b200``) never imports it.

Two libraries are wrapped:

* ``_ref/liborc.so`` — the plain-C restatement (``oracle.c``, ``gen.cpp``) of
  HPCC_FPGA LINPACK's CPU arithmetic for LU without pivoting.
* ``_ref/libref32.so`` / ``_ref/libref64.so`` — the reference's own
  ``LINPACK/src/host/linpack_data.cpp`` compiled unmodified (``Makefile``);
  present only where the reference sources were available at build time.

Storage convention throughout: ``S[r, c] = a[r*lda + c]`` (numpy row-major),
the factored matrix is ``M = S.T`` and ``b = M @ ones``.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(_HERE, "_ref")
_F32P = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_F64P = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_I32P = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
FLT_EPS = float(np.finfo(np.float32).eps)
DBL_EPS = float(np.finfo(np.float64).eps)

_orc = None
_ref32 = None
_ref64 = None


REFERENCE_ENV = "HPCC_FPGA_REFERENCE"


def reference_root(explicit: str | None = None) -> str | None:
    """Where the reference checkout is read from: the explicit argument, else
    $HPCC_FPGA_REFERENCE, else a checkout named ``reference`` beside this
    repository; None when none of them holds LINPACK's host sources."""
    repo = os.path.dirname(_HERE)
    for cand in (explicit, os.environ.get(REFERENCE_ENV), os.path.join(os.path.dirname(repo), "reference")):
        if cand and os.path.isdir(os.path.join(cand, "LINPACK", "src", "host")):
            return cand
    return None


def build(reference_root_dir: str | None = None) -> None:
    """Build the restatement and, when the reference sources are found
    (reference_root), the reference libraries (``make -C oracle``).  Without
    them the prebuilt files already in ``_ref/`` are used as they are."""
    subprocess.run(["make", "-s", "-C", _HERE, "orc"], check=True)
    root = reference_root(reference_root_dir)
    if root is not None:
        subprocess.run(["make", "-s", "-C", _HERE, "ref", f"REF_ROOT={root}"], check=True)


def _load(name):
    path = os.path.join(REF_DIR, name)
    if not os.path.exists(path):
        return None
    return ctypes.CDLL(path)


def orc():
    global _orc
    if _orc is None:
        lib = _load("liborc.so")
        if lib is None:
            raise RuntimeError("oracle/_ref/liborc.so is not built (run make -C oracle)")
        c_int, c_uint, c_double = ctypes.c_int, ctypes.c_uint, ctypes.c_double
        lib.orc_gefa_nopvt_f32.argtypes = [_F32P, c_int, c_int]
        lib.orc_gefa_nopvt_f64.argtypes = [_F64P, c_int, c_int]
        lib.orc_gesl_nopvt_f32.argtypes = [_F32P, _F32P, c_int, c_int]
        lib.orc_gesl_nopvt_f64.argtypes = [_F64P, _F64P, c_int, c_int]
        lib.orc_gefa_pvt_f32.argtypes = [_F32P, c_int, c_int, _I32P]
        lib.orc_gefa_pvt_f64.argtypes = [_F64P, c_int, c_int, _I32P]
        lib.orc_gesl_pvt_f32.argtypes = [_F32P, _F32P, _I32P, c_int, c_int]
        lib.orc_gesl_pvt_f64.argtypes = [_F64P, _F64P, _I32P, c_int, c_int]
        lib.orc_top_update_f32.argtypes = [_F32P, c_int, _F32P, c_int, c_int, c_int]
        lib.orc_left_update_f32.argtypes = [_F32P, c_int, _F32P, c_int, c_int, c_int]
        lib.orc_inner_update_f32.argtypes = [_F32P, c_int, _F32P, c_int, _F32P, c_int, c_int, c_int, c_int]
        lib.orc_blocked_gefa_f32.argtypes = [_F32P, c_int, c_int, c_int]
        lib.orc_residn_f32.argtypes = [_F32P, c_int, c_double, ctypes.POINTER(c_double)]
        lib.orc_residn_f32.restype = c_double
        lib.orc_hpl_resid_f32a.argtypes = [_F32P, c_int, c_int, _F64P, _F64P, c_double]
        lib.orc_hpl_resid_f32a.restype = c_double
        lib.orc_residual_f64.argtypes = [_F32P, c_int, c_int, _F64P, _F64P, _F64P]
        lib.orc_gen_reference_f32.argtypes = [_F32P, _F32P, c_int, c_int,
                                              ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float)]
        lib.orc_gen_baseline.argtypes = [_F32P, _F64P, _F32P, c_int, c_uint, c_double]
        _orc = lib
    return _orc


def ref(precision: str = "f32"):
    """The reference's own compiled routines, or None when not built."""
    global _ref32, _ref64
    if precision == "f32":
        if _ref32 is None:
            lib = _load("libref32.so")
            if lib is not None:
                lib.ref_gefa_nopvt_f32.argtypes = [_F32P, ctypes.c_uint, ctypes.c_uint]
                lib.ref_gesl_nopvt_f32.argtypes = [_F32P, _F32P, ctypes.c_uint, ctypes.c_uint]
                lib.ref_gefa_pvt_f32.argtypes = [_F32P, ctypes.c_uint, ctypes.c_uint, _I32P]
                lib.ref_gesl_pvt_f32.argtypes = [_F32P, _F32P, _I32P, ctypes.c_uint, ctypes.c_uint]
                lib.gmres_ref.argtypes = [ctypes.c_int, _F64P, ctypes.c_int, _F64P, _F64P, _F64P,
                                          ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double]
            _ref32 = lib
        return _ref32
    if _ref64 is None:
        lib = _load("libref64.so")
        if lib is not None:
            lib.ref_gefa_nopvt_f64.argtypes = [_F64P, ctypes.c_uint, ctypes.c_uint]
            lib.ref_gesl_nopvt_f64.argtypes = [_F64P, _F64P, ctypes.c_uint, ctypes.c_uint]
            lib.ref_gefa_pvt_f64.argtypes = [_F64P, ctypes.c_uint, ctypes.c_uint, _I32P]
            lib.ref_gesl_pvt_f64.argtypes = [_F64P, _F64P, _I32P, ctypes.c_uint, ctypes.c_uint]
        _ref64 = lib
    return _ref64


# ---------------------------------------------------------------- generators
def gen_reference(n: int, diag_dominant: bool = True):
    """Reference-mode input (linpack_benchmark.hpp:211-297, one rank).
    Returns (A float32 n x n, b float32 n, norma, normb)."""
    A = np.empty((n, n), np.float32)
    b = np.empty(n, np.float32)
    na, nb = ctypes.c_float(), ctypes.c_float()
    orc().orc_gen_reference_f32(A, b, n, int(diag_dominant), ctypes.byref(na), ctypes.byref(nb))
    return A, b, float(na.value), float(nb.value)


def gen_baseline(n: int, seed: int = 42, margin: float = 1.0):
    """Baseline-mode input.  Returns (A float32, b64 float64, b32 float32)."""
    A = np.empty((n, n), np.float32)
    b64 = np.empty(n, np.float64)
    b32 = np.empty(n, np.float32)
    orc().orc_gen_baseline(A, b64, b32, n, seed, float(margin))
    return A, b64, b32


# ---------------------------------------------------------------- algorithms
def gefa_nopvt(A: np.ndarray) -> np.ndarray:
    """Unblocked LU without pivoting in the reference encoding (copy)."""
    a = np.ascontiguousarray(A).copy()
    n = a.shape[0]
    if a.dtype == np.float32:
        orc().orc_gefa_nopvt_f32(a, n, a.shape[1])
    else:
        a = a.astype(np.float64)
        orc().orc_gefa_nopvt_f64(a, n, a.shape[1])
    return a


def gesl_nopvt(LU: np.ndarray, b: np.ndarray) -> np.ndarray:
    lu = np.ascontiguousarray(LU)
    n = lu.shape[0]
    if lu.dtype == np.float32:
        x = np.ascontiguousarray(b, dtype=np.float32).copy()
        orc().orc_gesl_nopvt_f32(lu, x, n, lu.shape[1])
    else:
        x = np.ascontiguousarray(b, dtype=np.float64).copy()
        orc().orc_gesl_nopvt_f64(lu, x, n, lu.shape[1])
    return x


def gefa_pvt(A: np.ndarray):
    """Unblocked LU with partial pivoting (LINPACK convention, reference
    encoding): returns (factors, ipvt) as copies."""
    a = np.ascontiguousarray(A).copy()
    n = a.shape[0]
    ipvt = np.zeros(max(n, 1), dtype=np.int32)
    if a.dtype == np.float32:
        orc().orc_gefa_pvt_f32(a, n, a.shape[1], ipvt)
    else:
        a = a.astype(np.float64)
        orc().orc_gefa_pvt_f64(a, n, a.shape[1], ipvt)
    return a, ipvt[:n]


def gesl_pvt(LU: np.ndarray, ipvt: np.ndarray, b: np.ndarray) -> np.ndarray:
    lu = np.ascontiguousarray(LU)
    n = lu.shape[0]
    piv = np.ascontiguousarray(ipvt, dtype=np.int32)
    if lu.dtype == np.float32:
        x = np.ascontiguousarray(b, dtype=np.float32).copy()
        orc().orc_gesl_pvt_f32(lu, x, piv, n, lu.shape[1])
    else:
        x = np.ascontiguousarray(b, dtype=np.float64).copy()
        orc().orc_gesl_pvt_f64(lu, x, piv, n, lu.shape[1])
    return x


def top_update(lu: np.ndarray, t: np.ndarray) -> np.ndarray:
    out = np.ascontiguousarray(t, dtype=np.float32).copy()
    lu = np.ascontiguousarray(lu, dtype=np.float32)
    orc().orc_top_update_f32(lu, lu.shape[1], out, out.shape[1], lu.shape[0], out.shape[1])
    return out


def left_update(lu: np.ndarray, l: np.ndarray) -> np.ndarray:
    out = np.ascontiguousarray(l, dtype=np.float32).copy()
    lu = np.ascontiguousarray(lu, dtype=np.float32)
    orc().orc_left_update_f32(lu, lu.shape[1], out, out.shape[1], lu.shape[0], out.shape[0])
    return out


def inner_update(c: np.ndarray, l: np.ndarray, t: np.ndarray) -> np.ndarray:
    out = np.ascontiguousarray(c, dtype=np.float32).copy()
    l = np.ascontiguousarray(l, dtype=np.float32)
    t = np.ascontiguousarray(t, dtype=np.float32)
    m, n = out.shape
    orc().orc_inner_update_f32(out, n, l, l.shape[1], t, t.shape[1], m, n, l.shape[1])
    return out


def blocked_gefa(A: np.ndarray, bs: int) -> np.ndarray:
    a = np.ascontiguousarray(A, dtype=np.float32).copy()
    orc().orc_blocked_gefa_f32(a, a.shape[0], a.shape[1], bs)
    return a


def residn(x: np.ndarray, normb: float):
    """Reference residual (linpack_benchmark.hpp:395-417): (residn, resid)."""
    r = ctypes.c_double()
    xv = np.ascontiguousarray(x, dtype=np.float32)
    val = orc().orc_residn_f32(xv, xv.size, float(normb), ctypes.byref(r))
    return float(val), float(r.value)


def hpl_resid(A: np.ndarray, x: np.ndarray, b: np.ndarray, eps: float = DBL_EPS / 2) -> float:
    """HPL-AI scaled residual (gmres.c:182-193) with M = S.T."""
    a = np.ascontiguousarray(A, dtype=np.float32)
    return float(orc().orc_hpl_resid_f32a(a, a.shape[1], a.shape[0],
                                          np.ascontiguousarray(x, dtype=np.float64),
                                          np.ascontiguousarray(b, dtype=np.float64), float(eps)))


def residual_f64(A: np.ndarray, x: np.ndarray, b: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(A, dtype=np.float32)
    r = np.empty(a.shape[0], np.float64)
    orc().orc_residual_f64(a, a.shape[1], a.shape[0], np.ascontiguousarray(x, dtype=np.float64),
                           np.ascontiguousarray(b, dtype=np.float64), r)
    return r


def ref_bench_path() -> str:
    return os.path.join(REF_DIR, "ref_bench")
