"""ctypes binding of liblpcuda.so (the C ABI declared in include/lpcuda.h).

This module only marshals arguments; all work is done by the CUDA library.
It raises if the library is missing — there is no fallback path.
"""
from __future__ import annotations

import ctypes
import os
import re

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "_lib", "liblpcuda.so")
HEADER_PATH = os.path.join(os.path.dirname(_PKG), "include", "lpcuda.h")

LP_OK = 0
LP_E_INVALID = -1
LP_E_CUDA = -2
LP_E_NOMEM = -3
LP_E_TIMEOUT = -4
LP_E_NUMERIC = -5
LP_E_STATE = -6
LP_E_BUDGET = -7
LP_E_NODEVICE = -8

LP_F32, LP_BF16_IR, LP_FP8_IR, LP_F32_BF16X6 = 0, 1, 2, 3
LP_STALL_NONE, LP_STALL_GESL = 0, 1
PRECISIONS = {"f32": LP_F32, "bf16": LP_BF16_IR, "fp8": LP_FP8_IR, "f32_bf16x6": LP_F32_BF16X6}

_F32P = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_F64P = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_I32P = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_VP = ctypes.c_void_p
_I = ctypes.c_int


class LpTiming(ctypes.Structure):
    _fields_ = [("gefa_s", ctypes.c_double), ("gesl_s", ctypes.c_double), ("ir_s", ctypes.c_double),
                ("h2d_s", ctypes.c_double), ("d2h_s", ctypes.c_double), ("ir_iters", ctypes.c_int),
                ("reserved", ctypes.c_int), ("hpl_resid", ctypes.c_double)]

    def as_dict(self) -> dict:
        return {f[0]: getattr(self, f[0]) for f in self._fields_ if f[0] != "reserved"}


STAGES = ["lu", "top", "left", "inner", "gesl", "other"]


class LpProfile(ctypes.Structure):
    _fields_ = [("stage_s", ctypes.c_double * 6), ("stage_flops", ctypes.c_double * 6),
                ("stage_bytes", ctypes.c_double * 6), ("stage_calls", ctypes.c_longlong * 6),
                ("kernel_launches", ctypes.c_longlong)]

    def as_dict(self) -> dict:
        d = {s: {"s": self.stage_s[i], "flops": self.stage_flops[i], "bytes": self.stage_bytes[i],
                 "calls": self.stage_calls[i]} for i, s in enumerate(STAGES)}
        d["kernel_launches"] = self.kernel_launches
        return d


class LpStageEvent(ctypes.Structure):
    _fields_ = [("stage", ctypes.c_int), ("stream", ctypes.c_int), ("t0_s", ctypes.c_double),
                ("t1_s", ctypes.c_double)]


class LpSystem(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int), ("nrhs", ctypes.c_int), ("lda", ctypes.c_int), ("ldb", ctypes.c_int),
                ("a_off", ctypes.c_longlong), ("b_off", ctypes.c_longlong)]


class LpBatchConfig(ctypes.Structure):
    _fields_ = [("small_n_max", ctypes.c_int), ("nb", ctypes.c_int * 5), ("ctas_per_sm", ctypes.c_int),
                ("use_graph", ctypes.c_int)]

    def as_dict(self) -> dict:
        return {"small_n_max": self.small_n_max, "nb": list(self.nb), "ctas_per_sm": self.ctas_per_sm,
                "use_graph": self.use_graph}


class LpBatchStats(ctypes.Structure):
    _fields_ = [("seconds", ctypes.c_double), ("flops", ctypes.c_double), ("gflops", ctypes.c_double),
                ("solves_per_s", ctypes.c_double), ("systems", ctypes.c_int), ("graph_replayed", ctypes.c_int)]

    def as_dict(self) -> dict:
        return {f[0]: getattr(self, f[0]) for f in self._fields_}


LP_SERVE_CONTINUOUS, LP_SERVE_PER_REQUEST = 0, 1


class LpServerConfig(ctypes.Structure):
    _fields_ = [("hbm_budget_bytes", ctypes.c_longlong), ("mode", ctypes.c_int), ("precision", ctypes.c_int),
                ("slots", ctypes.c_int), ("batch_workers", ctypes.c_int), ("batch_max_n", ctypes.c_int),
                ("batch_max_count", ctypes.c_int), ("max_refinements", ctypes.c_int), ("warm_n", ctypes.c_int),
                ("reserve_bytes", ctypes.c_longlong), ("large_n", ctypes.c_int), ("large_slots", ctypes.c_int)]

    def as_dict(self) -> dict:
        return {f[0]: getattr(self, f[0]) for f in self._fields_}


class LpRequest(ctypes.Structure):
    _fields_ = [("key", ctypes.c_longlong), ("n", ctypes.c_int), ("nrhs", ctypes.c_int), ("A", _VP),
                ("lda", ctypes.c_int), ("B", _VP), ("ldb", ctypes.c_int), ("X", _VP), ("ldx", ctypes.c_int)]


class LpResult(ctypes.Structure):
    _fields_ = [("id", ctypes.c_longlong), ("key", ctypes.c_longlong), ("status", ctypes.c_int),
                ("n", ctypes.c_int), ("nrhs", ctypes.c_int), ("reused", ctypes.c_int), ("batched", ctypes.c_int),
                ("ir_iters", ctypes.c_int), ("hpl_resid", ctypes.c_double), ("t_submit", ctypes.c_double),
                ("t_start", ctypes.c_double), ("t_done", ctypes.c_double)]

    def as_dict(self) -> dict:
        return {f[0]: getattr(self, f[0]) for f in self._fields_}


class LpServerInfo(ctypes.Structure):
    _fields_ = [("pending", ctypes.c_int), ("running", ctypes.c_int), ("resident", ctypes.c_int),
                ("used_bytes", ctypes.c_longlong), ("completed", ctypes.c_longlong), ("waves", ctypes.c_longlong),
                ("waved_systems", ctypes.c_longlong), ("evictions", ctypes.c_longlong),
                ("rejected", ctypes.c_longlong), ("pool_reserved_bytes", ctypes.c_longlong),
                ("slot_busy_s", ctypes.c_double), ("wave_busy_s", ctypes.c_double)]

    def as_dict(self) -> dict:
        return {f[0]: getattr(self, f[0]) for f in self._fields_}


class LpError(RuntimeError):
    def __init__(self, status: int, where: str, detail: str):
        self.status = status
        super().__init__(f"{where}: {strerror(status)} ({status}): {detail}")


_lib = None


def lib() -> ctypes.CDLL:
    """Load liblpcuda.so (built by hpcc_fpga_b200.build); raise if absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m hpcc_fpga_b200.build`")
    L = ctypes.CDLL(LIB_PATH)
    L.lp_strerror.restype = ctypes.c_char_p
    L.lp_strerror.argtypes = [_I]
    L.lp_last_error.restype = ctypes.c_char_p
    L.lp_last_error.argtypes = []
    L.lp_version.restype = _I
    L.lp_device_count.argtypes = [ctypes.POINTER(_I)]
    L.lp_ctx_create.argtypes = [_I, ctypes.POINTER(_VP)]
    L.lp_ctx_destroy.argtypes = [_VP]
    L.lp_ctx_stream.argtypes = [_VP, ctypes.POINTER(_VP)]
    L.lp_ctx_sync.argtypes = [_VP]
    L.lp_ctx_device_name.argtypes = [_VP, ctypes.c_char_p, _I]
    L.lp_ctx_set_profiling.argtypes = [_VP, _I]
    L.lp_ctx_read_profile.argtypes = [_VP, ctypes.POINTER(LpProfile), _I]
    L.lp_ctx_read_timeline.argtypes = [_VP, ctypes.POINTER(LpStageEvent), _I, ctypes.POINTER(_I)]
    L.lp_ctx_test_stall.argtypes = [_VP, _I]
    L.lp_host_alloc.argtypes = [ctypes.c_size_t, ctypes.POINTER(_VP)]
    L.lp_host_free.argtypes = [_VP]
    L.lp_lu_block_dev.argtypes = [_VP, _VP, _I, _I]
    L.lp_top_update_dev.argtypes = [_VP, _VP, _I, _VP, _I, _I, _I]
    L.lp_left_update_dev.argtypes = [_VP, _VP, _I, _VP, _I, _I, _I, _VP, _I]
    L.lp_inner_update_dev.argtypes = [_VP, _VP, _I, _VP, _I, _VP, _I, _I, _I, _I]
    L.lp_gefa_dev.argtypes = [_VP, _VP, _I, _I, _I]
    L.lp_gefa_prec_dev.argtypes = [_VP, _I, _VP, _I, _I, _I]
    L.lp_inner_update_tc_dev.argtypes = [_VP, _I, _VP, _I, _VP, _I, _VP, _I, _I, _I, _I]
    L.lp_refine_dev.argtypes = [_VP, _VP, _I, _VP, _I, _VP, _VP, _I, _I, ctypes.POINTER(LpTiming)]
    L.lp_gesl_dev.argtypes = [_VP, _VP, _I, _I, _VP, _I, _I]
    L.lp_gesl_dev_noalloc.argtypes = [_VP, _I, _I, _VP, _I, _I, _VP]
    L.lp_calculate.argtypes = [_VP, _I, _I, _I, _I, _F32P, _F32P, _F64P, _F64P]
    L.lp_gmres_dev.argtypes = [_VP, _VP, _I, _VP, _I, _VP, _VP, _I, _I, ctypes.c_double, ctypes.POINTER(LpTiming)]
    L.lp_gefa_f64_dev.argtypes = [_VP, _VP, _I, _I, _I]
    L.lp_gesl_f64_dev.argtypes = [_VP, _VP, _I, _I, _VP, _I, _I]
    L.lp_calculate_f64.argtypes = [_VP, _I, _I, _I, _I, _F64P, _F64P, _F64P, _F64P]
    L.lp_gefa_pvt_dev.argtypes = [_VP, _VP, _I, _I, _VP]
    L.lp_gesl_pvt_dev.argtypes = [_VP, _VP, _I, _I, _VP, _VP, _I, _I]
    L.lp_calculate_pvt.argtypes = [_VP, _I, _I, _I, _F32P, _F32P, _I32P, _F64P, _F64P]
    L.lp_solve_host.argtypes = [_VP, _I, _I, _I, _F32P, _I, _F64P, _I, _F64P, _I, ctypes.POINTER(LpTiming)]
    L.lp_factor.argtypes = [_VP, _I, _I, _I, _F32P, _I, ctypes.POINTER(LpTiming)]
    L.lp_solve.argtypes = [_VP, _I, _I, _F32P, _F64P, ctypes.POINTER(LpTiming)]
    L.lp_batch_default_config.argtypes = [ctypes.POINTER(LpBatchConfig)]
    L.lp_batch_solve_dev.argtypes = [_VP, _I, ctypes.POINTER(LpSystem), _VP, _VP, ctypes.POINTER(LpBatchConfig),
                                     ctypes.POINTER(LpBatchStats)]
    L.lp_batch_autotune.argtypes = [_VP, _I, ctypes.POINTER(LpSystem), _VP, _VP, ctypes.POINTER(LpBatchConfig)]
    L.lp_batch_solve_ir_dev.argtypes = [_VP, _I, _I, ctypes.POINTER(LpSystem), _VP, _VP, _VP, _I,
                                        ctypes.POINTER(LpBatchConfig), ctypes.POINTER(LpBatchStats), _VP, _VP]
    L.lp_batch_solve.argtypes = [_VP, _I, _I, ctypes.POINTER(LpSystem), _F32P, _F64P, _F64P, _I,
                                 ctypes.POINTER(LpBatchConfig), ctypes.POINTER(LpBatchStats), _VP, _VP]
    L.lp_generate_reference.argtypes = [_F32P, _F32P, _I, _I, ctypes.POINTER(ctypes.c_float),
                                        ctypes.POINTER(ctypes.c_float)]
    L.lp_generate_baseline.argtypes = [_F32P, _VP, _VP, _I, ctypes.c_uint, ctypes.c_double]
    L.lp_server_default_config.argtypes = [ctypes.POINTER(LpServerConfig)]
    L.lp_server_start.argtypes = [_I, ctypes.POINTER(LpServerConfig), ctypes.POINTER(_VP)]
    L.lp_server_stop.argtypes = [_VP]
    L.lp_server_submit.argtypes = [_VP, ctypes.POINTER(LpRequest), ctypes.POINTER(ctypes.c_longlong)]
    L.lp_server_poll.argtypes = [_VP, ctypes.POINTER(LpResult), _I, _I, ctypes.POINTER(_I)]
    L.lp_server_get_info.argtypes = [_VP, ctypes.POINTER(LpServerInfo)]
    L.lp_server_replay.argtypes = [_VP, _I, ctypes.POINTER(LpRequest), _F64P, ctypes.POINTER(LpResult), _I]
    _lib = L
    return L


def strerror(status: int) -> str:
    return lib().lp_strerror(status).decode()


def last_error() -> str:
    return lib().lp_last_error().decode()


def check(status: int, where: str) -> None:
    if status != LP_OK:
        raise LpError(status, where, last_error())


def header_functions(path: str = HEADER_PATH) -> list[str]:
    """Names of the functions include/lpcuda.h declares."""
    text = open(path).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(lp_[a-z0-9_]+)\s*\(", text)))


def device_count() -> int:
    n = _I(0)
    st = lib().lp_device_count(ctypes.byref(n))
    return n.value if st == LP_OK else 0


# ------------------------------------------------------------------ generators
def generate_reference(n: int, diag_dominant: bool = True):
    """LinpackBenchmark::generateInputData (one rank): (A, b, norma, normb)."""
    A = np.empty((n, n), np.float32)
    b = np.empty(n, np.float32)
    na, nb = ctypes.c_float(), ctypes.c_float()
    check(lib().lp_generate_reference(A, b, n, int(diag_dominant), ctypes.byref(na), ctypes.byref(nb)),
          "lp_generate_reference")
    return A, b, float(na.value), float(nb.value)


def generate_baseline(n: int, seed: int = 42, margin: float = 1.0):
    """Seeded workload matrix: (A float32, b64 float64, b32 float32)."""
    A = np.empty((n, n), np.float32)
    b64 = np.empty(n, np.float64)
    b32 = np.empty(n, np.float32)
    check(lib().lp_generate_baseline(A, b64.ctypes.data, b32.ctypes.data, n, seed, float(margin)),
          "lp_generate_baseline")
    return A, b64, b32


# ------------------------------------------------------------------ context
class Context:
    """One CUDA device, stream and workspace (lp_ctx)."""

    def __init__(self, device: int = 0):
        h = _VP()
        check(lib().lp_ctx_create(device, ctypes.byref(h)), "lp_ctx_create")
        self._h = h
        self.device = device

    @property
    def handle(self):
        return self._h

    def close(self) -> None:
        if self._h:
            lib().lp_ctx_destroy(self._h)
            self._h = _VP()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream(self) -> int:
        s = _VP()
        check(lib().lp_ctx_stream(self._h, ctypes.byref(s)), "lp_ctx_stream")
        return s.value or 0

    def sync(self) -> None:
        check(lib().lp_ctx_sync(self._h), "lp_ctx_sync")

    def device_name(self) -> str:
        buf = ctypes.create_string_buffer(256)
        check(lib().lp_ctx_device_name(self._h, buf, 256), "lp_ctx_device_name")
        return buf.value.decode()

    def set_profiling(self, on: bool) -> None:
        check(lib().lp_ctx_set_profiling(self._h, int(on)), "lp_ctx_set_profiling")

    def read_timeline(self, max_events: int = 1 << 16) -> list[tuple]:
        """(stage, stream, t0_s, t1_s) of every profiled stage launch since the last reset."""
        out = (LpStageEvent * max_events)()
        k = _I(0)
        check(lib().lp_ctx_read_timeline(self._h, out, max_events, ctypes.byref(k)), "lp_ctx_read_timeline")
        return [(STAGES[out[i].stage], out[i].stream, out[i].t0_s, out[i].t1_s) for i in range(k.value)]

    def test_stall(self, site: int) -> None:
        """Arm a bounded wait that runs out (failure-path tests): see lp_ctx_test_stall."""
        check(lib().lp_ctx_test_stall(self._h, site), "lp_ctx_test_stall")

    def read_profile(self, reset: bool = True) -> dict:
        p = LpProfile()
        check(lib().lp_ctx_read_profile(self._h, ctypes.byref(p), int(reset)), "lp_ctx_read_profile")
        return p.as_dict()

    # ---- device-pointer entry points (pointers as ints) -----------------
    def lu_block(self, dA: int, lda: int, bs: int) -> None:
        check(lib().lp_lu_block_dev(self._h, dA, lda, bs), "lp_lu_block_dev")

    def top_update(self, dLU: int, ldlu: int, dT: int, ldt: int, bs: int, ncols: int) -> None:
        check(lib().lp_top_update_dev(self._h, dLU, ldlu, dT, ldt, bs, ncols), "lp_top_update_dev")

    def left_update(self, dLU: int, ldlu: int, dL: int, ldl: int, bs: int, nrows: int,
                    dLt: int | None = None, ldlt: int = 0) -> None:
        check(lib().lp_left_update_dev(self._h, dLU, ldlu, dL, ldl, bs, nrows, dLt, ldlt), "lp_left_update_dev")

    def inner_update(self, dC: int, ldc: int, dLt: int, ldlt: int, dT: int, ldt: int, m: int, n: int,
                     bs: int) -> None:
        check(lib().lp_inner_update_dev(self._h, dC, ldc, dLt, ldlt, dT, ldt, m, n, bs), "lp_inner_update_dev")

    def gefa(self, dA: int, n: int, lda: int, bs: int) -> None:
        check(lib().lp_gefa_dev(self._h, dA, n, lda, bs), "lp_gefa_dev")

    def gefa_prec(self, precision: str, dA: int, n: int, lda: int, bs: int) -> None:
        check(lib().lp_gefa_prec_dev(self._h, PRECISIONS[precision], dA, n, lda, bs), "lp_gefa_prec_dev")

    def inner_update_tc(self, precision: str, dC: int, ldc: int, dL: int, ldl: int, dT: int, ldt: int, m: int,
                        n: int, bs: int) -> None:
        check(lib().lp_inner_update_tc_dev(self._h, PRECISIONS[precision], dC, ldc, dL, ldl, dT, ldt, m, n, bs),
              "lp_inner_update_tc_dev")

    def refine(self, dA0: int, lda: int, dLU: int, n: int, dB64: int, dX: int, nrhs: int = 1,
               max_iters: int = 50) -> dict:
        t = LpTiming()
        check(lib().lp_refine_dev(self._h, dA0, lda, dLU, n, dB64, dX, nrhs, max_iters, ctypes.byref(t)),
              "lp_refine_dev")
        return t.as_dict()

    def gesl(self, dLU: int, n: int, lda: int, dB: int, nrhs: int = 1, ldb: int | None = None) -> None:
        check(lib().lp_gesl_dev(self._h, dLU, n, lda, dB, nrhs, n if ldb is None else ldb), "lp_gesl_dev")

    def gmres(self, dA0: int, lda: int, dLU: int, n: int, dB64: int, dX: int, restart: int = 50, max_it: int = 1,
              tol: float = 1e-8) -> dict:
        """gmres_ref on the device: dX = initial guess in, solution out."""
        t = LpTiming()
        check(lib().lp_gmres_dev(self._h, dA0, lda, dLU, n, dB64, dX, restart, max_it, tol, ctypes.byref(t)),
              "lp_gmres_dev")
        return t.as_dict()

    # ---- FP64 (the reference's double build) ----------------------------------
    def gefa_f64(self, dA: int, n: int, lda: int, bs: int = 128) -> None:
        check(lib().lp_gefa_f64_dev(self._h, dA, n, lda, bs), "lp_gefa_f64_dev")

    def gesl_f64(self, dLU: int, n: int, lda: int, dB: int, nrhs: int = 1, ldb: int | None = None) -> None:
        check(lib().lp_gesl_f64_dev(self._h, dLU, n, lda, dB, nrhs, n if ldb is None else ldb), "lp_gesl_f64_dev")

    def calculate_f64(self, A: np.ndarray, b: np.ndarray, bs: int = 128, repetitions: int = 1):
        """Double build of the backend: A (float64) -> factors, b -> x."""
        n = A.shape[0]
        tg = np.zeros(repetitions, np.float64)
        ts = np.zeros(repetitions, np.float64)
        check(lib().lp_calculate_f64(self._h, n, A.shape[1], bs, repetitions, A, b, tg, ts), "lp_calculate_f64")
        return {"gefa": tg.tolist(), "gesl": ts.tolist()}

    # ---- partial pivoting (gefa_ref / gesl_ref) -------------------------------
    def gefa_pvt(self, dA: int, n: int, lda: int, dIpvt: int) -> None:
        """LU with partial pivoting in place (reference encoding); dIpvt: n ints."""
        check(lib().lp_gefa_pvt_dev(self._h, dA, n, lda, dIpvt), "lp_gefa_pvt_dev")

    def gesl_pvt(self, dLU: int, n: int, lda: int, dIpvt: int, dB: int, nrhs: int = 1,
                 ldb: int | None = None) -> None:
        check(lib().lp_gesl_pvt_dev(self._h, dLU, n, lda, dIpvt, dB, nrhs, n if ldb is None else ldb),
              "lp_gesl_pvt_dev")

    def calculate_pvt(self, A: np.ndarray, b: np.ndarray, repetitions: int = 1):
        """The backend for non-diagonally-dominant matrices: A -> factors
        (gefa_ref encoding), b -> x.  Returns ({"gefa": [...], "gesl": [...]}, ipvt)."""
        n = A.shape[0]
        tg = np.zeros(repetitions, np.float64)
        ts = np.zeros(repetitions, np.float64)
        ipvt = np.zeros(n, np.int32)
        check(lib().lp_calculate_pvt(self._h, n, A.shape[1], repetitions, A, b, ipvt, tg, ts), "lp_calculate_pvt")
        return {"gefa": tg.tolist(), "gesl": ts.tolist()}, ipvt

    # ---- batched solves ---------------------------------------------------
    def batch_solve(self, systems, dA: int, dB: int, cfg: "LpBatchConfig | None" = None) -> dict:
        arr = (LpSystem * len(systems))(*systems)
        st = LpBatchStats()
        check(lib().lp_batch_solve_dev(self._h, len(systems), arr, dA, dB,
                                       ctypes.byref(cfg) if cfg is not None else None, ctypes.byref(st)),
              "lp_batch_solve_dev")
        return st.as_dict()

    def batch_solve_ir(self, systems, dA: int, dB64: int, dX: int, precision: str = "bf16", max_iters: int = 10,
                       cfg: "LpBatchConfig | None" = None):
        """Refined batch on device buffers: (stats dict, ir_iters array, hpl_resid array)."""
        arr = (LpSystem * len(systems))(*systems)
        st = LpBatchStats()
        its = np.zeros(len(systems), np.int32)
        res = np.zeros(len(systems), np.float64)
        check(lib().lp_batch_solve_ir_dev(self._h, PRECISIONS[precision], len(systems), arr, dA, dB64, dX, max_iters,
                                          ctypes.byref(cfg) if cfg is not None else None, ctypes.byref(st),
                                          its.ctypes.data, res.ctypes.data), "lp_batch_solve_ir_dev")
        return st.as_dict(), its, res

    def batch_solve_host(self, systems, A: np.ndarray, B: np.ndarray, precision: str = "bf16", max_iters: int = 10,
                         cfg: "LpBatchConfig | None" = None):
        """Refined batch on host buffers: A (float32, factored in place), B (float64
        right-hand sides) -> (X float64, stats dict, ir_iters, hpl_resid)."""
        arr = (LpSystem * len(systems))(*systems)
        st = LpBatchStats()
        X = np.zeros_like(B)
        its = np.zeros(len(systems), np.int32)
        res = np.zeros(len(systems), np.float64)
        check(lib().lp_batch_solve(self._h, PRECISIONS[precision], len(systems), arr, A, B, X, max_iters,
                                   ctypes.byref(cfg) if cfg is not None else None, ctypes.byref(st), its.ctypes.data,
                                   res.ctypes.data), "lp_batch_solve")
        return X, st.as_dict(), its, res

    def batch_autotune(self, systems, dA: int, dB: int) -> LpBatchConfig:
        arr = (LpSystem * len(systems))(*systems)
        cfg = LpBatchConfig()
        check(lib().lp_batch_autotune(self._h, len(systems), arr, dA, dB, ctypes.byref(cfg)), "lp_batch_autotune")
        return cfg

    # ---- host entry points ------------------------------------------------
    def calculate(self, A: np.ndarray, b: np.ndarray, bs: int, repetitions: int = 1):
        """execution::pcie::calculate stand-in: factors A in place, b -> x.
        Returns {"gefa": [...], "gesl": [...]} in seconds."""
        n = A.shape[0]
        tg = np.zeros(repetitions, np.float64)
        ts = np.zeros(repetitions, np.float64)
        check(lib().lp_calculate(self._h, n, A.shape[1], bs, repetitions, A, b, tg, ts), "lp_calculate")
        return {"gefa": tg.tolist(), "gesl": ts.tolist()}

    def solve_host(self, A: np.ndarray, b64: np.ndarray, bs: int, precision: str = "f32",
                   max_iters: int = 0):
        """Factor + solve (+ FP64 refinement).  b64: (n,) or (nrhs, n)."""
        A = np.ascontiguousarray(A, dtype=np.float32)
        B = np.ascontiguousarray(np.atleast_2d(b64), dtype=np.float64)
        nrhs, n = B.shape
        x = np.empty_like(B)
        t = LpTiming()
        check(lib().lp_solve_host(self._h, PRECISIONS[precision], n, bs, A, A.shape[1], B, nrhs, x, max_iters,
                                  ctypes.byref(t)), "lp_solve_host")
        return (x[0] if np.ndim(b64) == 1 else x), t.as_dict()

    def factor(self, A: np.ndarray, bs: int, precision: str = "f32") -> dict:
        """Factor the host matrix A in place (factors in the reference encoding
        written back) and keep the factors resident for solve()."""
        if A.dtype != np.float32 or not A.flags.c_contiguous:
            raise ValueError("factor: A must be a C-contiguous float32 array (it is overwritten)")
        t = LpTiming()
        check(lib().lp_factor(self._h, PRECISIONS[precision], A.shape[0], bs, A, A.shape[1], ctypes.byref(t)),
              "lp_factor")
        return t.as_dict()

    def solve(self, B: np.ndarray):
        """Solve with the resident factors of the last factor(): B (n,) or
        (nrhs, n) float32 -> (x float64 of the same shape, timing dict)."""
        Bm = np.ascontiguousarray(np.atleast_2d(B), dtype=np.float32)
        nrhs, n = Bm.shape
        x = np.empty((nrhs, n), np.float64)
        t = LpTiming()
        check(lib().lp_solve(self._h, n, nrhs, Bm, x, ctypes.byref(t)), "lp_solve")
        return (x[0] if np.ndim(B) == 1 else x), t.as_dict()


# ------------------------------------------------------------------ pinned host memory
class Pinned:
    """Page-locked host buffer (lp_host_alloc) viewed as a numpy array."""

    def __init__(self, shape, dtype=np.float32):
        dtype = np.dtype(dtype)
        count = int(np.prod(shape))
        p = _VP()
        check(lib().lp_host_alloc(ctypes.c_size_t(max(1, count) * dtype.itemsize), ctypes.byref(p)),
              "lp_host_alloc")
        self._p = p
        buf = (ctypes.c_char * (max(1, count) * dtype.itemsize)).from_address(p.value)
        self.array = np.frombuffer(buf, dtype=dtype, count=count).reshape(shape)

    @property
    def ptr(self) -> int:
        return self._p.value

    def free(self) -> None:
        if self._p:
            self.array = None
            lib().lp_host_free(self._p)
            self._p = _VP()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


# ------------------------------------------------------------------ serving loop
def server_config(**kw) -> LpServerConfig:
    """Default lp_server_config with fields overridden by keyword (precision
    may be given as "f32" / "bf16" / "fp8", mode as "continuous" / "per_request")."""
    cfg = LpServerConfig()
    check(lib().lp_server_default_config(ctypes.byref(cfg)), "lp_server_default_config")
    for k, v in kw.items():
        if k == "precision" and isinstance(v, str):
            v = PRECISIONS[v]
        if k == "mode" and isinstance(v, str):
            v = {"continuous": LP_SERVE_CONTINUOUS, "per_request": LP_SERVE_PER_REQUEST}[v]
        setattr(cfg, k, int(v))
    return cfg


class Server:
    """lp_server: asynchronous solve requests with resident factors."""

    def __init__(self, device: int = 0, cfg: LpServerConfig | None = None, **kw):
        if cfg is None:
            cfg = server_config(**kw)
        h = _VP()
        check(lib().lp_server_start(device, ctypes.byref(cfg), ctypes.byref(h)), "lp_server_start")
        self._h = h
        self.cfg = cfg

    def stop(self) -> None:
        if self._h:
            lib().lp_server_stop(self._h)
            self._h = _VP()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.stop()

    def __del__(self):
        try:
            self.stop()
        except Exception:
            pass

    def submit(self, req: LpRequest) -> int:
        rid = ctypes.c_longlong()
        check(lib().lp_server_submit(self._h, ctypes.byref(req), ctypes.byref(rid)), "lp_server_submit")
        return rid.value

    def poll(self, max_results: int = 256, timeout_ms: int = 1000) -> list[dict]:
        """Finished results (possibly none when the wait times out)."""
        out = (LpResult * max_results)()
        k = _I(0)
        st = lib().lp_server_poll(self._h, out, max_results, timeout_ms, ctypes.byref(k))
        if st not in (LP_OK, LP_E_TIMEOUT):
            check(st, "lp_server_poll")
        return [out[i].as_dict() for i in range(k.value)]

    def wait(self, count: int, timeout_ms: int = 60000) -> list[dict]:
        """Poll until `count` results arrived; LpError(LP_E_TIMEOUT) if a wait expires."""
        got: list[dict] = []
        while len(got) < count:
            out = (LpResult * 256)()
            k = _I(0)
            check(lib().lp_server_poll(self._h, out, 256, timeout_ms, ctypes.byref(k)), "lp_server_poll")
            got += [out[i].as_dict() for i in range(k.value)]
        return got

    def info(self) -> dict:
        i = LpServerInfo()
        check(lib().lp_server_get_info(self._h, ctypes.byref(i)), "lp_server_get_info")
        return i.as_dict()

    def replay(self, reqs, arrival_s: np.ndarray, timeout_ms: int = 60000) -> list[dict]:
        """Submit reqs[i] at arrival_s[i] (seconds from the call) and collect all results, in order."""
        arr = (LpRequest * len(reqs))(*reqs)
        out = (LpResult * len(reqs))()
        t = np.ascontiguousarray(arrival_s, dtype=np.float64)
        check(lib().lp_server_replay(self._h, len(reqs), arr, t, out, timeout_ms), "lp_server_replay")
        return [out[i].as_dict() for i in range(len(reqs))]
