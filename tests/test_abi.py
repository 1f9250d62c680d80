"""The C-ABI boundary without a GPU: the library loads, exports every
function include/lpcuda.h declares, validates arguments before touching the
device, and its host-only generators match the oracle bit for bit."""
import ctypes
import subprocess

import numpy as np
import pytest

import oracle


def test_library_exports_every_header_function(lp):
    names = lp.header_functions()
    assert len(names) >= 19
    out = subprocess.run(["nm", "-D", "--defined-only", lp.LIB_PATH], capture_output=True, text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    missing = [f for f in names if f not in exported]
    assert not missing, f"declared but not exported: {missing}"
    for f in names:
        getattr(lp.lib(), f)


def test_strerror_and_version(lp):
    assert lp.lib().lp_version() == 100
    assert lp.strerror(0) == "ok"
    assert lp.strerror(lp.LP_E_INVALID) == "invalid argument"
    assert lp.strerror(lp.LP_E_TIMEOUT) == "timeout"
    assert lp.strerror(12345) == "unknown status"


def test_null_context_rejected(lp):
    L = lp.lib()
    assert L.lp_gefa_dev(None, None, 128, 128, 128) == lp.LP_E_INVALID
    assert L.lp_gesl_dev(None, None, 128, 128, None, 1, 128) == lp.LP_E_INVALID
    assert L.lp_ctx_sync(None) == lp.LP_E_INVALID
    A = np.zeros((16, 16), np.float32)
    assert L.lp_factor(None, 0, 16, 16, A, 16, None) == lp.LP_E_INVALID
    assert L.lp_solve(None, 16, 1, np.zeros(16, np.float32), np.zeros(16), None) == lp.LP_E_INVALID
    assert "null" in lp.last_error()
    assert L.lp_ctx_destroy(None) == 0


def test_context_without_gpu(lp):
    if lp.device_count() > 0:
        pytest.skip("a GPU is present")
    with pytest.raises(lp.LpError) as e:
        lp.Context(0)
    assert e.value.status == lp.LP_E_NODEVICE


@pytest.mark.parametrize("n", [1, 17, 128])
def test_reference_generator_bitexact(lp, n):
    A, b, na, nb = lp.generate_reference(n)
    oA, ob, ona, onb = oracle.gen_reference(n)
    assert np.array_equal(A.view(np.uint32), oA.view(np.uint32))
    assert np.array_equal(b.view(np.uint32), ob.view(np.uint32))
    assert (na, nb) == (ona, onb)


def test_reference_generator_uniform(lp):
    A, b, _, _ = lp.generate_reference(40, diag_dominant=False)
    oA, ob, _, _ = oracle.gen_reference(40, diag_dominant=False)
    assert np.array_equal(A, oA) and np.array_equal(b, ob)


@pytest.mark.parametrize("n,seed,margin", [(33, 42, 1.0), (128, 7, 0.1 * 128 ** 0.5), (64, 42, 64.0)])
def test_baseline_generator_bitexact(lp, n, seed, margin):
    A, b64, b32 = lp.generate_baseline(n, seed, margin)
    oA, ob64, ob32 = oracle.gen_baseline(n, seed, margin)
    assert np.array_equal(A.view(np.uint32), oA.view(np.uint32))
    assert np.array_equal(b64, ob64)
    assert np.array_equal(b32, ob32)


def test_generator_rejects_bad_size(lp):
    A = np.zeros((1, 1), np.float32)
    assert lp.lib().lp_generate_reference(A, np.zeros(1, np.float32), 0, 1, None, None) == lp.LP_E_INVALID
