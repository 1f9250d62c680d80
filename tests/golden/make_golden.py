"""Generate tests/golden/linpack_golden.npz from the REFERENCE's own code.

Inputs come from the oracle's generators (restatements of
LINPACK/src/host/linpack_benchmark.hpp:211-297 and of the seeded workload
generator); the factors and solutions come from gefa_ref_nopvt /
gesl_ref_nopvt compiled unmodified from LINPACK/src/host/linpack_data.cpp
into oracle/_ref/libref32.so (``make -C oracle``).

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
import oracle  # noqa: E402

SIZES = [16, 32, 128]
BSIZES = [64]


def main() -> None:
    ref = oracle.ref("f32")
    if ref is None:
        raise SystemExit("oracle/_ref/libref32.so missing: run `make -C oracle` where the reference sources exist")
    out = {"sizes": np.array(SIZES), "bsizes": np.array(BSIZES)}
    for n in SIZES:
        A, b, _, _ = oracle.gen_reference(n)
        lu = A.copy()
        ref.ref_gefa_nopvt_f32(lu, n, n)
        x = b.copy()
        ref.ref_gesl_nopvt_f32(lu, x, n, n)
        out.update({f"A_{n}": A, f"b_{n}": b, f"lu_{n}": lu, f"x_{n}": x})
    for n in BSIZES:
        A, b64, b32 = oracle.gen_baseline(n, seed=42, margin=1.0)
        lu = A.copy()
        ref.ref_gefa_nopvt_f32(lu, n, n)
        x = b32.copy()
        ref.ref_gesl_nopvt_f32(lu, x, n, n)
        out.update({f"BA_{n}": A, f"Bb64_{n}": b64, f"Blu_{n}": lu, f"Bx_{n}": x})
    path = os.path.join(HERE, "linpack_golden.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
