"""Building batches of independent systems for lp_batch_solve_dev.

A batch packs every system's matrix (row-major, leading dimension rounded up
to a multiple of 4) into one float32 array and its right-hand sides (nrhs
rows) into another, and describes them with lpcuda.LpSystem records.
"""
from __future__ import annotations

import math

import numpy as np

from . import lpcuda


def round4(n: int) -> int:
    return (n + 3) // 4 * 4


def log_uniform_sizes(count: int, lo: int, hi: int, seed: int) -> np.ndarray:
    """n_i = round(exp(U(ln lo, ln hi))) from a seeded generator."""
    rng = np.random.default_rng(seed)
    return np.clip(np.rint(np.exp(rng.uniform(math.log(lo), math.log(hi), count))), lo, hi).astype(np.int64)


class Batch:
    """Packed host arrays + descriptors.  mats[i] / rhs[i] are views."""

    def __init__(self, sizes, nrhs):
        self.sizes = [int(n) for n in sizes]
        self.nrhs = [int(r) for r in nrhs]
        self.systems = []
        a_off = b_off = 0
        for n, r in zip(self.sizes, self.nrhs):
            ld = round4(n)
            self.systems.append(lpcuda.LpSystem(n, r, ld, ld, a_off, b_off))
            a_off += n * ld
            b_off += r * ld
        self.A = np.zeros(max(a_off, 1), np.float32)
        self.B = np.zeros(max(b_off, 1), np.float32)

    def mat(self, i: int) -> np.ndarray:
        s = self.systems[i]
        return self.A[s.a_off:s.a_off + s.n * s.lda].reshape(s.n, s.lda)[:, :s.n]

    def rhs(self, i: int) -> np.ndarray:
        s = self.systems[i]
        return self.B[s.b_off:s.b_off + s.nrhs * s.ldb].reshape(s.nrhs, s.ldb)[:, :s.n]

    def flops(self) -> float:
        return float(sum(2.0 * n ** 3 / 3.0 + 2.0 * r * n * n for n, r in zip(self.sizes, self.nrhs)))


def make_batch(count: int = 4096, lo: int = 32, hi: int = 1024, seed: int = 7, rhs_max: int = 8,
               margin: float = 1.0) -> Batch:
    """The batched-solve workload: n log-uniform in [lo, hi] (seed), each
    matrix from the seeded diagonally dominant generator (seed + i), 1..rhs_max
    right-hand sides uniform in [-1, 1)."""
    sizes = log_uniform_sizes(count, lo, hi, seed)
    rng = np.random.default_rng(seed + 1)
    nrhs = rng.integers(1, rhs_max + 1, count)
    b = Batch(sizes, nrhs)
    for i, n in enumerate(b.sizes):
        A, _, _ = lpcuda.generate_baseline(int(n), seed + i, margin)
        b.mat(i)[:, :] = A
        b.rhs(i)[:, :] = rng.uniform(-1.0, 1.0, (b.nrhs[i], n)).astype(np.float32)
    return b
