"""hpcc_fpga_b200 — B200-native LINPACK (LU without pivoting + substitution).

The compute path is liblpcuda.so (hand-written sm_100a kernels behind the C
ABI of include/lpcuda.h); ``lpcuda`` is its ctypes binding and ``linpack``
the host-side mirror of the reference's LinpackBenchmark interface.
"""
from . import lpcuda  # noqa: F401

__all__ = ["lpcuda"]
