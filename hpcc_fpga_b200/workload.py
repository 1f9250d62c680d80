"""Device-side helpers for the seeded benchmark matrices (torch as plumbing).

The seeded workload generator (lp_generate_baseline) draws the off-diagonal
entries from mt19937(seed) and sets each storage-row diagonal to
fl32(sum |off-diagonal| + margin), with b64 = M * ones in FP64.  Only the
diagonal and b64 depend on the margin, so a matrix already on the device can
be moved to another margin without drawing it again: every off-diagonal entry
is a multiple of 2^-24 below 0.5 in magnitude, so the FP64 row sums of |off|
and the FP64 column sums are exact in any summation order, and
fl32(S + margin) rounds exactly as the host generator does.  The result is
bit-identical to lp_generate_baseline(n, seed, margin).
"""
from __future__ import annotations


def set_margin(torch, dA, n: int, margin: float, rows: int = 0):
    """Rewrite the diagonal of the n x n seeded matrix dA (float32, device or
    CPU tensor, row-major with leading dimension n) for `margin`; returns
    b64 = M * ones (float64 tensor on dA's device)."""
    if rows <= 0:
        rows = max(1, min(n, (1 << 28) // (8 * n)))  # FP64 temporaries of at most 2 GiB
    dev = dA.device
    off = torch.empty(n, dtype=torch.float64, device=dev)
    for r0 in range(0, n, rows):
        r1 = min(n, r0 + rows)
        blk = dA[r0:r1].to(torch.float64)
        idx = torch.arange(r1 - r0, device=dev)
        off[r0:r1] = blk.abs().sum(1) - blk[idx, idx + r0].abs()
        del blk
    dA.diagonal().copy_((off + float(margin)).to(torch.float32))
    b64 = torch.zeros(n, dtype=torch.float64, device=dev)
    for r0 in range(0, n, rows):
        b64 += dA[r0:min(n, r0 + rows)].to(torch.float64).sum(0)
    return b64
