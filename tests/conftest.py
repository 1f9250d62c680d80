import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def lp():
    from hpcc_fpga_b200 import lpcuda
    lpcuda.lib()
    return lpcuda


@pytest.fixture(scope="session")
def ctx(lp):
    c = lp.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="session")
def torch_cuda():
    import torch
    assert torch.cuda.is_available(), "GPU tests need CUDA"
    return torch


class Dev:
    """Device copies of numpy arrays through torch (plumbing only)."""

    def __init__(self, torch, ctx):
        self.torch = torch
        self.ctx = ctx

    def put(self, a: np.ndarray):
        t = self.torch.from_numpy(np.ascontiguousarray(a)).cuda()
        self.torch.cuda.synchronize()
        return t

    def get(self, t) -> np.ndarray:
        self.ctx.sync()
        self.torch.cuda.synchronize()
        return t.cpu().numpy()

    def empty(self, shape, dtype=np.float32):
        t = self.torch.zeros(shape, dtype=getattr(self.torch, np.dtype(dtype).name), device="cuda")
        self.torch.cuda.synchronize()
        return t


@pytest.fixture(scope="session")
def dev(torch_cuda, ctx):
    return Dev(torch_cuda, ctx)
