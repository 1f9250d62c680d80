"""The N > 1 path of bench.py on CPU: two ranks over gloo (127.0.0.1) run
independent replicas; the whole-job rate is the total work over the slowest
rank's time, and the only collective is that max-reduction."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist
    from hpcc_fpga_b200.replicas import job_rate, max_over_ranks

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        my_seconds = 1.0 + rank          # rank 1 is the slow one
        rate, t = job_rate(10.0, my_seconds)
        out[rank] = (rate, t, max_over_ranks(3.0 - rank))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_ranks_rate_is_total_work_over_slowest():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
            assert p.exitcode == 0
        for r in range(2):
            rate, t, other = out[r]
            assert t == 2.0 and rate == pytest.approx(2 * 10.0 / 2.0)
            assert other == 3.0


def test_single_process_without_group():
    from hpcc_fpga_b200.replicas import job_rate

    rate, t = job_rate(5.0, 2.0)
    assert (rate, t) == (2.5, 2.0)
