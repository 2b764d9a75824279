"""The replica path of bench.py (N > 1 ranks, one independent solver each):
the max-over-ranks timing and the whole-job rate, run as two gloo ranks on
CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from minicombust_app_b200 import replicas


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, times, out):
    import torch.distributed as dist
    from datetime import timedelta
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    slowest = replicas.max_over_ranks(times[rank], dist)
    out[rank] = (slowest, replicas.whole_job_rate(10, slowest, world))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_and_rate_with_two_gloo_ranks():
    world, times = 2, [0.25, 0.4]
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_rank, args=(world, _free_port(), times, out), nprocs=world, join=True,
                           start_method="spawn")
        res = dict(out)
    for r in range(world):
        slowest, rate = res[r]
        assert slowest == pytest.approx(0.4)
        assert rate == pytest.approx(world * 10 / 0.4)


def test_single_process_needs_no_group():
    assert replicas.max_over_ranks(1.5) == 1.5
    assert replicas.whole_job_rate(10, 2.0, 1) == 5.0
    with pytest.raises(ValueError):
        replicas.whole_job_rate(10, 0.0, 1)
