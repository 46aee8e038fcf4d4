"""The multi-GPU path of bench.py on the CPU: replicas on two gloo ranks.
Each rank relaxes or steps its own work with no data-path exchange; the only
collective is the max-over-ranks reduction of the timed region, and the
job's throughput is the units of all ranks over the slowest rank's time."""
from __future__ import annotations

import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, times, out):
    import datetime
    import sys

    import torch.distributed as dist

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    slowest = bench.max_over_ranks(times[rank], dist)
    out[rank] = slowest
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_replicas_take_the_slowest_rank():
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    out = manager.dict()
    times = [0.25, 0.4]
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, times, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    assert out[0] == out[1] == 0.4
    # whole-job throughput: both replicas' units over the slowest time
    units = 4000 * 200
    assert 2 * units / out[0] == pytest.approx(4.0e6)


def test_single_process_needs_no_collective():
    import bench

    assert bench.max_over_ranks(0.3, None) == 0.3
