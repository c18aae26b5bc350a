"""The N > 1 path of bench.py on the CPU: two gloo ranks, each an
independent replica, aggregate their step times (max over ranks) and their
units (sum) the way the GPU run does over NCCL."""

import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms_local = 2.0 + rank  # rank 1 is slower
        units = 1000.0 * (rank + 1)
        ms, value = bench.aggregate_replicas(ms_local, units, dist)
        dist.barrier()
        out[rank] = (ms, value)
    finally:
        dist.destroy_process_group()


def test_two_gloo_replicas_aggregate_max_time_and_total_units():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        ctx = mp.get_context("spawn")
        procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
            assert p.exitcode == 0
        res = dict(out)
    assert set(res) == {0, 1}
    for rank in range(world):
        ms, value = res[rank]
        assert ms == pytest.approx(3.0)
        assert value == pytest.approx(3000.0 / 3e-3)


def test_single_rank_needs_no_group():
    ms, value = bench.aggregate_replicas(4.0, 8.0e6)
    assert ms == 4.0 and value == pytest.approx(2.0e9)
