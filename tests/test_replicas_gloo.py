"""The N-GPU benchmark runs independent replicas (the path does not shard a
single instance).  Its only cross-rank step is the timing reduction: the max
of the per-rank device times and the sum of the per-rank particle counts.
Checked here with two gloo ranks on the CPU."""
from __future__ import annotations

import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    ms = [120.0, 150.0][rank]
    n = [1000.0, 1200.0][rank]
    t = torch.tensor([ms, n], dtype=torch.float64)
    mx = t.clone()
    dist.all_reduce(mx, op=dist.ReduceOp.MAX)
    tot = t.clone()
    dist.all_reduce(tot, op=dist.ReduceOp.SUM)
    steps = 10
    value = float(tot[1]) * steps / (float(mx[0]) / 1e3)
    out[rank] = value
    dist.barrier()
    dist.destroy_process_group()


def test_replica_timing_reduction():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
        vals = dict(out)
    expect = (1000.0 + 1200.0) * 10 / 0.150
    assert vals[0] == pytest.approx(expect) and vals[1] == pytest.approx(expect)
