"""Slab decomposition over ranks, host side (piernik_b200/slabs.py): the
layout, and the torch.distributed transport run as world_size 2 and 3 gloo
ranks on the CPU (point-to-point halo buffers in both directions, dt
minimum and c_all maximum)."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from piernik_b200.config import Setup
from piernik_b200.slabs import TorchTransport, slab_layout, split


def test_split_and_layout():
    assert split(10, 3) == [4, 3, 3]
    assert split(256, 4) == [64] * 4
    with pytest.raises(ValueError):
        split(2, 3)
    s = Setup(n=(16, 12, 10), magnetic=False, fluids=[("neu", 1.4)])
    lay = slab_layout(s, 3, axis=2)
    assert [l[0] for l in lay] == [(16, 12, 4), (16, 12, 3), (16, 12, 3)]
    assert [l[1] for l in lay] == [(0, 0, 0), (0, 0, 4), (0, 0, 7)]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        tr = TorchTransport(torch.device("cpu"))
        peers = sorted({(rank - 1) % world, (rank + 1) % world} - {rank})
        send = {p: torch.arange(5, dtype=torch.float64) + 100 * rank + 10 * p for p in peers}
        recv = {p: torch.empty(5, dtype=torch.float64) for p in peers}
        tr.exchange(rank, peers, send, recv)
        ok = all(torch.equal(recv[p], torch.arange(5, dtype=torch.float64) + 100 * p + 10 * rank) for p in peers)
        lo = tr.reduce(rank, 1.0 + rank, 0)
        hi = tr.reduce(rank, 1.0 + rank, 1)
        q.put((rank, ok, lo, hi))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_torch_transport_gloo(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ok, lo, hi in res:
        assert ok, f"rank {rank} received wrong halo buffers"
        assert lo == 1.0 and hi == float(world)
