"""Slab decomposition over ranks, host side (piernik_b200/slabs.py): the
layout, the torch.distributed transport run as world_size 2 and 3 gloo ranks
on the CPU (point-to-point halo buffers in both directions, dt minimum and
c_all maximum), and the exchange plan itself across processes: every rank
builds its per-peer segment lists with the library's planner
(piernik_b200/csrc/pk_exchange.cpp), packs its slab's cells in the order of
the device pack kernel, moves the buffers over gloo and unpacks them into its
guard cells, which must then equal the periodic images of the global field --
for the whole halo and for the z faces alone, which is all a z sweep reads
(and the x and y lists carry nothing between z slabs)."""
import ctypes as C
import os
import subprocess

import numpy as np

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


def _init(rank, world, store):
    """gloo over a file rendezvous (no TCP port to race for between tests)"""
    dist.init_process_group("gloo", init_method="file://" + store, rank=rank, world_size=world)


def _worker(rank, world, store, q):
    _init(rank, world, store)
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
def test_torch_transport_gloo(world, tmp_path):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    store = str(tmp_path / "rendezvous")
    procs = [ctx.Process(target=_worker, args=(r, world, store, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ok, lo, hi in res:
        assert ok, f"rank {rank} received wrong halo buffers"
        assert lo == 1.0 and hi == float(world)


HERE = os.path.dirname(os.path.abspath(__file__))
HSRC = os.path.join(HERE, "native", "xchg_harness.cpp")
HPLAN = os.path.join(HERE, "..", "piernik_b200", "csrc", "pk_exchange.cpp")
HLIB = os.path.join(HERE, "native", "libxchg_harness.so")


def _harness():
    if not os.path.exists(HLIB) or os.path.getmtime(HLIB) < max(os.path.getmtime(HSRC), os.path.getmtime(HPLAN)):
        subprocess.check_call(["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-o", HLIB, HSRC, HPLAN])
    return C.CDLL(HLIB)


def _segs(lib, layout, rank, peer, which, direction, nb=4):
    """This rank's view of the plan: its slab first, then the others."""
    order = [rank] + [r for r in range(len(layout)) if r != rank]
    own = [-1] + [r for r in order[1:]]
    k = len(order)
    n = (C.c_int * (3 * k))(*[x for r in order for x in layout[r][0]])
    g = (C.c_int * (3 * k))(*[(nb if layout[r][0][d] > 1 else 0) for r in order for d in range(3)])
    off = (C.c_longlong * (3 * k))(*[x for r in order for x in layout[r][1]])
    dom = (C.c_longlong * 3)(*[sum(layout[r][0][2] for r in range(len(layout))) if d == 2 else layout[0][0][d]
                               for d in range(3)])
    out = (C.c_int * (11 * 4096))()
    cnt = lib.xchg_peer_segs(k, 1, (C.c_int * k)(*own), n, g, off, dom, (C.c_int * 3)(1, 1, 1), peer, which,
                             direction, out, 4096)
    assert cnt >= 0
    return [tuple(out[11 * i:11 * i + 11]) for i in range(cnt)]


def _cells(seg):
    lo, hi = seg[2:5], seg[5:8]
    for k in range(lo[2], hi[2]):
        for j in range(lo[1], hi[1]):
            for i in range(lo[0], hi[0]):          # i fastest, as k_halo_copy
                yield i, j, k


def _plan_worker(rank, world, store, q):
    _init(rank, world, store)
    try:
        lib = _harness()
        s = Setup(n=(8, 6, 4 * world), magnetic=False, fluids=[("neu", 1.4)])
        layout = slab_layout(s, world, axis=2)
        nb, npl = 4, 3
        rng = np.random.default_rng(11)
        glob = rng.standard_normal((npl,) + tuple(s.n[::-1]))        # [plane, z, y, x], interior only
        (nz, ny, nx), (oz, oy, ox) = layout[rank][0][::-1], layout[rank][1][::-1]
        loc = np.full((npl, nz + 2 * nb, ny + 2 * nb, nx + 2 * nb), np.nan)
        loc[:, nb:nb + nz, nb:nb + ny, nb:nb + nx] = glob[:, oz:oz + nz, oy:oy + ny, ox:ox + nx]
        tr = TorchTransport(torch.device("cpu"))
        peers = sorted({(rank - 1) % world, (rank + 1) % world} - {rank})
        report = {}
        for direction in (-1, 2, 0, 1):
            send, recv, sl, rl = {}, {}, {}, {}
            for p in peers:
                sl[p] = _segs(lib, layout, rank, p, 1, direction)
                rl[p] = _segs(lib, layout, rank, p, 0, direction)
                cs = [c for sg in sl[p] for c in _cells(sg)]
                cr = sum(1 for sg in rl[p] for _ in _cells(sg))
                buf = np.empty((npl, len(cs)))
                at = 0
                for sg in sl[p]:
                    for i, j, k in _cells(sg):
                        buf[:, at] = loc[:, k + sg[10], j + sg[9], i + sg[8]]
                        at += 1
                send[p] = torch.tensor(buf.reshape(-1))
                recv[p] = torch.empty(npl * cr, dtype=torch.float64)
            report[direction] = sum(int(send[p].numel()) for p in peers)
            active = [p for p in peers if send[p].numel() or recv[p].numel()]
            tr.exchange(rank, active, send, recv)
            got = np.full_like(loc, np.nan)
            for p in active:
                buf = recv[p].numpy().reshape(npl, -1)
                at = 0
                for sg in rl[p]:
                    for i, j, k in _cells(sg):
                        got[:, k, j, i] = buf[:, at]
                        at += 1
            # every cell written is the periodic image of the global field
            zz, yy, xx = np.nonzero(~np.isnan(got[0]))
            want = glob[:, (zz - nb + oz) % s.n[2], (yy - nb + oy) % s.n[1], (xx - nb + ox) % s.n[0]]
            report[f"ok{direction}"] = bool(np.array_equal(got[:, zz, yy, xx], want))
            if direction == 2:   # the z faces: x and y interior, z guards, all of them
                face = got[:, list(range(nb)) + list(range(nb + nz, 2 * nb + nz)), nb:nb + ny, nb:nb + nx]
                report["zface_full"] = bool(not np.isnan(face).any()) and len(zz) == face[0].size
        q.put((rank, report))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_halo_plan_over_gloo(world, tmp_path):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    store = str(tmp_path / "rendezvous")
    procs = [ctx.Process(target=_plan_worker, args=(r, world, store, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=180) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, rep in res:
        assert all(rep[f"ok{d}"] for d in (-1, 2, 0, 1)), (rank, rep)
        assert rep["zface_full"], (rank, rep)
        assert rep[0] == 0 and rep[1] == 0, rep                 # x and y sweeps move nothing between z slabs
        assert 0 < rep[2] < rep[-1], rep                        # the z faces are part of the whole halo
