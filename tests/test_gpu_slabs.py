"""A periodic level split into slabs over ranks (piernik_b200/slabs.py):
ranks run as threads of this process on one GPU with the in-process
transport (the halo buffers cross between the ranks' handles on the host
side; no kernel waits for another rank).  The slabs together must evolve
exactly like the level held as one block."""
import threading

import numpy as np
import pytest

from helpers import assert_bitexact, random_state, setup_for
from piernik_b200.sim import Simulation
from piernik_b200.slabs import SlabRank, ThreadTransport

pytestmark = pytest.mark.gpu


def exact(setup):
    return setup.replace(xmin=(0.0, 0.0, 0.0), xmax=tuple(0.125 * setup.n[d] for d in range(3)))


def run_ranks(full, state, world, nsteps, axis=2):
    tr = ThreadTransport(world)
    ranks = [SlabRank(full, r, world, tr, axis=axis) for r in range(world)]
    for r in ranks:
        r.upload_global(*state)
    errors = []

    def go(r):
        try:
            r.run(nsteps)
        except Exception as e:          # noqa: BLE001 -- reported below
            errors.append(e)

    th = [threading.Thread(target=go, args=(r,)) for r in ranks]
    for t in th:
        t.start()
    for t in th:
        t.join(timeout=300)
    assert not errors, errors
    for r in ranks:
        r.detach()
    out = [(r.layout[r.rank], r.sim.download(), r.sim.time_state, (r.exchanges, r.skipped)) for r in ranks]
    for r in ranks:
        r.close()
    return out


@pytest.mark.parametrize("phys,world,axis,order", [("hd", 2, 2, 2), ("mhd", 2, 2, 2), ("mhd", 3, 1, 2),
                                                  ("hd", 2, 0, 1)])
def test_slabs_equal_one_block(gpu_lib, phys, world, axis, order):
    """RK2: fused sweeps with the halo from the guards; Euler (order 1): the
    per-stage path, exchanging after the stage."""
    full = exact(setup_for(phys, n=(24, 30, 32), lim="moncen", integration_order=order))
    state = random_state(full, seed=7)
    one = Simulation(full)
    one.upload(*state)
    one.run(3)
    ref = one.download()
    st = one.time_state
    one.close()
    g = full.guards
    for (n, off), arrs, st_r, nex in run_ranks(full, state, world, 3, axis):
        assert st_r.t == st.t and st_r.dt == st.dt
        moved, skipped = nex
        if order == 2:      # fused sweeps: only the two sweeps along the slab axis per step cross ranks
            assert moved == 3 * 2 and skipped == 3 * 4, nex
        else:               # per-stage path: the whole halo after every stage
            assert moved >= 3 * 6, nex
        for k in range(3):
            if arrs[k] is None:
                continue
            mine = arrs[k][g[2]:g[2] + n[2], g[1]:g[1] + n[1], g[0]:g[0] + n[0]]
            want = ref[k][tuple(slice(g[d] + off[d], g[d] + off[d] + n[d]) for d in (2, 1, 0))]
            assert_bitexact(mine, want, f"{phys} slab {off} array {k}")


@pytest.mark.parametrize("world", [2, 3])
def test_block_shards_equal_one_handle(gpu_lib, world):
    """Independent uneven blocks (ion MHD + neutral + dust) split into
    per-rank block lists, ranks as threads with the in-process transport:
    with dt reduced over ranks every block evolves bit for bit as in one
    handle holding them all."""
    from piernik_b200 import problems
    from piernik_b200.shard import BlockShard
    data = problems.batched_blocks(nblocks=7, seed=5, sizes=(8, 16, 24), n0=16)
    one = Simulation(data[0][0])
    for s, *_ in data[1:]:
        one.add_block(s)
    for i, (s, u, b, psi) in enumerate(data):
        one.upload(u, b, psi, block=i)
    one.run(3)
    ref = [one.download(block=i) for i in range(len(data))]
    st = one.time_state
    one.close()
    tr = ThreadTransport(world)
    shards = [BlockShard(data, r, world, tr) for r in range(world)]
    errors = []

    def go(sh):
        try:
            sh.run(3)
        except Exception as e:          # noqa: BLE001 -- reported below
            errors.append(e)

    th = [threading.Thread(target=go, args=(sh,)) for sh in shards]
    for t in th:
        t.start()
    for t in th:
        t.join(timeout=300)
    assert not errors, errors
    seen = set()
    for sh in shards:
        ts = sh.sim.time_state
        assert (ts.t, ts.dt, ts.nstep) == (st.t, st.dt, st.nstep)
        for i in sh.mine:
            for k, (x, y) in enumerate(zip(sh.download(i), ref[i])):
                if x is not None:
                    assert_bitexact(x, y, f"block {i} array {k} on rank {sh.rank}")
            seen.add(i)
        sh.close()
    assert seen == set(range(len(data)))
