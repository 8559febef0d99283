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
    out = [(r.layout[r.rank], r.sim.download(), r.sim.time_state, r.exchanges) for r in ranks]
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
        assert nex >= 3 * 6 * (1 if order == 2 else 1)
        for k in range(3):
            if arrs[k] is None:
                continue
            mine = arrs[k][g[2]:g[2] + n[2], g[1]:g[1] + n[1], g[0]:g[0] + n[0]]
            want = ref[k][tuple(slice(g[d] + off[d], g[d] + off[d] + n[d]) for d in (2, 1, 0))]
            assert_bitexact(mine, want, f"{phys} slab {off} array {k}")
