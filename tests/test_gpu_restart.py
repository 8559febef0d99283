"""Restart files (piernik_b200.restart, the reference's restart_hdf5_v2
contents in a NumPy archive): a run saved after some steps and resumed from
the file must continue exactly as the uninterrupted run -- states with guard
cells and time states bit for bit -- for one block, a refined domain and
stacked instances."""
import numpy as np
import pytest

from helpers import assert_bitexact, random_state, setup_for
from piernik_b200 import problems, restart
from piernik_b200.sim import Simulation
from test_gpu_instances import N1, NI, put, stack, states

pytestmark = pytest.mark.gpu

DOM3 = (16, 16, 16)
REG3 = [((8, 8, 8), (24, 24, 24)), ((24, 24, 24), (40, 40, 40))]


def same_run(a, b):
    assert sorted(a.blocks) == sorted(b.blocks)
    for i in a.blocks:
        for x, y, name in zip(a.download(block=i), b.download(block=i), ("u", "b", "psi")):
            if x is not None:
                assert_bitexact(x, y, f"{name} of block {i}")
    sa, sb = a.time_state, b.time_state
    for name, _ in type(sa)._fields_:
        assert getattr(sa, name) == getattr(sb, name), name


def resume_equals(sim, path, before=3, after=3):
    sim.run(before)
    restart.save(sim, path)
    sim.run(after)
    back = restart.load(path)
    back.run(after)
    same_run(sim, back)
    return back


def test_restart_one_block(gpu_lib, tmp_path):
    s = setup_for("mhd", n=(24, 20, 16), lim="moncen", cflcontrol="redo")
    sim = Simulation(s)
    sim.upload(*random_state(s, seed=4))
    resume_equals(sim, str(tmp_path / "one.npz")).close()
    sim.close()


def test_restart_refined(gpu_lib, tmp_path):
    layout = problems.refined_layout(DOM3, REG3, sizes=(8, 16), seed=3)
    setup = setup_for("mhd", n=(8, 8, 8))
    blocks = problems.refined_blocks(DOM3, layout, setup, problems.wave_fields(DOM3, seed=5))
    sim = Simulation(blocks[0][0])
    for s, *_ in blocks[1:]:
        sim.add_block(s)
    sim.set_domain(DOM3, (True, True, True))
    for i, (s, L, off, u, b, psi) in enumerate(blocks):
        sim.place_block(i, off, L)
        sim.upload(u, b, psi, block=i)
    sim.update_boundaries()
    back = resume_equals(sim, str(tmp_path / "refined.npz"), before=2, after=2)
    assert back.placement == sim.placement and back.domain == sim.domain
    back.close()
    sim.close()


def test_restart_instances(gpu_lib, tmp_path):
    s1 = setup_for("hd", n=N1)
    S = setup_for("hd", n=(N1[0], N1[1], NI * N1[2]))
    sim = Simulation(S)
    put(sim, stack(S, s1, states(s1, "random", [21, 22, 23], [1.0, 2.0, 0.7])))
    sim.set_instances(NI)
    back = resume_equals(sim, str(tmp_path / "inst.npz"), before=2, after=2)
    for k in range(NI):
        a, b = sim.instance_state(k), back.instance_state(k)
        assert (a.t, a.dt, a.nstep) == (b.t, b.dt, b.nstep)
    back.close()
    sim.close()


def test_restart_after_removing_block0(gpu_lib, tmp_path):
    """Block 0 removed (derefined) before the save: the new block 0 is a base
    block with another cell size and level than the Setup the run was made
    with, and the resumed run must still continue bit for bit."""
    layout = problems.refined_layout(DOM3, REG3[:1], sizes=(8, 16), seed=3)
    setup = setup_for("mhd", n=(8, 8, 8))
    blocks = problems.refined_blocks(DOM3, layout, setup, problems.wave_fields(DOM3, seed=5))
    fine = [i for i, x in enumerate(blocks) if x[1] == 1]
    assert fine
    order = [fine[0]] + [i for i in range(len(blocks)) if i != fine[0]]
    blocks = [blocks[i] for i in order]            # a level-1 block is block 0
    sim = Simulation(blocks[0][0])
    for s, *_ in blocks[1:]:
        sim.add_block(s)
    sim.set_domain(DOM3, (True, True, True))
    for i, (s, L, off, u, b, psi) in enumerate(blocks):
        sim.place_block(i, off, L)
        sim.upload(u, b, psi, block=i)
    sim.update_boundaries()
    sim.run(1)
    sim.restrict()
    sim.remove_block(0)
    sim.update_boundaries()
    assert sim.placement[0][1] == 0 and sim.blocks[0].dl != sim.setup.dl
    back = resume_equals(sim, str(tmp_path / "removed0.npz"), before=1, after=2)
    assert back.placement == sim.placement
    back.close()
    sim.close()
