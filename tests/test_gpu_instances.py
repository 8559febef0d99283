"""Independent instances stacked along z in one block (pk_set_instances).

Each instance is a fully periodic problem of its own; one launch per sweep
advances all of them, each with its own CFL time step, chspeed and damping.
The result of every instance must equal, bit for bit, a handle holding that
instance alone: states, time states and (on the differentiable path) the
gradient of the same loss.
"""
import numpy as np
import pytest

from helpers import assert_bitexact, random_state, setup_for, smooth_state, to_soa
from piernik_b200._lib import PK_LAYOUT_SOA, PkError
from piernik_b200.config import BND_OUT, BND_PER
from piernik_b200.sim import Simulation

pytestmark = pytest.mark.gpu

N1 = (16, 12, 10)     # one instance
NI = 3


def put(sim, x):
    s = sim.setup
    nv = s.nvar
    if s.magnetic:
        sim.upload(np.ascontiguousarray(x[:nv]), np.ascontiguousarray(x[nv:nv + 3]),
                   np.ascontiguousarray(x[nv + 3]), layout=PK_LAYOUT_SOA)
    else:
        sim.upload(np.ascontiguousarray(x[:nv]), layout=PK_LAYOUT_SOA)


def get(sim):
    u, b, psi = sim.download(layout=PK_LAYOUT_SOA)
    return np.concatenate([u] + ([b, psi[None]] if sim.setup.magnetic else []), 0)


def inner(s, x, i=None, seg=None):
    g, n = s.guards, s.n
    if i is None:
        return x[:, g[2]:g[2] + n[2], g[1]:g[1] + n[1], g[0]:g[0] + n[0]]
    return x[:, g[2] + i * seg:g[2] + (i + 1) * seg, g[1]:g[1] + n[1], g[0]:g[0] + n[0]]


def stack(S, s1, xs):
    """Per-instance SoA states -> the stacked block's SoA state."""
    X = np.zeros((xs[0].shape[0],) + tuple(S.ext[::-1]))
    for i, x in enumerate(xs):
        inner(S, X, i, s1.n[2])[...] = inner(s1, x)
    return X


def states(s1, kind, seeds, scale):
    xs = []
    for sd, f in zip(seeds, scale):
        u, b, psi = (random_state if kind == "random" else smooth_state)(s1, seed=sd)
        # a faster flow in some instances gives them clearly different time steps
        mom = slice(1, 4)
        ek0 = 0.5 * (u[..., mom] ** 2).sum(-1) / u[..., 0]
        u[..., mom] *= f
        u[..., 4] += 0.5 * (u[..., mom] ** 2).sum(-1) / u[..., 0] - ek0
        xs.append(to_soa(s1, u, b, psi))
    return xs


@pytest.mark.parametrize("phys", ["hd", "mhd"])
@pytest.mark.parametrize("graph", [False, True])
def test_instances_equal_separate_runs(gpu_lib, phys, graph):
    s1 = setup_for(phys, n=N1, lim="vanleer")
    S = setup_for(phys, n=(N1[0], N1[1], NI * N1[2]), lim="vanleer")
    xs = states(s1, "random", [11, 12, 13], [1.0, 2.5, 0.5])
    big = Simulation(S)
    put(big, stack(S, s1, xs))
    big.set_instances(NI)
    if graph:
        big.use_graph(True)
    big.run(6)
    out = get(big)
    dts = set()
    for i in range(NI):
        one = Simulation(s1)
        put(one, xs[i])
        one.run(6)
        assert_bitexact(inner(S, out, i, N1[2]), inner(s1, get(one)), f"instance {i}")
        a, b = big.instance_state(i), one.time_state
        assert (a.t, a.dt, a.nstep, a.chspeed, a.c_all) == (b.t, b.dt, b.nstep, b.chspeed, b.c_all), f"instance {i}"
        dts.add(a.dt)
        one.close()
    assert len(dts) == NI, "the instances should take different time steps"
    big.close()


def test_instances_rejects(gpu_lib):
    S = setup_for("mhd", n=(16, 12, 30), lim="vanleer")
    big = Simulation(S)
    with pytest.raises(PkError):
        big.set_instances(4)               # 30 planes do not split in 4
    with pytest.raises(PkError):
        big.set_instances(10)              # 3 planes per instance < nb
    big.close()
    S2 = setup_for("hd", n=(16, 12, 30), lim="vanleer", bnd=((BND_PER, BND_PER), (BND_PER, BND_PER), (BND_OUT, BND_OUT)))
    big = Simulation(S2)
    with pytest.raises(PkError):
        big.set_instances(3)               # outflow along z
    big.close()


def test_instances_gradient_equals_separate(gpu_lib):
    """The checkpointed adjoint over stacked instances (each with its own dt
    sequence) gives every instance the gradient of a separate handle."""
    s1 = setup_for("mhd", n=N1, lim="vanleer")
    S = setup_for("mhd", n=(N1[0], N1[1], NI * N1[2]), lim="vanleer")
    xs = states(s1, "smooth", [21, 22, 23], [1.0, 1.8, 0.6])
    rng = np.random.default_rng(5)
    ws = [rng.standard_normal(x.shape) for x in xs]
    K = 5
    big = Simulation(S)
    put(big, stack(S, s1, xs))
    big.set_instances(NI)
    dts = big.grad_forward(K, 2)
    assert dts.shape == (K, NI)
    big.adjoint_set(stack(S, s1, ws))
    big.grad_backward()
    g = big.adjoint_get()
    for i in range(NI):
        one = Simulation(s1)
        put(one, xs[i])
        d1 = one.grad_forward(K, 2)
        assert np.array_equal(d1, dts[:, i]), f"instance {i} dt sequence"
        one.adjoint_set(ws[i])
        one.grad_backward()
        assert_bitexact(inner(S, g, i, N1[2]), inner(s1, one.adjoint_get()), f"gradient of instance {i}")
        one.close()
    big.close()
