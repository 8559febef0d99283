"""Refinement criteria on the GPU (pk_mark_refinement, pk_refine_map,
pk_refine_candidates) against the oracle's restatement of URC_var.F90 and
refinemap2SFC_list, bit for bit: flag maps with guard cells, the per-block
derefinement inhibition and the candidate lists, on one periodic block and
on a three-level refined domain (leaf masks)."""
import numpy as np
import pytest

import amr
import oracle as O
import urc
from helpers import setup_for
from piernik_b200 import problems
from piernik_b200.sim import Simulation

pytestmark = pytest.mark.gpu

DOM3 = (16, 16, 16)
REG3 = [((8, 8, 8), (24, 24, 24)), ((24, 24, 24), (40, 40, 40))]
DOM2 = (16, 16, 1)
REG2 = [((8, 6, 0), (24, 22, 1)), ((22, 18, 0), (38, 34, 1))]


def pick(mark, target=0.3):
    """a threshold flagging about ``target`` of the interior (oracle side):
    bisection in log space, the flagged fraction falling as thr grows"""
    lo, hi = -9.0, 6.0
    for _ in range(50):
        mid = 0.5 * (lo + hi)
        if mark(10.0 ** mid) > target:
            lo = mid
        else:
            hi = mid
    thr = 10.0 ** hi
    assert 0.0 < mark(thr) < 1.0
    return float(thr)


def criteria_for(ob, has, nv):
    """one criterion of each kind on density, energy-like and psi / momentum planes"""
    s = ob.setup
    g, n = s.guards, s.n

    def fr(c):                  # fraction of the interior flagged
        f = urc.field_of(ob, c[1])
        m = urc.mark_block(f, s.n, s.guards, s.dl, has, 0, [(c[0], f, c[2], c[3])])
        return m[g[2]:g[2] + n[2], g[1]:g[1] + n[1], g[0]:g[0] + n[0]].mean()
    out = []
    for method, f, aux in [(urc.LOECHNER, 0, 0.01), (urc.GRAD, 1, 0.0), (urc.RELGRAD, nv - 1, 0.0),
                           (urc.THRESHOLD, 0, 0.0)]:
        out.append((method, f, pick(lambda t: fr((method, f, t, aux))), aux))
    return out


@pytest.mark.parametrize("phys,n", [("mhd", (24, 16, 20)), ("hd", (32, 24, 1))])
def test_mark_single_block(gpu_lib, phys, n):
    s = setup_for(phys, n=n)
    u, b, psi = problems.wave_fields(tuple(n), seed=7)(s, *np.meshgrid(*[np.arange(e, dtype=float) for e in
                                                                           (s.ext[2], s.ext[1], s.ext[0])],
                                                                         indexing="ij")[::-1])
    ob = O.OracleBlock(s, u, b, psi)
    ob.fill_guards()
    has = tuple(x > 1 for x in n)
    crits = criteria_for(ob, has, s.nvar)
    sim = Simulation(s)
    sim.upload(u, b, psi)
    for sel in ([0], [1], [2], [3], [0, 1, 2, 3]):
        cr = [crits[k] for k in sel]
        want = urc.mark_block(ob.u[..., 0], s.n, s.guards, s.dl, has, 0,
                              [(m, urc.field_of(ob, f), t, a) for m, f, t, a in cr])
        flagged = sim.mark_refinement(cr)
        got = sim.refine_map(0)
        assert np.array_equal(got, want), sel
        g = s.guards
        assert flagged[0] == int(want[g[2]:g[2] + n[2], g[1]:g[1] + n[1], g[0]:g[0] + n[0]].any())
        bs = tuple(8 if x > 1 else 0 for x in n)
        assert sim.refine_candidates(0, bs) == urc.candidates(want, None, s.n, g, (0, 0, 0), bs, has)
    sim.close()


@pytest.mark.parametrize("dom,reg", [(DOM3, REG3), (DOM2, REG2)])
def test_mark_refined(gpu_lib, dom, reg):
    layout = problems.refined_layout(dom, reg, sizes=(8, 16), seed=3)
    setup = setup_for("mhd", n=tuple(8 if d > 1 else 1 for d in dom))
    blocks = problems.refined_blocks(dom, layout, setup, problems.blast_fields(centre=(9.0, 8.0, 8.5 if dom[2] > 1
                                                                                        else 0.0), radius=2.5))
    a = amr.AmrOracle(dom, blocks)
    a.fill_guards()
    a.run(2)
    a.fill_guards()
    sim = Simulation(blocks[0][0])
    for s, *_ in blocks[1:]:
        sim.add_block(s)
    sim.set_domain(dom, (True, True, True))
    for i, (s, L, off, u, b, psi) in enumerate(blocks):
        sim.place_block(i, off, L)
        sim.upload(u, b, psi, block=i)
    sim.update_boundaries()
    sim.run(2)
    nv = blocks[0][0].nvar
    crits = [(urc.LOECHNER, 4, 0.8, 0.01), (urc.RELGRAD, 0, 0.05, 0.0), (urc.THRESHOLD, nv - 1 + 4, 1e-4, 2.0)]
    maps, flagged = urc.mark_amr(a, crits)
    got = sim.mark_refinement(crits)
    assert list(got) == flagged and sum(flagged) > 0
    bs = tuple(8 if d > 1 else 0 for d in dom)
    ncand = 0
    for i, ob in enumerate(a.blocks):
        assert np.array_equal(sim.refine_map(i), maps[i]), i
        s = ob.setup
        want = urc.candidates(maps[i], a.leaf[i], s.n, s.guards, a.off[i], bs, a.has)
        assert sim.refine_candidates(i, bs) == want, i
        ncand += len(want)
    assert ncand > 0
    sim.close()


def test_mark_rejects(gpu_lib):
    s = setup_for("hd", n=(8, 8, 8), nb=2)
    sim = Simulation(s)
    with pytest.raises(Exception, match="nb >= 4"):
        sim.mark_refinement([(urc.LOECHNER, 0, 0.5, 0.01)])
    with pytest.raises(Exception, match="field"):
        sim.mark_refinement([(urc.GRAD, 99, 0.5, 0.0)])
    with pytest.raises(Exception, match="pk_mark_refinement first"):
        sim.refine_map(0)
    sim.close()
