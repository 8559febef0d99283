"""The same-level guard exchange plan (piernik_b200/csrc/pk_exchange.cpp,
cg_list_bnd.F90:251-324) against a brute-force cell-by-cell construction:
every guard cell whose position, wrapped along periodic directions, lies in
some block's interior is filled exactly once, from exactly that cell; no
interior cell is ever a target; overlapping blocks are rejected."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "native", "xchg_harness.cpp")
PLAN = os.path.join(HERE, "..", "piernik_b200", "csrc", "pk_exchange.cpp")
LIB = os.path.join(HERE, "native", "libxchg_harness.so")


@pytest.fixture(scope="module")
def lib():
    if (not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(SRC), os.path.getmtime(PLAN))):
        subprocess.check_call(["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-o", LIB, SRC, PLAN])
    L = C.CDLL(LIB)
    L.xchg_plan.restype = C.c_int
    return L


def plan(lib, blocks, dom, periodic, g=4):
    nb = len(blocks)
    n = (C.c_int * (3 * nb))(*[x for b in blocks for x in b[0]])
    gg = (C.c_int * (3 * nb))(*[(g if b[0][d] > 1 else 0) for b in blocks for d in range(3)])
    off = (C.c_longlong * (3 * nb))(*[x for b in blocks for x in b[1]])
    dm = (C.c_longlong * 3)(*dom)
    per = (C.c_int * 3)(*[int(p) for p in periodic])
    cap = 64 * nb * nb + 64
    segs = (C.c_int * (11 * cap))()
    err = C.create_string_buffer(256)
    k = lib.xchg_plan(nb, n, gg, off, dm, per, segs, cap, err, 256)
    if k < 0:
        raise ValueError(err.value.decode())
    return np.array(segs[:11 * k]).reshape(k, 11)


def brute(blocks, dom, periodic, g=4):
    """{(dst, i, j, k): (src, si, sj, sk)} from cell-by-cell search."""
    out = {}
    for t, (n, off) in enumerate(blocks):
        gt = [g if n[d] > 1 else 0 for d in range(3)]
        for k in range(n[2] + 2 * gt[2]):
            for j in range(n[1] + 2 * gt[1]):
                for i in range(n[0] + 2 * gt[0]):
                    loc = (i, j, k)
                    if all(gt[d] <= loc[d] < gt[d] + n[d] for d in range(3)):
                        continue
                    glob = [off[d] - gt[d] + loc[d] for d in range(3)]
                    ok = True
                    for d in range(3):
                        if periodic[d]:
                            glob[d] %= dom[d]
                        elif not 0 <= glob[d] < dom[d]:
                            ok = False
                    if not ok:
                        continue
                    for s, (ns, offs) in enumerate(blocks):
                        if all(offs[d] <= glob[d] < offs[d] + ns[d] for d in range(3)):
                            gs = [g if ns[d] > 1 else 0 for d in range(3)]
                            out[(t,) + loc] = (s,) + tuple(glob[d] - offs[d] + gs[d] for d in range(3))
                            break
    return out


def expand(segs):
    out = {}
    for r in segs:
        dst, src = int(r[0]), int(r[1])
        lo, hi, sh = r[2:5], r[5:8], r[8:11]
        for k in range(lo[2], hi[2]):
            for j in range(lo[1], hi[1]):
                for i in range(lo[0], hi[0]):
                    key = (dst, i, j, k)
                    assert key not in out, f"guard cell {key} filled twice"
                    out[key] = (src, i + sh[0], j + sh[1], k + sh[2])
    return out


def tiling(xs, ys, zs):
    blocks = []
    oz = 0
    for bz in zs:
        oy = 0
        for by in ys:
            ox = 0
            for bx in xs:
                blocks.append(((bx, by, bz), (ox, oy, oz)))
                ox += bx
            oy += by
        oz += bz
    return blocks, (sum(xs), sum(ys), sum(zs))


@pytest.mark.parametrize("periodic", [(1, 1, 1), (0, 1, 1), (0, 0, 0)])
def test_plan_matches_brute_force_3d(lib, periodic):
    blocks, dom = tiling([6, 9], [5, 7], [8])
    got = expand(plan(lib, blocks, dom, periodic))
    assert got == brute(blocks, dom, periodic)


def test_plan_single_periodic_block_is_wrap(lib):
    blocks = [((7, 6, 5), (0, 0, 0))]
    got = expand(plan(lib, blocks, (7, 6, 5), (1, 1, 1)))
    want = brute(blocks, (7, 6, 5), (1, 1, 1))
    assert got == want
    # every guard cell of a periodic single block has a source
    assert len(got) == 15 * 14 * 13 - 7 * 6 * 5


def test_plan_2d_and_holes(lib):
    blocks = [((8, 6, 1), (0, 0, 0)), ((8, 6, 1), (8, 6, 0)), ((5, 6, 1), (16, 0, 0))]
    dom = (21, 12, 1)
    for periodic in [(1, 1, 0), (0, 1, 0)]:
        assert expand(plan(lib, blocks, dom, periodic)) == brute(blocks, dom, periodic)


def test_plan_rejects_overlap_and_escape(lib):
    with pytest.raises(ValueError, match="overlap"):
        plan(lib, [((8, 8, 8), (0, 0, 0)), ((8, 8, 8), (4, 0, 0))], (16, 8, 8), (1, 1, 1))
    with pytest.raises(ValueError, match="leaves the domain"):
        plan(lib, [((8, 8, 8), (12, 0, 0))], (16, 8, 8), (1, 1, 1))


def peer_lists(lib, blocks, owners, rank, peer, which, dom, periodic, g=4):
    """Rank `rank`'s view: its blocks first, then the others with owners."""
    order = [i for i in range(len(blocks)) if owners[i] == rank] + [i for i in range(len(blocks)) if owners[i] != rank]
    nl = sum(1 for o in owners if o == rank)
    bl = [blocks[i] for i in order]
    own = [(-1 if owners[i] == rank else owners[i]) for i in order]
    nb = len(bl)
    n = (C.c_int * (3 * nb))(*[x for b in bl for x in b[0]])
    gg = (C.c_int * (3 * nb))(*[(g if b[0][d] > 1 else 0) for b in bl for d in range(3)])
    off = (C.c_longlong * (3 * nb))(*[x for b in bl for x in b[1]])
    ow = (C.c_int * nb)(*own)
    out = (C.c_longlong * (12 * 4096))()
    k = lib.xchg_peer(nb, nl, ow, n, gg, off, (C.c_longlong * 3)(*dom), (C.c_int * 3)(*[int(p) for p in periodic]),
                      peer, which, out, 4096)
    assert k >= 0
    return [tuple(out[12 * i:12 * i + 12]) for i in range(k)]


@pytest.mark.parametrize("nranks", [2, 3])
def test_peer_order_agrees_between_ranks(lib, nranks):
    """What rank s sends to rank r is what r receives from s, in the same
    order, although each rank numbers the blocks differently."""
    lib.xchg_peer.restype = C.c_int
    blocks, dom = tiling([6, 9, 5], [5, 7], [8, 4])
    owners = [i % nranks for i in range(len(blocks))]
    for r in range(nranks):
        for s in range(nranks):
            if r == s:
                continue
            recv = peer_lists(lib, blocks, owners, r, s, 0, dom, (1, 1, 1))
            send = peer_lists(lib, blocks, owners, s, r, 1, dom, (1, 1, 1))
            assert recv == send and len(recv) > 0
