"""CPU emulation of the sweep kernels' index arithmetic.

For every launch shape the library can produce for the given block sizes
(fused tiles of every variant the autotuner tries, the whole-pencil and
chunked stage tiles), each thread's global offset and every shared-memory
slot it reads are computed exactly as the kernels do and checked to be in
bounds; owned cells must be updated.  This runs before any GPU sees a new
tile shape.  Mirrors k_sweep_fused / k_stage / k_stage_batched / k_unsplit_flux in
piernik_b200/csrc/pk_kernels.cuh and launch_fused / launch_stage /
launch_unsplit_flux / build_batch in pk_launch.cuh and pk_api.cu.
"""
import pytest

ORTHO1 = [1, 0, 0]
ORTHO2 = [2, 2, 1]
STAGE_MAXT = 320
UNSPLIT_MAXT = 256
SV_T = [320, 128, 192, 384]             # launch shapes of the batched stage kernel
VARIANT_T = [320, 256, 256, 128, 128, 192, 512]


def geom(n, nb, d):
    g = [nb if x > 1 else 0 for x in n]
    ext = [n[k] + 2 * g[k] for k in range(3)]
    st = [1, ext[0], ext[0] * ext[1]]
    o1, o2 = ORTHO1[d], ORTHO2[d]
    return dict(plane=ext[0] * ext[1] * ext[2], sd=st[d], s1=st[o1], s2=st[o2], ext_d=ext[d], n_d=n[d],
                g_d=g[d], n1=n[o1], g1=g[o1], n2=n[o2], g2=g[o2])


def fused_shape(n, d, P, L, maxt):
    G = geom(n, 4, d)
    L = min(L, n[d])
    P = min(P, G["n1"])
    circ = L == n[d] and n[d] <= maxt            # whole periodic pencil, no halo (Tile::circ)
    T = L if circ else L + 8
    while P * T > maxt and P > 1:
        P -= 1
    assert P * T <= maxt
    return G, P, L, T, circ


def check_fused(n, d, P, L, maxt):
    G, P, L, T, circ = fused_shape(n, d, P, L, maxt)
    PT = P * T
    xfast = d == 0
    covered = set()
    for bx in range((G["n1"] + P - 1) // P):
        for by in range((n[d] + L - 1) // L):
            for bz in sorted({0, G["n2"] - 1}):
                for tid in range(PT):
                    t, p = (tid % T, tid // T) if xfast else (tid // P, tid % P)
                    sp, st = (T, 1) if xfast else (1, P)
                    me = p * sp + t * st
                    assert 0 <= me < PT
                    i1 = bx * P + p
                    if i1 >= G["n1"]:
                        continue
                    s = t if circ else by * L - 4 + t
                    w = s % G["n_d"]
                    off = (G["g_d"] + w) * G["sd"] + (G["g1"] + i1) * G["s1"] + (G["g2"] + bz) * G["s2"]
                    assert 0 <= off < G["plane"]
                    if circ:
                        mp = p * sp + ((t - 1) % T) * st
                        mn = p * sp + ((t + 1) % T) * st
                        assert 0 <= mp < PT and 0 <= mn < PT
                        if bz == 0:
                            covered.add((i1, s))
                        continue
                    for lo, hi in ((0, T), (2, T - 2)):
                        if lo < t < hi - 1:
                            assert me - st >= 0 and me + st < PT
                        if lo + 1 <= t < hi - 2:
                            assert me + st < PT
                        if lo + 2 <= t < hi - 2:
                            assert me - st >= 0
                    if 4 <= t < T - 4 and s < by * L + L and s < G["n_d"] and bz == 0:
                        covered.add((i1, s))
    assert len(covered) == G["n1"] * G["n_d"]


def check_stage(n, d):
    G = geom(n, 4, d)
    ext = G["ext_d"]
    if ext <= STAGE_MAXT:
        P = STAGE_MAXT // ext
        if P >= 4:
            P -= P % 4
        P = min(P, G["n1"])
        T, L, halo = ext, ext, 0
    else:
        P, L, T, halo = 4, 64, 68, 2
    PT = P * T
    xfast = d == 0
    for bx in range((G["n1"] + P - 1) // P):
        for by in range((ext + L - 1) // L):
            for bz in sorted({0, G["n2"] - 1}):
                for tid in range(PT):
                    t, p = (tid % T, tid // T) if xfast else (tid // P, tid % P)
                    sp, st = (T, 1) if xfast else (1, P)
                    me = p * sp + t * st
                    i1 = bx * P + p
                    c0 = by * L
                    s = c0 - halo + t
                    if not (i1 < G["n1"] and 0 <= s < ext):
                        continue
                    off = s * G["sd"] + (G["g1"] + i1) * G["s1"] + (G["g2"] + bz) * G["s2"]
                    assert 0 <= off < G["plane"]
                    end = -1 if s == 0 else (1 if s == ext - 1 else 0)
                    slope = end != 0 or (1 <= t <= T - 2)
                    next_slope = s + 1 < ext and t + 1 <= T - 1 and (s + 1 == ext - 1 or t + 1 <= T - 2)
                    flux = slope and next_slope
                    prev_flux = t >= 1 and s >= 1 and (s - 1 == 0 or t - 1 >= 1)
                    upd = 1 <= s <= ext - 2 and prev_flux and flux
                    if slope:
                        if end < 0:
                            assert me + st < PT
                        elif end > 0:
                            assert me - st >= 0
                        else:
                            assert me - st >= 0 and me + st < PT
                    if flux:
                        assert me + st < PT
                    if upd:
                        assert me - st >= 0
                    if c0 <= s < c0 + L and 1 <= s <= ext - 2:
                        assert upd


def roles_ok(ext, T, t, s, me, st, PT):
    """the neighbour slots rk_stage reads for a tile cell are inside the tile"""
    end = -1 if s == 0 else (1 if s == ext - 1 else 0)
    slope = end != 0 or (1 <= t <= T - 2)
    next_slope = s + 1 < ext and t + 1 <= T - 1 and (s + 1 == ext - 1 or t + 1 <= T - 2)
    flux = slope and next_slope
    prev_flux = t >= 1 and s >= 1 and (s - 1 == 0 or t - 1 >= 1)
    upd = 1 <= s <= ext - 2 and prev_flux and flux
    if slope:
        if end < 0:
            assert me + st < PT
        elif end > 0:
            assert me - st >= 0
        else:
            assert me - st >= 0 and me + st < PT
    if flux:
        assert me + st < PT
    if upd:
        assert me - st >= 0
    return flux, upd


def check_stage_batched(n, d, maxt):
    """k_stage_batched: tiles [g-2, g+n+2) of P pencils taken in i1-fastest
    order across the rows of the block face; every interior cell updated"""
    G = geom(n, 4, d)
    ext, T = G["ext_d"], n[d] + 4
    face = G["n1"] * G["n2"]
    P = min(maxt // T, face)
    PT = P * T
    assert PT <= maxt and 3 * 18 * PT * 8 <= 220 * 1024
    xfast = d == 0
    updated = set()
    for q0 in range(0, face, P):
        for tid in range(PT):
            t, p = (tid % T, tid // T) if xfast else (tid // P, tid % P)
            sp, st = (T, 1) if xfast else (1, P)
            me = p * sp + t * st
            assert 0 <= me < PT
            q = q0 + p
            if q >= face:
                continue
            i2, i1 = divmod(q, G["n1"])
            s = G["g_d"] - 2 + t
            if not 0 <= s < ext:
                continue
            off = s * G["sd"] + (G["g1"] + i1) * G["s1"] + (G["g2"] + i2) * G["s2"]
            assert 0 <= off < G["plane"]
            _, upd = roles_ok(ext, T, t, s, me, st, PT)
            if upd and G["g_d"] <= s < G["g_d"] + n[d]:
                updated.add((i1, i2, s))
    assert len(updated) == face * n[d]


def check_unsplit(n, d):
    """k_unsplit_flux: whole pencils where they fit, else 4 x (60 + 4) chunks;
    the flux through every face between two cells of the pencil is stored once"""
    G = geom(n, 4, d)
    ext = G["ext_d"]
    if ext <= UNSPLIT_MAXT and (d == 0 or UNSPLIT_MAXT // ext >= 4 or G["n1"] < 4):
        P = UNSPLIT_MAXT // ext
        if P >= 4:
            P -= P % 4
        P = min(P, G["n1"])
        T, L, halo = ext, ext, 0
    else:
        P, L, halo = 4, UNSPLIT_MAXT // 4 - 4, 2
        T = L + 4
    PT = P * T
    assert PT <= UNSPLIT_MAXT
    xfast = d == 0
    stored = {}
    for bx in range((G["n1"] + P - 1) // P):
        for by in range((ext + L - 1) // L):
            for tid in range(PT):
                t, p = (tid % T, tid // T) if xfast else (tid // P, tid % P)
                sp, st = (T, 1) if xfast else (1, P)
                me = p * sp + t * st
                i1 = bx * P + p
                c0 = by * L
                s = c0 - halo + t
                if not (i1 < G["n1"] and 0 <= s < ext):
                    continue
                off = s * G["sd"] + (G["g1"] + i1) * G["s1"] + G["g2"] * G["s2"]
                assert 0 <= off < G["plane"]
                flux, _ = roles_ok(ext, T, t, s, me, st, PT)
                if flux and c0 <= s < c0 + L:
                    assert 0 <= off + G["sd"] < G["plane"]
                    stored[(i1, s)] = stored.get((i1, s), 0) + 1
    assert all(v == 1 for v in stored.values())
    assert len(stored) == G["n1"] * (ext - 1)


CASES = [(12, 10, 8), (20, 14, 11), (50, 37, 29), (400, 6, 5), (24, 17, 9), (32, 32, 1), (9, 8, 7),
         (64, 64, 64), (16, 24, 48)]


@pytest.mark.parametrize("n", CASES)
def test_stage_kernel_indexing(n):
    for d in range(3):
        if n[d] > 1:
            check_stage(n, d)


@pytest.mark.parametrize("n", CASES)
def test_fused_kernel_indexing(n):
    from piernik_b200.autotune import LENGTHS
    for d in range(3):
        if n[d] <= 1:
            continue
        balanced = tuple(sorted({-(-n[d] // k) for k in (2, 3, 5, 7) if -(-n[d] // k) >= 8}))
        for maxt in sorted(set(VARIANT_T)):
            for L in LENGTHS[:6] + (8, 16) + balanced:
                for P in (1, 2, 3, 4, 5, 7, 8):
                    if L + 8 <= maxt:
                        check_fused(n, d, P, L, maxt)


BATCH_CASES = [(16, 16, 16), (24, 64, 48), (64, 64, 64), (48, 16, 32), (40, 36, 28), (8, 8, 8), (16, 24, 1)]


@pytest.mark.parametrize("n", BATCH_CASES)
def test_stage_batched_kernel_indexing(n):
    for d in range(3):
        if n[d] > 1:
            for maxt in SV_T:
                if n[d] + 4 <= maxt:
                    check_stage_batched(n, d, maxt)


@pytest.mark.parametrize("n", [(12, 10, 8), (50, 37, 29), (264, 6, 5), (64, 64, 64), (16, 300, 6), (32, 32, 1)])
def test_unsplit_flux_kernel_indexing(n):
    for d in range(3):
        if n[d] > 1:
            check_unsplit(n, d)


# ---------------------------------------------------------------------------
# k_sweep_staged (pk_staged.cuh): TMA box per CTA and the shared-memory slots
# ---------------------------------------------------------------------------
def staged_ok(n, g, ext, nplanes, d):
    """staged_ok in pk_staged.cuh"""
    if n[d] > 256 or n[d] < 2 or nplanes > 256:
        return False
    if ext[0] % 2 or g[0] % 2:
        return False
    if d == 0 and n[0] % 2:
        return False
    return True


def check_staged(n, nb, d, nv):
    g = [nb if x > 1 else 0 for x in n]
    ext = [n[k] + 2 * g[k] for k in range(3)]
    if not staged_ok(n, g, ext, nv, d):
        return False
    o1, o2 = ORTHO1[d], ORTHO2[d]
    nd, n1, n2 = n[d], n[o1], n[o2]
    box = [0, 0, 0, nv]
    box[d], box[o1], box[o2] = nd, 2, 1
    # the tensor map: strides multiples of 16 bytes, the inner box row a multiple of 16 bytes
    assert (ext[0] * 8) % 16 == 0 and (ext[0] * ext[1] * 8) % 16 == 0
    assert (box[0] * 8) % 16 == 0 and all(1 <= b <= 256 for b in box)
    threads = (nd + 31) // 32 * 32
    assert threads <= 256
    smem_doubles = 5 * nv * nd
    bar_off = 5 * nv * nd * 8
    assert bar_off % 8 == 0 and bar_off + 8 <= smem_doubles * 8 + 16
    st_t, st_p = (1, nd) if d == 0 else (2, 1)
    stored = set()
    nbx = (n1 + 1) // 2
    full = n[0] * n[1] * n[2] <= 200000          # larger blocks: the edge CTAs only
    for bx in (range(nbx) if full else sorted({0, 1, nbx - 1})):
        for bz in (range(n2) if full else sorted({0, n2 - 1})):
            c = [0, 0, 0, 0]
            c[d], c[o1], c[o2] = g[d], g[o1] + 2 * bx, g[o2] + bz
            assert (c[0] * 8) % 16 == 0                      # TMA: x coordinate on a 16-byte boundary
            for k in range(3):                               # the box lies inside the array (guards included)
                assert 0 <= c[k] and c[k] + box[k] <= ext[k], (c, box, ext)
            for p in range(2):
                if 2 * bx + p >= n1:
                    break
                for t in range(threads):
                    if t >= nd:
                        continue
                    for v in range(nv):
                        idx = v * 2 * nd + t * st_t + p * st_p
                        assert 0 <= idx < 2 * nv * nd
                        # the box element order (x fastest, then y, z, plane) holds this cell there
                        e = [0, 0, 0, v]
                        e[d], e[o1], e[o2] = t, p, 0
                        assert idx == ((e[3] * box[2] + e[2]) * box[1] + e[1]) * box[0] + e[0]
                    for nb_ in ((t - 1) % nd, (t + 1) % nd):          # circular neighbours in the Q/L/R planes
                        assert 0 <= nb_ < nd
                    cell = [0, 0, 0]
                    cell[d], cell[o1], cell[o2] = t, 2 * bx + p, bz
                    assert tuple(cell) not in stored
                    stored.add(tuple(cell))
    if full:
        assert len(stored) == n[0] * n[1] * n[2]
    return True


@pytest.mark.parametrize("n", [(256, 256, 256), (50, 37, 29), (48, 31, 20), (64, 48, 1), (36, 30, 22), (8, 8, 8)])
@pytest.mark.parametrize("d", [0, 1, 2])
@pytest.mark.parametrize("nv", [5, 9, 18])
def test_staged_indexing(n, d, nv):
    if n[d] == 1:
        return
    if n == (256, 256, 256) and nv != 9:
        return
    ok = check_staged(n, 4, d, nv)
    assert ok == staged_ok(n, [4 if x > 1 else 0 for x in n], [x + 8 if x > 1 else 1 for x in n], nv, d)


def test_staged_refused_for_odd_x():
    """An odd x extent or guard width would put a TMA row off a 16-byte boundary."""
    assert not staged_ok((51, 40, 40), (4, 4, 4), (59, 48, 48), 9, 1)
    assert not staged_ok((50, 40, 40), (3, 3, 3), (56, 46, 46), 9, 2)
    assert not staged_ok((300, 40, 40), (4, 4, 4), (308, 48, 48), 9, 0)
