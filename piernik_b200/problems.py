"""Seeded synthetic initial conditions for the benchmark configurations.

Arrays are returned in the reference's guard-cell layout (Fortran ``cg%u(v,i,j,k)``
seen from C as ``u[k, j, i, v]``, ``b[k, j, i, d]``, ``psi[k, j, i]``) with the
guard cells already filled periodically.  The recipes follow the reference's
problem setups where one exists (problems/sedov/initproblem.F90:179-292,
problems/otvortex/initproblem.F90:99-166); no external dataset is involved.
"""
from __future__ import annotations

import math
from typing import Optional, Tuple

import numpy as np

from .config import BND_PER, Setup


def _empty(setup: Setup):
    ez, ey, ex = setup.ext[2], setup.ext[1], setup.ext[0]
    u = np.zeros((ez, ey, ex, setup.nvar))
    b = np.zeros((ez, ey, ex, 3)) if setup.magnetic else None
    psi = np.zeros((ez, ey, ex)) if setup.magnetic else None
    return u, b, psi


def _centres(setup: Setup, d: int) -> np.ndarray:
    g = setup.guards[d]
    dl = setup.dl[d]
    i = np.arange(setup.ext[d]) - g
    return setup.xmin[d] + (i + 0.5) * dl


def fill_periodic(setup: Setup, arr: Optional[np.ndarray]) -> None:
    """Copy interior cells into guard cells periodically, x then y then z."""
    if arr is None:
        return
    g = setup.guards
    for d in range(3):
        if g[d] == 0:
            continue
        ax = 2 - d                    # array axis of direction d (k, j, i order)
        n = setup.n[d]
        sl = [slice(None)] * arr.ndim
        for ib in range(g[d]):
            lo_dst, lo_src = g[d] - 1 - ib, g[d] + n - 1 - ib
            hi_dst, hi_src = g[d] + n + ib, g[d] + ib
            for dst, src in ((lo_dst, lo_src), (hi_dst, hi_src)):
                a = list(sl)
                bsl = list(sl)
                a[ax] = dst
                bsl[ax] = src
                arr[tuple(a)] = arr[tuple(bsl)]


def _set_fluid(setup, u, f, rho, vx, vy, vz, p, emag=None):
    """Conservative variables of fluid index f from primitives (broadcasting)."""
    beg = sum(4 if k == "dst" else 5 for k, _ in setup.fluids[:f])
    kind, gam = setup.fluids[f]
    u[..., beg + 0] = rho
    u[..., beg + 1] = rho * vx
    u[..., beg + 2] = rho * vy
    u[..., beg + 3] = rho * vz
    if kind != "dst":
        e = p / (gam - 1.0) + 0.5 * rho * (vx * vx + vy * vy + vz * vz)
        if emag is not None:
            e = e + emag
        u[..., beg + 4] = e


def sedov(n: int = 64, r_cells: float = 3.5, e_total: float = 1.0, p0: float = 1.0e-5,
          gamma: float = 5.0 / 3.0, setup: Optional[Setup] = None):
    """3D Sedov blast, plain hydro (neutral fluid, no B), periodic box [-1,1]^3.

    Total energy ``e_total`` is deposited as thermal energy in cells whose 4^3
    sub-samples lie within ``r_cells`` cells of the centre, weighted per
    sub-sample as in problems/sedov/initproblem.F90:226-255.
    """
    if setup is None:
        setup = Setup(n=(n, n, n), fluids=[("neu", gamma)], magnetic=False, limiter="vanleer",
                      limiter_b="vanleer", cfl=0.7, cfl_glm=0.7, smalld=1.0e-3)
    u, _, _ = _empty(setup)
    x, y, z = (_centres(setup, d) for d in range(3))
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    _set_fluid(setup, u, 0, 1.0, 0.0, 0.0, 0.0, p0)
    dx = setup.dl[0]
    r0 = r_cells * dx
    isub = 4
    offs = (2 * np.arange(1, isub + 1) - isub - 1) / (2.0 * isub)
    frac = np.zeros(X.shape)
    for ox in offs:
        for oy in offs:
            for oz in offs:
                r = np.sqrt((X + ox * dx) ** 2 + (Y + oy * dx) ** 2 + (Z + oz * dx) ** 2)
                frac += (r < r0)
    frac /= isub ** 3
    g = setup.guards
    interior = frac[g[2]:g[2] + setup.n[2], g[1]:g[1] + setup.n[1], g[0]:g[0] + setup.n[0]]
    vol = float(np.prod(setup.dl))
    eexpl = e_total / (interior.sum() * vol)        # energy density of the deposit
    ien = 4
    u[..., ien] += eexpl * frac
    fill_periodic(setup, u)
    return setup, u, None, None


def _rng(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64(seed))


def _fourier_field(n: Tuple[int, int, int], kmin: float, kmax: float, slope: float,
                   rng: np.random.Generator, ncomp: int = 3) -> np.ndarray:
    """Real periodic field on an (nz, ny, nx) grid with random-phase modes of
    integer wavenumber kmin <= |k| <= kmax and amplitude |k|**slope."""
    nx, ny, nz = n
    kz = np.fft.fftfreq(nz, 1.0 / nz)[:, None, None]
    ky = np.fft.fftfreq(ny, 1.0 / ny)[None, :, None]
    kx = np.fft.rfftfreq(nx, 1.0 / nx)[None, None, :]
    kk = np.sqrt(kx * kx + ky * ky + kz * kz)
    mask = (kk >= kmin) & (kk <= kmax)
    out = np.empty((ncomp, nz, ny, nx))
    amp = np.where(mask, np.where(kk > 0, kk, 1.0) ** slope, 0.0)
    for c in range(ncomp):
        ph = rng.uniform(0.0, 2.0 * np.pi, size=kk.shape)
        spec = amp * np.exp(1j * ph)
        out[c] = np.fft.irfftn(spec, s=(nz, ny, nx), axes=(0, 1, 2))
    return out, (kx, ky, kz, mask)


def mhd_turbulence_fields(n: int = 256, seed: int = 1, mach: float = 1.0, b0: float = 0.2,
                          db_frac: float = 0.1, gamma: float = 5.0 / 3.0):
    """Interior fields (rho, v[3], B[3]; each (n, n, n) as [k, j, i]) and the
    uniform pressure p0 of the decaying-turbulence recipe: rho = 1 + 1% white
    noise (seed); v from random-phase Fourier modes with 1 <= |k| <= 4,
    amplitude ~ k^-2 (seed+1), scaled to rms Mach ``mach`` for the sound speed
    of p0 = 1/gamma (c_s = 1); B = (b0, 0, 0) + curl of a random vector
    potential (seed+2) scaled to rms ``db_frac * b0``."""
    p0 = 1.0 / gamma
    shp = (n, n, n)
    rho = 1.0 + 0.01 * _rng(seed).standard_normal((n, n, n))
    v, _ = _fourier_field(shp, 1.0, 4.0, -2.0, _rng(seed + 1))
    vrms = math.sqrt(float(np.mean(v[0] ** 2 + v[1] ** 2 + v[2] ** 2)))
    v *= mach * 1.0 / vrms
    a, (kx, ky, kz, mask) = _fourier_field(shp, 1.0, 4.0, -2.0, _rng(seed + 2))
    # curl of A, spectrally
    ah = [np.fft.rfftn(a[c]) for c in range(3)]
    bh = [1j * (ky * ah[2] - kz * ah[1]), 1j * (kz * ah[0] - kx * ah[2]), 1j * (kx * ah[1] - ky * ah[0])]
    db = np.stack([np.fft.irfftn(bh[c], s=shp, axes=(0, 1, 2)) for c in range(3)])
    dbrms = math.sqrt(float(np.mean(db[0] ** 2 + db[1] ** 2 + db[2] ** 2)))
    db *= db_frac * b0 / dbrms
    bf = np.stack([b0 + db[0], db[1], db[2]])
    return rho, v, bf, p0


def turbulence_setup(n: int, nz: Optional[int] = None, gamma: float = 5.0 / 3.0, limiter: str = "moncen",
                     cfl: float = 0.5) -> Setup:
    """The decaying-turbulence run on [0,1]^3 cells of 1/n (nz cells along z,
    default n: nz = count * n stacks count instances along z)."""
    nz = n if nz is None else nz
    return Setup(n=(n, n, nz), xmin=(0.0, 0.0, 0.0), xmax=(1.0, 1.0, nz / n),
                 fluids=[("ion", gamma)], magnetic=True, limiter=limiter, limiter_b=limiter,
                 cfl=cfl, cfl_glm=0.7, smalld=1.0e-3)


def mhd_turbulence(n: int = 256, seed: int = 1, mach: float = 1.0, b0: float = 0.2,
                   db_frac: float = 0.1, gamma: float = 5.0 / 3.0, limiter: str = "moncen",
                   cfl: float = 0.5):
    """3D ideal-MHD decaying turbulence on one periodic block (the fields of
    mhd_turbulence_fields, psi = 0)."""
    setup = turbulence_setup(n, gamma=gamma, limiter=limiter, cfl=cfl)
    rho, v, bf, p0 = mhd_turbulence_fields(n, seed, mach, b0, db_frac, gamma)
    g = setup.guards
    u, b, psi = _empty(setup)
    emag = 0.5 * (bf[0] * bf[0] + bf[1] * bf[1] + bf[2] * bf[2])
    sl = (slice(g[2], g[2] + n), slice(g[1], g[1] + n), slice(g[0], g[0] + n))
    ui = u[sl]
    _set_fluid(setup, ui, 0, rho, v[0], v[1], v[2], p0, emag)
    b[sl + (0,)] = bf[0]
    b[sl + (1,)] = bf[1]
    b[sl + (2,)] = bf[2]
    fill_periodic(setup, u)
    fill_periodic(setup, b)
    return setup, u, b, psi


def turbulence_ensemble(count: int = 64, n: int = 128, seed: int = 1):
    """Parameters of the batched-adjoint ensemble: instance i is the
    decaying-turbulence recipe at n^3 with seed seed + 10 i, rms Mach drawn
    log-uniform in [0.5, 5] and B0 uniform in [0.05, 0.5] (one generator
    seeded with ``seed``).  Returns a list of (seed, mach, b0)."""
    rng = _rng(seed + 7919)
    mach = np.exp(rng.uniform(math.log(0.5), math.log(5.0), size=count))
    b0 = rng.uniform(0.05, 0.5, size=count)
    return [(seed + 10 * i, float(mach[i]), float(b0[i])) for i in range(count)]


def orszag_tang(n: int = 512, seed: int = 1, amp: float = 1.0e-3, corr_cells: float = 8.0,
                limiter: str = "vanleer"):
    """2D Orszag-Tang vortex (problems/otvortex/initproblem.F90:99-166) on [0,1]^2
    with a seeded Gaussian-random density perturbation (amplitude ``amp``,
    Gaussian correlation length ``corr_cells`` cells)."""
    gamma = 5.0 / 3.0
    setup = Setup(n=(n, n, 1), xmin=(0.0, 0.0, -0.5), xmax=(1.0, 1.0, 0.5),
                  fluids=[("ion", gamma)], magnetic=True, limiter=limiter, limiter_b=limiter,
                  cfl=0.8, cfl_glm=0.7, smalld=1.0e-3, smallei=1.0e-5)
    u, b, psi = _empty(setup)
    x, y = _centres(setup, 0), _centres(setup, 1)
    Y, X = np.meshgrid(y, x, indexing="ij")
    rho0 = 25.0 / (36.0 * math.pi)
    pre = 5.0 / (12.0 * math.pi)
    b0 = 1.0 / math.sqrt(4.0 * math.pi)
    pert = gaussian_random_field((n, n), corr_cells, _rng(seed))
    g = setup.guards
    rho = np.full(X.shape, rho0)
    rho[g[1]:g[1] + n, g[0]:g[0] + n] *= 1.0 + amp * pert
    vx = -np.sin(2 * math.pi * Y)
    vy = np.sin(2 * math.pi * X)
    bx = b0 * vx
    by = b0 * np.sin(4 * math.pi * X)
    emag = 0.5 * (bx * bx + by * by)
    _set_fluid(setup, u[0], 0, rho, vx, vy, 0.0, pre, emag)
    b[0, ..., 0] = bx
    b[0, ..., 1] = by
    fill_periodic(setup, u)
    fill_periodic(setup, b)
    return setup, u, b, psi


def orszag_tang_fields(n: int):
    """Interior (ny, nx) fields of the unperturbed Orszag-Tang vortex and its
    scalars: (setup, rho0, pre, vx, vy, bx, by)."""
    gamma = 5.0 / 3.0
    setup = Setup(n=(n, n, 1), xmin=(0.0, 0.0, -0.5), xmax=(1.0, 1.0, 0.5),
                  fluids=[("ion", gamma)], magnetic=True, limiter="vanleer", limiter_b="vanleer",
                  cfl=0.8, cfl_glm=0.7, smalld=1.0e-3, smallei=1.0e-5)
    g = setup.guards
    x = _centres(setup, 0)[g[0]:g[0] + n]
    y = _centres(setup, 1)[g[1]:g[1] + n]
    Y, X = np.meshgrid(y, x, indexing="ij")
    b0 = 1.0 / math.sqrt(4.0 * math.pi)
    vx = -np.sin(2 * math.pi * Y)
    vy = np.sin(2 * math.pi * X)
    return setup, 25.0 / (36.0 * math.pi), 5.0 / (12.0 * math.pi), vx, vy, b0 * vx, b0 * np.sin(4 * math.pi * X)


def orszag_tang_perturbation(n: int, seed: int = 1, corr_cells: float = 8.0) -> np.ndarray:
    """The seeded unit-rms density perturbation field of the Orszag-Tang setup."""
    return gaussian_random_field((n, n), corr_cells, _rng(seed))


def gaussian_random_field(shape, corr_cells: float, rng: np.random.Generator) -> np.ndarray:
    """Unit-rms periodic Gaussian random field with a Gaussian correlation kernel."""
    w = rng.standard_normal(shape)
    ks = np.meshgrid(*[np.fft.fftfreq(s) for s in shape], indexing="ij")
    k2 = sum(k * k for k in ks)
    f = np.fft.ifftn(np.fft.fftn(w) * np.exp(-2.0 * (math.pi ** 2) * (corr_cells ** 2) * k2)).real
    f = f - f.mean()
    return f / f.std()


def random_state(setup: Setup, seed: int = 0, dv: float = 0.3, db: float = 0.3):
    """Small random MHD/HD state for parity tests: smooth background plus noise,
    positive density and pressure."""
    rng = _rng(seed)
    u, b, psi = _empty(setup)
    g = setup.guards
    sl = (slice(g[2], g[2] + setup.n[2]), slice(g[1], g[1] + setup.n[1]), slice(g[0], g[0] + setup.n[0]))
    shp = (setup.n[2], setup.n[1], setup.n[0])
    emag = None
    if setup.magnetic:
        bi = rng.uniform(-db, db, size=shp + (3,))
        bi[..., 0] += 0.4
        b[sl] = bi
        emag = 0.5 * (bi ** 2).sum(-1)
        psi[sl] = rng.uniform(-0.01, 0.01, size=shp)
    for f, (kind, gam) in enumerate(setup.fluids):
        rho = rng.uniform(0.5, 1.5, size=shp)
        vel = rng.uniform(-dv, dv, size=shp + (3,))
        p = rng.uniform(0.3, 1.0, size=shp)
        _set_fluid(setup, u[sl], f, rho, vel[..., 0], vel[..., 1], vel[..., 2], p,
                   emag if kind == "ion" else None)
    fill_periodic(setup, u)
    fill_periodic(setup, b)
    fill_periodic(setup, psi)
    return u, b, psi


def batched_blocks(nblocks: int = 512, seed: int = 1, sizes=(16, 24, 32, 48, 64), levels: int = 3,
                   fluids=(("ion", 5.0 / 3.0), ("neu", 7.0 / 5.0), ("dst", -1.0)), magnetic: bool = True,
                   n0: int = 64, limiter: str = "vanleer", centre=(0.3, -0.2, 0.1)):
    """Many independent periodic blocks of uneven sizes sampling an off-centre
    Sedov blast at three refinement levels.

    Block edges are drawn per axis from ``sizes`` (seeded).  A block's level l
    has cell size 2/n0 / 2**l; level-2 blocks are placed within 0.25 of the
    blast centre, level-1 blocks within 0.6, level-0 blocks anywhere in
    [-1,1]^3, each block's cells sampling the same analytic initial state:
    every fluid at rest with density 1 (dust 0.01) and pressure 1e-5, the
    gaseous fluids carrying a thermal energy density 10 inside r < 0.12 of the
    centre; uniform B = (0.1, 0.05, 0) with psi = 0 when magnetised.
    Returns a list of (Setup, u, b, psi).
    """
    rng = _rng(seed)
    out = []
    fl = list(fluids)
    for ib in range(nblocks):
        n = tuple(int(x) for x in rng.choice(sizes, size=3))
        lev = int(rng.integers(0, levels))
        dl = 2.0 / n0 / 2 ** lev
        reach = (0.25, 0.6, 1.0)[min(lev, 2)]
        origin = [centre[d] + rng.uniform(-reach, reach) - 0.5 * n[d] * dl for d in range(3)]
        setup = Setup(n=n, xmin=tuple(origin), xmax=tuple(origin[d] + n[d] * dl for d in range(3)),
                      fluids=fl, magnetic=magnetic, limiter=limiter, limiter_b=limiter, cfl=0.7, cfl_glm=0.7,
                      smalld=1.0e-4)
        u, b, psi = _empty(setup)
        x, y, z = (_centres(setup, d) for d in range(3))
        Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
        r = np.sqrt((X - centre[0]) ** 2 + (Y - centre[1]) ** 2 + (Z - centre[2]) ** 2)
        hot = np.where(r < 0.12, 10.0, 0.0)
        emag = None
        if magnetic:
            b[..., 0] = 0.1
            b[..., 1] = 0.05
            emag = 0.5 * (0.1 ** 2 + 0.05 ** 2)
        for f, (kind, gam) in enumerate(fl):
            rho = 0.01 if kind == "dst" else 1.0
            _set_fluid(setup, u, f, rho, 0.0, 0.0, 0.0, 1.0e-5, emag if kind == "ion" else None)
            if kind != "dst":
                beg = sum(4 if k == "dst" else 5 for k, _ in fl[:f])
                u[..., beg + 4] += hot
        fill_periodic(setup, u)
        out.append((setup, u, b, psi))
    return out


def _composition(total: int, sizes, rng: np.random.Generator):
    """Split total cells into consecutive pieces with sizes from ``sizes``."""
    for _ in range(1000):
        parts, left = [], total
        while left > 0:
            fit = [s for s in sizes if s <= left]
            if not fit:
                break
            s = int(rng.choice(fit))
            parts.append(s)
            left -= s
        if left == 0:
            return parts
    raise ValueError(f"{total} cells cannot be split into pieces from {sizes}")


def refined_layout(dom, regions, sizes=(16, 24, 32, 48, 64), seed: int = 1):
    """Blocks of a refined periodic domain.  dom: base cells per direction;
    regions[L-1] = (lo, hi): the box of level L >= 1 on the level-L grid
    (even bounds, two coarse cells inside level L-1).  Every level is cut
    into blocks by per-axis compositions drawn from ``sizes`` (seeded).
    Returns a list of (level, off, n)."""
    rng = _rng(seed)
    boxes = [((0, 0, 0), tuple(dom))] + [tuple(r) for r in regions]
    out = []
    for L, (lo, hi) in enumerate(boxes):
        cuts = []
        for d in range(3):
            ext = hi[d] - lo[d]
            if dom[d] == 1:
                cuts.append([(0, 1)])
                continue
            parts = _composition(ext, [s for s in sizes if L == 0 or s % 2 == 0], rng)
            edges = np.concatenate([[0], np.cumsum(parts)]) + lo[d]
            cuts.append([(int(edges[k]), int(parts[k])) for k in range(len(parts))])
        for oz, nz in cuts[2]:
            for oy, ny in cuts[1]:
                for ox, nx in cuts[0]:
                    out.append((L, (ox, oy, oz), (nx, ny, nz)))
    return out


def refined_blocks(dom, layout, setup: Setup, fields, dl0: float = 0.125):
    """Setups and states of the blocks of ``refined_layout``: block cells of
    level L have size dl0 / 2**L (dl0 a power of two keeps every cell size
    exact); ``fields(setup, X, Y, Z)`` returns (u, b, psi) at cell centres
    (guard cells included), with X, Y, Z in base-cell units.  Returns a list
    of (setup, level, off, u, b, psi)."""
    out = []
    for L, off, n in layout:
        dl = dl0 / 2 ** L
        s = setup.replace(n=tuple(n), xmin=tuple(off[d] * dl if dom[d] > 1 else -0.5 * dl0 for d in range(3)),
                          xmax=tuple((off[d] + n[d]) * dl if dom[d] > 1 else 0.5 * dl0 for d in range(3)))
        X, Y, Z = (_centres(s, d) / dl0 for d in range(3))
        Zg, Yg, Xg = np.meshgrid(Z, Y, X, indexing="ij")
        u, b, psi = fields(s, Xg, Yg, Zg)
        out.append((s, L, tuple(off), u, b, psi))
    return out


def blast_fields(centre, radius: float, e_in: float = 10.0, p0: float = 1.0e-5, b0=(0.1, 0.05, 0.0),
                 dust_rho: float = 0.01):
    """(u, b, psi) at cell centres: every fluid at rest with density 1 (dust
    ``dust_rho``) and pressure p0, the gaseous fluids with thermal energy
    density e_in inside ``radius`` base cells of ``centre``; uniform B = b0,
    psi = 0 when magnetised."""
    def f(setup, X, Y, Z):
        u, b, psi = _empty(setup)
        r = np.sqrt((X - centre[0]) ** 2 + (Y - centre[1]) ** 2 + (Z - centre[2]) ** 2)
        hot = np.where(r < radius, e_in, 0.0)
        emag = None
        if setup.magnetic:
            for c in range(3):
                b[..., c] = b0[c]
            emag = 0.5 * (b0[0] ** 2 + b0[1] ** 2 + b0[2] ** 2)
        for fl, (kind, gam) in enumerate(setup.fluids):
            rho = dust_rho if kind == "dst" else 1.0
            _set_fluid(setup, u, fl, rho, 0.0, 0.0, 0.0, p0, emag if kind == "ion" else None)
            if kind != "dst":
                beg = sum(4 if k == "dst" else 5 for k, _ in setup.fluids[:fl])
                u[..., beg + 4] += hot
        return u, b, psi
    return f


def wave_fields(dom, seed: int = 1, amp: float = 0.2):
    """Smooth periodic (u, b, psi) at cell centres: a few seeded sinusoids
    with the period of the base domain (``dom`` base cells) per field, a
    function of position only, so that every level samples the same state."""
    rng = _rng(seed)
    per = [float(max(n, 1)) for n in dom]

    def f(setup, X, Y, Z):
        u, b, psi = _empty(setup)

        def wave(a):
            k = rng.integers(1, 3, size=3)
            ph = rng.uniform(0, 2 * np.pi, size=3)
            return a * (np.sin(2 * np.pi * k[0] * X / per[0] + ph[0]) * np.cos(2 * np.pi * k[1] * Y / per[1] + ph[1])
                        + np.sin(2 * np.pi * k[2] * Z / per[2] + ph[2]))
        state = rng.bit_generator.state
        emag = None
        if setup.magnetic:
            for c in range(3):
                b[..., c] = (0.5 if c == 0 else 0.2) + wave(0.15)
            psi[...] = wave(0.02)
            emag = 0.5 * (b ** 2).sum(-1)
        for fl, (kind, gam) in enumerate(setup.fluids):
            rho = 1.0 + wave(amp)
            p = 0.8 + wave(0.15)
            _set_fluid(setup, u, fl, rho, wave(0.3), wave(0.3), wave(0.3), p, emag if kind == "ion" else None)
        rng.bit_generator.state = state
        return u, b, psi
    return f


def refined_blast(seed: int = 4, base: int = 128, centre=(70, 58, 66), r1: int = 104, r2: int = 120,
                  sizes=(16, 24, 32, 48, 64), radius: float = 4.0, dl0: float = 2.0 ** -6,
                  fluids=(("ion", 5.0 / 3.0), ("neu", 7.0 / 5.0), ("dst", -1.0)), magnetic: bool = True):
    """The uneven-blocks workload on a real three-level refinement: a
    periodic base^3 domain cut into blocks with edges from ``sizes`` (seeded),
    a level-1 box of (2 r1)^3 level-1 cells and a level-2 box of (2 r2)^3
    level-2 cells centred on the blast at ``centre`` (base cells), each cut the
    same way; ion MHD + neutral + dust at rest, thermal energy density 10
    inside ``radius`` base cells of the centre, uniform B = (0.1, 0.05, 0).
    Returns (dom, blocks) for refined_blocks' block list."""
    dom = (base, base, base)
    c1 = [2 * c for c in centre]
    c2 = [4 * c for c in centre]
    regions = [(tuple(c - r1 for c in c1), tuple(c + r1 for c in c1)),
               (tuple(c - r2 for c in c2), tuple(c + r2 for c in c2))]
    layout = refined_layout(dom, regions, sizes=sizes, seed=seed)
    setup = Setup(n=(16, 16, 16), fluids=list(fluids), magnetic=magnetic, limiter="vanleer", limiter_b="vanleer",
                  cfl=0.7, cfl_glm=0.7, smalld=1.0e-4)
    return dom, refined_blocks(dom, layout, setup, blast_fields(centre, radius), dl0=dl0)


def cpaw(nx: int = 128, ny: int = 64, A: float = 0.1, d0: float = 1.0, p0: float = 0.1, vA: float = 1.0,
         kx: float = 6.283185307, ky: float = 12.566370614, gamma: float = 5.0 / 3.0):
    """Circularly polarised Alfvén wave (problems/cpaw/initproblem.F90:
    problem_initial_conditions, problem.par): [0,1] x [0,0.5] periodic, one
    ionised fluid, the wave rotated by atan(ky/kx) in the x-y plane, run with
    the unsplit solver, vanleer, CFL 0.3, cfl_glm 0.3, smalld = smallei = 1e-5
    to tend = 0.447213595 (one period).  Returns (setup, u, b, psi, ini_b)
    with ini_b the initial field (the reference compares B with it)."""
    setup = Setup(n=(nx, ny, 1), xmin=(0.0, 0.0, 0.0), xmax=(1.0, 0.5, 1.0), fluids=[("ion", gamma)],
                  magnetic=True, limiter="vanleer", limiter_b="vanleer", cfl=0.3, cfl_glm=0.3, smalld=1.0e-5,
                  smallei=1.0e-5, solver="unsplit", cflcontrol="redo", tend=0.447213595)
    u, b, psi = _empty(setup)
    g = setup.guards
    # cell centres: fbnd + dl * (i - is + 1/2) over the guard-inclusive range (grid_container_base.F90:377)
    x = setup.xmin[0] + setup.dl[0] * (np.arange(setup.ext[0]) - g[0] + 0.5)
    y = setup.xmin[1] + setup.dl[1] * (np.arange(setup.ext[1]) - g[1] + 0.5)
    z = 0.5 * (setup.xmin[2] + setup.xmax[2])
    aa = math.atan(ky / kx)
    gg = math.atan(math.cos(aa) * (0.0 / kx))
    kp = math.sqrt(kx ** 2 + ky ** 2)
    rot = np.array([[math.cos(aa) * math.cos(gg), -math.sin(aa), -math.cos(aa) * math.sin(gg)],
                    [math.sin(aa) * math.cos(gg), math.cos(aa), -math.sin(aa) * math.sin(gg)],
                    [math.sin(gg), 0.0, math.cos(gg)]])
    Y, X = np.meshgrid(y, x, indexing="ij")
    xp = (rot[0, 0] * X + rot[1, 0] * Y) + rot[2, 0] * z       # first row of rot^T . (x, y, z)
    phi = kp * xp
    s, c = np.sin(phi), np.cos(phi)
    vp = [np.zeros_like(phi), A * s, A * c]
    bp = [np.full_like(phi, vA * math.sqrt(d0)), -math.sqrt(d0) * A * s, -math.sqrt(d0) * A * c]
    v = [(rot[i, 0] * vp[0] + rot[i, 1] * vp[1]) + rot[i, 2] * vp[2] for i in range(3)]
    bf = [(rot[i, 0] * bp[0] + rot[i, 1] * bp[1]) + rot[i, 2] * bp[2] for i in range(3)]
    ek = (0.5 * ((v[0] ** 2 + v[1] ** 2) + v[2] ** 2)) / d0
    em = 0.5 * ((bf[0] ** 2 + bf[1] ** 2) + bf[2] ** 2)
    gam_1 = gamma - 1.0
    for k in range(setup.ext[2]):
        u[k, :, :, 0] = d0
        for dd in range(3):
            u[k, :, :, 1 + dd] = v[dd]
            b[k, :, :, dd] = bf[dd]
        u[k, :, :, 4] = (p0 / gam_1 + ek) + em
    return setup, u, b, psi, b.copy()


def cpaw_error(setup, b, ini_b):
    """verify_test (problems/cpaw/initproblem.F90): sqrt of the summed squared
    deviation of B from its initial field over the interior, directions with
    extent only, over the summed squares of the initial field."""
    g, n = setup.guards, setup.n
    sl = (slice(g[2], g[2] + n[2]), slice(g[1], g[1] + n[1]), slice(g[0], g[0] + n[0]))
    num = den = 0.0
    for d in range(3):
        if n[d] > 1:
            num += float(((ini_b[sl + (d,)] - b[sl + (d,)]) ** 2).sum())
            den += float((ini_b[sl + (d,)] ** 2).sum())
    return math.sqrt(num / den)
