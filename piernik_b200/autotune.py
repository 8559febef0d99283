"""Autotuner for the fused sweep's tile shape and launch-bound variant.

For each sweep direction it times ``pk_sweep`` on the simulation's own state
for every candidate (pencils per CTA P, output cells per pencil L, kernel
variant V) whose CTA fits the variant's thread budget, using the library's
CUDA-event kernel timing, keeps the fastest, and restores the state and time
state afterwards.  Every candidate computes the same bits (the tile shape only
changes which CTA computes a cell), so tuning never changes results.
"""
from __future__ import annotations

import ctypes as C
import json
import os
from typing import Dict, Iterable, List, Optional, Tuple

from . import _lib as L

LENGTHS = (24, 32, 40, 48, 56, 64, 88, 120, 184, 248)


def variants() -> List[Tuple[int, int]]:
    lib = L.load()
    n = C.c_int32()
    t = (C.c_int32 * 16)()
    b = (C.c_int32 * 16)()
    lib.pk_tile_variants(C.byref(n), t, b)
    return [(t[i], b[i]) for i in range(n.value)]


def candidates(n_dir: int, n_ortho: int) -> Iterable[Tuple[int, int, int]]:
    """(P, L, variant) tiles: chunks of L owned cells with a 4-cell halo, and the
    whole pencil without halo (L = n_dir) where it fits the CTA, and the
    TMA-staged whole-pencil kernel (two pencils per CTA) for pencils of up to
    256 cells.  Besides the
    fixed lengths, the balanced ones ceil(n_dir / k) split the pencil into k
    nearly equal chunks, so that no short last chunk runs a full tile."""
    balanced = {-(-n_dir // k) for k in range(2, 13) if -(-n_dir // k) >= 16}
    for v, (maxt, _) in enumerate(variants()):
        if v == L.PK_VARIANT_STAGED:             # whole pencils, two per CTA, staged by TMA
            if n_dir <= 256:
                yield 2, n_dir, v
            continue
        lengths = sorted(set(min(Lc, n_dir) for Lc in LENGTHS) | balanced | ({n_dir} if n_dir <= maxt else set()))
        for Lc in lengths:
            T = Lc if (Lc == n_dir and n_dir <= maxt) else Lc + 8
            for P in (1, 2, 3, 4, 5, 6, 7, 8, 10, 12, 14, 16):
                if P > n_ortho:
                    continue
                if P * T <= maxt and 2 * P * T > maxt:
                    yield P, Lc, v


def _time_sweep(sim, d: int, dt: float, ch: float, reps: int) -> float:
    sim.profile(True)
    sim.profile_read()
    for _ in range(reps):
        sim.sweep(d + 1, dt, ch)
    _, nl, ms = sim.profile_read()
    sim.profile(False)
    return ms / max(nl, 1)


def autotune(sim, reps: int = 2, cache: Optional[str] = None, verbose: bool = False) -> Dict[int, dict]:
    """Pick the fastest fused-sweep tile per direction for ``sim`` and apply it."""
    setup = sim.setup
    key = f"{'mhd' if setup.magnetic else 'hd'}-{setup.limiter}-{setup.limiter_b}-{setup.n}"
    if cache and os.path.exists(cache):
        with open(cache) as f:
            known = json.load(f)
        if key in known:
            best = {int(d): v for d, v in known[key].items()}
            for d, b in best.items():
                sim.set_tile(d, b["P"], b["L"], b["V"])
            return best
    state = sim.download(layout=L.PK_LAYOUT_SOA)
    ts = sim.time_state
    dt, _ = sim.timestep_raw()
    ch = (setup.cfl_glm * min(setup.dl)) / dt if setup.magnetic else 0.0
    best: Dict[int, dict] = {}
    for d in range(3):
        if setup.n[d] <= 1:
            continue
        o = [x for x in range(3) if x != d]
        n1 = setup.n[1] if d == 0 else setup.n[0]
        results = []
        for P, Lc, v in candidates(setup.n[d], n1):
            sim.set_tile(d, P, Lc, v)
            ms = _time_sweep(sim, d, dt, ch, reps)
            results.append((ms, P, Lc, v))
            if verbose:
                print(f"dir {d} P={P} L={Lc} V={v}: {ms:.3f} ms")
        results.sort()
        ms, P, Lc, v = results[0]
        best[d] = {"P": P, "L": Lc, "V": v, "ms": ms, "candidates": len(results),
                   "default_ms": next((r[0] for r in results if (r[1], r[2], r[3]) == (4 if d else 2, min(64, setup.n[d]), 0)), None)}
        sim.set_tile(d, P, Lc, v)
    sim.upload(*state, layout=L.PK_LAYOUT_SOA)
    sim.time_state = ts
    if cache:
        known = {}
        if os.path.exists(cache):
            with open(cache) as f:
                known = json.load(f)
        known[key] = best
        with open(cache, "w") as f:
            json.dump(known, f, indent=1)
    return best
