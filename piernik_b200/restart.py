"""Restart files: the whole state of a run in one ``.npz`` file.

The reference writes its vital named arrays (u, b, psi) and the time
variables to an HDF5 restart file (src/IO/hdf5/restart_hdf5_v2.F90) and reads
them back to resume a run bit for bit.  No HDF5 library exists on this
platform, so the same contents go to a NumPy archive instead: every block's
u, b and psi in the reference's array layout (guard cells included), the
block layout (extents, cell sizes, boundaries, placement and refinement
level, the domain), the run configuration, the time state (t, dt, dt_old,
chspeed, nstep, the retry state) and, for stacked instances, each
instance's time state.  ``load`` rebuilds a Simulation that continues
exactly as the saved one would have.  Launch tuning (tiles, stage shape,
graphs) is not part of the state and is not saved.
"""
from __future__ import annotations

import dataclasses
import json

import numpy as np

from . import _lib as L
from .config import Setup
from .sim import Simulation

FORMAT = 1
_TUPLE_FIELDS = ("n", "xmin", "xmax", "skip_sweep")


def _setup_dict(s: Setup) -> dict:
    return dataclasses.asdict(s)


def _setup_from(d: dict) -> Setup:
    d = dict(d)
    for k in _TUPLE_FIELDS:
        d[k] = tuple(d[k])
    d["bnd"] = tuple(tuple(x) for x in d["bnd"])
    d["fluids"] = [tuple(x) for x in d["fluids"]]
    return Setup(**d)


def _ts_dict(st: L.PkTimeState) -> dict:
    return {name: getattr(st, name) for name, _ in L.PkTimeState._fields_}


def _ts_from(d: dict) -> L.PkTimeState:
    st = L.PkTimeState()
    for name, _ in L.PkTimeState._fields_:
        setattr(st, name, d[name])
    return st


def save(sim: Simulation, path: str) -> None:
    """Write the run held by ``sim`` to ``path`` (a .npz archive)."""
    ids = sorted(sim.blocks)
    meta = {
        "format": FORMAT,
        "setup": _setup_dict(sim.setup),
        "blocks": [{"setup": _setup_dict(sim.blocks[i]), "placement": sim.placement.get(i)} for i in ids],
        "domain": sim.domain,
        "instances": sim.instances,
        "time_state": _ts_dict(sim.time_state),
        "instance_states": [_ts_dict(sim.instance_state(k)) for k in range(sim.instances)] if sim.instances > 1 else [],
    }
    arrays = {}
    for i in ids:
        u, b, psi = sim.download(block=i)
        arrays[f"u{i}"] = u
        if b is not None:
            arrays[f"b{i}"] = b
            arrays[f"psi{i}"] = psi
    np.savez(path, meta=np.array(json.dumps(meta)), **arrays)


def load(path: str) -> Simulation:
    """A Simulation resuming the run saved in ``path``."""
    with np.load(path, allow_pickle=False) as z:
        meta = json.loads(str(z["meta"]))
        if meta.get("format") != FORMAT:
            raise ValueError(f"{path}: restart format {meta.get('format')} (this library reads {FORMAT})")
        arrays = {k: z[k] for k in z.files if k != "meta"}
    setups = [_setup_from(b["setup"]) for b in meta["blocks"]]
    phys = _setup_from(meta["setup"])
    # block 0 takes its own extent, cell size and boundaries (after a
    # remove_block(0) it is not the block the run was created with); the
    # physics comes from the run's Setup, which the Simulation keeps
    s0 = setups[0]
    sim = Simulation(phys.replace(n=s0.n, nb=s0.nb, xmin=s0.xmin, xmax=s0.xmax, bnd=s0.bnd))
    sim.setup = phys
    sim.blocks[0] = s0
    for s in setups[1:]:
        sim.add_block(s)
    if meta["domain"] is not None:
        sim.set_domain(*meta["domain"])
    for i, b in enumerate(meta["blocks"]):
        if b["placement"] is not None:
            off, level = b["placement"]
            sim.place_block(i, off, level)
    for i in range(len(setups)):
        sim.upload(arrays[f"u{i}"], arrays.get(f"b{i}"), arrays.get(f"psi{i}"), block=i)
    if meta["instances"] > 1:
        sim.set_instances(meta["instances"])
    sim.time_state = _ts_from(meta["time_state"])      # (with instances this sets every instance's) ...
    for k, d in enumerate(meta["instance_states"]):     # ... so each instance's own state comes after it
        sim.set_instance_state(k, _ts_from(d))
    return sim
