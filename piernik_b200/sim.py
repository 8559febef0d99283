"""Host-side mirror of the reference's interface for the split Riemann path.

``Simulation`` owns one library handle and exposes the reference's routine
names with their argument meaning:

=====================  ==============================================================
``solve_cg``            solve_cg_riemann(cg, ddim, istep)  src/scheme/Riemann_Solver/solve_cg_riemann.F90:68
``update_boundaries``   update_boundaries                  src/scheme/sweeps.F90:66
``sweep``               sweep(cdim)                        src/scheme/sweeps.F90:114
``glmdamping``          glmdamping                         src/scheme/Riemann_Solver/hdc.F90:289
``time_step``           time_step(dt, flind, .true.)       src/base/timestep.F90:112
``fluid_update``        fluid_update -> fluid_update_full  src/scheme/fluidupdate.F90:60,99
``run``                 main loop body                     src/base/piernik.F90:125-213
=====================  ==============================================================

Directions are 1-based (xdim=1, ydim=2, zdim=3) as in the reference.  Arrays
use the reference's memory layout: a C-ordered numpy array ``u[k, j, i, v]`` is
Fortran's ``cg%u(v, i, j, k)`` (guard cells included), ``b[k, j, i, d]`` is
``cg%b(d, i, j, k)`` and ``psi[k, j, i]`` is ``cg%q(psi)%arr(i, j, k)``.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Tuple

import numpy as np

from . import _lib as L
from .config import Setup


def _check(lib, h, rc, what):
    if rc != L.PK_OK:
        msg = lib.pk_last_error(h).decode() if h else ""
        raise L.PkError(f"{what} failed: {L.ERRORS.get(rc, rc)} {msg}")


def make_config(setup: Setup) -> L.PkConfig:
    setup.validate()
    lib = L.load()
    c = L.PkConfig()
    lib.pk_config_default(C.byref(c))
    c.nfluids = len(setup.fluids)
    for i, (kind, gam) in enumerate(setup.fluids):
        c.fluid_kind[i] = L.PK_FLUID[kind]
        c.gamma[i] = gam
    c.magnetic = int(setup.magnetic)
    c.limiter = L.PK_LIM[setup.limiter]
    c.limiter_b = L.PK_LIM[setup.limiter_b]
    c.use_smalld = int(setup.use_smalld)
    c.use_smallei = int(setup.use_smallei)
    c.disallow_negatives = int(setup.disallow_negatives)
    c.smalld = setup.smalld
    c.smallei = setup.smallei
    c.cfl = setup.cfl
    c.cfl_glm = setup.cfl_glm
    c.glm_alpha = setup.glm_alpha
    c.integration_order = setup.integration_order
    c.nb = setup.nb
    c.dt_initial = setup.dt_initial
    c.dt_max_grow = setup.dt_max_grow
    c.dt_min = setup.dt_min
    c.dt_max = setup.dt_max
    c.tend = setup.tend
    for d in range(3):
        c.skip_sweep[d] = int(setup.skip_sweep[d])
    c.cflcontrol = L.PK_CFL[setup.cflcontrol]
    c.cfl_max = setup.cfl_max
    c.dt_shrink = setup.dt_shrink
    c.max_redostep_attempts = setup.max_redostep_attempts
    c.interpolation = {"linear": 0, "weno3": 1}[setup.interpolation]
    c.w_epsilon = setup.w_epsilon
    c.solver = {"split": 0, "unsplit": 1}[setup.solver]
    c.ord_fluid_prolong = setup.ord_fluid_prolong
    c.ord_mag_prolong = setup.ord_mag_prolong
    c.ch_grid = int(setup.ch_grid)
    c.use_eglm = int(setup.use_eglm)
    return c


class Simulation:
    """One device-resident block of a PIERNIK run, swept by the CUDA library."""

    def __init__(self, setup: Setup):
        self.setup = setup
        self.lib = L.load()
        cfg = make_config(setup)
        h = C.c_void_p()
        rc = self.lib.pk_create(C.byref(cfg), C.byref(h))
        if rc != L.PK_OK:
            raise L.PkError(f"pk_create failed: {L.ERRORS.get(rc, rc)}")
        self.h = h
        n = (C.c_int32 * 3)(*setup.n)
        dl = (C.c_double * 3)(*setup.dl)
        bnd = (C.c_int32 * 6)(*[setup.bnd[d][s] for d in range(3) for s in range(2)])
        self.blocks = {}
        self.instances = 1
        self.domain = None          # (cells of the base grid, periodic flags) after set_domain
        self.placement = {}         # block -> (offset, level) after place_block
        self.block = self.add_block(setup)

    def add_block(self, setup: Setup) -> int:
        """Register one more block (grid_container) with its own extent, cell
        size and boundaries; physics parameters come from the first Setup."""
        n = (C.c_int32 * 3)(*setup.n)
        dl = (C.c_double * 3)(*setup.dl)
        bnd = (C.c_int32 * 6)(*[setup.bnd[d][s] for d in range(3) for s in range(2)])
        bid = C.c_int32()
        self._chk(self.lib.pk_block_add(self.h, n, dl, bnd, C.byref(bid)), "pk_block_add")
        self.blocks[bid.value] = setup
        return bid.value

    # -- plumbing ---------------------------------------------------------
    def _chk(self, rc, what):
        _check(self.lib, self.h, rc, what)

    def close(self):
        if getattr(self, "h", None):
            self.lib.pk_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _shapes(self, block: int = 0):
        s = self.blocks.get(block, self.setup)
        ez, ey, ex = s.ext[2], s.ext[1], s.ext[0]
        return (ez, ey, ex, self.setup.nvar), (ez, ey, ex, 3), (ez, ey, ex)

    # -- state transfer ------------------------------------------------------
    def upload(self, u: np.ndarray, b: Optional[np.ndarray] = None, psi: Optional[np.ndarray] = None,
               layout: int = L.PK_LAYOUT_FORTRAN, block: int = 0) -> None:
        su, sb, sp = self._shapes(block)
        u = np.ascontiguousarray(u, dtype=np.float64)
        if u.size != int(np.prod(su)):
            raise ValueError(f"u has {u.size} elements, expected {int(np.prod(su))}")
        bp = pp = None
        if self.setup.magnetic:
            b = np.ascontiguousarray(b, dtype=np.float64)
            psi = np.ascontiguousarray(psi, dtype=np.float64)
            if b.size != int(np.prod(sb)) or psi.size != int(np.prod(sp)):
                raise ValueError("b / psi have the wrong size")
            bp, pp = b.ctypes.data, psi.ctypes.data
        self._keep = (u, b, psi)
        self._chk(self.lib.pk_upload(self.h, block, u.ctypes.data, bp, pp, layout), "pk_upload")
        self.sync()

    def download(self, layout: int = L.PK_LAYOUT_FORTRAN, out=None,
                 block: int = 0) -> Tuple[np.ndarray, Optional[np.ndarray], Optional[np.ndarray]]:
        su, sb, sp = self._shapes(block)
        if layout == L.PK_LAYOUT_SOA:
            su = (su[3],) + su[:3]
            sb = (3,) + sb[:3]
        if out is None:
            u = np.empty(su)
            b = np.empty(sb) if self.setup.magnetic else None
            psi = np.empty(sp) if self.setup.magnetic else None
        else:
            u, b, psi = out
        self._chk(self.lib.pk_download(self.h, block, u.ctypes.data,
                                       b.ctypes.data if b is not None else None,
                                       psi.ctypes.data if psi is not None else None, layout), "pk_download")
        return u, b, psi

    def sync(self):
        self._chk(self.lib.pk_sync(self.h), "pk_sync")

    # -- the reference's routines ------------------------------------------
    def solve_cg(self, ddim: int, istep: int, dt: float, chspeed: float = 0.0, block: int = 0) -> None:
        self._chk(self.lib.pk_solve_cg(self.h, block, ddim, istep, dt, chspeed), "pk_solve_cg")

    def update_boundaries(self) -> None:
        self._chk(self.lib.pk_fill_guards(self.h), "pk_fill_guards")

    def sweep(self, cdim: int, dt: float, chspeed: float = 0.0) -> None:
        self._chk(self.lib.pk_sweep(self.h, cdim, dt, chspeed), "pk_sweep")

    def glmdamping(self, fac: float) -> None:
        self._chk(self.lib.pk_glm_damp(self.h, fac), "pk_glm_damp")

    def timestep_raw(self) -> Tuple[float, float]:
        dt, c = C.c_double(), C.c_double()
        self._chk(self.lib.pk_timestep_raw(self.h, C.byref(dt), C.byref(c)), "pk_timestep_raw")
        return dt.value, c.value

    def time_step(self) -> float:
        dt = C.c_double()
        self._chk(self.lib.pk_time_step(self.h, C.byref(dt)), "pk_time_step")
        return dt.value

    def fluid_update(self) -> None:
        self._chk(self.lib.pk_fluid_update(self.h), "pk_fluid_update")

    def run(self, nsteps: int) -> None:
        self._chk(self.lib.pk_run(self.h, nsteps), "pk_run")

    @property
    def time_state(self) -> L.PkTimeState:
        st = L.PkTimeState()
        self._chk(self.lib.pk_get_time_state(self.h, C.byref(st)), "pk_get_time_state")
        return st

    @time_state.setter
    def time_state(self, st: L.PkTimeState) -> None:
        self._chk(self.lib.pk_set_time_state(self.h, C.byref(st)), "pk_set_time_state")

    def status(self) -> int:
        s = C.c_uint32()
        self._chk(self.lib.pk_status(self.h, C.byref(s)), "pk_status")
        return s.value

    def profile(self, on: bool = True) -> None:
        self._chk(self.lib.pk_profile_enable(self.h, int(on)), "pk_profile_enable")

    def profile_read(self):
        """(kernel launches since creation, sweep launches timed, their device ms)."""
        a, b, ms = C.c_int64(), C.c_int64(), C.c_double()
        self._chk(self.lib.pk_profile_read(self.h, C.byref(a), C.byref(b), C.byref(ms)), "pk_profile_read")
        return a.value, b.value, ms.value

    @property
    def stream(self) -> int:
        return self.lib.pk_stream(self.h) or 0

    def set_batch(self, enable: bool = True, length: int = 0, variant: int = -1) -> None:
        """Sweep all blocks in one persistent launch over a tile work list."""
        self._chk(self.lib.pk_set_batch(self.h, int(enable), length, variant), "pk_set_batch")

    def set_stage_variant(self, variant: int) -> None:
        """Launch-bound variant of the batched stage kernel (0: 320 x 1,
        1: 128 x 3, 2: 192 x 2, 3: 384 x 1 threads x CTAs per SM)."""
        self._chk(self.lib.pk_set_stage_variant(self.h, variant), "pk_set_stage_variant")

    def use_graph(self, enable: bool = True) -> None:
        """Replay each step's sweeps as a captured CUDA graph."""
        self._chk(self.lib.pk_use_graph(self.h, int(enable)), "pk_use_graph")

    def set_refined_launch(self, one_launch: bool = True) -> None:
        """Refined domains: sweep every level of an RK stage in one persistent
        launch, or level by level (the default)."""
        self._chk(self.lib.pk_set_refined_launch(self.h, int(one_launch)), "pk_set_refined_launch")

    # -- independent instances stacked along z -------------------------------
    def set_instances(self, count: int) -> None:
        """Run ``count`` independent periodic problems, stacked along z in the
        single block, with one launch per sweep and a time step each."""
        self._chk(self.lib.pk_set_instances(self.h, count), "pk_set_instances")
        self.instances = count

    def instance_state(self, i: int) -> L.PkTimeState:
        st = L.PkTimeState()
        self._chk(self.lib.pk_get_instance_state(self.h, i, C.byref(st)), "pk_get_instance_state")
        return st

    def set_instance_state(self, i: int, st: L.PkTimeState) -> None:
        self._chk(self.lib.pk_set_instance_state(self.h, i, C.byref(st)), "pk_set_instance_state")

    # -- connected blocks of one level --------------------------------------
    def set_domain(self, ncells, periodic=(True, True, True)) -> None:
        """Declare the level's cell grid; placed blocks then exchange guards."""
        n = (C.c_int64 * 3)(*[int(x) for x in ncells])
        p = (C.c_int32 * 3)(*[int(bool(x)) for x in periodic])
        self._chk(self.lib.pk_set_domain(self.h, n, p), "pk_set_domain")
        self.domain = (tuple(int(x) for x in ncells), tuple(bool(x) for x in periodic))

    def restrict(self) -> None:
        """Covered coarse cells take the mean of their children, finest level
        first (restrict_to_base)."""
        self._chk(self.lib.pk_restrict(self.h), "pk_restrict")

    def mark_refinement(self, criteria) -> np.ndarray:
        """Flag cells by the refinement criteria (URC_var.F90) on every leaf
        block; ``criteria`` = [(method, field, thr, aux)], method one of
        ``_lib.URC_METHODS`` (or its number), field a plane of the state.
        Returns, per block, 1 where a leaf interior cell is flagged."""
        arr = (L.PkUrc * max(len(criteria), 1))()
        for k, (m, f, thr, aux) in enumerate(criteria):
            arr[k] = L.PkUrc(L.URC_METHODS[m] if isinstance(m, str) else int(m), int(f), float(thr), float(aux))
        out = (C.c_int32 * len(self.blocks))()
        self._chk(self.lib.pk_mark_refinement(self.h, arr, len(criteria), out), "pk_mark_refinement")
        return np.array(out[:], dtype=np.int32)

    def refine_map(self, block: int = 0) -> np.ndarray:
        """The flag map of ``block`` after mark_refinement, [z, y, x] with guard cells."""
        s = self.blocks.get(block, self.setup)
        m = np.zeros((s.ext[2], s.ext[1], s.ext[0]), dtype=np.uint8)
        self._chk(self.lib.pk_refine_map(self.h, block, m.ctypes.data), "pk_refine_map")
        return m

    def refine_candidates(self, block: int, bsize) -> list:
        """Offsets (level + 1 grid) of the bsize blocks refinemap2SFC_list would create."""
        bs = (C.c_int32 * 3)(*bsize)
        cnt = C.c_int32()
        self._chk(self.lib.pk_refine_candidates(self.h, block, bs, None, 0, C.byref(cnt)), "pk_refine_candidates")
        offs = (C.c_int64 * (3 * max(cnt.value, 1)))()
        self._chk(self.lib.pk_refine_candidates(self.h, block, bs, offs, cnt.value, C.byref(cnt)),
                  "pk_refine_candidates")
        return [tuple(offs[3 * k:3 * k + 3]) for k in range(cnt.value)]

    def remove_block(self, block: int) -> None:
        """Free ``block``; the ids above it move down by one."""
        self._chk(self.lib.pk_block_remove(self.h, block), "pk_block_remove")
        self.blocks = {(k if k < block else k - 1): v for k, v in self.blocks.items() if k != block}
        self.placement = {(k if k < block else k - 1): v for k, v in self.placement.items() if k != block}

    def prolong_block(self, block: int) -> None:
        """Fill every cell of ``block`` (a refined level's) from the coarser level."""
        self._chk(self.lib.pk_prolong_block(self.h, block), "pk_prolong_block")

    def place_block(self, block: int, off, level: int = 0) -> None:
        """Put the block's first interior cell at ``off`` on the grid of its
        refinement level (the base grid refined ``level`` times)."""
        o = (C.c_int64 * 3)(*[int(x) for x in off])
        self._chk(self.lib.pk_block_place_level(self.h, block, level, o), "pk_block_place_level")
        self.placement[block] = (tuple(int(x) for x in off), int(level))

    # -- differentiable path (one periodic block, one fluid, RK2) -------------
    @property
    def nplanes(self) -> int:
        """Component planes of the device state: u, then bx, by, bz, psi."""
        return self.setup.nvar + (4 if self.setup.magnetic else 0)

    def state_shape(self, block: int = 0) -> Tuple[int, int, int, int]:
        """Shape of the structure-of-arrays state with guard cells."""
        su, _, _ = self._shapes(block)
        return (self.nplanes,) + su[:3]

    def upload_device(self, ptr: int, block: int = 0) -> None:
        """Copy a device SoA state (``state_shape()`` doubles at ``ptr``) in."""
        self._chk(self.lib.pk_upload_device(self.h, block, ptr), "pk_upload_device")

    def download_device(self, ptr: int, block: int = 0) -> None:
        self._chk(self.lib.pk_download_device(self.h, block, ptr), "pk_download_device")

    def adjoint_set(self, lam, block: int = 0, on_device: bool = False) -> None:
        """Set dL/dU (SoA with guard cells; guard values are ignored).  ``lam``
        is a numpy array, or a device address when ``on_device``."""
        if on_device:
            self._chk(self.lib.pk_adjoint_set(self.h, block, lam, 1), "pk_adjoint_set")
            return
        lam = np.ascontiguousarray(lam, dtype=np.float64)
        if lam.shape != self.state_shape(block):
            raise ValueError(f"adjoint has shape {lam.shape}, expected {self.state_shape(block)}")
        self._chk(self.lib.pk_adjoint_set(self.h, block, lam.ctypes.data, 0), "pk_adjoint_set")

    def adjoint_get(self, out=None, block: int = 0, on_device: bool = False):
        if on_device:
            self._chk(self.lib.pk_adjoint_get(self.h, block, out, 1), "pk_adjoint_get")
            return out
        if out is None:
            out = np.empty(self.state_shape(block))
        self._chk(self.lib.pk_adjoint_get(self.h, block, out.ctypes.data, 0), "pk_adjoint_get")
        return out

    def adjoint_sweep(self, cdim: int, dt: float, chspeed: float = 0.0) -> None:
        """lam <- (d sweep(cdim) / dU)^T lam at the current state."""
        self._chk(self.lib.pk_adjoint_sweep(self.h, cdim, dt, chspeed), "pk_adjoint_sweep")

    def grad_forward(self, nsteps: int, every: int = 0, dts=None) -> np.ndarray:
        """Advance ``nsteps`` steps recording what the adjoint needs; checkpoint
        every ``every`` steps (0: about sqrt(nsteps)).  ``dts`` replays a
        prescribed dt sequence.  Returns the dt of each step
        (with stacked instances: an array [step, instance], and ``dts`` holds
        that many values)."""
        if every <= 0:
            every = max(1, int(round(np.sqrt(max(nsteps, 1)))))
        ni = getattr(self, "instances", 1)
        out = np.empty(max(nsteps, 1) * ni)
        dp = None
        if dts is not None:
            dts = np.ascontiguousarray(dts, dtype=np.float64)
            if dts.size < nsteps * ni:
                raise ValueError("dts has fewer than nsteps values (per instance)")
            dp = dts.ctypes.data
        self._chk(self.lib.pk_grad_forward(self.h, nsteps, every, dp, out.ctypes.data), "pk_grad_forward")
        out = out[:nsteps * ni]
        return out.reshape(nsteps, ni) if ni > 1 else out

    def grad_backward(self) -> None:
        self._chk(self.lib.pk_grad_backward(self.h), "pk_grad_backward")

    def set_adjoint_tile(self, direction: int = -1, length: int = 0, variant: int = -1) -> None:
        """Owned cells per pencil and launch-bound variant of the adjoint
        kernels along ``direction`` (0..2, -1: all)."""
        self._chk(self.lib.pk_set_adjoint_tile(self.h, direction, length, variant), "pk_set_adjoint_tile")

    def grad_release(self) -> None:
        self._chk(self.lib.pk_grad_release(self.h), "pk_grad_release")

    def set_arithmetic(self, mode: str = "bitexact") -> None:
        """Arithmetic of the fused / batched sweeps: 'bitexact' (the
        reference's rounding, the default) or 'fma' (contracted multiply-adds
        and hoisted reciprocals; agrees to ~1e-15 relative per step)."""
        self._chk(self.lib.pk_set_arithmetic(self.h, L.PK_ARITH[mode]), "pk_set_arithmetic")

    def set_tile(self, direction: int, pencils: int, length: int, variant: int = -1) -> None:
        """Tile of the fused sweep along ``direction`` (0..2): pencils per CTA,
        output cells per pencil, launch-bound variant (-1: default)."""
        self._chk(self.lib.pk_set_tile(self.h, direction, pencils, length, variant), "pk_set_tile")
