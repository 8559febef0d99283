"""ctypes front end of the CPU oracle -- TEST INFRASTRUCTURE, NOT PRODUCT CODE.

Only tests/, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
import this module.  It drives ``liboracle.so`` (oracle/pk_oracle.c), a C
restatement of PIERNIK's RIEMANN_SPLIT sweep.  No Fortran compiler exists
here, so it cannot be run against the reference itself; it is pinned by the
reference's own known answers instead (the CPAW test's tabulated L2 errors,
reproduced to the 8 printed decimals, tests/test_cpaw.py) and, where the
reference holds none, by exact solutions (tests/test_exact_riemann_cpu.py,
tests/test_stationary_discontinuities_cpu.py, tests/test_dust_advection_cpu.py);
see pk_oracle.h.

Arrays use the reference's guard-cell layout:
``u[k, j, i, v]`` (= Fortran ``cg%u(v, i, j, k)``), ``b[k, j, i, d]``,
``psi[k, j, i]``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")

ION, NEU, DST = 0, 1, 2
LIMITERS = {"vanleer": 0, "minmod": 1, "moncen": 2, "superbee": 3}


class OCfg(C.Structure):
    _fields_ = [
        ("nfluids", C.c_int),
        ("kind", C.c_int * 3),
        ("gamma", C.c_double * 3),
        ("magnetic", C.c_int),
        ("limiter", C.c_int),
        ("limiter_b", C.c_int),
        ("use_smalld", C.c_int),
        ("use_smallei", C.c_int),
        ("disallow_negatives", C.c_int),
        ("smalld", C.c_double),
        ("smallei", C.c_double),
        ("cfl", C.c_double),
        ("cfl_glm", C.c_double),
        ("glm_alpha", C.c_double),
        ("ch_grid", C.c_int),
        ("integration_order", C.c_int),
        ("dt_initial", C.c_double),
        ("dt_max_grow", C.c_double),
        ("dt_min", C.c_double),
        ("dt_max", C.c_double),
        ("tend", C.c_double),
        ("skip_sweep", C.c_int * 3),
        ("cflcontrol", C.c_int),
        ("cfl_max", C.c_double),
        ("dt_shrink", C.c_double),
        ("max_redostep_attempts", C.c_int),
        ("interpolation", C.c_int),
        ("w_epsilon", C.c_double),
        ("solver", C.c_int),
        ("use_eglm", C.c_int),
    ]


class OBlock(C.Structure):
    _fields_ = [
        ("n", C.c_int * 3),
        ("nb", C.c_int),
        ("dl", C.c_double * 3),
        ("bnd", (C.c_int * 2) * 3),
        ("u", C.POINTER(C.c_double)),
        ("uh", C.POINTER(C.c_double)),
        ("b", C.POINTER(C.c_double)),
        ("bh", C.POINTER(C.c_double)),
        ("psi", C.POINTER(C.c_double)),
        ("psih", C.POINTER(C.c_double)),
        ("dn_negative", C.c_int),
        ("ei_negative", C.c_int),
        ("uh_retry", C.POINTER(C.c_double)),
        ("leaf", C.c_void_p),
        ("eflx", C.c_void_p * 3),
    ]


class OState(C.Structure):
    _fields_ = [
        ("t", C.c_double),
        ("dt", C.c_double),
        ("dt_old", C.c_double),
        ("c_all", C.c_double),
        ("chspeed", C.c_double),
        ("nstep", C.c_int),
        ("dt_full", C.c_double),
        ("c_all_old", C.c_double),
        ("dt_cur_shrink", C.c_double),
        ("stepcfl", C.c_double),
        ("t_saved", C.c_double),
        ("nstep_saved", C.c_int),
        ("tstep_attempt", C.c_int),
        ("repeat", C.c_int),
        ("redone", C.c_int),
        ("cfl_c", C.c_double),
    ]


def build(force: bool = False) -> str:
    """Compile liboracle.so with the flags that keep the reference's operation order."""
    src = os.path.join(HERE, "pk_oracle.c")
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(src):
        subprocess.check_call(
            ["gcc", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-fPIC", "-shared",
             "-Wall", "-o", LIB, src, "-lm"], cwd=HERE)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB)
        P, B, S = C.POINTER(OCfg), C.POINTER(OBlock), C.POINTER(OState)
        L.o_solve_cg.argtypes = [P, B, C.c_int, C.c_int, C.c_double, C.c_double]
        L.o_fill_guards.argtypes = [P, B]
        L.o_sweep.argtypes = [P, B, C.c_int, C.c_double, C.c_double]
        L.o_glm_fac.argtypes = [P, B, C.c_double, C.c_double]
        L.o_glm_fac.restype = C.c_double
        L.o_glm_apply.argtypes = [P, B, C.c_double]
        L.o_eglm.argtypes = [P, B, C.c_double]
        L.o_chspeed.argtypes = [P, B, C.c_double]
        L.o_chspeed.restype = C.c_double
        L.o_timestep_raw.argtypes = [P, B, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.o_time_step.argtypes = [P, B, S]
        L.o_fluid_update.argtypes = [P, B, S]
        L.o_run.argtypes = [P, B, S, C.c_int]
        L.o_nvar.argtypes = [P]
        L.o_run_multi.argtypes = [P, C.POINTER(B), C.c_int, S, C.c_int]
        L.o_time_step_multi.argtypes = [P, C.POINTER(B), C.c_int, S]
        L.o_unsplit_stage.argtypes = [P, B, C.c_int, C.c_double, C.c_double]
        L.o_set_threads.argtypes = [C.c_int]
        L.o_run_fixed.argtypes = [P, B, S, C.POINTER(C.c_double), C.c_int]
        L.o_cfl_max.argtypes = [P]
        L.o_cfl_max.restype = C.c_double
        L.o_get_threads.restype = C.c_int
        _lib = L
    return _lib


def make_cfg(setup) -> OCfg:
    """Fill the oracle configuration from a ``piernik_b200.Setup``-like object."""
    c = OCfg()
    c.nfluids = len(setup.fluids)
    for i, (kind, gam) in enumerate(setup.fluids):
        c.kind[i] = {"ion": ION, "neu": NEU, "dst": DST}[kind]
        c.gamma[i] = gam
    c.magnetic = int(setup.magnetic)
    c.limiter = LIMITERS[setup.limiter]
    c.limiter_b = LIMITERS[setup.limiter_b]
    c.use_smalld = int(setup.use_smalld)
    c.use_smallei = int(setup.use_smallei)
    c.disallow_negatives = int(setup.disallow_negatives)
    c.smalld = setup.smalld
    c.smallei = setup.smallei
    c.cfl = setup.cfl
    c.cfl_glm = setup.cfl_glm
    c.glm_alpha = setup.glm_alpha
    c.ch_grid = int(getattr(setup, "ch_grid", True))
    c.integration_order = setup.integration_order
    c.dt_initial = setup.dt_initial
    c.dt_max_grow = setup.dt_max_grow
    c.dt_min = setup.dt_min
    c.dt_max = setup.dt_max
    c.tend = setup.tend
    for d in range(3):
        c.skip_sweep[d] = int(setup.skip_sweep[d])
    c.cflcontrol = {"none": 0, "warn": 1, "redo": 2, "repeat": 2, "flex": 3, "flexible": 3, "auto": 4,
                    "adaptive": 4}[setup.cflcontrol]
    c.cfl_max = setup.cfl_max
    c.dt_shrink = setup.dt_shrink
    c.max_redostep_attempts = setup.max_redostep_attempts
    c.interpolation = {"linear": 0, "weno3": 1}[setup.interpolation]
    c.w_epsilon = setup.w_epsilon
    c.solver = {"split": 0, "unsplit": 1}[setup.solver]
    c.use_eglm = int(getattr(setup, "use_eglm", False))
    return c


def _ptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double)) if a is not None else None


class OracleBlock:
    """One block with guard cells, in the reference's array layout."""

    def __init__(self, setup, u, b=None, psi=None):
        self.setup = setup
        self.cfg = make_cfg(setup)
        self.u = np.ascontiguousarray(u, dtype=np.float64).copy()
        self.uh = np.zeros_like(self.u)
        mag = setup.magnetic
        self.b = np.ascontiguousarray(b, dtype=np.float64).copy() if mag else None
        self.bh = np.zeros_like(self.b) if mag else None
        self.psi = np.ascontiguousarray(psi, dtype=np.float64).copy() if mag else None
        self.psih = np.zeros_like(self.psi) if mag else None
        self.blk = OBlock()
        for d in range(3):
            self.blk.n[d] = setup.n[d]
            self.blk.dl[d] = setup.dl[d]
            for s in range(2):
                self.blk.bnd[d][s] = setup.bnd[d][s]
        self.blk.nb = setup.nb
        self.blk.u, self.blk.uh = _ptr(self.u), _ptr(self.uh)
        self.blk.b, self.blk.bh = _ptr(self.b), _ptr(self.bh)
        self.blk.psi, self.blk.psih = _ptr(self.psi), _ptr(self.psih)
        ez, ey, ex = [setup.ext[d] for d in (2, 1, 0)]
        self.retry = np.zeros((setup.nvar + 4) * ez * ey * ex)
        self.blk.uh_retry = _ptr(self.retry)
        self.state = OState()
        self.state.dt = 0.0
        self.state.dt_old = -1.0
        self.state.dt_cur_shrink = 1.0
        self.state.cfl_c = 1.0

    def fill_guards(self):
        lib().o_fill_guards(C.byref(self.cfg), C.byref(self.blk))

    def solve_cg(self, ddim, istep, dt, ch):
        return lib().o_solve_cg(C.byref(self.cfg), C.byref(self.blk), ddim, istep, dt, ch)

    def sweep(self, cdim, dt, ch):
        return lib().o_sweep(C.byref(self.cfg), C.byref(self.blk), cdim, dt, ch)

    def eglm(self, dt):
        """E-GLM sources for dt and the boundary update (a no-op unless the
        setup has use_eglm)."""
        lib().o_eglm(C.byref(self.cfg), C.byref(self.blk), dt)

    def timestep_raw(self):
        dt, c = C.c_double(), C.c_double()
        lib().o_timestep_raw(C.byref(self.cfg), C.byref(self.blk), C.byref(dt), C.byref(c))
        return dt.value, c.value

    def time_step(self):
        return lib().o_time_step(C.byref(self.cfg), C.byref(self.blk), C.byref(self.state))

    def fluid_update(self):
        return lib().o_fluid_update(C.byref(self.cfg), C.byref(self.blk), C.byref(self.state))

    def run(self, nsteps):
        return lib().o_run(C.byref(self.cfg), C.byref(self.blk), C.byref(self.state), nsteps)

    def run_fixed(self, dts):
        """fluid_update at the prescribed dt sequence (no CFL)."""
        d = np.ascontiguousarray(dts, dtype=np.float64)
        return lib().o_run_fixed(C.byref(self.cfg), C.byref(self.blk), C.byref(self.state), _ptr(d), len(d))

    def glm_fac(self, dt, ch):
        return lib().o_glm_fac(C.byref(self.cfg), C.byref(self.blk), dt, ch)

    def chspeed(self, dt):
        return lib().o_chspeed(C.byref(self.cfg), C.byref(self.blk), dt)


def run_multi(blocks, nsteps: int, state: OState = None) -> OState:
    """Advance several OracleBlocks (same Setup apart from n/dl) with one
    global dt, as the reference's leaves loop does."""
    if state is None:
        state = OState()
        state.dt_old = -1.0
        state.dt_cur_shrink = 1.0
        state.cfl_c = 1.0
    arr = (C.POINTER(OBlock) * len(blocks))(*[C.pointer(b.blk) for b in blocks])
    rc = lib().o_run_multi(C.byref(blocks[0].cfg), arr, len(blocks), C.byref(state), nsteps)
    if rc:
        raise RuntimeError(f"o_run_multi failed: {rc}")
    return state


def set_threads(n: int) -> None:
    lib().o_set_threads(int(n))


def get_threads() -> int:
    return lib().o_get_threads()
