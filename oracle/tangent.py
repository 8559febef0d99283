"""Tangent-linear oracle (forward mode) -- TEST INFRASTRUCTURE, NOT PRODUCT CODE.

``liboracle_tangent.so`` is pk_oracle.c compiled with every double replaced
by a dual number (oracle/pk_tangent.cpp).  ``jvp`` runs the oracle's
fluid_update at a prescribed dt sequence on (state, seed direction) and
returns the final state and J v, the directional derivative of the final
state along v.  Only tests import this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle_tangent.so")


class Dual(C.Structure):
    _fields_ = [("v", C.c_double), ("d", C.c_double)]


def _dualize(fields):
    out = []
    for name, t in fields:
        if t is C.c_double:
            out.append((name, Dual))
        elif isinstance(t, type) and issubclass(t, C.Array) and t._type_ is C.c_double:
            out.append((name, Dual * t._length_))
        elif t == C.POINTER(C.c_double):
            out.append((name, C.c_void_p))
        else:
            out.append((name, t))
    return out


class TCfg(C.Structure):
    _fields_ = _dualize(O.OCfg._fields_)


class TBlock(C.Structure):
    _fields_ = _dualize(O.OBlock._fields_)


class TState(C.Structure):
    _fields_ = _dualize(O.OState._fields_)


def build(force: bool = False) -> str:
    srcs = [os.path.join(HERE, f) for f in ("pk_tangent.cpp", "pk_oracle.c", "pk_oracle.h")]
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(s) for s in srcs):
        subprocess.check_call(["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fpermissive",
                               "-fPIC", "-shared", "-w", "-o", LIB, os.path.join(HERE, "pk_tangent.cpp")], cwd=HERE)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB)
        assert L.t_dual_size() == 16
        L.o_run_fixed.argtypes = [C.POINTER(TCfg), C.POINTER(TBlock), C.POINTER(TState), C.c_void_p, C.c_int]
        L.o_fill_guards.argtypes = [C.POINTER(TCfg), C.POINTER(TBlock)]
        _lib = L
    return _lib


def _tcfg(setup) -> TCfg:
    oc = O.make_cfg(setup)
    tc = TCfg()
    for name, t in O.OCfg._fields_:
        val = getattr(oc, name)
        if t is C.c_double:
            setattr(tc, name, Dual(val, 0.0))
        elif isinstance(t, type) and issubclass(t, C.Array) and t._type_ is C.c_double:
            arr = getattr(tc, name)
            for i in range(t._length_):
                arr[i] = Dual(val[i], 0.0)
        else:
            setattr(tc, name, val)
    return tc


def _dual(val, der):
    return np.ascontiguousarray(np.stack([np.asarray(val, np.float64), np.asarray(der, np.float64)], axis=-1))


def jvp(setup, u, b, psi, du, db, dpsi, dts):
    """Run len(dts) steps of fluid_update from (u, b, psi) with the seed
    (du, db, dpsi); returns ((u, b, psi), (du, db, dpsi)) at the end, all in
    the guard-cell layout of the oracle (u[k, j, i, v]).  The guard cells of
    the input (and of the seed) are replaced by the boundary rules' images
    of the interior first."""
    L = lib()
    cfg = _tcfg(setup)
    mag = setup.magnetic
    U = _dual(u, du)
    B = _dual(b, db) if mag else None
    P = _dual(psi, dpsi) if mag else None
    UH = np.zeros_like(U)
    BH = np.zeros_like(B) if mag else None
    PH = np.zeros_like(P) if mag else None
    ez, ey, ex = [setup.ext[d] for d in (2, 1, 0)]
    RT = np.zeros(((setup.nvar + 4) * ez * ey * ex, 2))
    blk = TBlock()
    for d in range(3):
        blk.n[d] = setup.n[d]
        blk.dl[d] = Dual(setup.dl[d], 0.0)
        for s in range(2):
            blk.bnd[d][s] = setup.bnd[d][s]
    blk.nb = setup.nb
    ptr = lambda a: a.ctypes.data if a is not None else None
    blk.u, blk.uh, blk.b, blk.bh, blk.psi, blk.psih = ptr(U), ptr(UH), ptr(B), ptr(BH), ptr(P), ptr(PH)
    blk.uh_retry = ptr(RT)
    st = TState()
    st.dt_old = Dual(-1.0, 0.0)
    st.dt_cur_shrink = Dual(1.0, 0.0)
    D = _dual(np.asarray(dts, np.float64), np.zeros(len(dts)))
    # guard cells start as the images the block's boundary rules give (values and
    # derivatives alike): the map is interior -> interior, as on the fused path
    L.o_fill_guards(C.byref(cfg), C.byref(blk))
    rc = L.o_run_fixed(C.byref(cfg), C.byref(blk), C.byref(st), D.ctypes.data, len(dts))
    if rc:
        raise RuntimeError(f"o_run_fixed failed: {rc}")
    L.o_fill_guards(C.byref(cfg), C.byref(blk))
    vals = (U[..., 0], B[..., 0] if mag else None, P[..., 0] if mag else None)
    ders = (U[..., 1], B[..., 1] if mag else None, P[..., 1] if mag else None)
    return vals, ders
