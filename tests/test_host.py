"""Host-side logic on CPU: namelists, configuration, initial conditions, and
the C-ABI library's exported symbols (loaded without running any kernel)."""
import ctypes
import os
import re

import numpy as np
import pytest

from piernik_b200 import build, problems, read_problem_par
from piernik_b200 import _lib as L
from piernik_b200.config import BND_OUT, BND_PER, Setup

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SEDOV_PAR = """
 $BASE_DOMAIN
    n_d = 64, 64, 64
    bnd_xl = 'per'
    bnd_xr = 'out'   ! outflow on one side
    xmin   =-1.0
    xmax   = 1.0
 /
 $FLUID_NEUTRAL
    gamma = 1.666666666
 /
 $NUMERICAL_SETUP
    cfl    = 0.8
    smalld = 1.e-3
    smallei= 1.e-5
    limiter = 'moncen'
 /
 $END_CONTROL
    tend   = 1.0d-3
 /
"""


def test_namelist_reader():
    s = read_problem_par(SEDOV_PAR, fluids=["neu"], magnetic=False)
    assert s.n == (64, 64, 64)
    assert s.bnd[0] == (BND_PER, BND_OUT)
    assert s.cfl == 0.8 and s.smalld == 1e-3 and s.smallei == 1e-5
    assert s.limiter == "moncen" and s.limiter_b == "moncen"     # limiter_b follows limiter
    assert s.tend == 1e-3
    assert s.fluids == [("neu", 1.666666666)]
    assert s.dl[0] == 2.0 / 64


def test_namelist_cmdline_override():
    s = read_problem_par(SEDOV_PAR, cmdline="&NUMERICAL_SETUP cfl=0.5, limiter_b='vanleer'/", fluids=["neu"])
    assert s.cfl == 0.5 and s.limiter == "moncen" and s.limiter_b == "vanleer"


def test_namelist_logical_switches():
    s = read_problem_par(SEDOV_PAR, fluids=["neu"])
    assert s.use_eglm is False and s.ch_grid is True                 # global.F90:252, :254
    s = read_problem_par(SEDOV_PAR, cmdline="&NUMERICAL_SETUP use_eglm=.true., ch_grid=.false./", fluids=["neu"])
    assert s.use_eglm is True and s.ch_grid is False


def test_namelist_rejects_other_solvers():
    with pytest.raises(ValueError):
        read_problem_par("&NUMERICAL_SETUP solver_str='rtvd' /")


def test_setup_validation():
    with pytest.raises(ValueError):
        Setup(cfl=1.5).validate()
    with pytest.raises(ValueError):
        Setup(fluids=[("neu", 1.4), ("ion", 5 / 3)]).validate()
    with pytest.raises(ValueError):
        Setup(magnetic=True, bnd=((BND_OUT, BND_OUT),) * 3).validate()
    Setup().validate()


def test_sedov_ic_energy():
    setup, u, _, _ = problems.sedov(n=32)
    g = setup.guards
    ui = u[g[2]:-g[2], g[1]:-g[1], g[0]:-g[0]]
    vol = np.prod(setup.dl)
    e_th0 = 1.0e-5 / (5.0 / 3.0 - 1.0)
    excess = (ui[..., 4] - e_th0).sum() * vol
    assert abs(excess - 1.0) < 1e-12
    assert np.all(ui[..., 0] == 1.0)


def test_turbulence_ic_properties():
    setup, u, b, psi = problems.mhd_turbulence(n=16, seed=7)
    g = setup.guards
    sl = (slice(g[2], -g[2]), slice(g[1], -g[1]), slice(g[0], -g[0]))
    rho = u[sl][..., 0]
    v = u[sl][..., 1:4] / rho[..., None]
    assert abs(np.sqrt((v ** 2).sum(-1).mean()) - 1.0) < 0.05
    bi = b[sl]
    assert abs(bi[..., 0].mean() - 0.2) < 1e-12
    # spectral divergence of B vanishes
    n = 16
    k = np.fft.fftfreq(n, 1.0 / n)
    kz, ky, kx = np.meshgrid(k, k, k, indexing="ij")
    div = kx * np.fft.fftn(bi[..., 0]) + ky * np.fft.fftn(bi[..., 1]) + kz * np.fft.fftn(bi[..., 2])
    assert np.abs(div).max() < 1e-10 * np.abs(np.fft.fftn(bi[..., 1])).max()
    # periodic guards
    assert np.array_equal(u[:, :, 0], u[:, :, n])
    assert np.all(psi == 0.0)


def test_orszag_tang_ic():
    setup, u, b, psi = problems.orszag_tang(n=16)
    assert setup.n == (16, 16, 1) and setup.ext[2] == 1
    assert u.shape == (1, 24, 24, 5)
    rho = u[0, 4:-4, 4:-4, 0]
    assert abs(rho.mean() - 25.0 / (36.0 * np.pi)) < 1e-4


def _header_symbols():
    text = open(os.path.join(ROOT, "include", "piernik_b200.h")).read()
    return sorted(set(re.findall(r"\b(pk_[a-z0-9_]+)\s*\(", text)))


def test_header_symbols_listed():
    assert sorted(L.EXPORTS) == _header_symbols()


def test_library_builds_and_exports():
    path = build.build()
    lib = ctypes.CDLL(path)
    for name in _header_symbols():
        assert hasattr(lib, name), name
    lib.pk_abi_version.restype = ctypes.c_int
    assert lib.pk_abi_version() == 6
    cfg = L.PkConfig()
    lib.pk_config_default(ctypes.byref(cfg))
    assert cfg.cfl == 0.7 and cfg.glm_alpha == 0.1 and cfg.nb == 4 and cfg.integration_order == 2


def test_create_rejects_bad_config():
    lib = L.load(build.build())
    cfg = L.PkConfig()
    lib.pk_config_default(ctypes.byref(cfg))
    cfg.cfl = 2.0
    h = ctypes.c_void_p()
    assert lib.pk_create(ctypes.byref(cfg), ctypes.byref(h)) == -1
    lib.pk_config_default(ctypes.byref(cfg))
    cfg.nfluids = 2
    cfg.fluid_kind[1] = 0          # ion after ion: not flind order
    assert lib.pk_create(ctypes.byref(cfg), ctypes.byref(h)) == -1


def test_missing_library_fails_loudly(tmp_path, monkeypatch):
    monkeypatch.setattr(L, "_lib", None)
    with pytest.raises(L.PkError):
        L.load(str(tmp_path / "absent.so"))
