"""Run configuration of the sweep path, with PIERNIK's names and defaults.

The fields mirror the reference namelists the split Riemann path reads:
``NUMERICAL_SETUP`` (src/base/global.F90:118-120, defaults :196-260),
``FLUID_IONIZED`` / ``FLUID_NEUTRAL`` / ``FLUID_DUST`` (gamma), ``BASE_DOMAIN``
(n_d, bnd_*, xmin..zmax; src/grid/domain.F90:139) and ``END_CONTROL`` (tend).
"""
from __future__ import annotations

import dataclasses
import sys
from dataclasses import dataclass, field
from typing import List, Tuple

BND_PER, BND_OUT, BND_REF = 0, 1, 2
BND_NAMES = {"per": BND_PER, "out": BND_OUT, "ref": BND_REF}
LIMITER_NAMES = ("vanleer", "minmod", "moncen", "superbee")
FLT_TINY = 1.1754943508222875e-38        # tiny(real(1.0,4))  (constants.F90:104)
DBL_HUGE = sys.float_info.max            # huge(1.)
DBL_TINY = sys.float_info.min            # tiny(1.)


@dataclass
class Setup:
    # BASE_DOMAIN
    n: Tuple[int, int, int] = (64, 64, 64)
    nb: int = 4
    xmin: Tuple[float, float, float] = (-1.0, -1.0, -1.0)
    xmax: Tuple[float, float, float] = (1.0, 1.0, 1.0)
    bnd: Tuple[Tuple[int, int], ...] = ((BND_PER, BND_PER),) * 3
    # fluids, in flind order (ionized, neutral, dust): (kind, gamma)
    fluids: List[Tuple[str, float]] = field(default_factory=lambda: [("ion", 5.0 / 3.0)])
    magnetic: bool = True            # MAGNETIC with divB_0 = 'HDC' (global.F90:189)
    # NUMERICAL_SETUP
    cfl: float = 0.7
    cfl_glm: float = 0.7             # set from the default cfl before the namelist is read (:253)
    glm_alpha: float = 0.1
    limiter: str = "vanleer"
    limiter_b: str = "vanleer"       # limiter_b = limiter (:212-213)
    smalld: float = 1.0e-3
    smallei: float = 1.0e-10
    use_smalld: bool = True
    use_smallei: bool = True
    disallow_negatives: bool = True
    integration_order: int = 2
    dt_initial: float = -1.0
    dt_max_grow: float = 2.0
    dt_min: float = DBL_TINY
    dt_max: float = DBL_HUGE
    cflcontrol: str = "none"         # the reference defaults to 'redo' (:218); 'none' keeps parity runs unforked
    ch_grid: bool = True             # :254 (psi speed from the grid; False: from the gas, hdc.F90:118-131)
    use_eglm: bool = False           # :252 (E-GLM sources after each triple of sweeps, hdc.F90:355-457)
    cfl_max: float = 0.9             # :233
    dt_shrink: float = 0.5           # :245
    max_redostep_attempts: int = 10  # :258
    interpolation: str = "linear"    # interpol_str (:220): linear or weno3
    w_epsilon: float = 1.0e-10       # :255
    solver: str = "split"            # solver_str (:423-437): split (RIEMANN_SPLIT) or unsplit (RIEMANN_UNSPLIT)
    ord_fluid_prolong: int = 0       # :260 O_INJ (refined domains' guard cells; 0 or 1, others degrade to 0)
    ord_mag_prolong: int = 2         # :259 O_I2 (-6..6 but -1: the orders of grid_container_prolong.F90)
    skip_sweep: Tuple[bool, bool, bool] = (False, False, False)
    # END_CONTROL
    tend: float = DBL_HUGE
    nend: int = 0

    @property
    def dl(self) -> Tuple[float, float, float]:
        return tuple((self.xmax[d] - self.xmin[d]) / self.n[d] for d in range(3))

    @property
    def guards(self) -> Tuple[int, int, int]:
        return tuple(self.nb if self.n[d] > 1 else 0 for d in range(3))

    @property
    def ext(self) -> Tuple[int, int, int]:
        g = self.guards
        return tuple(self.n[d] + 2 * g[d] for d in range(3))

    @property
    def nvar(self) -> int:
        return sum(4 if k == "dst" else 5 for k, _ in self.fluids)

    def replace(self, **kw) -> "Setup":
        return dataclasses.replace(self, **kw)

    def validate(self) -> None:
        if self.limiter not in LIMITER_NAMES or self.limiter_b not in LIMITER_NAMES:
            raise ValueError(f"unknown limiter {self.limiter!r}/{self.limiter_b!r}")
        if not (0.0 < self.cfl <= 1.0):
            raise ValueError("CFL value should be >0. and <=1.")      # global.F90:303
        if self.integration_order not in (1, 2):
            raise ValueError("integration_order must be 1 or 2")
        if self.ord_mag_prolong not in (-6, -5, -4, -3, -2, 0, 1, 2, 3, 4, 5, 6):
            raise ValueError(f"ord_mag_prolong {self.ord_mag_prolong}: unknown prolongation order")
        if self.solver not in ("split", "unsplit"):
            raise ValueError(f"solver {self.solver!r}: this library implements split and unsplit")
        if self.interpolation not in ("linear", "weno3"):
            raise ValueError(f"interpol_str {self.interpolation!r}: this library implements linear and weno3")
        if self.cflcontrol not in ("none", "warn", "redo", "repeat", "flex", "flexible", "auto", "adaptive"):
            raise ValueError(f"cflcontrol {self.cflcontrol!r}: this library implements none, warn, redo, flex "
                             f"and auto")
        kinds = [k for k, _ in self.fluids]
        if kinds != sorted(kinds, key=("ion", "neu", "dst").index) or len(set(kinds)) != len(kinds):
            raise ValueError("fluids must be a subset of (ion, neu, dst) in that order")
        if self.magnetic and "ion" not in kinds:
            raise ValueError("a magnetised run needs the ionized fluid")
        if self.magnetic and any(b != (BND_PER, BND_PER) for d, b in enumerate(self.bnd) if self.n[d] > 1):
            raise ValueError("magnetised runs support periodic boundaries only")
