"""piernik_b200 -- PIERNIK's split HLLD/HLLC sweep on NVIDIA B200 (sm_100a).

The hot path (pencil reconstruction, Riemann fluxes with GLM, RK2 stages,
guard cells, CFL reduction) runs in hand-written CUDA kernels in
``libpiernik_b200.so``; this package holds the host-side mirror of the
reference's routines (``Simulation``), the run configuration with the
reference's parameter names (``Setup``, ``read_problem_par``) and seeded
initial conditions (``problems``).
"""
from .config import Setup
from .namelist import read_problem_par
from .sim import Simulation

__all__ = ["Setup", "Simulation", "read_problem_par"]
