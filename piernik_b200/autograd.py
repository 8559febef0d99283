"""PyTorch binding of the differentiable sweep path.

``advance(sim, state, nsteps, dts=None, every=0)`` maps the interior state
``(nplanes, nz, ny, nx)`` (float64, CUDA) to the state after ``nsteps`` steps
of the split RK2 sweeps and is differentiable with respect to ``state``.
The forward pass runs the library's fused sweeps while recording each step's
dt, chspeed and psi damping and checkpointing the state every ``every``
steps (about sqrt(nsteps) by default); the backward pass recomputes one
segment at a time and runs the hand-written adjoint sweep kernel in reverse.
The time steps are those of the forward pass, held fixed: the derivative is
taken at a fixed dt sequence (dt's own dependence on the state through the
CFL condition is not differentiated).

Only memory management goes through torch; every sweep and adjoint kernel is
the library's.  The handle must hold one periodic block of one fluid.
"""
from __future__ import annotations

import numpy as np
import torch

from .sim import Simulation


def _interior(sim: Simulation):
    s = sim.setup
    g = s.guards
    return (slice(None), slice(g[2], g[2] + s.n[2]), slice(g[1], g[1] + s.n[1]), slice(g[0], g[0] + s.n[0]))


def _padded(sim: Simulation, x: torch.Tensor) -> torch.Tensor:
    full = torch.zeros(sim.state_shape(), dtype=torch.float64, device=x.device)
    full[_interior(sim)] = x
    return full


class _Advance(torch.autograd.Function):
    @staticmethod
    def forward(ctx, state, sim, nsteps, dts, every):
        if state.dtype != torch.float64 or not state.is_cuda:
            raise TypeError("state must be a float64 CUDA tensor")
        full = _padded(sim, state.detach())
        torch.cuda.current_stream().synchronize()
        sim.upload_device(full.data_ptr())
        ctx.dts = sim.grad_forward(nsteps, every, dts)
        out = torch.empty_like(full)
        sim.download_device(out.data_ptr())
        ctx.sim = sim
        return out[_interior(sim)].contiguous()

    @staticmethod
    def backward(ctx, grad_out):
        sim = ctx.sim
        lam = _padded(sim, grad_out.to(torch.float64))
        torch.cuda.current_stream().synchronize()
        sim.adjoint_set(lam.data_ptr(), on_device=True)
        sim.grad_backward()
        res = torch.empty_like(lam)
        sim.adjoint_get(res.data_ptr(), on_device=True)
        return res[_interior(sim)].contiguous(), None, None, None, None


def advance(sim: Simulation, state: torch.Tensor, nsteps: int, dts=None, every: int = 0) -> torch.Tensor:
    """Differentiable ``nsteps`` steps of the sweep path from ``state``."""
    if dts is not None:
        dts = np.asarray(dts, dtype=np.float64)
    return _Advance.apply(state, sim, int(nsteps), dts, int(every))


def orszag_tang_state(sim: Simulation, pert: torch.Tensor) -> torch.Tensor:
    """Interior state of the Orszag-Tang vortex with density rho0 (1 + pert),
    as a differentiable function of the (n, n) relative density perturbation
    field ``pert`` (problems/otvortex/initproblem.F90:99-166 with the
    perturbation on top; the seeded workload uses pert = 1e-3 x a unit-rms
    Gaussian random field)."""
    from .problems import orszag_tang_fields
    n = sim.setup.n[0]
    _, rho0, pre, vx, vy, bx, by = orszag_tang_fields(n)
    gam = sim.setup.fluids[0][1]
    t = lambda a: torch.as_tensor(a, dtype=torch.float64, device=pert.device)
    vx, vy, bx, by = t(vx), t(vy), t(bx), t(by)
    rho = rho0 * (1.0 + pert)
    emag = 0.5 * (bx * bx + by * by)
    zero = torch.zeros_like(rho)
    ene = ((pre / (gam - 1.0)) + 0.5 * rho * (vx * vx + vy * vy + zero * zero)) + emag
    planes = [rho, rho * vx, rho * vy, zero, ene, bx, by, zero, zero]
    return torch.stack(planes, 0)[:, None]


def central_magnetic_energy(sim: Simulation, state: torch.Tensor, frac: float = 0.25) -> torch.Tensor:
    """Magnetic energy integrated over the central ``frac`` x ``frac`` of a 2D
    block (the central 128^2 cells of a 512^2 block for frac = 1/4)."""
    s = sim.setup
    nv = s.nvar
    ny, nx = s.n[1], s.n[0]
    cy, cx = int(round(ny * frac)), int(round(nx * frac))
    y0, x0 = (ny - cy) // 2, (nx - cx) // 2
    b = state[nv:nv + 3, 0, y0:y0 + cy, x0:x0 + cx]
    return 0.5 * (b * b).sum() * float(np.prod(s.dl))


def turbulence_state(sim: Simulation, rho: torch.Tensor, v: torch.Tensor, b: torch.Tensor,
                     p0: float) -> torch.Tensor:
    """Interior MHD state (nplanes, nz, ny, nx) from density, velocity and
    magnetic field (each component-first), pressure p0 and psi = 0: a
    differentiable function of the fields (the conversion of the turbulence
    recipe: m = rho v, e = p0/(gamma-1) + rho |v|^2 / 2 + |B|^2 / 2)."""
    gam = sim.setup.fluids[0][1]
    emag = 0.5 * ((b[0] * b[0] + b[1] * b[1]) + b[2] * b[2])
    ene = ((p0 / (gam - 1.0)) + 0.5 * rho * ((v[0] * v[0] + v[1] * v[1]) + v[2] * v[2])) + emag
    planes = [rho, rho * v[0], rho * v[1], rho * v[2], ene, b[0], b[1], b[2], torch.zeros_like(rho)]
    return torch.stack(planes, 0)


def spectrum_power(sim: Simulation, state: torch.Tensor, kmin: float = 8.0, kmax: float = 16.0,
                   instances: int = 1) -> torch.Tensor:
    """Kinetic-energy spectrum power in the shell kmin <= |k| <= kmax of each
    of ``instances`` cubes stacked along z in ``state`` (interior,
    (nplanes, nz, ny, nx)): P = sum over the shell of |v_hat(k)|^2 / 2 with
    v = m / rho and v_hat the unitary-mean DFT (sum_k |v_hat|^2 = mean |v|^2).
    Returns a tensor of ``instances`` powers."""
    nz, ny, nx = state.shape[1:]
    seg = nz // instances
    rho = state[0].reshape(instances, seg, ny, nx)
    v = state[1:4].reshape(3, instances, seg, ny, nx) / rho
    vh = torch.fft.rfftn(v, dim=(-3, -2, -1)) / float(seg * ny * nx)
    kz = torch.fft.fftfreq(seg, 1.0 / seg, dtype=torch.float64, device=state.device)[:, None, None]
    ky = torch.fft.fftfreq(ny, 1.0 / ny, dtype=torch.float64, device=state.device)[None, :, None]
    kx = torch.fft.rfftfreq(nx, 1.0 / nx, dtype=torch.float64, device=state.device)[None, None, :]
    kk = torch.sqrt(kx * kx + ky * ky + kz * kz)
    # the half spectrum holds each pair (k, -k) once except the kx = 0 and Nyquist planes
    wgt = torch.full(kk.shape, 2.0, dtype=torch.float64, device=state.device)
    wgt[..., 0] = 1.0
    if nx % 2 == 0:
        wgt[..., -1] = 1.0
    wgt = torch.where((kk >= kmin) & (kk <= kmax), wgt, torch.zeros_like(wgt))
    pw = (vh.real * vh.real + vh.imag * vh.imag) * wgt
    return 0.5 * pw.sum(dim=(0, 2, 3, 4))


def last_dts(out: torch.Tensor):
    """The dt sequence recorded by the ``advance`` call that produced ``out``."""
    fn = out.grad_fn
    return None if fn is None else getattr(fn, "dts", None)
