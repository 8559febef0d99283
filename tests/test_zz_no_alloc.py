"""pk_timestep_raw_noalloc: the CFL time step for callers that cannot let the
library allocate device memory (their device memory is all reserved for their
own pool, or a cudaMalloc inside their step loop would synchronise the
device), so they cannot create a handle.  It must give pk_timestep_raw's
result bit for bit on the same states; its reduction slots are a fixed device
array shared by all calls, so two calls in a row, the first on faster states,
also check that each call starts from cleared slots.

This file is collected last on purpose: a run that stops at the first
failure has then already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from helpers import random_state, setup_for
from piernik_b200 import _lib as L
from piernik_b200.sim import Simulation, make_config

PK_E_ARG = -1            # include/piernik_b200.h


PK_E_STATE = -5


def call_noalloc(lib, setup, blocks, err_len=256, stream=None):
    """blocks: list of (n, dl, device pointer); stream: a cudaStream_t handle
    (int) or None; returns (rc, dt, c_all, message)."""
    cfg = make_config(setup)
    nb = len(blocks)
    n = (C.c_int32 * (3 * nb))(*[x for b in blocks for x in b[0]])
    dl = (C.c_double * (3 * nb))(*[x for b in blocks for x in b[1]])
    ptrs = (C.c_void_p * nb)(*[b[2] for b in blocks])
    dt, c_all = C.c_double(-1.0), C.c_double(-1.0)
    err = C.create_string_buffer(err_len)
    rc = lib.pk_timestep_raw_noalloc(C.byref(cfg), nb, n, dl, ptrs, C.c_void_p(stream), C.byref(dt),
                                     C.byref(c_all), err, err_len)
    return rc, dt.value, c_all.value, err.value.decode()


def test_noalloc_rejects_too_many_blocks():
    """Beyond PK_NOALLOC_MAX_BLOCKS the call fails before touching a GPU."""
    lib = L.load()
    s = setup_for("hd", n=(8, 8, 8))
    blocks = [(s.n, s.dl, 1)] * 65
    rc, _, _, msg = call_noalloc(lib, s, blocks)
    assert rc == PK_E_ARG
    assert "PK_NOALLOC_MAX_BLOCKS" in msg and "65" in msg


@pytest.mark.gpu
@pytest.mark.parametrize("phys,shape,on_stream", [
    ("hd", "3d", False), ("mhd", "3d", False), ("mhd", "3d", True),
    ("hd", "2d", False), ("mhd", "2d", True)])
def test_noalloc_matches_timestep_raw(gpu_lib, phys, shape, on_stream):
    """Blocks of 3D and 2D (n_z = 1: no z guard cells) extents, on the legacy
    default stream and on a stream of the caller's."""
    import torch

    n1, n2 = ((20, 14, 11), (9, 16, 12)) if shape == "3d" else ((16, 12, 1), (10, 18, 1))
    s1 = setup_for(phys, n=n1, lim="moncen")
    s2 = setup_for(phys, n=n2, lim="moncen")
    stream = torch.cuda.Stream() if on_stream else None
    handle = stream.cuda_stream if on_stream else None
    slow = [random_state(s1, seed=1), random_state(s2, seed=2)]
    fast = []
    for (u, b, psi), s in zip(slow, (s1, s2)):
        u = u.copy()
        u[..., 1:4] *= 3.0          # faster flow: larger signal speeds
        fast.append((u, b, psi))

    def on_handle(states):
        sim = Simulation(s1)
        sim.upload(*states[0])
        bid = sim.add_block(s2)
        sim.upload(*states[1], block=bid)
        dt, c_all = sim.timestep_raw()
        soa = [sim.download(layout=L.PK_LAYOUT_SOA, block=i) for i in (0, bid)]
        sim.close()
        dev = []
        for u, b, psi in soa:
            planes = [u] + ([b, psi[None]] if s1.magnetic else [])
            dev.append(torch.tensor(np.concatenate(planes, 0), device="cuda"))
        return dt, c_all, dev

    for states in (fast, slow):                     # two calls in a row, the faster state first
        dt_ref, c_ref, dev = on_handle(states)
        torch.cuda.synchronize()
        blocks = [(s1.n, s1.dl, dev[0].data_ptr()), (s2.n, s2.dl, dev[1].data_ptr())]
        rc, dt, c_all, msg = call_noalloc(gpu_lib, s1, blocks, stream=handle)
        assert rc == L.PK_OK, msg
        assert np.float64(dt).view(np.uint64) == np.float64(dt_ref).view(np.uint64), (dt, dt_ref)
        assert np.float64(c_all).view(np.uint64) == np.float64(c_ref).view(np.uint64), (c_all, c_ref)
        # one block alone
        sim = Simulation(s1)
        sim.upload(*states[0])
        dt1, c1 = sim.timestep_raw()
        sim.close()
        rc, dt, c_all, msg = call_noalloc(gpu_lib, s1, blocks[:1], stream=handle)
        assert rc == L.PK_OK, msg
        assert (dt, c_all) == (dt1, c1)


@pytest.mark.gpu
def test_noalloc_rejects_host_memory(gpu_lib):
    """A state in host memory is refused before any launch (a kernel given it
    would fault or read the wrong memory)."""
    s = setup_for("hd", n=(8, 8, 8))
    host = np.zeros(s.nvar * 16 ** 3)
    rc, _, _, msg = call_noalloc(gpu_lib, s, [(s.n, s.dl, host.ctypes.data)])
    assert rc == PK_E_ARG and "device memory" in msg


@pytest.mark.gpu
def test_noalloc_refuses_capture(gpu_lib):
    """The call synchronises its stream, so it refuses to run while that
    stream is capturing (the caller's graph stays valid)."""
    import torch

    s = setup_for("hd", n=(8, 8, 8))
    x = torch.zeros(s.nvar * 16 ** 3, dtype=torch.float64, device="cuda")
    # first call outside any capture
    rc, _, _, msg = call_noalloc(gpu_lib, s, [(s.n, s.dl, x.data_ptr())])
    assert rc == L.PK_OK, msg
    stream = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=stream):
        x.add_(1.0)
        rc, _, _, msg = call_noalloc(gpu_lib, s, [(s.n, s.dl, x.data_ptr())], stream=stream.cuda_stream)
    assert rc == PK_E_STATE and "capturing" in msg
    g.replay()
    torch.cuda.synchronize()
    assert float(x[0]) == 1.0
