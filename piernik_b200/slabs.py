"""One level split into slabs over ranks (one process per GPU).

The reference runs one MPI rank per block set and exchanges guard cells
between ranks inside ``internal_boundaries`` (src/grid/cg_list_bnd.F90:251-324,
isend/irecv of packed segments) and reduces dt with MPI_MIN
(src/base/timestep.F90:173).  Here each rank holds one slab of a periodic
domain as one block; the library plans the segments, packs the cells a peer
needs and unpacks what it receives (``pk_halo_*``), and this module moves the
buffers between ranks through a transport:

* ``TorchTransport`` -- ``torch.distributed`` point-to-point
  (``batch_isend_irecv``) and ``all_reduce``: NCCL over NVLink between GPUs,
  gloo for CPU tests of the transport itself;
* ``ThreadTransport`` -- ranks as threads of one process sharing one GPU
  (tests): buffers handed over in host memory order, a barrier between the
  pack and the unpack.  No kernel ever waits for another rank's kernel.

Every exchange is host-driven, so all ranks take the same steps in the same
order: the library calls the halo callback after each local guard exchange
(once before every fused sweep, with the sweep's direction) and the reduce
callback twice per time step (dt minimum, c_all maximum).  Before a sweep
only the face boxes along its direction are moved (``pk_halo_*_dir``): for z
slabs the x and y sweeps move nothing and post no message, and the z sweeps
move the z faces only.  The pack and unpack kernels and the NCCL transfers
are ordered on the library's stream (NCCL waits on it for the pack, the
stream waits on NCCL for the unpack), so no exchange stops the host.
"""
from __future__ import annotations

import ctypes as C
import threading
from typing import Dict, List, Optional, Sequence, Tuple

import torch

from . import _lib as L
from .config import BND_PER, Setup
from .sim import Simulation


def split(n: int, parts: int) -> List[int]:
    """Slab thicknesses: n cells into ``parts`` nearly equal slabs."""
    if parts < 1 or n < parts:
        raise ValueError(f"cannot split {n} cells into {parts} slabs")
    base, extra = divmod(n, parts)
    return [base + (1 if i < extra else 0) for i in range(parts)]


def slab_layout(setup: Setup, world: int, axis: int = 2) -> List[Tuple[Tuple[int, int, int], Tuple[int, int, int]]]:
    """(n, off) of every rank's slab of the level described by ``setup``."""
    sizes = split(setup.n[axis], world)
    out = []
    o = 0
    for s in sizes:
        n = list(setup.n)
        n[axis] = s
        off = [0, 0, 0]
        off[axis] = o
        out.append((tuple(n), tuple(off)))
        o += s
    return out


def slab_setup(setup: Setup, n, off) -> Setup:
    """The slab's own Setup; its cell size must equal the level's bit for bit
    (true for power-of-two extents of a power-of-two box, checked here)."""
    dl = setup.dl
    s = setup.replace(n=tuple(n),
                      xmin=tuple(setup.xmin[d] + off[d] * dl[d] for d in range(3)),
                      xmax=tuple(setup.xmin[d] + (off[d] + n[d]) * dl[d] for d in range(3)))
    if s.dl != dl:
        raise ValueError("slab cell size differs from the level's in the last bit; choose a box and "
                         "extents whose cell size and slab edges are exact in binary")
    return s


class TorchTransport:
    """Halo buffers and reductions over ``torch.distributed``."""

    def __init__(self, device: torch.device):
        self.device = device

    def exchange(self, rank: int, peers: Sequence[int], send: Dict[int, torch.Tensor],
                 recv: Dict[int, torch.Tensor], stream: Optional[int] = None) -> None:
        """Post every peer's send and receive (empty buffers are skipped; both
        sides of a pair agree on which are empty) and wait for them.  With
        ``stream`` (a cudaStream_t), NCCL is ordered after the work queued
        there and that stream waits for the transfers; the host does not."""
        import torch.distributed as dist
        ops = []
        for p in peers:
            if send[p].numel():
                ops.append(dist.P2POp(dist.isend, send[p], p))
            if recv[p].numel():
                ops.append(dist.P2POp(dist.irecv, recv[p], p))
        if not ops:
            return
        if stream is not None and self.device.type == "cuda":
            with torch.cuda.stream(torch.cuda.ExternalStream(stream, device=self.device)):
                for r in dist.batch_isend_irecv(ops):
                    r.wait()
        else:
            for r in dist.batch_isend_irecv(ops):
                r.wait()
            if self.device.type == "cuda":
                torch.cuda.synchronize(self.device)

    def reduce(self, rank: int, x: float, op: int) -> float:
        import torch.distributed as dist
        t = torch.tensor([x], dtype=torch.float64, device=self.device)
        dist.all_reduce(t, op=dist.ReduceOp.MIN if op == 0 else dist.ReduceOp.MAX)
        return float(t.item())


class ThreadTransport:
    """Ranks as threads of one process (one device): hand-over through a
    shared table, a barrier on each side of every exchange."""

    def __init__(self, world: int):
        self.world = world
        self.barrier = threading.Barrier(world)
        self.box: Dict[Tuple[int, int], torch.Tensor] = {}
        self.vals: Dict[int, float] = {}

    def exchange(self, rank, peers, send, recv, stream=None):
        torch.cuda.synchronize()                  # every rank's pack has landed
        for p in peers:
            self.box[(rank, p)] = send[p]
        self.barrier.wait()
        for p in peers:
            recv[p].copy_(self.box[(p, rank)])
        torch.cuda.synchronize()
        self.barrier.wait()

    def reduce(self, rank, x, op):
        self.vals[rank] = x
        self.barrier.wait()
        vals = [self.vals[r] for r in range(self.world)]
        r = min(vals) if op == 0 else max(vals)
        self.barrier.wait()
        return r


class SlabRank:
    """This rank's slab of a periodic level as a connected block of one
    handle, with the other ranks' slabs declared remote and the transport
    wired into the library's halo and reduce callbacks."""

    def __init__(self, setup: Setup, rank: int, world: int, transport, axis: int = 2,
                 device: Optional[torch.device] = None):
        for d in range(3):
            if setup.n[d] > 1 and setup.bnd[d] != (BND_PER, BND_PER):
                raise ValueError("slab domains are periodic in every direction")
        self.setup, self.rank, self.world, self.transport = setup, rank, world, transport
        self.device = device or torch.device("cuda", torch.cuda.current_device())
        self.layout = slab_layout(setup, world, axis)
        n, off = self.layout[rank]
        self.local = slab_setup(setup, n, off)
        self.sim = Simulation(self.local)
        self.sim.set_domain(setup.n, (True, True, True))
        self.sim.place_block(0, off)
        lib, h = self.sim.lib, self.sim.h
        for r, (nr, offr) in enumerate(self.layout):
            if r == rank:
                continue
            rc = lib.pk_block_remote(h, r, (C.c_int32 * 3)(*nr), (C.c_int64 * 3)(*offr))
            if rc != L.PK_OK:
                raise L.PkError(lib.pk_last_error(h).decode())
        cnt = C.c_int32()
        self.sim._chk(lib.pk_halo_peers(h, None, 0, C.byref(cnt)), "pk_halo_peers")
        arr = (C.c_int32 * max(cnt.value, 1))()
        self.sim._chk(lib.pk_halo_peers(h, arr, cnt.value, C.byref(cnt)), "pk_halo_peers")
        self.peers = [arr[i] for i in range(cnt.value)]
        # buffers per direction: -1 the whole halo (guard refreshes), 0..2 the
        # face boxes a sweep along that direction reads
        self.bufs = {}
        for direction in (-1, 0, 1, 2):
            send, recv = {}, {}
            for p in self.peers:
                s, r = C.c_int64(), C.c_int64()
                self.sim._chk(lib.pk_halo_sizes_dir(h, p, direction, C.byref(s), C.byref(r)), "pk_halo_sizes_dir")
                send[p] = torch.empty(s.value, dtype=torch.float64, device=self.device)
                recv[p] = torch.empty(r.value, dtype=torch.float64, device=self.device)
            active = [p for p in self.peers if send[p].numel() or recv[p].numel()]
            self.bufs[direction] = (send, recv, active)
        self.send, self.recv, _ = self.bufs[-1]
        self.exchanges = 0
        self.skipped = 0
        self.error = None
        self._halo_cb = L.HALO_FN(self._halo)
        self._reduce_cb = L.REDUCE_FN(self._reduce)
        self.attach()

    def attach(self) -> None:
        """Install the halo and reduce callbacks (done at construction)."""
        self.sim._chk(self.sim.lib.pk_set_comm(self.sim.h, C.cast(self._halo_cb, C.c_void_p),
                                               C.cast(self._reduce_cb, C.c_void_p), None), "pk_set_comm")

    # callbacks (called by the library on this rank's host thread); an error
    # cannot cross the C boundary, so it is kept and raised by check()
    def _halo(self, ctx, direction):
        lib, h = self.sim.lib, self.sim.h
        send, recv, active = self.bufs[direction if direction in self.bufs else -1]
        if not active:                  # nothing crosses ranks for this sweep (the same on every rank)
            self.skipped += 1
            return
        for p in active:
            if send[p].numel():
                rc = lib.pk_halo_pack_dir(h, p, direction, send[p].data_ptr())
                if rc != L.PK_OK and self.error is None:
                    self.error = f"pk_halo_pack_dir: {lib.pk_last_error(h).decode()}"
        self.transport.exchange(self.rank, active, send, recv, self.sim.stream)
        for p in active:
            if recv[p].numel():
                rc = lib.pk_halo_unpack_dir(h, p, direction, recv[p].data_ptr())
                if rc != L.PK_OK and self.error is None:
                    self.error = f"pk_halo_unpack_dir: {lib.pk_last_error(h).decode()}"
        self.exchanges += 1

    def check(self):
        if self.error:
            raise L.PkError(self.error)

    def _reduce(self, ctx, x, op):
        return self.transport.reduce(self.rank, x, op)

    def upload_global(self, u, b=None, psi=None):
        """Take this rank's window (interior plus guards) of global arrays in
        the reference's layout."""
        n, off = self.layout[self.rank]
        g = self.setup.guards
        sl = tuple(slice(off[d], off[d] + n[d] + 2 * g[d]) for d in (2, 1, 0))
        win = lambda a: None if a is None else a[sl].copy()
        self.sim.upload(win(u), win(b), win(psi))

    def detach(self) -> None:
        """Drop the callbacks: later guard refreshes (a download after fused
        sweeps refreshes guards, which with callbacks is collective) stay on
        this rank and leave the cells taken from other ranks as they are."""
        self.sim._chk(self.sim.lib.pk_set_comm(self.sim.h, None, None, None), "pk_set_comm")

    def run(self, nsteps: int) -> None:
        self.sim.run(nsteps)
        self.check()

    def close(self):
        self.sim.close()
