"""Independent blocks and independent instances spread over ranks (one
process per GPU).

The reference distributes the leaves of a grid over MPI ranks and reduces
the time step over all of them (src/base/timestep.F90:173, MPI_MIN); blocks
that share no guard cells need no other exchange.  Two shardings follow:

* ``BlockShard`` -- a list of independent periodic blocks (the uneven-blocks
  workload) split into per-rank block lists balanced by cell count; each
  rank sweeps its list with one batched launch per sweep, and the step's dt
  (and c_all) are reduced over ranks through the library's reduce callback,
  so every rank advances with the dt one handle holding all blocks would
  take.
* ``instance_ranges`` -- stacked independent instances (the batched-adjoint
  workload): contiguous groups per rank; each instance keeps its own dt, so
  the ranks never communicate (replicas).
"""
from __future__ import annotations

import ctypes as C
from typing import List, Sequence, Tuple

from . import _lib as L
from .sim import Simulation


def balance(cells: Sequence[int], world: int) -> List[List[int]]:
    """Block indices per rank: the largest block first to the least loaded
    rank (ties to the lower rank); every rank's list in ascending block order.
    Deterministic, so every rank derives the same assignment."""
    if world < 1:
        raise ValueError("world must be at least 1")
    load = [0] * world
    out: List[List[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(cells)), key=lambda k: (-cells[k], k)):
        r = min(range(world), key=lambda q: (load[q], q))
        out[r].append(i)
        load[r] += cells[i]
    return [sorted(x) for x in out]


def instance_ranges(count: int, world: int) -> List[Tuple[int, int]]:
    """[first, end) of the instances each rank stacks: contiguous, sizes
    differing by at most one."""
    if world < 1 or count < world:
        raise ValueError(f"cannot spread {count} instances over {world} ranks")
    base, extra = divmod(count, world)
    out, o = [], 0
    for r in range(world):
        k = base + (1 if r < extra else 0)
        out.append((o, o + k))
        o += k
    return out


class BlockShard:
    """This rank's share of independent blocks in one handle; the time step
    is reduced over ranks by ``transport.reduce`` (MIN for dt, MAX for
    c_all).  ``blocks``: the whole list of (setup, u, b, psi), the same on
    every rank."""

    def __init__(self, blocks, rank: int, world: int, transport):
        self.rank, self.world, self.transport = rank, world, transport
        cells = [s.n[0] * s.n[1] * s.n[2] for s, *_ in blocks]
        self.assign = balance(cells, world)
        self.mine = self.assign[rank]
        if not self.mine:
            raise ValueError(f"rank {rank} has no block: fewer blocks than ranks")
        first = blocks[self.mine[0]]
        self.sim = Simulation(first[0])
        for i in self.mine[1:]:
            self.sim.add_block(blocks[i][0])
        for k, i in enumerate(self.mine):
            _, u, b, psi = blocks[i]
            self.sim.upload(u, b, psi, block=k)
        self._reduce_cb = L.REDUCE_FN(self._reduce)
        self.sim._chk(self.sim.lib.pk_set_comm(self.sim.h, None, C.cast(self._reduce_cb, C.c_void_p), None),
                      "pk_set_comm")

    def _reduce(self, ctx, x, op):
        return self.transport.reduce(self.rank, x, op)

    def run(self, nsteps: int) -> None:
        self.sim.run(nsteps)

    def download(self, index: int):
        """The state of global block ``index`` (held by this rank)."""
        return self.sim.download(block=self.mine.index(index))

    def close(self) -> None:
        self.sim.close()
