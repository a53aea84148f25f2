"""Slab decomposition of one uniform 3D grid across ranks (one process per
GPU): the last axis z is split into contiguous slabs, each rank steps its
slab with two ghost planes on every side that has a neighbour, and per RK2
stage the ranks exchange those planes.  The CFL maximum is all-reduced
(max), the conserved totals all-reduced (sum).

The reference has no distributed path (a single host); its flux loop
(src/driver.jl:209-223 over lib/RefMesh/src/RefMesh.jl:187-197) is what the
ghost planes feed: a PLM face flux needs two cells on each side, so two
planes of the neighbouring slab make every face of a slab computable
locally, and each cell's face sum keeps the reference's order because the
stage kernels classify a slab's planes by their global position.

`Halo` is the exchange plan and protocol, independent of where the planes
live: `get(first, count)` returns the `count` local planes starting at
`first` as a tensor, `put(first, tensor)` stores planes, and the transfers
go through `torch.distributed` point-to-point operations (NCCL on GPUs,
gloo in the CPU tests).  A rank that is its own neighbour (one rank with a
periodic z axis) copies locally.
"""
from __future__ import annotations

from typing import Callable, Optional

GHOST = 2  # planes of the neighbouring slab a PLM face flux reaches


def split(nz: int, world: int, rank: int) -> tuple:
    """Global planes [z0, z1) of `rank`: contiguous, sizes differing by at most
    one, the larger slabs first."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank")
    base, extra = divmod(nz, world)
    z0 = rank * base + min(rank, extra)
    return z0, z0 + base + (1 if rank < extra else 0)


class Halo:
    """Ghost-plane plan of one rank's slab.

    Local planes: `g_lo` ghosts, the `nact` active planes (global z0..z1-1),
    `g_hi` ghosts.  A side has ghosts when a neighbour lies across it: always
    on a periodic z axis, otherwise everywhere but the domain's ends."""

    def __init__(self, nz: int, world: int, rank: int, periodic: bool):
        self.world, self.rank, self.periodic = world, rank, periodic
        self.z0, self.z1 = split(nz, world, rank)
        self.nact = self.z1 - self.z0
        if nz < GHOST * world:  # the smallest slab has nz // world planes
            raise ValueError(f"every slab needs at least {GHOST} planes "
                             f"(nz = {nz} over {world} ranks)")
        self.lo_nbr = (rank - 1) % world if (periodic or rank > 0) else None
        self.hi_nbr = (rank + 1) % world if (periodic or rank < world - 1) else None
        self.g_lo = GHOST if self.lo_nbr is not None else 0
        self.g_hi = GHOST if self.hi_nbr is not None else 0
        self.nloc = self.g_lo + self.nact + self.g_hi
        # local index of the first active plane, and whether it is the
        # domain's first plane (its lo face is then the periodic wrap or a wall)
        self.act0 = self.g_lo
        self.holds_z0 = self.z0 == 0

    def global_planes(self, nz: int) -> list:
        """Global plane index of every local plane (ghosts wrap when periodic)."""
        return [(self.z0 - self.g_lo + i) % nz for i in range(self.nloc)]

    def exchange(self, get: Callable, put: Callable, make_like: Callable,
                 group=None) -> None:
        """Fill this rank's ghost planes from its neighbours' active planes.

        Every rank posts its operations in the same order: sends of its lowest
        active planes to lo_nbr (tag 0) and its highest to hi_nbr (tag 1), then
        the receive of its hi ghosts from hi_nbr (tag 0) and of its lo ghosts
        from lo_nbr (tag 1); between one pair of ranks the messages then match
        in order whether or not the backend honours tags."""
        import torch.distributed as dist
        lo_send = get(self.act0, GHOST) if self.lo_nbr is not None else None
        hi_send = get(self.act0 + self.nact - GHOST, GHOST) if self.hi_nbr is not None else None
        lo_recv = hi_recv = None
        ops = []
        if self.lo_nbr is not None and self.lo_nbr != self.rank:
            ops.append(dist.P2POp(dist.isend, lo_send, self.lo_nbr, group, 0))
        if self.hi_nbr is not None and self.hi_nbr != self.rank:
            ops.append(dist.P2POp(dist.isend, hi_send, self.hi_nbr, group, 1))
        if self.hi_nbr is not None:
            if self.hi_nbr == self.rank:
                hi_recv = lo_send  # one periodic rank: its own lowest planes
            else:
                hi_recv = make_like(lo_send if lo_send is not None else hi_send)
                ops.append(dist.P2POp(dist.irecv, hi_recv, self.hi_nbr, group, 0))
        if self.lo_nbr is not None:
            if self.lo_nbr == self.rank:
                lo_recv = hi_send
            else:
                lo_recv = make_like(hi_send if hi_send is not None else lo_send)
                ops.append(dist.P2POp(dist.irecv, lo_recv, self.lo_nbr, group, 1))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        if hi_recv is not None:
            put(self.act0 + self.nact, hi_recv)
        if lo_recv is not None:
            put(0, lo_recv)


def allreduce_max_bits(t, group=None) -> None:
    """In-place max over ranks of CFL maxima held as the bit patterns of
    non-negative doubles (which order like unsigned integers)."""
    import torch.distributed as dist
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)


def allreduce_sum(t, group=None) -> None:
    import torch.distributed as dist
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
