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

import math
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


# z-lo face order classes of the tiled kernels (the reference's emission order)
_LO_AFTER = 2  # emitted by the periodic partner at the domain's far end


class SlabSimulation:
    """One rank's slab of a z-split uniform 3D grid, stepped on its GPU.

    The rank's grid holds its planes plus the ghost planes of `Halo`; the
    tiled kernels compute every local plane, the ghosts' results are
    replaced by the exchange before anything reads them, and the window set
    with vb_grid_set_zwindow keeps the CFL maximum and the totals to the
    rank's own planes and gives the domain's first plane its global face
    order.  Per step: CFL maximum all-reduced (max), dt, stage 1, stage-1
    ghosts exchanged, stage 2, clock, state ghosts exchanged.  The results
    equal one grid stepped alone, bit for bit.

    `group`: the torch.distributed group of the ranks (None: the default
    group, or a single rank when torch.distributed is not initialised).
    `world`/`rank` override the group's size and rank: slabs of one process
    then move their planes themselves (phase / get_planes / put_planes /
    cfl_bits), which is how a single GPU runs several slabs.
    """

    def __init__(self, problem, *, precision: str = "fp64", group=None, ctx=None,
                 initial=None, kz: Optional[int] = None, world: Optional[int] = None,
                 rank: Optional[int] = None):
        import numpy as np
        import torch
        import torch.distributed as dist
        from . import problem as P
        from .simulation import B200Mesh, Simulation
        from ._lib import default_context
        if problem.ndim != 3:
            raise ValueError("slab decomposition splits 3D grids along z")
        self.group = group
        dist_on = dist.is_available() and dist.is_initialized()
        self.world = world if world is not None else (dist.get_world_size(group) if dist_on else 1)
        self.rank = rank if rank is not None else (dist.get_rank(group) if dist_on else 0)
        nx, ny, nz = problem.dims
        pairs = problem.bc_pairs()
        periodic = pairs[2][0] == P.Periodic.code
        self.halo = h = Halo(nz, self.world, self.rank, periodic)
        self.global_dims = (nx, ny, nz)
        code_bc = {P.Outflow.code: P.Outflow, P.Periodic.code: P.Periodic,
                   P.Reflecting.code: P.Reflecting}
        # a side with ghosts is an ordinary outflow side to the local grid:
        # only ghost planes see it, and the exchange overwrites them
        zlo = code_bc[pairs[2][0]] if h.g_lo == 0 else P.Outflow
        zhi = code_bc[pairs[2][1]] if h.g_hi == 0 else P.Outflow
        bcs = tuple((code_bc[a], code_bc[b]) for a, b in pairs[:2]) + ((zlo, zhi),)
        (x0, x1), (y0, y1), (zd0, zd1) = problem.domain
        wz = (zd1 - zd0) / nz
        local = P.Problem(name=problem.name + f"[slab {self.rank}/{self.world}]",
                          dims=(nx, ny, h.nloc), domain=((x0, x1), (y0, y1),
                                                         (zd0 + (h.z0 - h.g_lo) * wz,
                                                          zd0 + (h.z0 - h.g_lo + h.nloc) * wz)),
                          gamma=problem.gamma, bcs=bcs, tfinal=math.inf, cfl=problem.cfl,
                          # the slab's state comes from the whole domain's (below)
                          init=lambda x, y, z: (1.0, 0.0, 0.0, 0.0, 1.0))
        self.ctx = ctx or default_context()
        self.planes = h.global_planes(nz)
        if initial is None:
            initial = P.initial_state(problem)
        Ug = np.asarray(initial).reshape(5, nz, ny, nx)
        Ul = np.ascontiguousarray(Ug[:, self.planes].reshape(5, -1))
        self.sim = Simulation(B200Mesh(local.dims, local.domain), local, precision=precision,
                              ctx=self.ctx, initial=Ul)
        self.sim.set_kernel("tiled", kz=kz)
        zcls0 = _LO_AFTER if (periodic and h.holds_z0 and nz > 1) else -1
        self._call("vb_grid_set_zwindow", h.act0, h.act0 + h.nact, zcls0, wz)
        dev = torch.device("cuda", self.ctx.device)
        self._bits = torch.zeros(1, dtype=torch.int64, device=dev)
        n = 5 * GHOST * nx * ny
        self._bufs = {k: torch.empty(n, dtype=torch.float64, device=dev) for k in ("lo", "hi")}
        self._stream = torch.cuda.ExternalStream(self.ctx.stream, device=dev)
        self.t = 0.0
        self.step_count = 0

    # -- library calls on the rank's grid --
    def _call(self, name, *args):
        from . import _lib
        _lib.call(name, self.sim.handle, *args)

    def phase(self, p: int) -> None:
        """One phase of a step (_lib.PHASE_*), queued on the library's stream."""
        self._call("vb_grid_step_phase", p)

    def get_planes(self, which: int, first: int, count: int, out=None):
        """Local planes [first, first + count) of the state (0) or stage-1 state
        (1) as a (5, count, ny * nx) device tensor (queued on the library's stream)."""
        import torch
        nx, ny, _ = self.global_dims
        if out is None:
            out = torch.empty(5 * count * nx * ny, dtype=torch.float64, device=self._bits.device)
        self._call("vb_grid_planes", which, first, count, out.data_ptr(), 0)
        return out.view(5, count, nx * ny)

    def put_planes(self, which: int, first: int, t) -> None:
        t = t.contiguous()
        self._call("vb_grid_planes", which, first, t.shape[1], t.data_ptr(), 1)

    def cfl_bits(self, t=None, put: bool = False):
        """The running CFL maximum as an int64 device word (read, or written back)."""
        t = self._bits if t is None else t
        self._call("vb_grid_cfl_bits", t.data_ptr(), 1 if put else 0)
        return t

    def _exchange(self, which):
        import torch
        h = self.halo

        def get(first, count):
            buf = self._bufs["lo" if first == h.act0 else "hi"]
            return self.get_planes(which, first, count, out=buf)

        def put(first, t):
            self.put_planes(which, first, t)

        # the collectives order themselves after the library's stream work
        with torch.cuda.stream(self._stream):
            h.exchange(get, put, torch.empty_like, self.group)

    def _allreduce_cfl(self):
        import torch
        with torch.cuda.stream(self._stream):
            self.cfl_bits()
            if self.world > 1:
                allreduce_max_bits(self._bits, self.group)
            self.cfl_bits(put=True)

    def step(self, nsteps: int = 1) -> None:
        """nsteps CFL steps of the whole domain (every rank calls it)."""
        from . import _lib
        for _ in range(nsteps):
            self.phase(_lib.PHASE_CFL)
            self._allreduce_cfl()
            self.phase(_lib.PHASE_FINALIZE)
            self.phase(_lib.PHASE_STAGE1)
            self._exchange(1)
            self.phase(_lib.PHASE_STAGE2)
            self.phase(_lib.PHASE_ADVANCE)
            self._exchange(0)
            self.step_count += 1

    def time(self) -> tuple:
        return self.sim.t, self.sim.step

    def own_state(self):
        """This rank's planes of the conserved state, (5, nact * ny * nx)."""
        nx, ny, _ = self.global_dims
        U = self.sim.state().reshape(5, self.halo.nloc, ny, nx)
        a = self.halo.act0
        return U[:, a:a + self.halo.nact].reshape(5, -1)

    def conserved_totals(self):
        """Totals of the whole domain (all-reduced sum; every rank calls it)."""
        import numpy as np
        import torch
        tot = np.array(self.sim_totals())
        if self.world > 1:
            t = torch.tensor(tot, dtype=torch.float64, device=self._bits.device)
            allreduce_sum(t, self.group)
            tot = t.cpu().numpy()
        return tot

    def sim_totals(self):
        from .simulation import conserved_totals
        return conserved_totals(self.sim)

    def close(self):
        self.sim.close()
