"""Slab decomposition of one grid across ranks, on CPU: gloo ranks, each
stepping its z slab with the oracle's per-cell gather and exchanging two
ghost planes per side per RK2 stage through vespa_b200.slab.Halo (the same
protocol the device path runs over NCCL), the CFL maximum all-reduced.
After several steps the assembled slabs must be bit-identical to the
single-domain oracle: periodic and walled z axes, even and uneven splits,
two and three ranks."""
import math
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path[:0] = [ROOT, os.path.join(ROOT, "vespa.jl_b200")]

from vespa_b200 import slab as S  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _problem(dims, zbc):
    from vespa_b200 import problem as P
    prob = P.smooth_random_problem(dims, seed=9)
    prob.bcs = ((P.Periodic, P.Periodic), (P.Outflow, P.Reflecting), zbc)
    return prob


def _rank_main(rank, world, port, dims, zbc_name, nsteps, out):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path[:0] = [ROOT, os.path.join(ROOT, "vespa.jl_b200")]
    import datetime
    import torch
    import torch.distributed as dist
    from oracle import oracle as O
    from vespa_b200 import problem as P
    from vespa_b200 import slab as S
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        zbc = {"periodic": (P.Periodic, P.Periodic), "walls": (P.Reflecting, P.Outflow)}[zbc_name]
        prob = _problem(dims, zbc)
        nx, ny, nz = dims
        g = O.grid_from_problem(prob)
        halo = S.Halo(nz, world, rank, periodic=zbc_name == "periodic")
        Ug = P.initial_state(prob).reshape(5, nz, ny, nx)
        # this rank's view: only its slab and ghost planes hold data
        work = np.full((5, nz, ny, nx), np.nan)
        planes = halo.global_planes(nz)
        work[:, planes] = Ug[:, planes]
        flat = work.reshape(5, -1)
        lin0, lin1 = halo.z0 * nx * ny, halo.z1 * nx * ny

        def get(first, count):
            return torch.from_numpy(np.ascontiguousarray(work[:, planes[first:first + count]]))

        def put(first, t):
            work[:, planes[first:first + t.shape[1]]] = t.numpy()

        w = [(b - a) / n for (a, b), n in zip(prob.domain, dims)]
        vol = w[0] * w[1] * w[2]
        acc = np.zeros_like(flat)
        t = 0.0
        for _ in range(nsteps):
            inv = torch.tensor([O.invdt_range(g, flat, lin0, lin1)], dtype=torch.float64)
            S.allreduce_max_bits(inv)
            dt = prob.cfl / float(inv[0]) if float(inv[0]) > 0 else math.inf
            invV = dt / (1.0 * vol)
            u0 = flat[:, lin0:lin1].copy()
            O.accumulate_flux_range(g, flat, acc, lin0, lin1)
            flat[:, lin0:lin1] = u0 - invV * acc[:, lin0:lin1]
            halo.exchange(get, put, torch.empty_like)
            O.accumulate_flux_range(g, flat, acc, lin0, lin1)
            flat[:, lin0:lin1] = 0.5 * u0 + 0.5 * (flat[:, lin0:lin1] - invV * acc[:, lin0:lin1])
            halo.exchange(get, put, torch.empty_like)
            t += dt
        mine = torch.from_numpy(np.ascontiguousarray(flat[:, lin0:lin1]))
        parts = [None] * world
        dist.all_gather_object(parts, (halo.z0, halo.z1, mine.numpy(), t))
        if rank == 0:
            out.put(parts)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("dims,zbc,world", [((6, 5, 12), "periodic", 2),
                                            ((5, 4, 11), "walls", 3),
                                            ((4, 6, 9), "periodic", 3),
                                            ((6, 4, 8), "walls", 2)])
def test_slabs_bit_identical_to_single_domain(dims, zbc, world):
    import multiprocessing as mp
    from oracle import oracle as O
    from vespa_b200 import problem as P
    nsteps = 4
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, dims, zbc, nsteps, q))
             for r in range(world)]
    for p in procs:
        p.start()
    parts = q.get(timeout=180)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    zb = {"periodic": (P.Periodic, P.Periodic), "walls": (P.Reflecting, P.Outflow)}[zbc]
    prob = _problem(dims, zb)
    U = P.initial_state(prob)
    t, n = O.evolve(O.grid_from_problem(prob), U, math.inf, max_steps=nsteps)
    nx, ny, nz = dims
    got = np.full_like(U, np.nan).reshape(5, nz, ny, nx)
    for z0, z1, part, tr in parts:
        got[:, z0:z1] = part.reshape(5, z1 - z0, ny, nx)
        assert tr == t
    assert np.array_equal(got.reshape(U.shape), U)


def test_split_and_halo_plan():
    assert [S.split(11, 3, r) for r in range(3)] == [(0, 4), (4, 8), (8, 11)]
    h = S.Halo(11, 3, 0, periodic=False)
    assert (h.lo_nbr, h.hi_nbr, h.g_lo, h.g_hi, h.nloc, h.act0) == (None, 1, 0, 2, 6, 0)
    h = S.Halo(11, 3, 2, periodic=True)
    assert (h.lo_nbr, h.hi_nbr, h.g_lo, h.g_hi, h.nloc) == (1, 0, 2, 2, 7)
    assert h.global_planes(11) == [6, 7, 8, 9, 10, 0, 1]
    h = S.Halo(8, 1, 0, periodic=True)
    assert (h.lo_nbr, h.hi_nbr) == (0, 0) and h.global_planes(8) == [6, 7] + list(range(8)) + [0, 1]
    with pytest.raises(ValueError):
        S.Halo(5, 3, 0, periodic=True)  # slabs of fewer than two planes
