"""The N > 1 path of bench.py on CPU: two gloo ranks, each integrating its own
independent instance (the oracle stands in for the device), combined the way
the benchmark combines them (max of the per-rank times, whole-job value)."""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path[:0] = [ROOT, os.path.join(ROOT, "vespa.jl_b200")]
    import bench
    import vespa_b200 as vb
    from oracle import oracle as O
    ranks = bench.Ranks(world, backend="gloo")
    try:
        # each rank: its own seed, its own instance, no data-path exchange
        prob = vb.smooth_random_problem((16, 16, 8), seed=vb.problem.DEFAULT_SEED + ranks.rank)
        U = vb.initial_state(prob)
        g = O.grid_from_problem(prob)
        t, n = O.evolve(g, U, float("inf"), max_steps=3)
        ms = 10.0 * (ranks.rank + 1)          # a synthetic per-rank time
        ms_max = ranks.max(ms)
        cells = ranks.sum(float(prob.ncell))
        ranks.barrier()
        out.put((ranks.rank, n, float((U[0] ** 2).sum()), ms_max, cells,
                 bench.weak_scaling_value(prob.ncell, ranks.world, 3, ms_max)))
    finally:
        ranks.close()


def test_two_gloo_ranks_weak_scaling():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    (r0, n0, m0, ms0, c0, v0), (r1, n1, m1, ms1, c1, v1) = res
    assert n0 == n1 == 3
    assert m0 != m1                       # independent instances (different seeds)
    assert ms0 == ms1 == 20.0             # max over ranks on every rank
    assert c0 == c1 == 2 * 16 * 16 * 8    # whole-job cells
    assert v0 == v1 == pytest.approx(2 * 16 * 16 * 8 * 3 / 0.020 / 1e6)
