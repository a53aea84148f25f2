"""Batches of independent problems: one persistent launch per stage over all
boxes, per-box clocks and CFL dt, graph-replayed steps.  Each box must step
exactly as the same problem stepped alone (which the parity tests pin to the
oracle), in both precision modes."""
import math

import numpy as np
import pytest

import vespa_b200 as vb
from vespa_b200 import problem as P

pytestmark = pytest.mark.gpu


def box_problems():
    out = []
    specs = [((32, 32, 32), P.Periodic, 1), ((48, 32, 40), P.Outflow, 2),
             ((16, 16, 9), P.Reflecting, 3), ((64, 48, 20), P.Periodic, 4)]
    for dims, bc, seed in specs:
        p = P.smooth_random_problem(dims, seed=seed)
        p.bcs = bc
        out.append(p)
    out.append(P.riemann_box_problem(7, side=32))  # outflow, strong discontinuity
    return out


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_boxes_equal_single_runs(vb, precision):
    probs = box_problems()
    batch = vb.Batch(probs, precision=precision)
    batch.run_steps(3)
    batch.run_steps(2)  # a second graph (different length), continuing the clocks
    for i, p in enumerate(probs):
        sim = vb.Simulation(vb.B200Mesh(p.dims, p.domain), p, precision=precision)
        sim.set_kernel("tiled")  # the batch always runs the tiled kernel
        vb.evolve(sim, tfinal=math.inf, max_steps=5)
        t, n = batch.time(i)
        assert n == 5 and t == sim.t, (i, t, sim.t)
        a, b = batch.state(i), sim.state()
        assert np.array_equal(a, b), (i, float(np.abs(a - b).max()))


def test_batch_graph_replay_is_deterministic(vb):
    probs = box_problems()[:3]
    a = vb.Batch(probs, precision="mixed")
    b = vb.Batch(probs, precision="mixed")
    for _ in range(3):
        a.run_steps(2)
    b.run_steps(6)
    for i in range(len(probs)):
        assert a.time(i) == b.time(i)
        assert np.array_equal(a.state(i), b.state(i))


def test_batch_of_riemann_boxes_stays_physical(vb):
    probs = [P.riemann_box_problem(i, sides=(32, 48, 64)) for i in range(6)]
    batch = vb.Batch(probs, precision="mixed")
    batch.run_steps(10)
    for i, p in enumerate(probs):
        W = P.cons2prim(batch.state(i), p.gamma)
        assert np.all(np.isfinite(W)) and np.all(W[0] > 0) and np.all(W[4] > 0)
        assert batch.time(i)[1] == 10


def test_batch_rejects_untileable_boxes(vb):
    bad = P.smooth_random_problem((24, 16, 8))
    with pytest.raises(vb.VespaB200Error) as e:
        vb.Batch([bad])
    assert e.value.status == 6
