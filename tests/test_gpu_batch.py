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


def test_seeded_64_box_batch_equals_single_runs_and_oracle(vb, oracle):
    """The benchmark's batch (64 seeded Riemann boxes, sides from
    {32, ..., 256}, about 282 M cells): after 3 mixed-precision steps every
    box equals its single-grid run bit for bit; in float64 every box of side
    64 or less equals the oracle bit for bit."""
    probs = [P.riemann_box_problem(i, seed=P.DEFAULT_SEED) for i in range(64)]
    assert len({p.dims[0] for p in probs}) >= 5  # the draw spans the side list
    steps = 3
    batch = vb.Batch(probs, precision="mixed")
    batch.run_steps(steps)
    for i, p in enumerate(probs):
        U0 = P.initial_state(p)
        sim = vb.Simulation(vb.B200Mesh(p.dims, p.domain), p, precision="mixed", initial=U0)
        sim.set_kernel("tiled")
        vb.evolve(sim, tfinal=math.inf, max_steps=steps)
        assert batch.time(i) == (sim.t, steps), i
        a = batch.state(i)
        b = sim.state()
        sim.close()
        assert np.array_equal(a, b), (i, p.dims, float(np.abs(a - b).max()))
    batch.close()

    batch = vb.Batch(probs, precision="fp64")
    batch.run_steps(steps)
    checked = 0
    for i, p in enumerate(probs):
        if p.dims[0] > 64:
            continue
        U = P.initial_state(p)
        t, n = oracle.evolve(oracle.grid_from_problem(p), U, math.inf, max_steps=steps, mode=1)
        assert batch.time(i) == (t, n), i
        a = batch.state(i)
        assert np.array_equal(a, U), (i, p.dims, float(np.abs(a - U).max()))
        checked += 1
    batch.close()
    assert checked >= 10


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_autotune_restores_state_and_keeps_bits(vb, precision):
    """vb_batch_autotune times every work-item depth on the batch itself,
    then restores states and clocks; the chosen layout steps to the same
    bits as the default one."""
    probs = box_problems()
    a = vb.Batch(probs, precision=precision)
    b = vb.Batch(probs, precision=precision)
    a.run_steps(1)
    b.run_steps(1)
    s0 = [a.state(i) for i in range(len(probs))]
    cap, ms = a.autotune(2)
    assert cap in (0, 16, 24, 32, 48, 64, 96, 128) and ms > 0
    for i in range(len(probs)):
        assert a.time(i) == b.time(i)
        assert np.array_equal(a.state(i), s0[i])
    a.run_steps(3)
    b.run_steps(3)
    for i in range(len(probs)):
        assert a.time(i) == b.time(i)
        assert np.array_equal(a.state(i), b.state(i)), (i, cap)
    a.close()
    b.close()
