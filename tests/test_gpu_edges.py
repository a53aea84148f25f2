"""Edge cases and error paths of the device library: empty face batches,
1- and 2-cell axes, the maximum-size guards, and the configurations the
adjoint, batch and AMR entry points refuse."""
import math

import numpy as np
import pytest

import vespa_b200 as vb
from vespa_b200 import amr as A
from vespa_b200 import problem as P

from test_gpu_parity import assert_bit_identical, make_sim, problem_from

pytestmark = pytest.mark.gpu


def test_empty_face_batch_is_a_no_op(vb):
    F = np.zeros((0, 5))
    out = vb.compute_face_fluxes(vb.B200Flux(), vb.IdealHydro(1.4), F, np.zeros((0, 5)),
                                 np.zeros((0, 5)), np.zeros(0, dtype=np.int32))
    assert out.shape == (0, 5)


@pytest.mark.parametrize("dims,bc", [((1,), 1), ((2,), 1), ((1,), 0), ((1, 3), 2), ((2, 1, 2), 1)])
def test_one_and_two_cell_axes_bit_identical(vb, oracle, dims, bc):
    nd = len(dims)
    prob = problem_from(dims, [(0.0, 1.0)] * nd, [bc] * nd, [bc] * nd, 1.4, 0.4)
    U0 = P.initial_state(P.smooth_random_problem(dims, seed=77))
    sim = make_sim(prob, U0)
    vb.evolve(sim, max_steps=4)
    U = U0.copy()
    g = oracle.make_grid(dims, [0] * nd, [1] * nd, [bc] * nd, [bc] * nd, 1.4, 0.4)
    t, n = oracle.evolve(g, U, math.inf, max_steps=4, mode=1)
    assert sim.step == n and sim.t == t
    assert_bit_identical(sim.state(), U)


def test_tiled_kernel_refused_where_it_does_not_apply(vb):
    prob = P.smooth_random_problem((24, 16, 4))       # nx not a multiple of 16
    sim = make_sim(prob, P.initial_state(prob))
    with pytest.raises(vb.VespaB200Error) as e:
        sim.set_kernel("tiled")
    assert "VB_ENOTSUP" in str(e.value)
    with pytest.raises(vb.VespaB200Error):
        sim.set_kernel("cell", kz=0)                    # chunk out of range


def test_adjoint_refuses_mixed_and_non_periodic_grids(vb):
    prob = P.kelvin_helmholtz_problem(n=16)
    mixed = make_sim(prob, P.initial_state(prob), "mixed")
    with pytest.raises(vb.VespaB200Error) as e:
        vb.Adjoint(mixed, 4, 2)
    assert "VB_ENOTSUP" in str(e.value)
    sod = vb.sod_problem_defaults(32)
    s = make_sim(sod, P.initial_state(sod))
    with pytest.raises(vb.VespaB200Error) as e:
        vb.Adjoint(s, 4, 2)
    assert "VB_ENOTSUP" in str(e.value)
    fp = make_sim(prob, P.initial_state(prob))
    adj = vb.Adjoint(fp, 4, 2)
    with pytest.raises(vb.VespaB200Error) as e:  # no recorded forward run yet
        adj.backward(np.zeros((5, fp.ncell)))
    assert "VB_EINVAL" in str(e.value)
    adj.close()


def test_amr_rejects_bad_leaves_and_keeps_state_without_tags(vb):
    prob = vb.sedov_problem(n=8)
    sim = A.AmrSimulation(A.AmrMesh(prob.dims, prob.domain), prob)
    with pytest.raises(vb.VespaB200Error) as e:
        sim.refine([64])
    assert "VB_EINVAL" in str(e.value)
    U0 = sim.state()
    # max_level 0: nothing may refine
    assert A.regrid(sim, A.RefinementPolicy(0.0, 0, 1)) == 0
    assert sim.nleaf == 64 and np.array_equal(sim.state(), U0)
    # refining the same leaf twice in one call is refining it once
    sim.refine([9, 9])
    assert sim.nleaf == 64 + 3


def test_batch_rejects_boxes_the_tiled_kernel_cannot_take(vb):
    good = P.riemann_box_problem(0, side=32)
    bad = P.Problem(name="b", dims=(24, 32, 8), domain=((0, 1),) * 3, gamma=1.4,
                    bcs=P.Outflow, init=good.init)
    with pytest.raises(vb.VespaB200Error) as e:
        vb.Batch([good, bad])
    assert "VB_ENOTSUP" in str(e.value)


def test_bounded_wait_gives_up_and_reports_a_timeout(vb, oracle):
    """The failure path of the tiled kernels' TMA stage waits, made to run out
    without faulting anything: a block waits (limit 1 ms) on an mbarrier that
    nothing completes, takes the stage kernels' abandon path and raises the
    grid's timeout flag; the host returns VB_ETIMEOUT, the state and clock are
    untouched, and the grid (and context) keep working afterwards."""
    from vespa_b200 import _lib
    prob = P.smooth_random_problem((32, 32, 16), seed=5)
    U0 = P.initial_state(prob)
    sim = make_sim(prob, U0)
    sim.set_kernel("tiled")
    rc = _lib.load().vb_grid_selftest_wait(sim.handle, 1_000_000)
    assert rc == _lib.VB_ETIMEOUT
    assert "gave up" in _lib.last_error()
    assert sim.t == 0.0 and sim.step == 0
    assert np.array_equal(sim.state(), U0)
    vb.evolve(sim, max_steps=2)  # no stale flag: the next steps run and match the oracle
    U = U0.copy()
    t, n = oracle.evolve(oracle.grid_from_problem(prob), U, math.inf, max_steps=2, mode=1)
    assert sim.step == n == 2 and sim.t == t
    assert_bit_identical(sim.state(), U)
    with pytest.raises(vb.VespaB200Error) as e:
        _lib.call("vb_grid_selftest_wait", sim.handle, 0)
    assert e.value.status == _lib.VB_EINVAL


def test_autotune_cache_file(vb, tmp_path, monkeypatch):
    """VB_AUTOTUNE_CACHE: a tuning is appended as "key kz taper" (key: GPU
    model, precision, dims and boundaries), and a grid created later starts
    from the file's entry for its key."""
    path = tmp_path / "tune.txt"
    monkeypatch.setenv("VB_AUTOTUNE_CACHE", str(path))
    prob = P.smooth_random_problem((64, 64, 40), seed=3)
    sim = make_sim(prob, P.initial_state(prob))
    sim.set_kernel("tiled")
    kz, _ = sim.autotune(1)
    sim.close()
    key, kz_file, taper_file = path.read_text().split()
    assert int(kz_file) == kz and int(taper_file) in (0, 1)
    parts = key.split(":")
    assert len(parts) == 5 and parts[2:] == ["64/11", "64/11", "40/11"]
    # an entry for a shape this process never tuned: the new grid takes it
    parts[4] = "36/11"
    with open(path, "a") as f:
        f.write(f"{':'.join(parts)} 24 1\n")
    prob2 = P.smooth_random_problem((64, 64, 36), seed=4)
    sim2 = make_sim(prob2, P.initial_state(prob2))
    sim2.set_kernel("tiled")
    assert sim2.kz == 24 and sim2.taper
    sim2.close()
