"""The device AMR path (vb_amr_*) against the AMR oracle (bit for bit) and
against the reference's AMR gates (test/test_sedov.jl, test/test_reflux.jl,
test/test_amr_ka_flux.jl)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _pair(vb, oracle, prob):
    from vespa_b200 import amr as A
    dev = A.AmrSimulation(A.AmrMesh(prob.dims, prob.domain), prob)
    ora = oracle.Amr(oracle.grid_from_problem(prob))
    ora.set_state(vb.initial_state(prob))
    return dev, ora


def _same(dev, ora):
    lev_d, cx_d = dev.leaves()
    lev_o, cx_o = ora.leaves()
    assert np.array_equal(lev_d, lev_o)
    assert np.array_equal(cx_d, cx_o)
    assert np.array_equal(dev.state(), ora.state())


@pytest.mark.parametrize("case", ["sod64", "mixed2d", "periodic3d", "sedov16"])
def test_unrefined_amr_matches_uniform_oracle(vb, oracle, case):
    from vespa_b200 import amr as A
    if case == "sod64":
        prob = vb.sod_problem_defaults(n=64)
    elif case == "mixed2d":
        prob = vb.Problem(name="m2", dims=(12, 9), domain=((0, 1), (0, 0.75)), gamma=1.4,
                          bcs=((vb.Outflow, vb.Reflecting), (vb.Reflecting, vb.Outflow)),
                          init_prim=lambda p: vb.initial_primitive(vb.smooth_random_problem((12, 9))))
    elif case == "periodic3d":
        prob = vb.smooth_random_problem((6, 5, 4))
    else:
        prob = vb.sedov_problem(n=16)
    dev, _ = _pair(vb, oracle, prob)
    g = oracle.grid_from_problem(prob)
    ref = np.ascontiguousarray(vb.initial_state(prob))
    for _ in range(5):
        dt = oracle.compute_dt(g, ref)
        assert A.compute_dt(dev) == dt
        oracle.step(g, ref, dt)
        A.step(dev, dt)
    assert np.array_equal(dev.state(), ref)
    ref_tot = oracle.conserved_totals(g, ref)
    np.testing.assert_allclose(A.conserved_totals(dev), ref_tot, rtol=1e-13,
                               atol=1e-13 * np.abs(ref_tot).max())
    dev.close()


def test_refined_steps_match_oracle(vb, oracle):
    from vespa_b200 import amr as A
    prob = vb.sedov_problem(n=16)
    dev, ora = _pair(vb, oracle, prob)
    for leaves in ([119, 120, 135, 136], [0, 255], [3]):
        dev.refine(leaves)
        ora.refine(leaves)
        _same(dev, ora)
    for _ in range(6):
        dt = ora.compute_dt()
        assert A.compute_dt(dev) == dt
        for lev in (None, 1):
            assert A.compute_dt(dev, 1 if lev else None) == ora.compute_dt(1 if lev else -1)
        ora.step(dt)
        A.step(dev, dt)
    _same(dev, ora)
    np.testing.assert_array_equal(dev.indicator(), ora.indicator())
    # one level alone (step!(sim, dt; level))
    dt = ora.compute_dt(1)
    ora.step(dt, 1)
    A.step(dev, dt, level=1)
    _same(dev, ora)
    dev.close()


@pytest.mark.parametrize("subcycle", [False, True])
def test_refined_sod_evolve_matches_oracle(vb, oracle, subcycle):
    """test/test_amr_ka_flux.jl:36-55 / test/test_reflux.jl:13-35 on the device:
    the whole evolve! with regrids, bit for bit, conserving to 1e-9."""
    from vespa_b200 import amr as A
    prob = vb.sod_problem_defaults(n=64)
    dev, ora = _pair(vb, oracle, prob)
    t0 = A.conserved_totals(dev)
    pol = A.RefinementPolicy(refine_above=0.1, max_level=2, every=4)
    A.evolve(dev, policy=pol, subcycle=subcycle)
    ora.evolve(prob.tfinal, refine_above=0.1, max_level=2, every=4, subcycle=subcycle)
    assert dev.max_level >= 1
    assert dev.step == ora.step_count and dev.t == ora.t
    _same(dev, ora)
    t1 = A.conserved_totals(dev)
    assert abs(t1.mass - t0.mass) <= 1e-9 * t0.mass
    assert abs(t1.energy - t0.energy) <= 1e-9 * t0.energy
    dev.close()


def test_nested_registers_match_oracle(vb, oracle):
    """test/test_reflux.jl:37-51: three levels, nested registers."""
    from vespa_b200 import amr as A
    prob = vb.sod_problem_defaults(n=64)
    dev, ora = _pair(vb, oracle, prob)
    A.evolve(dev, policy=A.RefinementPolicy(0.05, 3, 3), subcycle=True)
    ora.evolve(prob.tfinal, refine_above=0.05, max_level=3, every=3, subcycle=True)
    assert dev.max_level >= 2
    _same(dev, ora)
    dev.close()


def test_small_sedov_matches_oracle(vb, oracle):
    from vespa_b200 import amr as A
    prob = vb.sedov_problem(n=32, tfinal=0.02)
    dev, ora = _pair(vb, oracle, prob)
    A.evolve(dev, policy=A.RefinementPolicy(0.05, 2, 4))
    ora.evolve(prob.tfinal, refine_above=0.05, max_level=2, every=4)
    _same(dev, ora)
    dev.close()


def _shock_radius(sim):
    rho = sim.state()[0]
    x, y = sim.cell_centers()
    v = sim.cell_volumes()
    thresh = 0.5 * (1.0 + rho.max())
    m = rho >= thresh
    r = np.hypot(x - 0.5, y - 0.5)
    return float(np.sum(r[m] * v[m]) / np.sum(v[m]))


def test_sedov_reference_gates(vb):
    """test/test_sedov.jl: 64^2, refine_above 0.2, max_level 2, every 4."""
    from vespa_b200 import amr as A
    radii = []
    for tf in (0.02, 0.04):
        prob = vb.sedov_problem(n=64, tfinal=tf)
        sim = A.AmrSimulation(A.AmrMesh(prob.dims, prob.domain), prob)
        n0 = sim.nleaf
        t0 = A.conserved_totals(sim)
        A.evolve(sim, policy=A.RefinementPolicy(0.2, 2, 4))
        t1 = A.conserved_totals(sim)
        radii.append(_shock_radius(sim))
        if tf == 0.04:
            assert sim.nleaf > n0 and sim.max_level >= 1
            assert abs(t1.mass - t0.mass) <= 1e-9 * t0.mass
            assert abs(t1.energy - t0.energy) <= 1e-9 * t0.energy
            W = vb.cons2prim(sim.state(), prob.gamma)
            assert np.all(W[0] > 0) and np.all(W[4] > 0)
            x, y = sim.cell_centers()
            q = (x >= 0.5).astype(int) + 2 * (y >= 0.5).astype(int)
            mass = W[0] * sim.cell_volumes()
            quad = np.array([mass[q == k].sum() for k in range(4)])
            assert quad.max() - quad.min() < 1e-2 * quad.max()
        sim.close()
    ratio = radii[1] / radii[0]
    assert 0.7 * np.sqrt(2.0) < ratio < 1.3 * np.sqrt(2.0)


def test_sedov48_config_matches_oracle_first_steps(vb, oracle):
    """The benchmark configuration (48^2 base, 3-cell hot spot, refine above
    0.2 up to 4 levels every 4 steps): first 120 steps bit for bit."""
    from vespa_b200 import amr as A
    prob = vb.sedov_problem(n=48, r0=3.0 / 48, tfinal=0.05)
    dev, ora = _pair(vb, oracle, prob)
    A.evolve(dev, policy=A.RefinementPolicy(0.2, 4, 4), max_steps=120)
    ora.evolve(prob.tfinal, max_steps=120, refine_above=0.2, max_level=4, every=4)
    assert dev.step == 120
    _same(dev, ora)
    dev.close()
