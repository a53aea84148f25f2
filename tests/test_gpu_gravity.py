"""GPU self-gravity (src/gravity.jl on the device) against the oracle and
against the reference's gravity gates (test/test_gravity_poisson.jl,
test/test_gravity_hydro.jl).

What is bit-identical and what is not:
- the operator A x = -lap(x) V: bit-identical to the oracle (the reference's
  CSR row order, every operation rounded separately);
- the field g = -grad phi, the stage source and the free-fall dt: bit-identical
  for a given phi;
- a Poisson solve: the device's CG inner products are tree sums, the
  reference's serial sums, so phi agrees to the solver tolerance.
"""
import math

import numpy as np
import pytest

import vespa_b200 as vb
from vespa_b200 import problem as P
from test_gpu_parity import BC_OF, assert_bit_identical, make_sim

pytestmark = pytest.mark.gpu

PER, OUT, REF = 1, 0, 2


def problem(dims, domain, bcs, init, gamma=5.0 / 3.0, cfl=0.4):
    return P.Problem(name="grav", dims=dims, domain=domain, gamma=gamma, bcs=bcs, init=init, cfl=cfl)


def bcs_from(codes):
    return tuple((BC_OF[lo], BC_OF[hi]) for lo, hi in codes)


def random_density_problem(dims, seed, gamma=5.0 / 3.0, bcs=P.Periodic, cfl=0.4):
    rng = np.random.default_rng(seed)
    nd = len(dims)
    n = int(np.prod(dims))
    W = np.zeros((5, n))
    W[0] = 1.0 + 0.3 * rng.random(n)
    for d in range(nd):
        W[1 + d] = 0.2 * (rng.random(n) - 0.5)
    W[4] = 0.5 + 0.5 * rng.random(n)
    prob = P.Problem(name="grav_rand", dims=dims, domain=tuple((0.0, 1.0 + 0.25 * d) for d in range(nd)),
                     gamma=gamma, bcs=bcs, init_prim=lambda pr: W, cfl=cfl)
    return prob, np.ascontiguousarray(P.prim2cons(W, gamma))


def oracle_pair(oracle, prob, gcodes, G=1.0, maxiter=500, tol=1e-8, project_mean=True):
    g = oracle.grid_from_problem(prob)
    Pg = oracle.make_gravity(G, [c[0] for c in gcodes], [c[1] for c in gcodes], maxiter, tol,
                             project_mean)
    return g, Pg


LAP_CASES = {
    "1d_periodic16": ((16,), ((PER, PER),)),
    "2d_per_x_wall_y": ((24, 16), ((PER, PER), (OUT, REF))),
    "3d_periodic": ((16, 12, 10), ((PER, PER),) * 3),
    "3d_two_cell_axis": ((8, 6, 2), ((PER, PER), (OUT, OUT), (PER, PER))),
    "3d_one_cell_axis": ((6, 5, 1), ((PER, PER), (PER, PER), (PER, PER))),
}


@pytest.mark.parametrize("case", sorted(LAP_CASES))
def test_laplacian_bit_identical_to_oracle(vb, oracle, case):
    dims, gcodes = LAP_CASES[case]
    prob, U0 = random_density_problem(dims, seed=11)
    sim = make_sim(prob, U0)
    grav = vb.enable_gravity(sim, bcs=bcs_from(gcodes))
    g, Pg = oracle_pair(oracle, prob, gcodes)
    x = np.random.default_rng(5).standard_normal(sim.ncell)
    assert_bit_identical(vb.apply_laplacian(sim, grav, x), oracle.grav_laplacian(g, Pg, x))


def test_o1_operator_symmetric_null_space(vb):
    """test/test_gravity_poisson.jl O1 on the device operator."""
    n = 16
    prob = problem((n,), ((0.0, 1.0),), P.Periodic, lambda x, y, z: (1.0, 0.0, 0.0, 0.0, 1.0))
    sim = make_sim(prob, P.initial_state(prob))
    grav = vb.enable_gravity(sim)
    x = (np.arange(n) + 0.5) / n
    a = np.sin(2 * math.pi * x) + 0.3 * np.cos(6 * math.pi * x)
    b = np.cos(2 * math.pi * x) - 0.7 * np.sin(4 * math.pi * x)
    Aa, Ab = vb.apply_laplacian(sim, grav, a), vb.apply_laplacian(sim, grav, b)
    assert np.dot(a, Ab) == pytest.approx(np.dot(b, Aa), rel=1e-12, abs=1e-12)
    assert np.max(np.abs(vb.apply_laplacian(sim, grav, np.ones(n)))) < 1e-12
    s = np.sin(2 * math.pi * x)
    assert np.dot(s, vb.apply_laplacian(sim, grav, s)) > 0


def _fourier_l1(vb, n, A=0.1, G=1.0):
    k = 2 * math.pi
    prob = problem((n,), ((0.0, 1.0),), P.Periodic,
                   lambda x, y, z: (1.0 + A * np.cos(k * x), 0.0, 0.0, 0.0, 1.0))
    sim = make_sim(prob, P.initial_state(prob))
    grav = vb.enable_gravity(sim, G=G, tol=1e-12, maxiter=5000)
    its, rr = vb.solve_poisson(sim, grav)
    x = (np.arange(n) + 0.5) / n
    err = float(np.mean(np.abs(grav.phi - (-4 * math.pi * G * A / k ** 2) * np.cos(k * x))))
    return err, its, rr


def test_o2_fourier_mode_second_order(vb):
    e64, _, rr64 = _fourier_l1(vb, 64)
    e128, _, _ = _fourier_l1(vb, 128)
    assert rr64 < 1e-10
    assert e64 < 5e-3
    assert e64 / e128 > 3.5


def test_o2b_fourier_mode_2d(vb):
    n, A, G, k = 64, 0.1, 1.0, 2 * math.pi
    prob = problem((n, n), ((0.0, 1.0), (0.0, 1.0)), P.Periodic,
                   lambda x, y, z: (1.0 + A * np.cos(k * x) * np.cos(k * y), 0.0, 0.0, 0.0, 1.0))
    sim = make_sim(prob, P.initial_state(prob))
    grav = vb.enable_gravity(sim, G=G, tol=1e-11, maxiter=5000)
    _, rr = vb.solve_poisson(sim, grav)
    c = (np.arange(n) + 0.5) / n
    X, Y = np.meshgrid(c, c, indexing="ij")
    exact = (-4 * math.pi * G * A / (2 * k ** 2) * np.cos(k * X) * np.cos(k * Y)).reshape(-1, order="F")
    assert rr < 1e-9
    assert np.mean(np.abs(grav.phi - exact)) < 1e-2


@pytest.mark.parametrize("case", ["3d_periodic24", "2d_walls"])
def test_solve_matches_oracle_to_tolerance(vb, oracle, case):
    """Device CG vs the oracle's (serial inner products) at tol 1e-10.  A
    periodic or Neumann box is singular: the mean projection makes the
    right-hand side consistent only up to its rounding, which puts a residual
    floor between 1e-12 and 1e-11 under the serial sums on these grids (a
    tighter tol then never stops and the iteration drifts, in the reference's
    algorithm as in the oracle)."""
    if case == "3d_periodic24":
        dims, gcodes = (24, 24, 24), ((PER, PER),) * 3
    else:
        dims, gcodes = (40, 24), ((OUT, OUT), (REF, OUT))
    pm = True
    prob, U0 = random_density_problem(dims, seed=2)
    sim = make_sim(prob, U0)
    grav = vb.enable_gravity(sim, bcs=bcs_from(gcodes), tol=1e-10, maxiter=3000, project_mean=pm)
    its, rr = vb.solve_poisson(sim, grav)
    g, Pg = oracle_pair(oracle, prob, gcodes, tol=1e-10, maxiter=3000, project_mean=pm)
    phi = np.zeros(sim.ncell)
    its_o, rr_o = oracle.grav_solve(g, Pg, U0, phi)
    assert rr <= 1e-10 and rr_o <= 1e-10
    assert abs(its - its_o) <= 3
    scale = np.max(np.abs(phi))
    assert np.max(np.abs(grav.phi - phi)) <= 1e-8 * scale


STEP_CASES = {
    "3d_periodic": ((16, 16, 12), ((PER, PER),) * 3, ((PER, PER),) * 3),
    "2d_walls": ((32, 16), ((REF, OUT), (REF, REF)), ((OUT, OUT), (REF, REF))),
    "1d_periodic": ((64,), ((PER, PER),), ((PER, PER),)),
}


@pytest.mark.parametrize("precision", ["fp64"])
@pytest.mark.parametrize("case", sorted(STEP_CASES))
def test_step_with_given_phi_bit_identical(vb, oracle, case, precision):
    """For a given phi: g, compute_dt and a step with the source are
    bit-identical to the oracle (step!, src/driver.jl:343-351)."""
    dims, gas, gcodes = STEP_CASES[case]
    prob, U0 = random_density_problem(dims, seed=7, bcs=bcs_from(gas))
    sim = make_sim(prob, U0, precision)
    grav = vb.enable_gravity(sim, G=2.0, bcs=bcs_from(gcodes), project_mean=True)
    vb.solve_poisson(sim, grav)
    phi = grav.phi
    g, Pg = oracle_pair(oracle, prob, gcodes, G=2.0, project_mean=True)
    gacc = oracle.grav_accel(g, Pg, phi)
    assert_bit_identical(grav.accel(), gacc)
    dt = vb.compute_dt(sim)
    assert dt == oracle.compute_dt_gravity(g, 2.0, U0)
    vb.step(sim, dt)
    U = U0.copy()
    oracle.step_gravity(g, gacc, U, dt)
    assert_bit_identical(sim.state(), U)
    # a second step from set_phi (the field recomputed from an uploaded phi)
    grav.phi = phi * 0.5
    vb.step(sim, dt)
    oracle.step_gravity(g, oracle.grav_accel(g, Pg, phi * 0.5), U, dt)
    assert_bit_identical(sim.state(), U)


def test_evolve_equals_host_loop_and_tracks_oracle(vb, oracle):
    """evolve! with gravity (solve per step on the device loop) equals the host
    loop solve_poisson / compute_dt / step bit for bit, and follows the oracle's
    loop to the solver tolerance."""
    prob, U0 = random_density_problem((16, 16, 16), seed=9)
    a = make_sim(prob, U0)
    b = make_sim(prob, U0)
    ga = vb.enable_gravity(a, tol=1e-10, maxiter=2000)
    gb = vb.enable_gravity(b, tol=1e-10, maxiter=2000)
    vb.evolve(a, tfinal=math.inf, max_steps=6)
    for _ in range(6):
        vb.solve_poisson(b, gb)
        vb.step(b, vb.compute_dt(b))
    assert a.t == b.t and a.step == 6
    assert_bit_identical(a.state(), b.state())
    assert_bit_identical(ga.phi, gb.phi)
    g, Pg = oracle_pair(oracle, prob, ((PER, PER),) * 3, tol=1e-10, maxiter=2000)
    U = U0.copy()
    phi = np.zeros(a.ncell)
    t = 0.0
    for _ in range(6):
        oracle.grav_solve(g, Pg, U, phi)
        dt = oracle.compute_dt_gravity(g, 1.0, U)
        oracle.step_gravity(g, oracle.grav_accel(g, Pg, phi), U, dt)
        t += dt
    assert a.t == pytest.approx(t, rel=1e-12)
    rel = np.max(np.abs(a.state() - U)) / np.max(np.abs(U))
    assert rel < 1e-9, rel


def _jeans_sim(vb, n, A, p0, k, m_cfl=0.3):
    prob = problem((n,), ((0.0, 1.0),), P.Periodic,
                   lambda x, y, z: (1.0 + A * np.cos(k * x), 0.0, 0.0, 0.0, p0), cfl=m_cfl)
    sim = make_sim(prob, P.initial_state(prob))
    vb.enable_gravity(sim, G=1.0)
    return sim


def _mode_amp(sim, k):
    n = sim.ncell
    x = (np.arange(n) + 0.5) / n
    ck = np.cos(k * x)
    return float(np.sum((sim.state()[0] - 1.0) * ck) / np.sum(ck * ck))


def test_s1_overdensity_collapses(vb):
    k = 2 * math.pi
    sim = _jeans_sim(vb, 128, 1e-3, 0.06, k)
    a0 = _mode_amp(sim, k)
    for _ in range(40):
        vb.solve_poisson(sim)
        vb.step(sim, vb.compute_dt(sim))
    assert _mode_amp(sim, k) / a0 > 1.05


def test_s2_jeans_growth_rate(vb):
    gamma, p0, G, k = 5.0 / 3.0, 0.06, 1.0, 2 * math.pi
    s_exact = math.sqrt(-(gamma * p0 * k ** 2 - 4 * math.pi * G))
    sim = _jeans_sim(vb, 256, 1e-4, p0, k)
    a0 = abs(_mode_amp(sim, k))
    tmax = 2.0 / s_exact
    ts, logamp = [], []
    while sim.t < tmax:
        vb.solve_poisson(sim)
        vb.step(sim, min(vb.compute_dt(sim), tmax - sim.t))
        ts.append(sim.t)
        logamp.append(math.log(abs(_mode_amp(sim, k)) / a0))
    half = len(ts) // 2
    s_meas = np.polyfit(ts[half:], logamp[half:], 1)[0]
    assert abs(s_meas - s_exact) / s_exact < 0.08


def test_s2b_jeans_stable_mode_bounded(vb):
    gamma, p0, G, k = 5.0 / 3.0, 0.5, 1.0, 2 * math.pi * 4
    w2 = gamma * p0 * k ** 2 - 4 * math.pi * G
    sim = _jeans_sim(vb, 256, 1e-4, p0, k)
    a0 = abs(_mode_amp(sim, k))
    amax = a0
    tend = 2 * 2 * math.pi / math.sqrt(w2)
    while sim.t < tend:
        vb.solve_poisson(sim)
        vb.step(sim, min(vb.compute_dt(sim), tend - sim.t))
        amax = max(amax, abs(_mode_amp(sim, k)))
    assert amax / a0 < 1.5


def test_gravity_off_is_a_no_op(vb):
    """A grid that had gravity enabled and then disabled steps exactly as one
    that never had it (and on the tiled kernel again)."""
    prob = P.smooth_random_problem((32, 32, 32), seed=4)
    U0 = P.initial_state(prob)
    a = make_sim(prob, U0)
    b = make_sim(prob, U0)
    vb.enable_gravity(b)
    vb.solve_poisson(b)
    vb.disable_gravity(b)
    vb.evolve(a, max_steps=5)
    vb.evolve(b, max_steps=5)
    assert a.t == b.t
    assert_bit_identical(a.state(), b.state())


def test_mixed_precision_with_gravity_conserves_mass(vb):
    prob, U0 = random_density_problem((32, 32, 16), seed=8)
    sim = make_sim(prob, U0, "mixed")
    vb.enable_gravity(sim)
    m0 = vb.conserved_totals(sim).mass
    vb.evolve(sim, tfinal=math.inf, max_steps=8)
    assert sim.step == 8
    assert vb.conserved_totals(sim).mass == pytest.approx(m0, rel=1e-12)


TILED_CASES = {
    "periodic": (((PER, PER),) * 3, ((PER, PER),) * 3),
    "walls_z": (((PER, PER), (PER, PER), (REF, REF)), ((PER, PER), (PER, PER), (REF, REF))),
}


@pytest.mark.parametrize("case", sorted(TILED_CASES))
def test_tiled_fp64_with_gravity_bit_identical_to_cell(vb, case):
    """The 3D tiled float64 kernel carries the gravity source and the free-fall
    dt term: evolve! through it equals the cell-centric kernel (itself
    bit-identical to the oracle) bit for bit."""
    gas, gcodes = TILED_CASES[case]
    prob, U0 = random_density_problem((32, 32, 24), seed=21, bcs=bcs_from(gas))
    a = make_sim(prob, U0)
    b = make_sim(prob, U0)
    a.set_kernel("cell")
    b.set_kernel("tiled")
    assert b.kernel == "tiled"
    for sim in (a, b):
        vb.enable_gravity(sim, G=2.0, bcs=bcs_from(gcodes), tol=1e-10, maxiter=3000,
                          project_mean=True)
        vb.evolve(sim, tfinal=math.inf, max_steps=5)
    assert a.step == b.step == 5 and a.t == b.t
    assert_bit_identical(a.state(), b.state())


def test_tiled_mixed_with_gravity_tracks_fp64(vb):
    prob, U0 = random_density_problem((32, 32, 32), seed=22)
    a = make_sim(prob, U0)
    b = make_sim(prob, U0, "mixed")
    b.set_kernel("tiled")
    assert b.kernel == "tiled"
    m0 = vb.conserved_totals(b).mass
    for sim in (a, b):
        vb.enable_gravity(sim, G=2.0, tol=1e-10, maxiter=3000, precond="mg")
        vb.evolve(sim, tfinal=math.inf, max_steps=8)
    assert b.step == 8
    assert b.t == pytest.approx(a.t, rel=1e-6)
    ra, rb = a.state()[0], b.state()[0]
    l1 = float(np.sum(np.abs(ra - rb)) / np.sum(np.abs(ra)))
    assert l1 <= 1e-6, l1
    assert vb.conserved_totals(b).mass == pytest.approx(m0, rel=1e-12)


def test_adjoint_refuses_gravity_grid(vb):
    prob, U0 = random_density_problem((16, 16), seed=1)
    sim = make_sim(prob, U0)
    vb.enable_gravity(sim)
    with pytest.raises(vb.VespaB200Error) as e:
        vb.Adjoint(sim, 4, 2)
    assert e.value.status == 6


def test_gravity_api_errors(vb):
    prob, U0 = random_density_problem((16, 16), seed=1)
    sim = make_sim(prob, U0)
    with pytest.raises(vb.VespaB200Error):
        vb.solve_poisson(sim)  # not enabled
    with pytest.raises(vb.VespaB200Error):
        vb.enable_gravity(sim, bcs=((P.Periodic, P.Outflow), (P.Periodic, P.Periodic)))
    grav = vb.enable_gravity(sim)
    with pytest.raises(ValueError):
        grav.phi = np.zeros(3)


# ------------------------------------------------ multigrid-preconditioned CG
@pytest.mark.parametrize("n", [32, 24])
def test_mg_pcg_matches_oracle_cg_in_few_iterations(vb, oracle, n):
    """precond="mg" (ext/mg_pcg.jl) converges to the plain-CG potential of the
    oracle in a handful of iterations; n = 24 coarsens 24, 12, 6, 3."""
    prob, U0 = random_density_problem((n, n, n), seed=12)
    sim = make_sim(prob, U0)
    grav = vb.enable_gravity(sim, tol=1e-10, maxiter=3000, precond="mg")
    its, rr = vb.solve_poisson(sim, grav)
    g, Pg = oracle_pair(oracle, prob, ((PER, PER),) * 3, tol=1e-10, maxiter=3000)
    phi = np.zeros(sim.ncell)
    its_o, _ = oracle.grav_solve(g, Pg, U0, phi)
    assert rr <= 1e-10
    assert its <= 25 and its * 4 < its_o, (its, its_o)
    assert np.max(np.abs(grav.phi - phi)) <= 1e-8 * np.max(np.abs(phi))


def test_mg_evolve_tracks_plain_cg(vb):
    prob, U0 = random_density_problem((32, 32, 32), seed=13)
    a = make_sim(prob, U0)
    b = make_sim(prob, U0)
    vb.enable_gravity(a, tol=1e-10, maxiter=3000)
    vb.enable_gravity(b, tol=1e-10, maxiter=3000, precond="mg")
    vb.evolve(a, tfinal=math.inf, max_steps=5)
    vb.evolve(b, tfinal=math.inf, max_steps=5)
    assert a.t == pytest.approx(b.t, rel=1e-12)
    rel = np.max(np.abs(a.state() - b.state())) / np.max(np.abs(a.state()))
    assert rel < 1e-9, rel


def test_mg_refuses_unsupported_grids(vb):
    prob, U0 = random_density_problem((32, 32, 16), seed=1)
    sim = make_sim(prob, U0)
    with pytest.raises(vb.VespaB200Error) as e:
        vb.enable_gravity(sim, precond="mg")
    assert e.value.status == 6
    prob, U0 = random_density_problem((16, 16, 16), seed=1)
    sim = make_sim(prob, U0)
    with pytest.raises(vb.VespaB200Error) as e:
        vb.enable_gravity(sim, precond="mg", bcs=P.Outflow)
    assert e.value.status == 6
