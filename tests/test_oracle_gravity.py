"""The self-gravity restatement in the oracle (oracle/vespa_oracle.c, after
src/gravity.jl) against the reference's own gates: test/test_gravity_poisson.jl
(O1 operator symmetry and null space, O2/O2b Fourier-mode Poisson with second
order convergence) and test/test_gravity_hydro.jl (S1 sign gate, S2 Jeans
growth rate, S2b stable mode), re-expressed for the CPU."""
import math

import numpy as np
import pytest

PER, OUT, REF = 1, 0, 2


def _grid1d(O, n, L=1.0, gamma=5.0 / 3.0, cfl=0.4):
    return O.make_grid((n,), (0.0,), (L,), (PER,), (PER,), gamma, cfl)


def _state_1d(n, rho, p0, gamma, L=1.0):
    x = (np.arange(n) + 0.5) * (L / n)
    U = np.zeros((5, n))
    U[0] = rho(x)
    U[4] = p0 / (gamma - 1.0)
    return x, U


def test_o1_operator_symmetric_with_constant_null_space(oracle):
    O = oracle
    n = 16
    g = _grid1d(O, n)
    P = O.make_gravity(1.0, (PER,), (PER,))
    x = (np.arange(n) + 0.5) / n
    a = np.sin(2 * math.pi * x) + 0.3 * np.cos(6 * math.pi * x)
    b = np.cos(2 * math.pi * x) - 0.7 * np.sin(4 * math.pi * x)
    Aa, Ab = O.grav_laplacian(g, P, a), O.grav_laplacian(g, P, b)
    assert np.dot(a, Ab) == pytest.approx(np.dot(b, Aa), rel=1e-12, abs=1e-12)
    assert np.max(np.abs(O.grav_laplacian(g, P, np.ones(n)))) < 1e-12
    s = np.sin(2 * math.pi * x)
    assert np.dot(s, O.grav_laplacian(g, P, s)) > 0


def test_o1_operator_3d_walls_and_periodic_wrap(oracle):
    """Symmetric and constant-annihilating with Neumann walls too (3D)."""
    O = oracle
    dims = (6, 5, 4)
    g = O.make_grid(dims, (0, 0, 0), (1.0, 2.0, 0.5), (PER, OUT, PER), (PER, OUT, PER), 1.4)
    P = O.make_gravity(1.0, (PER, OUT, REF), (PER, OUT, REF))
    rng = np.random.default_rng(3)
    a, b = rng.standard_normal(120), rng.standard_normal(120)
    Aa, Ab = O.grav_laplacian(g, P, a), O.grav_laplacian(g, P, b)
    assert np.dot(a, Ab) == pytest.approx(np.dot(b, Aa), rel=1e-12)
    assert np.max(np.abs(O.grav_laplacian(g, P, np.full(120, 2.5)))) < 1e-12
    assert np.dot(a, Aa) > 0


def _fourier_l1(O, n, m=1, A=0.1, rhobar=1.0, G=1.0, L=1.0):
    k = 2 * math.pi * m / L
    g = _grid1d(O, n, L)
    x, U = _state_1d(n, lambda x: rhobar + A * np.cos(k * x), 1.0, 5.0 / 3.0, L)
    P = O.make_gravity(G, (PER,), (PER,), maxiter=5000, tol=1e-12)
    phi = np.zeros(n)
    its, rr = O.grav_solve(g, P, U, phi)
    coef = -4 * math.pi * G * A / k ** 2
    return float(np.mean(np.abs(phi - coef * np.cos(k * x)))), its, rr


def test_o2_fourier_mode_second_order(oracle):
    e64, _, rr64 = _fourier_l1(oracle, 64)
    e128, _, _ = _fourier_l1(oracle, 128)
    assert rr64 < 1e-10
    assert e64 < 5e-3
    assert e64 / e128 > 3.5


def test_o2b_fourier_mode_2d(oracle):
    O = oracle
    n, A, G = 64, 0.1, 1.0
    k = 2 * math.pi
    g = O.make_grid((n, n), (0, 0), (1.0, 1.0), (PER, PER), (PER, PER), 5.0 / 3.0)
    c = (np.arange(n) + 0.5) / n
    X, Y = np.meshgrid(c, c, indexing="ij")
    rho = (1.0 + A * np.cos(k * X) * np.cos(k * Y)).reshape(-1, order="F")
    U = np.zeros((5, n * n))
    U[0] = rho
    U[4] = 1.5
    P = O.make_gravity(G, (PER, PER), (PER, PER), maxiter=5000, tol=1e-11)
    phi = np.zeros(n * n)
    _, rr = O.grav_solve(g, P, U, phi)
    exact = (-4 * math.pi * G * A / (2 * k ** 2) * np.cos(k * X) * np.cos(k * Y)).reshape(-1, order="F")
    assert rr < 1e-9
    assert np.mean(np.abs(phi - exact)) < 1e-2


def _mode_amp(U, x, k, rhobar):
    ck = np.cos(k * x)
    return float(np.sum((U[0] - rhobar) * ck) / np.sum(ck * ck))


def _run_jeans(O, n, A, p0, k, tmax, G=1.0, gamma=5.0 / 3.0, cfl=0.3):
    g = _grid1d(O, n, gamma=gamma, cfl=cfl)
    x, U = _state_1d(n, lambda x: 1.0 * (1 + A * np.cos(k * x)), p0, gamma)
    P = O.make_gravity(G, (PER,), (PER,))
    phi = np.zeros(n)
    t, ts, amps = 0.0, [], []
    a0 = abs(_mode_amp(U, x, k, 1.0))
    while t < tmax:
        O.grav_solve(g, P, U, phi)
        gacc = O.grav_accel(g, P, phi)
        dt = min(O.compute_dt_gravity(g, G, U), tmax - t)
        O.step_gravity(g, gacc, U, dt)
        t += dt
        ts.append(t)
        amps.append(abs(_mode_amp(U, x, k, 1.0)) / a0)
    return np.array(ts), np.array(amps)


def test_s1_overdensity_collapses(oracle):
    O = oracle
    n, k = 128, 2 * math.pi
    g = _grid1d(O, n, cfl=0.3)
    x, U = _state_1d(n, lambda x: 1.0 + 1e-3 * np.cos(k * x), 0.06, 5.0 / 3.0)
    P = O.make_gravity(1.0, (PER,), (PER,))
    phi = np.zeros(n)
    a0 = _mode_amp(U, x, k, 1.0)
    for _ in range(40):
        O.grav_solve(g, P, U, phi)
        gacc = O.grav_accel(g, P, phi)
        O.step_gravity(g, gacc, U, O.compute_dt_gravity(g, 1.0, U))
    assert _mode_amp(U, x, k, 1.0) / a0 > 1.05


def test_s2_jeans_growth_rate(oracle):
    gamma, p0, G = 5.0 / 3.0, 0.06, 1.0
    k = 2 * math.pi
    w2 = gamma * p0 * k ** 2 - 4 * math.pi * G
    assert w2 < 0
    s_exact = math.sqrt(-w2)
    ts, amps = _run_jeans(oracle, 256, 1e-4, p0, k, 2.0 / s_exact)
    half = len(ts) // 2
    s_meas = np.polyfit(ts[half:], np.log(amps[half:]), 1)[0]
    assert abs(s_meas - s_exact) / s_exact < 0.08


def test_s2b_jeans_stable_mode_bounded(oracle):
    gamma, p0, G = 5.0 / 3.0, 0.5, 1.0
    k = 2 * math.pi * 4
    w2 = gamma * p0 * k ** 2 - 4 * math.pi * G
    assert w2 > 0
    _, amps = _run_jeans(oracle, 256, 1e-4, p0, k, 2 * 2 * math.pi / math.sqrt(w2))
    assert amps.max() < 1.5


def test_accel_is_central_difference_with_wall_halves(oracle):
    """g = -(phi_hi - phi_lo) / (d_lo + d_hi); at a Neumann wall the missing
    neighbour is the cell itself at half a width (_gax)."""
    O = oracle
    g = O.make_grid((5,), (0.0,), (1.0,), (OUT,), (OUT,), 1.4)
    P = O.make_gravity(1.0, (OUT,), (OUT,))
    phi = np.array([1.0, 2.0, 4.0, 8.0, 16.0])
    acc = O.grav_accel(g, P, phi)[0]
    w = 0.2
    assert acc[0] == -(2.0 - 1.0) / (0.5 * w + w)
    assert acc[2] == -(8.0 - 2.0) / (w + w)
    assert acc[4] == -(16.0 - 8.0) / (w + 0.5 * w)
