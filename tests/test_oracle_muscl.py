"""The unsplit MUSCL restatement in the oracle (lib/PPMKernels muscl_step_3d!,
src/muscl_grid.jl) against the reference's own driver checks
(lib/PPMKernels/test/test_muscl_grid.jl): a 3-D step on a state that varies
along one axis only equals a 1-D SSP-RK2 built from the flux line, for x, y
and z (this exercises the cyclic momentum roles), and a contained blob keeps
mass, momentum and energy to round-off."""
import numpy as np
import pytest

NG, GAMMA, THETA, DT, DX = 3, 1.4, 1.5, 0.02, 1.0


def _rk2_line_ref(O, D, Sn, St1, St2, Tau, na):
    """test_muscl_grid.jl _rk2_line_ref: 1-D SSP-RK2 from the flux line."""
    active, dtdx = na - 2 * NG, DT / DX

    def L(U):
        D, S1, S2, S3, Tau = U
        vx, vy, vz = S1 / D, S2 / D, S3 / D
        prim = np.array([D, Tau / D - 0.5 * (vx * vx + vy * vy + vz * vz), vx, vy, vz])
        F = O.muscl_flux_line(prim, NG, GAMMA, THETA)
        dU = np.zeros((5, na))
        for m in range(active):
            dU[:, NG + m] = -(F[:, m + 1] - F[:, m]) * dtdx
        return dU

    U0 = np.array([D, Sn, St1, St2, Tau])
    U1 = U0 + L(U0)
    return 0.5 * (U0 + U1 + L(U1))


@pytest.mark.parametrize("axis", [0, 1, 2])
def test_reduces_to_1d_rk2_along_axis(oracle, axis):
    O = oracle
    na = 22
    dims = [(na, 8, 7), (7, na, 8), (8, 7, na)][axis]
    m = np.arange(1, na + 1)
    t = np.tanh((m - 11.0) * 0.8)
    rho, pr, vn = 0.6 - 0.35 * t, 0.6 - 0.45 * t, 0.15 - 0.10 * t
    vt1, vt2 = np.full(na, 0.05), np.full(na, -0.03)
    eint = pr / ((GAMMA - 1) * rho)
    etot = eint + 0.5 * (vn ** 2 + vt1 ** 2 + vt2 ** 2)
    line = (rho, rho * vn, rho * vt1, rho * vt2, rho * etot)
    ref = _rk2_line_ref(O, *line, na)
    N = int(np.prod(dims))
    mn, mt1, mt2 = [(1, 2, 3), (2, 3, 1), (3, 1, 2)][axis]
    U = np.zeros((5, N))
    idx = np.arange(N)
    coord = (idx // [1, dims[0], dims[0] * dims[1]][axis]) % dims[axis]
    U[0] = line[0][coord]
    U[mn] = line[1][coord]
    U[mt1] = line[2][coord]
    U[mt2] = line[3][coord]
    U[4] = line[4][coord]
    O.muscl_step(dims, NG, U, DT, GAMMA, THETA, DX)
    st = [1, dims[0], dims[0] * dims[1]]
    base = sum(3 * st[d] for d in range(3) if d != axis)
    pencil = base + np.arange(na) * st[axis]
    for f, r in ((0, ref[0]), (mn, ref[1]), (mt1, ref[2]), (mt2, ref[3]), (4, ref[4])):
        np.testing.assert_allclose(U[f, pencil], r, rtol=1e-14, atol=1e-15)


def _blob(m):
    idx = np.arange(m ** 3)
    i, j, k = idx % m + 1, (idx // m) % m + 1, idx // (m * m) + 1
    x, y, z = (i - 13.5) / 2.2, (j - 13.5) / 2.2, (k - 13.5) / 2.2
    b = np.exp(-(x ** 2 + y ** 2 + z ** 2))
    rho = 1.0 + 0.4 * b
    pr = 0.6 + 0.3 * b
    vx, vy, vz = 0.10 * x * b, 0.08 * y * b, -0.06 * z * b
    etot = pr / ((GAMMA - 1) * rho) + 0.5 * (vx ** 2 + vy ** 2 + vz ** 2)
    return np.ascontiguousarray(np.array([rho, rho * vx, rho * vy, rho * vz, rho * etot]))


def _total(U, m):
    A = U.reshape(5, m, m, m)  # (k, j, i) ordering: x fastest
    return A[:, NG:m - NG, NG:m - NG, NG:m - NG].reshape(5, -1).sum(axis=1) * DX ** 3


def test_conservation_contained_blob(oracle):
    m = 26
    U = _blob(m)
    t0 = _total(U, m)
    for _ in range(3):
        oracle.muscl_step((m, m, m), NG, U, DT, GAMMA, THETA, DX)
    t1 = _total(U, m)
    assert abs(t1[0] - t0[0]) / abs(t0[0]) < 1e-12
    assert np.all(np.abs(t1[1:4] - t0[1:4]) < 1e-11)
    assert abs(t1[4] - t0[4]) / abs(t0[4]) < 1e-12


def test_periodic_fill_conserves_exactly_shaped_totals(oracle):
    """With periodic ghost fill the active region is a periodic box: totals stay
    to round-off for a state that touches the ghosts."""
    m = 16
    rng = np.random.default_rng(4)
    N = m ** 3
    rho = 1.0 + 0.3 * rng.random(N)
    v = 0.2 * (rng.random((3, N)) - 0.5)
    p = 0.5 + 0.5 * rng.random(N)
    U = np.ascontiguousarray(np.array([rho, rho * v[0], rho * v[1], rho * v[2],
                                       p / (GAMMA - 1) + 0.5 * rho * (v ** 2).sum(axis=0)]))
    oracle.muscl_step((m, m, m), NG, U, 0.0, GAMMA, THETA, DX, bc=1)  # fill, dt = 0
    t0 = _total(U, m)
    for _ in range(4):
        oracle.muscl_step((m, m, m), NG, U, 0.05, GAMMA, THETA, DX, bc=1)
    t1 = _total(U, m)
    assert np.allclose(t1, t0, rtol=1e-12, atol=1e-12)
