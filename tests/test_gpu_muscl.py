"""GPU unsplit MUSCL step (lib/PPMKernels muscl_step_3d! on the device)
against the oracle's restatement, bit for bit, and against the reference's
driver checks (lib/PPMKernels/test/test_muscl_grid.jl: one-axis reduction,
conservation)."""
import numpy as np
import pytest

import vespa_b200 as vb
from test_gpu_parity import assert_bit_identical

pytestmark = pytest.mark.gpu

NG, GAMMA, THETA, DT, DX = 3, 1.4, 1.5, 0.02, 1.0


def random_state(dims, seed):
    rng = np.random.default_rng(seed)
    N = int(np.prod(dims))
    rho = 0.5 + rng.random(N)
    v = 0.4 * (rng.random((3, N)) - 0.5)
    p = 0.3 + rng.random(N)
    etot = p / ((GAMMA - 1) * rho) + 0.5 * (v ** 2).sum(axis=0)
    return np.ascontiguousarray(np.array([rho, rho * v[0], rho * v[1], rho * v[2], rho * etot]))


def shock_state(dims, axis):
    N = int(np.prod(dims))
    idx = np.arange(N)
    c = (idx // [1, dims[0], dims[0] * dims[1]][axis]) % dims[axis]
    left = c < dims[axis] // 2
    rho = np.where(left, 1.0, 0.125)
    p = np.where(left, 1.0, 0.1)
    v = np.zeros((3, N))
    v[axis] = np.where(left, 0.3, -0.1)
    v[(axis + 1) % 3] = 0.05
    etot = p / ((GAMMA - 1) * rho) + 0.5 * (v ** 2).sum(axis=0)
    return np.ascontiguousarray(np.array([rho, rho * v[0], rho * v[1], rho * v[2], rho * etot]))


CASES = {
    "random_none": ((12, 10, 9), lambda d: random_state(d, 1), None, 3),
    "random_periodic": ((18, 15, 12), lambda d: random_state(d, 2), "periodic", 4),
    "shock_x_periodic": ((24, 9, 10), lambda d: shock_state(d, 0), "periodic", 3),
    "shock_z_none": ((9, 10, 24), lambda d: shock_state(d, 2), None, 3),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_step_bit_identical_to_oracle(vb, oracle, case):
    dims, make, bc, steps = CASES[case]
    U0 = make(dims)
    g = vb.MusclGrid(dims, NG)
    g.upload(U0)
    U = U0.copy()
    for _ in range(steps):
        g.step(dt=DT, gamma=GAMMA, theta=THETA, dx=DX, bc=bc)
        oracle.muscl_step(dims, NG, U, DT, GAMMA, THETA, DX, bc=0 if bc is None else 1)
    assert_bit_identical(g.state(), U)


def test_long_z_chunks_bit_identical_to_oracle(vb, oracle):
    """A grid large enough for multi-plane z chunks (about 20 planes per CTA,
    the five-plane ring wrapping several times), periodic ghosts."""
    dims = (134, 70, 128)
    U0 = random_state(dims, 4)
    g = vb.MusclGrid(dims, NG)
    g.upload(U0)
    g.step(dt=DT, gamma=GAMMA, theta=THETA, dx=DX, bc="periodic")
    U = U0.copy()
    oracle.muscl_step(dims, NG, U, DT, GAMMA, THETA, DX, bc=1)
    assert_bit_identical(g.state(), U)


def test_step_fields_on_caller_arrays_equals_owned_state(vb):
    """vb_muscl_step_fields on five device arrays the caller owns (here torch
    tensors) does what vb_muscl_step does on the handle's own state."""
    import torch
    dims = (14, 12, 10)
    U0 = random_state(dims, 3)
    g = vb.MusclGrid(dims, NG)
    g.upload(U0)
    g.step(dt=DT, gamma=GAMMA, theta=THETA, dx=DX, bc="periodic")
    fields = [torch.tensor(U0[f], dtype=torch.float64, device="cuda") for f in range(5)]
    torch.cuda.synchronize()
    g2 = vb.MusclGrid(dims, NG)
    g2.step_fields([t.data_ptr() for t in fields], dt=DT, gamma=GAMMA, theta=THETA, dx=DX,
                   bc="periodic")
    got = np.array([t.cpu().numpy() for t in fields])
    assert_bit_identical(got, g.state())


def test_muscl_step_3d_host_mirror(vb, oracle):
    dims = (10, 11, 12)
    U0 = random_state(dims, 5)
    D, S1, S2, S3, Tau = (U0[f].copy() for f in range(5))
    vb.muscl_step_3d(D, S1, S2, S3, Tau, dims, NG, dt=DT, gamma=GAMMA)
    U = U0.copy()
    oracle.muscl_step(dims, NG, U, DT, GAMMA, 1.5, 1.0)
    assert_bit_identical(np.array([D, S1, S2, S3, Tau]), U)


def _total(U, dims):
    A = U.reshape(5, dims[2], dims[1], dims[0])
    return A[:, NG:dims[2] - NG, NG:dims[1] - NG, NG:dims[0] - NG].reshape(5, -1).sum(axis=1) * DX ** 3


def test_conservation_blob(vb):
    """test_muscl_grid.jl conservation: a contained blob, 3 steps."""
    m = 26
    idx = np.arange(m ** 3)
    i, j, k = idx % m + 1, (idx // m) % m + 1, idx // (m * m) + 1
    x, y, z = (i - 13.5) / 2.2, (j - 13.5) / 2.2, (k - 13.5) / 2.2
    b = np.exp(-(x ** 2 + y ** 2 + z ** 2))
    rho, pr = 1.0 + 0.4 * b, 0.6 + 0.3 * b
    vx, vy, vz = 0.10 * x * b, 0.08 * y * b, -0.06 * z * b
    etot = pr / ((GAMMA - 1) * rho) + 0.5 * (vx ** 2 + vy ** 2 + vz ** 2)
    U0 = np.ascontiguousarray(np.array([rho, rho * vx, rho * vy, rho * vz, rho * etot]))
    g = vb.MusclGrid((m, m, m), NG)
    g.upload(U0)
    t0 = _total(U0, (m, m, m))
    for _ in range(3):
        g.step(dt=DT, gamma=GAMMA, theta=THETA, dx=DX)
    t1 = _total(g.state(), (m, m, m))
    assert abs(t1[0] - t0[0]) / abs(t0[0]) < 1e-12
    assert np.all(np.abs(t1[1:4] - t0[1:4]) < 1e-11)
    assert abs(t1[4] - t0[4]) / abs(t0[4]) < 1e-12


def test_refusals(vb):
    with pytest.raises(vb.VespaB200Error):
        vb.MusclGrid((6, 10, 10), 3)  # 6 < 2 ng + 1
    g = vb.MusclGrid((8, 10, 10), 3)
    with pytest.raises(vb.VespaB200Error):
        g.step(dt=DT, gamma=GAMMA, bc="periodic")  # 8 < 3 ng
    with pytest.raises(vb.VespaB200Error):
        g.step(dt=DT, gamma=1.0)
