"""The boundary-flux register on the device (BoundaryFluxRegister,
src/reflux.jl:113-191) against the oracle.

- Outer faces are recorded by the tiled kernels themselves (no fallback to
  the cell-centric kernel): in float64 state and register are bit-identical
  to the oracle's step!(sim, dt; bflux) on boxes with walls and outflow
  sides, in 3D and 2D.
- Mixed precision records the float32 fluxes its update used, so the
  register satisfies the conservation identity of
  test/test_boundary_flux.jl (change of each total = sum of lo-side minus
  hi-side boundary fluxes) to round-off, and agrees with the float64
  register to float32 accuracy.
- record_interior (VB_BFLUX_INTERIOR) captures every interior face too,
  bit-identical to the oracle.
- bflux_plane on the device equals the oracle's restatement bit for bit.
"""
import math

import numpy as np
import pytest

from vespa_b200 import problem as P

from test_gpu_parity import assert_bit_identical, make_sim, problem_from

pytestmark = pytest.mark.gpu

# dims, bc_lo, bc_hi (0 outflow, 1 periodic, 2 reflecting)
CASES_3D = [((32, 16, 9), [0, 2, 1], [2, 0, 1]), ((16, 32, 20), [2, 0, 0], [0, 2, 2])]
CASES_2D = [((256, 9), [0, 2], [2, 0]), ((512, 6), [2, 1], [0, 1])]


def run_pair(vb, oracle, dims, lo, hi, nsteps, kernel, mode, precision="fp64"):
    nd = len(dims)
    prob = problem_from(dims, [(0.0, 1.0)] * nd, lo, hi, 1.4, 0.4)
    U0 = P.initial_state(P.smooth_random_problem(dims, seed=31))
    sim = make_sim(prob, U0, precision)
    sim.set_kernel(kernel)
    sim.bflux_enable(mode)
    g = oracle.make_grid(dims, [0] * nd, [1] * nd, lo, hi, 1.4, 0.4)
    reg = oracle.BoundaryFluxRegister(g, record_interior=(mode == "interior"))
    U = U0.copy()
    for _ in range(nsteps):
        dt = oracle.compute_dt(g, U)
        vb.step(sim, dt)
        oracle.step_breg(g, U, dt, reg)
    return sim, g, reg, U, U0


@pytest.mark.parametrize("dims,lo,hi", CASES_3D + CASES_2D)
def test_tiled_kernels_record_outer_fluxes_bit_identical(vb, oracle, dims, lo, hi):
    sim, g, reg, U, _ = run_pair(vb, oracle, dims, lo, hi, 3, "tiled", True)
    assert sim.kernel == "tiled"
    assert_bit_identical(sim.state(), U)
    assert_bit_identical(sim.bflux_read(), reg.dense())
    assert reg.seen.any()
    sim.close()


@pytest.mark.parametrize("dims,lo,hi", CASES_3D[:1] + CASES_2D[:1])
def test_interior_register_bit_identical(vb, oracle, dims, lo, hi):
    sim, g, reg, U, _ = run_pair(vb, oracle, dims, lo, hi, 2, "auto", "interior")
    assert_bit_identical(sim.state(), U)
    assert_bit_identical(sim.bflux_read(), reg.dense())
    sim.close()


@pytest.mark.parametrize("dims,lo,hi", [((32, 16, 9), [0, 0, 0], [0, 0, 0]), ((256, 9), [0, 0], [0, 0])])
def test_mixed_tiled_register_conservation_identity(vb, oracle, dims, lo, hi):
    nd = len(dims)
    prob = problem_from(dims, [(0.0, 1.0)] * nd, lo, hi, 1.4, 0.4)
    U0 = P.initial_state(P.smooth_random_problem(dims, seed=32))
    m = make_sim(prob, U0, "mixed")
    m.set_kernel("tiled")
    m.bflux_enable(True)
    f = make_sim(prob, U0, "fp64")
    f.set_kernel("tiled")
    f.bflux_enable(True)
    t0 = np.array(vb.conserved_totals(m))
    for _ in range(4):
        dt = vb.compute_dt(f)
        vb.step(m, dt)
        vb.step(f, dt)
    assert m.kernel == "tiled"
    t1 = np.array(vb.conserved_totals(m))
    bm, bf = m.bflux_read(), f.bflux_read()
    # per axis and side: [5][plane] blocks; lo minus hi summed over the planes
    ncell = int(np.prod(dims))
    net = np.zeros(5)
    off = 0
    for d in range(nd):
        pl = ncell // dims[d]
        lo_b = bm[off:off + 5 * pl].reshape(5, pl).sum(axis=1)
        hi_b = bm[off + 5 * pl:off + 10 * pl].reshape(5, pl).sum(axis=1)
        net += lo_b - hi_b
        off += 10 * pl
    assert np.any(np.abs(net) > 1e-6)  # flux did cross the domain faces
    # the totals are sums of U * V; the register integrates F * area * dt
    assert np.allclose(t1 - t0, net, rtol=0, atol=1e-12 * np.abs(t0).max())
    np.testing.assert_allclose(bm, bf, rtol=0, atol=1e-5 * np.abs(bf).max())
    m.close()
    f.close()


def test_bflux_plane_on_device_bit_identical(vb, oracle):
    dims, lo, hi = (32, 16, 9), [0, 2, 1], [2, 0, 1]
    sim, g, reg, U, _ = run_pair(vb, oracle, dims, lo, hi, 2, "auto", "interior")
    g0 = (101, 7, 1)
    cases = [
        (0, "lo", (101, 7, 1), (101, 22, 9), 1, 1), (0, "hi", (132, 7, 1), (132, 22, 9), 32, 5),
        (1, "lo", (101, 7, 1), (132, 7, 9), 1, 2), (1, "hi", (101, 22, 1), (132, 22, 9), 16, 3),
        (2, "lo", (101, 7, 1), (132, 22, 1), 1, 1),                # periodic axis: zeros
        (0, "lo", (101, 5, 0), (101, 24, 10), 1, 4),               # wider than the grid
        (0, "interior", (110, 7, 1), (110, 22, 9), 10, 1),
        (2, "interior", (101, 7, 9), (132, 22, 9), 9, 5),          # periodic wrap faces
        (1, "interior", (101, 22, 1), (132, 22, 9), 16, 2),        # wall above: zeros
        (0, "hi", (132, 7, 1), (132, 22, 9), 32, 0),               # comp 0
    ]
    src = {"lo": 0, "hi": 1, "interior": 2}
    for dim, s, st, sp, off, comp in cases:
        got = sim.bflux_plane(dim, s, st, sp, g0, off, comp, 0.5)
        ref = oracle.bflux_plane(g, reg, dim, src[s], st, sp, g0, off, comp, 0.5)
        assert_bit_identical(got, ref)
    sim.close()


def test_bflux_modes_and_errors(vb):
    prob = problem_from((32, 16, 9), [(0.0, 1.0)] * 3, [0, 0, 0], [0, 0, 0], 1.4, 0.4)
    sim = make_sim(prob, P.initial_state(P.smooth_random_problem((32, 16, 9), seed=2)))
    sim.bflux_enable(True)
    n_outer = sim.bflux_read().size
    with pytest.raises(vb.VespaB200Error):
        sim.bflux_plane(0, "interior", (1, 1, 1), (1, 16, 9), (1, 1, 1), 1, 1, 1.0)
    with pytest.raises(vb.VespaB200Error):
        sim.bflux_plane(0, "lo", (1, 1, 1), (1, 16, 9), (1, 1, 1), 1, 6, 1.0)
    vb.step(sim, 1e-3)
    a = sim.bflux_read()
    sim.bflux_enable(False)  # stops recording, keeps the values
    vb.step(sim, 1e-3)
    assert np.array_equal(sim.bflux_read(), a)
    sim.bflux_enable("interior")  # new layout: zeroed, interior block appended
    b = sim.bflux_read()
    assert b.size == n_outer + 3 * 5 * 32 * 16 * 9 and not b.any()
    sim.close()
