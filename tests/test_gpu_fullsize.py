"""Cell-by-cell parity at the benchmark's full sizes.

The headline workloads run at sizes where the serial oracle would take
minutes per step, so these tests use the oracle's per-cell gather form
(``mode=1``: each cell sums its faces in the reference's enumeration order,
bit-identical to the serial face loop) on all host threads:

- 256^3 periodic, VB_FP64 on the tiled kernel with the autotuned z chunk, and
  the same run on the tapered work queue that the mixed-precision headline
  uses (chunks of 128, 64, 32, 16, 8, 8 planes): 2 steps, bit-identical;
- 4096^2 periodic, VB_FP64 on the tiled 2D kernel: 2 steps, bit-identical;
- 256^3 VB_MIXED: the tapered queue (at the autotuned chunk) is
  bit-identical to uniform chunks, and
  after the benchmark's 3 + 20 steps the density L1 error against VB_FP64 is
  at most 1e-6 relative, with the five totals conserved to 1e-12.

The VB_FP64 bar is exact equality, stronger than the relative 1e-12 per
cell that the GPU-versus-host comparison of the reference allows
(test/gpu/test_ka_flux_gpu.jl:102).
"""
import math

import numpy as np
import pytest

from vespa_b200 import problem as P

pytestmark = pytest.mark.gpu

BENCH_STEPS = 3 + 20  # warm-up + timed steps of the default benchmark line


def max_rel(a, b):
    scale = np.maximum(np.abs(a), np.abs(b))
    with np.errstate(invalid="ignore", divide="ignore"):
        r = np.where(scale > 0, np.abs(a - b) / scale, 0.0)
    return float(np.max(r))


def assert_bit_identical(a, b):
    assert a.shape == b.shape
    if not np.array_equal(a, b):
        raise AssertionError(f"not bit-identical: max rel diff {max_rel(a, b):.3e}, "
                             f"{int(np.sum(a != b))} of {a.size} values differ")


def make_sim(vb, prob, U0, precision):
    return vb.Simulation(vb.B200Mesh(prob.dims, prob.domain), prob, precision=precision,
                         initial=U0)


@pytest.fixture(scope="module")
def cube():
    prob = P.smooth_random_problem((256, 256, 256))
    return prob, P.initial_state(prob)


@pytest.fixture(scope="module")
def cube_oracle_2steps(oracle, cube):
    prob, U0 = cube
    U = U0.copy()
    t, n = oracle.evolve(oracle.grid_from_problem(prob), U, math.inf, max_steps=2, mode=1)
    assert n == 2
    return t, U


def test_cube256_fp64_autotuned_tiled_bit_identical(vb, cube, cube_oracle_2steps):
    prob, U0 = cube
    t_ref, U_ref = cube_oracle_2steps
    sim = make_sim(vb, prob, U0, "fp64")
    sim.set_kernel("tiled")
    kz, _ = sim.autotune(3)  # the benchmark's setup (chunk and queue shape); state restored
    assert sim.kz == kz
    vb.evolve(sim, max_steps=2)
    assert sim.step == 2 and sim.t == t_ref
    assert_bit_identical(sim.state(), U_ref)
    sim.close()


def test_cube256_fp64_on_the_tapered_queue_bit_identical(vb, cube, cube_oracle_2steps):
    """The mixed headline's queue shape (kz 128, tapered) in float64."""
    prob, U0 = cube
    t_ref, U_ref = cube_oracle_2steps
    sim = make_sim(vb, prob, U0, "fp64")
    sim.set_kernel("tiled", kz=128, taper=True)
    assert sim.taper and sim.kz == 128
    vb.evolve(sim, max_steps=2)
    assert sim.t == t_ref
    assert_bit_identical(sim.state(), U_ref)
    sim.close()


def test_plane4096_fp64_tiled_bit_identical(vb, oracle):
    prob = P.smooth_random_problem((4096, 4096))
    U0 = P.initial_state(prob)
    sim = make_sim(vb, prob, U0, "fp64")
    sim.set_kernel("tiled")
    sim.autotune(3)
    vb.evolve(sim, max_steps=2)
    U = U0.copy()
    t, n = oracle.evolve(oracle.grid_from_problem(prob), U, math.inf, max_steps=2, mode=1)
    assert n == 2 and sim.t == t
    assert_bit_identical(sim.state(), U)
    sim.close()


def test_cube256_mixed_taper_bits_and_l1_against_fp64(vb, cube):
    prob, U0 = cube
    tap = make_sim(vb, prob, U0, "mixed")
    tap.set_kernel("tiled")
    kz, _ = tap.autotune(3)
    tap.set_kernel("tiled", kz=kz, taper=True)
    assert tap.taper
    t0 = np.array(vb.conserved_totals(tap))
    vb.evolve(tap, max_steps=BENCH_STEPS)
    t1 = np.array(vb.conserved_totals(tap))
    Um = tap.state()
    tap.close()
    assert np.allclose(t1, t0, rtol=1e-12, atol=1e-12 * np.abs(t0).max())

    uni = make_sim(vb, prob, U0, "mixed")
    uni.set_kernel("tiled", kz=kz, taper=False)
    assert not uni.taper
    vb.evolve(uni, max_steps=BENCH_STEPS)
    assert_bit_identical(uni.state(), Um)
    uni.close()

    ref = make_sim(vb, prob, U0, "fp64")
    ref.set_kernel("tiled")
    vb.evolve(ref, max_steps=BENCH_STEPS)
    rho = ref.state()[0]
    ref.close()
    l1 = float(np.sum(np.abs(Um[0] - rho)) / np.sum(np.abs(rho)))
    assert l1 <= 1e-6, l1
