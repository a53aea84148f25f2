"""The tiled 2D kernel (256-cell row segments marching y) against the CPU
oracle (float64, bit for bit), the cell-centric kernel, and the float64 path
(mixed precision)."""
import math

import numpy as np
import pytest

import vespa_b200 as vb
from vespa_b200 import problem as P

from test_gpu_parity import BC_OF, assert_bit_identical, make_sim, problem_from

pytestmark = pytest.mark.gpu

TILED2D_CASES = [
    # dims, bc_lo, bc_hi, ky
    ((256, 16), [1, 1], [1, 1], None),
    ((512, 9), [0, 2], [2, 0], 3),
    ((256, 2), [1, 0], [1, 2], 1),
    ((768, 33), [2, 1], [2, 1], 8),
    ((256, 40), [0, 0], [0, 0], 40),
]


@pytest.mark.parametrize("dims,bclo,bchi,ky", TILED2D_CASES)
def test_tiled2d_bit_identical_to_oracle(vb, oracle, dims, bclo, bchi, ky):
    prob = problem_from(dims, [(0.0, 1.0)] * 2, bclo, bchi, 1.4, 0.4)
    U0 = P.initial_state(P.smooth_random_problem(dims, seed=sum(dims) + 3))
    sim = make_sim(prob, U0)
    sim.set_kernel("tiled", kz=ky)
    assert sim.kernel == "tiled"
    vb.evolve(sim, tfinal=math.inf, max_steps=5)
    U = U0.copy()
    g = oracle.make_grid(dims, [0] * 2, [1] * 2, bclo, bchi, 1.4, 0.4)
    t_ref, n_ref = oracle.evolve(g, U, math.inf, max_steps=5, mode=1)
    assert sim.step == n_ref and sim.t == t_ref
    assert_bit_identical(sim.state(), U)


def test_tiled2d_equals_cell_kernel_on_kh(vb):
    """Kelvin-Helmholtz (sharp shear layer, all HLLC branches): tiled and
    cell-centric float64 kernels agree to the bit over 20 steps."""
    prob = P.kelvin_helmholtz_problem(n=256)
    U0 = P.initial_state(prob)
    a = make_sim(prob, U0)
    b = make_sim(prob, U0)
    a.set_kernel("tiled", kz=16)
    b.set_kernel("cell")
    vb.evolve(a, max_steps=20)
    vb.evolve(b, max_steps=20)
    assert a.t == b.t
    assert_bit_identical(a.state(), b.state())


def test_tiled2d_sharp_walls_bit_identical(vb, oracle):
    """A 2D Riemann problem in a reflecting/outflow box: every boundary path."""
    dims = (256, 24)
    prob = P.Problem(name="r2", dims=dims, domain=((0.0, 1.0), (0.0, 0.1)), gamma=1.4,
                     bcs=((P.Reflecting, P.Outflow), (P.Outflow, P.Reflecting)),
                     init=lambda x, y, z: (np.where(x + 2 * y < 0.5, 1.0, 0.125),
                                           np.where(x < 0.3, 0.5, -0.25), 0.1, 0.0,
                                           np.where(x + 2 * y < 0.5, 1.0, 0.1)))
    U0 = P.initial_state(prob)
    sim = make_sim(prob, U0)
    sim.set_kernel("tiled")
    assert sim.kernel == "tiled"
    vb.evolve(sim, max_steps=12)
    g = oracle.grid_from_problem(prob)
    U = U0.copy()
    t_ref, n_ref = oracle.evolve(g, U, math.inf, max_steps=12, mode=1)
    assert sim.t == t_ref
    assert_bit_identical(sim.state(), U)


def test_tiled2d_mixed_accuracy_and_conservation(vb):
    prob = P.smooth_random_problem((512, 384), seed=9)
    U0 = P.initial_state(prob)
    a = make_sim(prob, U0, "fp64")
    b = make_sim(prob, U0, "mixed")
    a.set_kernel("tiled")
    b.set_kernel("tiled")
    assert a.kernel == "tiled" and b.kernel == "tiled"
    t0 = np.array(vb.conserved_totals(b))
    vb.evolve(a, max_steps=20)
    vb.evolve(b, max_steps=20)
    ra, rb = a.state()[0], b.state()[0]
    l1 = float(np.sum(np.abs(ra - rb)) / np.sum(np.abs(ra)))
    assert l1 <= 1e-6, l1
    t1 = np.array(vb.conserved_totals(b))
    assert np.allclose(t1, t0, rtol=1e-12, atol=1e-12 * np.abs(t0).max())


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_plane4096_properties(vb, precision):
    """The 4096^2 throughput configuration: a few steps conserve and stay finite;
    the result does not depend on the row chunk."""
    prob = P.smooth_random_problem((4096, 4096))
    U0 = P.initial_state(prob)
    a = make_sim(prob, U0, precision)
    t0 = np.array(vb.conserved_totals(a))
    a.set_kernel("tiled", kz=32)
    vb.evolve(a, max_steps=3)
    Ua = a.state()
    assert np.all(np.isfinite(Ua))
    t1 = np.array(vb.conserved_totals(a))
    assert np.allclose(t1, t0, rtol=1e-12, atol=1e-12 * np.abs(t0).max())
    a.close()
    b = make_sim(prob, U0, precision)
    b.set_kernel("tiled", kz=96)
    vb.evolve(b, max_steps=3)
    assert_bit_identical(b.state(), Ua)
