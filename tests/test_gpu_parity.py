"""GPU parity: the CUDA library against the CPU oracle and the golden fixtures.

The VB_FP64 path is bit-identical to the oracle (a float64 evaluation in the
reference's operation order), which is stronger than the 1e-12 relative per
cell the tier asks for; the tests assert exact equality and report the max
relative difference on failure.  The VB_MIXED path is checked against the
VB_FP64 path by its density L1 error (<= 1e-6 relative) and by conservation.
"""
import math
import os

import numpy as np
import pytest

import vespa_b200 as vb
from vespa_b200 import problem as P

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
BC_OF = {0: P.Outflow, 1: P.Periodic, 2: P.Reflecting}


def max_rel(a, b):
    scale = np.maximum(np.abs(a), np.abs(b))
    d = np.abs(a - b)
    with np.errstate(invalid="ignore", divide="ignore"):
        r = np.where(scale > 0, d / scale, 0.0)
    return float(np.max(r))


def assert_bit_identical(a, b):
    assert a.shape == b.shape
    if not np.array_equal(a, b):
        raise AssertionError(f"not bit-identical: max rel diff {max_rel(a, b):.3e}, "
                             f"{int(np.sum(a != b))} of {a.size} values differ")


def problem_from(dims, domain, bc_lo, bc_hi, gamma, cfl, tfinal=math.inf):
    bcs = tuple((BC_OF[int(l)], BC_OF[int(h)]) for l, h in zip(bc_lo, bc_hi))
    return P.Problem(name="case", dims=tuple(int(n) for n in dims),
                     domain=tuple((float(a), float(b)) for a, b in domain), gamma=float(gamma),
                     bcs=bcs, init=lambda x, y, z: (1.0, 0.0, 0.0, 0.0, 1.0), tfinal=tfinal,
                     cfl=float(cfl))


def make_sim(prob, U0, precision="fp64"):
    return vb.Simulation(vb.B200Mesh(prob.dims, prob.domain), prob, precision=precision,
                         initial=U0)


def golden_names():
    return sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz") and f != "hllc_faces.npz")


# ------------------------------------------------------------ face batches
def test_hllc_faces_golden_bit_identical(vb):
    d = np.load(os.path.join(GOLDEN, "hllc_faces.npz"))
    F = np.zeros_like(d["F"])
    out = vb.compute_face_fluxes(vb.B200Flux(), vb.IdealHydro(float(d["gamma"])), F,
                                 np.ascontiguousarray(d["WL"]), np.ascontiguousarray(d["WR"]),
                                 d["axis"])
    assert out is F
    assert_bit_identical(F, d["F"])


def test_hllc_faces_large_batch_vs_oracle(vb, oracle):
    from tests.golden.make_golden import random_faces
    WL, WR, axis = random_faces(300_001, seed=99)
    F = np.zeros_like(WL)
    vb.compute_face_fluxes(vb.B200Flux(), 5.0 / 3.0, F, WL, WR, axis)
    assert_bit_identical(F, oracle.compute_face_fluxes(WL, WR, axis, 5.0 / 3.0))
    # empty batch: F untouched (ext/VespaKAFluxExt.jl:40 returns early)
    E = np.zeros((0, 5))
    assert vb.compute_face_fluxes(vb.B200Flux(), 1.4, E, E.copy(), E.copy(), []) is E


def test_hllc_faces_rejects_bad_axis(vb):
    W = np.ones((3, 5))
    with pytest.raises(vb.VespaB200Error):
        vb.compute_face_fluxes(vb.B200Flux(), 1.4, np.zeros((3, 5)), W, W.copy(), [1, 4, 2])


# ------------------------------------------------------------ stepping
@pytest.mark.parametrize("name", golden_names())
def test_golden_steps_bit_identical(vb, name):
    d = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    prob = problem_from(d["dims"], d["domain"], d["bc_lo"], d["bc_hi"], d["gamma"], d["cfl"])
    sim = make_sim(prob, d["U0"])
    for dt_ref in d["dts"]:
        dt = vb.compute_dt(sim)
        assert dt == dt_ref
        vb.step(sim, dt)
    assert sim.step == len(d["dts"])
    assert sim.t == pytest.approx(float(np.sum(d["dts"])), rel=1e-14)
    assert_bit_identical(sim.state(), d["U"])


CASES = [
    ((16,), [0], [0]), ((16,), [2], [0]), ((9,), [1], [1]), ((1,), [1], [1]),
    ((6, 5), [1, 2], [1, 2]), ((7, 4), [0, 1], [2, 1]), ((1, 5), [1, 0], [1, 0]),
    ((2, 3), [1, 1], [1, 1]), ((4, 3, 3), [1, 0, 2], [1, 2, 0]),
    ((3, 1, 2), [0, 1, 1], [0, 1, 1]), ((2, 2, 2), [1, 1, 1], [1, 1, 1]),
    ((64, 48), [1, 1], [1, 1]), ((33, 17), [2, 0], [0, 2]),
    ((24, 20, 16), [1, 2, 0], [1, 2, 0]), ((17, 9, 11), [0, 0, 0], [0, 0, 0]),
]


@pytest.mark.parametrize("dims,bclo,bchi", CASES)
def test_random_grids_bit_identical_to_oracle(vb, oracle, dims, bclo, bchi):
    nd = len(dims)
    prob = problem_from(dims, [(0.0, 1.0)] * nd, bclo, bchi, 1.4, 0.4)
    U0 = np.ascontiguousarray(P.initial_state(P.smooth_random_problem(dims, seed=sum(dims))))
    g = oracle.make_grid(dims, [0] * nd, [1] * nd, bclo, bchi, 1.4, 0.4)
    sim = make_sim(prob, U0)
    # device-resident loop: dt computed and consumed on the GPU
    vb.evolve(sim, tfinal=math.inf, max_steps=6)
    U = U0.copy()
    t_ref, n_ref = oracle.evolve(g, U, math.inf, max_steps=6, mode=1)
    assert sim.step == n_ref == 6
    assert sim.t == t_ref
    assert_bit_identical(sim.state(), U)


def test_sod400_full_run_bit_identical(vb, oracle):
    prob = P.sod_problem_defaults(400, cfl=0.8)
    sim = vb.Simulation(vb.B200Mesh(prob.dims, prob.domain), prob)
    vb.evolve(sim)
    U = P.initial_state(prob)
    t, n = oracle.evolve(oracle.grid_from_problem(prob), U, prob.tfinal)
    assert sim.step == n and sim.t == t == pytest.approx(0.2, rel=1e-12)
    assert_bit_identical(sim.state(), U)


def test_sod_vs_exact_and_conservation_on_gpu(vb, oracle):
    """test/test_sod.jl:20-44 on the device path."""
    prob = P.sod_problem_defaults(256)
    sim = vb.Simulation(vb.B200Mesh(prob.dims, prob.domain), prob)
    t0 = vb.conserved_totals(sim)
    vb.evolve(sim)
    t1 = vb.conserved_totals(sim)
    assert t1.mass == pytest.approx(t0.mass, rel=1e-12)
    assert t1.energy == pytest.approx(t0.energy, rel=1e-12)
    d = vb.dump_fields(sim)
    ex = np.array([oracle.exact_riemann_sample((1.0, 0.0, 1.0), (0.125, 0.0, 0.1), 1.4,
                                               (x - 0.5) / sim.t)[0] for x in d["x"]])
    assert float(np.mean(np.abs(d["density"] - ex))) < 0.01
    assert np.all(d["density"] > 0) and np.all(d["pressure"] > 0)


def test_host_loop_equals_device_loop(vb):
    prob = P.smooth_random_problem((20, 18, 6), seed=4, tfinal=0.05)
    U0 = P.initial_state(prob)
    a = make_sim(prob, U0)
    vb.evolve(a)
    b = make_sim(prob, U0)
    t = 0.0
    while t < prob.tfinal * (1 - 1e-12):  # evolve! written out (src/driver.jl:493-500)
        dt = min(vb.compute_dt(b), prob.tfinal - t)
        vb.step(b, dt)
        t += dt
    assert a.step == b.step and a.t == b.t == t
    assert_bit_identical(a.state(), b.state())


def test_conserved_totals_match_serial_sum(vb, oracle):
    prob = P.smooth_random_problem((40, 36, 30), seed=8)
    U0 = P.initial_state(prob)
    sim = make_sim(prob, U0)
    got = np.array(vb.conserved_totals(sim))
    ref = oracle.conserved_totals(oracle.grid_from_problem(prob), U0)
    assert np.allclose(got, ref, rtol=1e-13, atol=1e-15 * np.abs(ref).max())
    assert np.array_equal(got, np.array(vb.conserved_totals(sim)))  # deterministic


def test_boundary_flux_identity_on_gpu(vb):
    """test/test_boundary_flux.jl:9-35 on the device register."""
    prob = P.Problem(name="ramp", dims=(64,), domain=((0.0, 1.0),), gamma=1.4, bcs=P.Outflow,
                     init=lambda x, y, z: (1.0 + x, 1.0, 0.0, 0.0, 2.0), tfinal=1.0, cfl=0.3)
    sim = vb.Simulation(vb.B200Mesh(prob.dims, prob.domain), prob)
    sim.bflux_enable(True)
    m0 = vb.conserved_totals(sim).mass
    lo = hi = 0.0
    for _ in range(20):
        sim.bflux_clear()
        vb.step(sim, 5e-4)
        bf = sim.bflux_read()
        lo += bf[0]
        hi += bf[5]
    dm = vb.conserved_totals(sim).mass - m0
    assert abs(dm) > 1e-3
    assert abs(dm - (lo - hi)) < 1e-12


def test_bflux_planes_match_oracle(vb, oracle):
    prob = problem_from((6, 5, 4), [(0.0, 1.0)] * 3, [0, 2, 1], [2, 0, 1], 1.4, 0.4)
    U0 = P.initial_state(P.smooth_random_problem((6, 5, 4), seed=21))
    sim = make_sim(prob, U0)
    sim.bflux_enable(True)
    g = oracle.make_grid((6, 5, 4), [0] * 3, [1] * 3, [0, 2, 1], [2, 0, 1], 1.4, 0.4)
    bf = np.zeros(oracle.bflux_size(g))
    U = U0.copy()
    for _ in range(3):
        dt = vb.compute_dt(sim)
        vb.step(sim, dt)
        oracle.step(g, U, dt, bflux=bf)
    assert_bit_identical(sim.bflux_read(), bf)


# ------------------------------------------------------------ tiled 3D kernel
TILED_CASES = [
    # dims, bc_lo, bc_hi, kz
    ((32, 16, 9), [1, 1, 1], [1, 1, 1], None),
    ((16, 32, 20), [0, 2, 1], [2, 0, 1], 3),
    ((48, 32, 11), [2, 1, 0], [2, 1, 0], 4),
    ((32, 48, 2), [1, 0, 2], [1, 2, 0], 1),
    ((16, 16, 7), [0, 0, 0], [0, 0, 0], 2),
    ((64, 32, 33), [1, 1, 1], [1, 1, 1], 8),
]


@pytest.mark.parametrize("dims,bclo,bchi,kz", TILED_CASES)
def test_tiled_kernel_bit_identical_to_oracle(vb, oracle, dims, bclo, bchi, kz):
    prob = problem_from(dims, [(0.0, 1.0)] * 3, bclo, bchi, 1.4, 0.4)
    U0 = P.initial_state(P.smooth_random_problem(dims, seed=sum(dims) + 1))
    sim = make_sim(prob, U0)
    sim.set_kernel("tiled", kz=kz)
    assert sim.kernel == "tiled"
    vb.evolve(sim, tfinal=math.inf, max_steps=5)
    U = U0.copy()
    g = oracle.make_grid(dims, [0] * 3, [1] * 3, bclo, bchi, 1.4, 0.4)
    t_ref, n_ref = oracle.evolve(g, U, math.inf, max_steps=5, mode=1)
    assert sim.step == n_ref and sim.t == t_ref
    assert_bit_identical(sim.state(), U)


def test_autotune_restores_state_and_keeps_results(vb):
    prob = P.smooth_random_problem((64, 48, 80), seed=31)
    U0 = P.initial_state(prob)
    a = make_sim(prob, U0)
    a.set_kernel("tiled")
    kz, ms = a.autotune(nsteps=2)
    assert kz in (16, 24, 32, 40, 48, 64) and ms > 0
    assert a.kz == kz
    assert a.step == 0 and a.t == 0.0
    assert_bit_identical(a.state(), U0)
    # the chunking changes the schedule, never the float64 result
    b = make_sim(prob, U0)
    b.set_kernel("tiled", kz=7)
    vb.evolve(a, tfinal=math.inf, max_steps=4)
    vb.evolve(b, tfinal=math.inf, max_steps=4)
    assert_bit_identical(a.state(), b.state())
    c = make_sim(prob, U0)  # a new grid of the same kind starts from the tuned kz
    assert c.kz == kz


def test_tiled_equals_cell_kernel_on_sharp_data(vb):
    """A strong planar discontinuity (all HLLC branches, both star sides) on
    outflow walls: tiled and cell-centric float64 kernels agree to the bit."""
    prob = P.riemann_box_problem(3, side=32)
    U0 = P.initial_state(prob)
    a = make_sim(prob, U0)
    b = make_sim(prob, U0)
    a.set_kernel("tiled", kz=5)
    b.set_kernel("cell")
    vb.evolve(a, tfinal=math.inf, max_steps=8)
    vb.evolve(b, tfinal=math.inf, max_steps=8)
    assert a.t == b.t
    assert_bit_identical(a.state(), b.state())


def test_tiled_mixed_precision_conserves(vb):
    prob = P.smooth_random_problem((64, 48, 40), seed=6)
    U0 = P.initial_state(prob)
    a = make_sim(prob, U0, "fp64")
    b = make_sim(prob, U0, "mixed")
    a.set_kernel("tiled")
    b.set_kernel("tiled")
    assert b.kernel == "tiled"
    t0 = np.array(vb.conserved_totals(b))
    vb.evolve(a, max_steps=20)
    vb.evolve(b, max_steps=20)
    ra, rb = a.state()[0], b.state()[0]
    l1 = float(np.sum(np.abs(ra - rb)) / np.sum(np.abs(ra)))
    assert l1 <= 1e-6, l1
    t1 = np.array(vb.conserved_totals(b))
    assert np.allclose(t1, t0, rtol=1e-12, atol=1e-12 * np.abs(t0).max())


@pytest.mark.parametrize("bcs", [((2, 2), (2, 2), (2, 2)), ((0, 2), (2, 0), (1, 1))])
def test_tiled_mixed_on_sharp_data(vb, bcs):
    """Mixed tiled kernel on a strong planar discontinuity with walls.  Interior
    faces telescope exactly; a reflecting wall's mass and energy flux is zero
    only analytically, and the float32 Riemann solve leaves a ~1e-7 relative
    residue there, so a closed box conserves to the reference's own
    closed-box tolerance (rtol 1e-9, test/test_sedov.jl:63-64) rather than to
    1e-12.  The density stays within a float32-level distance of float64."""
    base = P.riemann_box_problem(5, side=32)
    prob = P.Problem(name="box", dims=base.dims, domain=base.domain, gamma=base.gamma,
                     bcs=tuple((BC_OF[l], BC_OF[h]) for l, h in bcs), init=base.init, cfl=0.4)
    U0 = P.initial_state(prob)
    a = make_sim(prob, U0, "fp64")
    b = make_sim(prob, U0, "mixed")
    a.set_kernel("tiled")
    b.set_kernel("tiled")
    assert b.kernel == "tiled"
    t0 = np.array(vb.conserved_totals(b))
    vb.evolve(a, tfinal=math.inf, max_steps=15)
    vb.evolve(b, tfinal=math.inf, max_steps=15)
    ra, rb = a.state()[0], b.state()[0]
    assert np.all(rb > 0)
    l1 = float(np.sum(np.abs(ra - rb)) / np.sum(np.abs(ra)))
    assert l1 <= 1e-4, l1
    if bcs == ((2, 2), (2, 2), (2, 2)):
        t1 = np.array(vb.conserved_totals(b))
        assert t1[0] == pytest.approx(t0[0], rel=1e-9)
        assert t1[4] == pytest.approx(t0[4], rel=1e-9)


# ------------------------------------------------------------ mixed precision
def test_mixed_precision_accuracy_and_conservation(vb):
    prob = P.smooth_random_problem((48, 40, 32), seed=5)
    U0 = P.initial_state(prob)
    a = make_sim(prob, U0, "fp64")
    b = make_sim(prob, U0, "mixed")
    ta = vb.conserved_totals(b)
    vb.evolve(a, max_steps=20)
    vb.evolve(b, max_steps=20)
    ra, rb = a.state()[0], b.state()[0]
    l1 = float(np.sum(np.abs(ra - rb)) / np.sum(np.abs(ra)))
    assert l1 <= 1e-6, l1
    tb = vb.conserved_totals(b)
    assert tb.mass == pytest.approx(ta.mass, rel=1e-12)
    assert tb.energy == pytest.approx(ta.energy, rel=1e-12)


# ------------------------------------------------------------ failure detection
def test_nonfinite_state_is_reported(vb):
    prob = P.smooth_random_problem((16, 16), seed=2)
    U0 = P.initial_state(prob)
    U0[0, 37] = -1.0  # negative density: sound speed NaN
    sim = make_sim(prob, U0)
    with pytest.raises(vb.VespaB200Error) as e:
        vb.compute_dt(sim)
    assert e.value.status == 4
    with pytest.raises(vb.VespaB200Error) as e:
        vb.evolve(sim, max_steps=3)
    assert e.value.status == 4


def test_invalid_descriptors_rejected(vb):
    prob = problem_from((8, 8), [(0.0, 1.0)] * 2, [1, 0], [0, 0], 1.4, 0.4)
    with pytest.raises(vb.VespaB200Error) as e:
        make_sim(prob, P.initial_state(P.smooth_random_problem((8, 8))))
    assert e.value.status == 1


# ------------------------------------------------------------ full-size properties
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_full_size_256cubed_conservation_and_determinism(vb, precision):
    """At the benchmark's full size (256^3 periodic) the oracle is too slow to
    compare cell by cell, so check size-independent properties: periodic
    conservation of all five totals and bitwise run-to-run determinism."""
    prob = P.smooth_random_problem((256, 256, 256))
    U0 = P.initial_state(prob)
    a = make_sim(prob, U0, precision)
    t0 = np.array(vb.conserved_totals(a))
    vb.evolve(a, max_steps=3)
    t1 = np.array(vb.conserved_totals(a))
    assert np.allclose(t1, t0, rtol=1e-12, atol=1e-12 * np.abs(t0).max())
    Ua = a.state()
    a.close()
    b = make_sim(prob, U0, precision)
    vb.evolve(b, max_steps=3)
    assert np.array_equal(Ua, b.state())
