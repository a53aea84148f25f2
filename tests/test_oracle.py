"""The CPU oracle, pinned before it is trusted.

1. Known answers the reference's own tests hold for this path:
   Sod vs the exact Riemann solution and conservation (test/test_sod.jl:20-44),
   the boundary-flux identity (test/test_boundary_flux.jl:9-35), and Toro's
   published Sod star state (Riemann Solvers and Numerical Methods for Fluid
   Dynamics, Table 4.2, test 1).
2. An independent pure-Python transcription of the Julia source
   (oracle/pyref.py) agrees with the C oracle bit for bit on small grids with
   every boundary combination.
3. The parallel per-cell gather variant used as the timed CPU baseline is
   bit-identical to the faithful serial face enumeration.
4. The committed golden fixtures are reproduced exactly.
"""
import os

import numpy as np
import pytest

import vespa_b200.problem as P

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
SOD_L = (1.0, 0.0, 1.0)
SOD_R = (0.125, 0.0, 0.1)


def sod_l1(O, x, rho, t, gamma=1.4):
    ex = np.array([O.exact_riemann_sample(SOD_L, SOD_R, gamma, (xi - 0.5) / t)[0] for xi in x])
    return float(np.mean(np.abs(rho - ex)))


def test_toro_star_state(oracle):
    p, u = oracle.exact_riemann_star(SOD_L, SOD_R, 1.4)
    assert abs(p - 0.30313) < 5e-6 and abs(u - 0.92745) < 5e-6


@pytest.mark.parametrize("n,cfl,l1max", [(256, 0.4, 0.01), (400, 0.8, 0.01)])
def test_sod_vs_exact(oracle, n, cfl, l1max):
    prob = P.sod_problem_defaults(n, cfl=cfl)
    U = P.initial_state(prob)
    g = oracle.grid_from_problem(prob)
    t0 = oracle.conserved_totals(g, U)
    t, nsteps = oracle.evolve(g, U, prob.tfinal)
    t1 = oracle.conserved_totals(g, U)
    assert t == pytest.approx(0.2, rel=1e-12)
    # test/test_sod.jl:32-33
    assert t1[0] == pytest.approx(t0[0], rel=1e-12)
    assert t1[4] == pytest.approx(t0[4], rel=1e-12)
    W = P.cons2prim(U, 1.4)
    l1 = sod_l1(oracle, prob.cell_centers()[0], W[0], t)
    assert l1 < l1max  # test/test_sod.jl:37
    assert np.all(W[0] > 0) and np.all(W[4] > 0)
    assert W[0].max() <= 1.0 + 1e-6 and W[0].min() >= 0.125 - 1e-6


def test_boundary_flux_identity(oracle):
    """test/test_boundary_flux.jl:9-35: the time-integrated boundary flux
    accounts exactly for the change of total mass."""
    prob = P.Problem(name="ramp", dims=(64,), domain=((0.0, 1.0),), gamma=1.4, bcs=P.Outflow,
                     init=lambda x, y, z: (1.0 + x, 1.0, 0.0, 0.0, 2.0), tfinal=1.0, cfl=0.3)
    U = P.initial_state(prob)
    g = oracle.grid_from_problem(prob)
    V = 1 / 64
    mass = lambda: float(np.sum(U[0]) * V)
    m0 = mass()
    tot_lo = tot_hi = 0.0
    for _ in range(20):
        bf = np.zeros(oracle.bflux_size(g))
        oracle.step(g, U, 5e-4, bflux=bf)
        # layout: axis 1, side lo (5 comps x 1 plane cell), then side hi
        tot_lo += bf[0]
        tot_hi += bf[5]
    dm = mass() - m0
    assert abs(dm) > 1e-3
    assert abs(dm - (tot_lo - tot_hi)) < 1e-12


CASES = [
    ((16,), [0], [0]), ((16,), [2], [0]), ((9,), [1], [1]),
    ((6, 5), [1, 2], [1, 2]), ((7, 4), [0, 1], [2, 1]), ((1, 5), [1, 0], [1, 0]),
    ((2, 3), [1, 1], [1, 1]), ((4, 3, 3), [1, 0, 2], [1, 2, 0]),
    ((3, 1, 2), [0, 1, 1], [0, 1, 1]), ((2, 2, 2), [1, 1, 1], [1, 1, 1]),
]


def random_state(dims, seed, gamma=1.4):
    rng = np.random.default_rng(seed)
    n = int(np.prod(dims))
    W = np.empty((5, n))
    W[0] = rng.uniform(0.5, 2.0, n)
    W[1:4] = rng.uniform(-1.0, 1.0, (3, n))
    W[4] = rng.uniform(0.5, 2.0, n)
    W[1 + len(dims):4] = 0.0
    return np.ascontiguousarray(P.prim2cons(W, gamma))


@pytest.mark.parametrize("dims,bclo,bchi", CASES)
def test_oracle_matches_python_transcription(oracle, dims, bclo, bchi):
    from oracle import pyref as R
    nd = len(dims)
    U = random_state(dims, seed=3)
    g = oracle.make_grid(dims, [0] * nd, [1] * nd, bclo, bchi, 1.4, 0.4)
    m = R.UniformGrid(dims, [0.0] * nd, [1.0] * nd, bclo, bchi, 1.4, 0.4)
    cells = list(m.cells())
    Ud = {I: tuple(U[:, i]) for i, I in enumerate(cells)}
    acc_p = np.array([R.accumulate_flux(m, Ud)[I] for I in cells]).T
    assert np.array_equal(oracle.accumulate_flux(g, U), acc_p)
    assert oracle.compute_dt(g, U) == R.compute_dt(m, Ud)
    Uc = U.copy()
    for _ in range(2):
        dt = oracle.compute_dt(g, Uc)
        oracle.step(g, Uc, dt)
        Ud = R.step(m, Ud, dt)
    assert np.array_equal(Uc, np.array([Ud[I] for I in cells]).T)


@pytest.mark.parametrize("dims,bclo,bchi", CASES + [((33, 17), [1, 0], [1, 2]),
                                                    ((12, 9, 7), [1, 2, 0], [1, 0, 2])])
def test_gather_variant_is_bit_identical(oracle, dims, bclo, bchi):
    nd = len(dims)
    U = random_state(dims, seed=5)
    g = oracle.make_grid(dims, [0] * nd, [1] * nd, bclo, bchi, 1.4, 0.4)
    assert np.array_equal(oracle.accumulate_flux(g, U),
                          oracle.accumulate_flux(g, U, gather=True, nthreads=4))
    A, B = U.copy(), U.copy()
    for _ in range(3):
        dt = oracle.compute_dt(g, A)
        oracle.step(g, A, dt, mode=0)
        oracle.step(g, B, dt, mode=1, nthreads=3)
    assert np.array_equal(A, B)


def test_batched_faces_match_per_face(oracle):
    from oracle import pyref as R
    d = np.load(os.path.join(GOLDEN, "hllc_faces.npz"))
    F = oracle.compute_face_fluxes(d["WL"], d["WR"], d["axis"], 1.4)
    for f in range(0, len(F), 37):
        ref = R.hllc_flux(tuple(d["WL"][f]), tuple(d["WR"][f]), 1.4, int(d["axis"][f]))
        assert tuple(F[f]) == ref


def golden_names():
    return sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz") and f != "hllc_faces.npz")


def test_golden_faces_reproduced(oracle):
    d = np.load(os.path.join(GOLDEN, "hllc_faces.npz"))
    assert np.array_equal(oracle.compute_face_fluxes(d["WL"], d["WR"], d["axis"], float(d["gamma"])),
                          d["F"])


@pytest.mark.parametrize("name", golden_names())
def test_golden_steps_reproduced(oracle, name):
    d = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    dims = tuple(int(n) for n in d["dims"])
    g = oracle.make_grid(dims, d["domain"][:, 0], d["domain"][:, 1], d["bc_lo"], d["bc_hi"],
                         float(d["gamma"]), float(d["cfl"]))
    U = d["U0"].copy()
    for dt_ref in d["dts"]:
        dt = oracle.compute_dt(g, U)
        assert dt == dt_ref
        oracle.step(g, U, dt)
    assert np.array_equal(U, d["U"])


def test_interior_register_accounts_for_every_cell(oracle):
    """With record_interior the register holds every face's time-integrated
    flux (src/reflux.jl:138-146), so on a periodic box each cell's change
    over a step is minus the net integrated flux through its faces over its
    volume (the per-cell form of the conservation identity of
    test/test_boundary_flux.jl)."""
    dims = (6, 5, 4)
    g = oracle.make_grid(dims, [0] * 3, [1] * 3, [1] * 3, [1] * 3, 1.4, 0.4)
    U = P.initial_state(P.smooth_random_problem(dims, seed=4))
    U0 = U.copy()
    reg = oracle.BoundaryFluxRegister(g, record_interior=True)
    oracle.step_breg(g, U, oracle.compute_dt(g, U), reg)
    assert reg.iseen.all() and not reg.seen.any()   # periodic: no outer faces
    nc = U.size // 5
    R = reg.ivals.reshape(3, 5, *dims[::-1])        # [axis][comp][z][y][x]
    net = np.zeros((5,) + dims[::-1])
    for d in range(3):
        ax = 2 - d                                   # array axis of grid axis d
        net += R[d] - np.roll(R[d], 1, axis=1 + ax)  # out through hi face, in through lo face
    V = 1.0 / nc
    dU = (U - U0).reshape((5,) + dims[::-1])
    scale = np.abs(U0).reshape((5,) + dims[::-1]).max(axis=(1, 2, 3), keepdims=True)
    assert np.max(np.abs(dU + net / V) / scale) < 1e-12


def _plane_restated(reg, g, dims, dim, source, start, stop, g0, flux_off, comp, vcell):
    """bflux_plane (src/reflux.jl:171-191) transcribed over Dict registers built
    from the dense one, with the lookups of lib/EnzoLib/test/reflux_common.jl."""
    R = len(dims)
    nc = int(np.prod(dims))
    flux, interior = {}, {}
    P_ = lambda d: nc // dims[d]
    base = 0
    for d in range(R):
        for side in (0, 1):
            for idx in range(P_(d)):
                if reg.seen[base + idx]:
                    rest, mul, cell = idx, 1, [0] * R
                    for e in range(R):
                        if e == d:
                            continue
                        cell[e] = rest % dims[e]
                        rest //= dims[e]
                    cell[d] = 0 if side == 0 else dims[d] - 1
                    key = (d + 1, "lo" if side == 0 else "hi", tuple(c + 1 for c in cell))
                    flux[key] = [reg.vals[base + k * P_(d) + idx] for k in range(5)]
            base += 5 * P_(d)
    if reg.ivals is not None:
        for d in range(R):
            for lin in range(nc):
                if reg.iseen[d * nc + lin]:
                    cell, rest = [], lin
                    for e in range(R):
                        cell.append(rest % dims[e] + 1)
                        rest //= dims[e]
                    interior[(d + 1, tuple(cell))] = [reg.ivals[(d * 5 + k) * nc + lin] for k in range(5)]
    ax = dim + 1
    if source == 2:
        lookup = lambda I: interior.get((ax, I))
    else:
        lookup = lambda I: flux.get((ax, "lo" if source == 0 else "hi", I))
    D = [stop[d] - start[d] + 1 for d in range(R)]
    out = []
    for lin in range(int(np.prod(D))):
        rem, act = lin, []
        for d in range(R):
            od = rem % D[d]
            rem //= D[d]
            act.append(flux_off if d == dim else start[d] + od - g0[d] + 1)
        F = lookup(tuple(act))
        out.append(F[comp - 1] / vcell if (F is not None and comp > 0) else 0.0)
    return np.array(out)


def test_bflux_plane_matches_a_dict_restatement(oracle):
    dims = (6, 5, 4)
    g = oracle.make_grid(dims, [0] * 3, [1] * 3, [0, 2, 1], [2, 0, 1], 1.4, 0.4)
    U = P.initial_state(P.smooth_random_problem(dims, seed=21))
    reg = oracle.BoundaryFluxRegister(g, record_interior=True)
    for _ in range(2):
        oracle.step_breg(g, U, oracle.compute_dt(g, U), reg)
    g0 = (11, 21, 31)  # the grid's first active cell in global indices
    cases = [
        (0, 0, (11, 21, 31), (11, 25, 34), 1, 1), (0, 1, (16, 21, 31), (16, 25, 34), 6, 2),
        (1, 0, (11, 21, 31), (16, 21, 34), 1, 5), (1, 1, (11, 25, 31), (16, 25, 34), 5, 3),
        (2, 0, (11, 21, 31), (16, 25, 31), 1, 1),                  # periodic axis: nothing recorded
        (0, 0, (11, 19, 30), (11, 26, 35), 1, 4),                  # plane wider than the grid
        (0, 1, (16, 21, 31), (16, 25, 34), 3, 2),                  # flux_off off the boundary cell
        (0, 2, (13, 21, 31), (13, 25, 34), 2, 1), (2, 2, (11, 21, 34), (16, 25, 34), 4, 5),
        (1, 2, (11, 25, 31), (16, 25, 34), 5, 2),                  # hi y is a wall: no interior key
        (0, 0, (11, 21, 31), (11, 25, 34), 1, 0),                  # comp 0: zeros
    ]
    for dim, src, st, sp, off, comp in cases:
        got = oracle.bflux_plane(g, reg, dim, src, st, sp, g0, off, comp, 0.125)
        ref = _plane_restated(reg, g, dims, dim, src, st, sp, g0, off, comp, 0.125)
        assert np.array_equal(got, ref), (dim, src, st, sp, off, comp)
    assert np.any(oracle.bflux_plane(g, reg, 0, 0, (11, 21, 31), (11, 25, 34), g0, 1, 1, 0.125))
