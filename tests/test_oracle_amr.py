"""The AMR oracle (oracle/vespa_oracle_amr.c) against the uniform oracle and
against the reference's own AMR gates (test/test_amr_ka_flux.jl,
test/test_reflux.jl, test/test_sedov.jl), re-expressed for the CPU."""
import itertools

import numpy as np
import pytest


def _amr(O, prob, U=None):
    import vespa_b200 as vb
    a = O.Amr(O.grid_from_problem(prob))
    a.set_state(vb.initial_state(prob) if U is None else U)
    return a


def _levels_balanced(a, nd, dims):
    """Every pair of face-adjacent leaves differs by at most one level."""
    lev, cx = a.leaves()
    cells = {}
    L = int(lev.max())
    for l, c in zip(lev, cx):
        # mark the finest-level footprint of each leaf
        s = 1 << (L - l)
        rng = [range(int(c[d]) * s, (int(c[d]) + 1) * s) if d < nd else range(1) for d in range(3)]
        for p in itertools.product(*rng):
            cells[p] = int(l)
    for p, l in cells.items():
        for d in range(nd):
            q = list(p)
            q[d] += 1
            q = tuple(q)
            if q in cells and abs(cells[q] - l) > 1:
                return False
    return True


@pytest.mark.parametrize("case", ["sod64", "mixed2d", "periodic3d", "sedov16"])
def test_unrefined_amr_is_the_uniform_path(oracle, case):
    """With no refinement the composite mesh is RefMesh in the same order:
    the AMR restatement reproduces the uniform oracle bit for bit."""
    import vespa_b200 as vb
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
    U = vb.initial_state(prob)
    g = oracle.grid_from_problem(prob)
    a = _amr(oracle, prob, U)
    ref = np.ascontiguousarray(U.copy())
    for _ in range(5):
        dt = oracle.compute_dt(g, ref)
        assert a.compute_dt() == dt
        oracle.step(g, ref, dt)
        a.step(dt)
    assert np.array_equal(a.state(), ref)
    assert np.array_equal(a.totals(), oracle.conserved_totals(g, ref))


def test_refine_keeps_balance_and_totals(oracle):
    import vespa_b200 as vb
    prob = vb.sedov_problem(n=8)
    a = _amr(oracle, prob)
    t0 = a.totals()
    a.refine([27])          # one interior leaf
    a.refine([0])           # a corner leaf
    lev, cx = a.leaves()
    target = int(np.where((lev == 1) & (cx[:, 0] == 6) & (cx[:, 1] == 6))[0][0])
    a.refine([target])      # level 2 next to level-0 cells: balance must cascade
    assert a.max_level == 2
    assert _levels_balanced(a, 2, prob.dims)
    np.testing.assert_allclose(a.totals(), t0, rtol=1e-15, atol=1e-300)
    # leaves tile the domain exactly once
    lev, cx = a.leaves()
    area = np.sum(0.25 ** lev)
    assert area == 64.0


def _conserved(t0, t1, rtol=1e-9):
    assert abs(t1[0] - t0[0]) <= rtol * abs(t0[0])
    assert abs(t1[4] - t0[4]) <= rtol * abs(t0[4])


def test_refined_sod_single_rate_conserves(oracle):
    """test/test_amr_ka_flux.jl:36-45: refined Sod, single rate."""
    import vespa_b200 as vb
    prob = vb.sod_problem_defaults(n=64)
    a = _amr(oracle, prob)
    t0 = a.totals()
    a.evolve(prob.tfinal, refine_above=0.1, max_level=2, every=4)
    assert a.max_level >= 1
    assert abs(a.t - 0.2) < 1e-14
    _conserved(t0, a.totals())


def test_subcycled_sod_conserves(oracle):
    """test/test_reflux.jl:13-35 and :37-51 (nested registers)."""
    import vespa_b200 as vb
    prob = vb.sod_problem_defaults(n=64)
    for above, lmax, every, need in ((0.1, 2, 4, 1), (0.05, 3, 3, 2)):
        a = _amr(oracle, prob)
        t0 = a.totals()
        a.evolve(prob.tfinal, refine_above=above, max_level=lmax, every=every, subcycle=True)
        assert a.max_level >= need
        _conserved(t0, a.totals())
        U = a.state()
        W = vb.cons2prim(U, prob.gamma)
        assert np.all(W[0] > 0) and np.all(W[4] > 0)


def test_subcycled_matches_single_rate_accuracy(oracle):
    """test/test_reflux.jl:53-93: both runs against the exact solution."""
    import vespa_b200 as vb
    prob = vb.sod_problem_defaults(n=64)

    def l1(sub):
        a = _amr(oracle, prob)
        a.evolve(prob.tfinal, refine_above=0.1, max_level=2, every=4, subcycle=sub)
        lev, cx = a.leaves()
        w = (1.0 / 64) * 0.5 ** lev
        x = (cx[:, 0] + 0.5) * w
        rho = a.state()[0]
        ex = np.array([oracle.exact_riemann_sample((1.0, 0.0, 1.0), (0.125, 0.0, 0.1), 1.4,
                                                   (xi - 0.5) / a.t)[0] for xi in x])
        return float(np.sum(np.abs(rho - ex) * w) / np.sum(w))

    e_flat, e_sub = l1(False), l1(True)
    assert e_sub < 0.02
    assert e_sub < 1.5 * e_flat


def test_small_sedov_conserves(oracle):
    """test/test_amr_ka_flux.jl:57-66: 2D Sedov 32^2 to t = 0.02 with AMR."""
    import vespa_b200 as vb
    prob = vb.sedov_problem(n=32, tfinal=0.02)
    a = _amr(oracle, prob)
    t0 = a.totals()
    a.evolve(prob.tfinal, refine_above=0.05, max_level=2, every=4)
    assert a.max_level >= 1
    _conserved(t0, a.totals())
    assert _levels_balanced(a, 2, prob.dims)
