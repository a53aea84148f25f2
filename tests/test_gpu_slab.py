"""The slab decomposition's device path (vespa_b200.slab.SlabSimulation) on
one GPU, against one grid stepped alone:

- one rank with a periodic z axis: its ghost planes are copies of its own
  far planes, exchanged locally each stage;
- two and three slabs of one process, the planes moved between them by the
  test in place of the NCCL exchange (the exchange protocol itself is
  covered by the gloo tests in tests/test_slab.py), the CFL maxima combined
  as the all-reduce combines them.

In float64 every slab's planes and the clock must equal the single grid's
bit for bit (periodic and walled z axes); the mixed path must match the
single mixed grid bit for bit too, because each face is still solved once,
by the same formulas, in the same lane.
"""
import math

import numpy as np
import pytest

from vespa_b200 import problem as P
from vespa_b200 import slab as S

pytestmark = pytest.mark.gpu


def _problem(dims, zbc):
    prob = P.smooth_random_problem(dims, seed=12)
    prob.bcs = ((P.Periodic, P.Periodic), (P.Outflow, P.Reflecting), zbc)
    return prob


def _single(vb, prob, U0, precision, nsteps):
    sim = vb.Simulation(vb.B200Mesh(prob.dims, prob.domain), prob, precision=precision,
                        initial=U0)
    sim.set_kernel("tiled")
    vb.evolve(sim, tfinal=math.inf, max_steps=nsteps)
    out = sim.state(), sim.t, np.array(vb.conserved_totals(sim))
    sim.close()
    return out


def _step_emulated(slabs, nsteps):
    """Lockstep phases of all slabs of one process; ghost planes and the CFL
    maximum move as Halo.exchange and the all-reduce would move them.  The
    slabs share the library's stream, and the torch operations here run on
    it too, so every copy is ordered after the work that produced its data."""
    import torch
    from vespa_b200 import _lib
    stream = slabs[0]._stream
    assert all(s.ctx.stream == slabs[0].ctx.stream for s in slabs)

    def exchange(which):
        sends = {}
        for r, s in enumerate(slabs):
            h = s.halo
            sends[r] = (s.get_planes(which, h.act0, S.GHOST),
                        s.get_planes(which, h.act0 + h.nact - S.GHOST, S.GHOST))
        for r, s in enumerate(slabs):
            h = s.halo
            if h.hi_nbr is not None:
                s.put_planes(which, h.act0 + h.nact, sends[h.hi_nbr][0])
            if h.lo_nbr is not None:
                s.put_planes(which, 0, sends[h.lo_nbr][1])

    with torch.cuda.stream(stream):
        for _ in range(nsteps):
            for s in slabs:
                s.phase(_lib.PHASE_CFL)
            bits = [s.cfl_bits(torch.zeros(1, dtype=torch.int64, device=s._bits.device))
                    for s in slabs]
            m = torch.stack(bits).max(dim=0).values
            for s in slabs:
                s.cfl_bits(m, put=True)
                s.phase(_lib.PHASE_FINALIZE)
                s.phase(_lib.PHASE_STAGE1)
            exchange(1)
            for s in slabs:
                s.phase(_lib.PHASE_STAGE2)
                s.phase(_lib.PHASE_ADVANCE)
            exchange(0)
    slabs[0].ctx.synchronize()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("world,zbc", [(1, "periodic"), (2, "periodic"), (3, "periodic"),
                                       (2, "walls"), (3, "walls")])
def test_slabs_equal_one_grid(vb, world, zbc, precision):
    zb = {"periodic": (P.Periodic, P.Periodic), "walls": (P.Reflecting, P.Outflow)}[zbc]
    dims = (32, 32, 26)
    prob = _problem(dims, zb)
    U0 = P.initial_state(prob)
    nsteps = 4
    ref, t_ref, tot_ref = _single(vb, prob, U0, precision, nsteps)
    slabs = [S.SlabSimulation(prob, precision=precision, initial=U0, world=world, rank=r)
             for r in range(world)]
    if world == 1:
        slabs[0].step(nsteps)  # the exchange of one periodic rank is local
    else:
        _step_emulated(slabs, nsteps)
    nx, ny, nz = dims
    got = np.full((5, nz, ny, nx), np.nan)
    tot = np.zeros(5)
    for s in slabs:
        h = s.halo
        got[:, h.z0:h.z1] = s.own_state().reshape(5, h.nact, ny, nx)
        assert s.time() == (t_ref, nsteps)
        tot += np.array(s.sim_totals())
        s.close()
    assert np.array_equal(got.reshape(ref.shape), ref)
    np.testing.assert_allclose(tot, tot_ref, rtol=1e-13, atol=1e-15 * np.abs(tot_ref).max())


def test_slab_window_refuses_what_it_cannot_do(vb):
    from vespa_b200 import _lib
    prob = _problem((32, 32, 8), (P.Periodic, P.Periodic))
    sim = vb.Simulation(vb.B200Mesh(prob.dims, prob.domain), prob)
    sim.set_kernel("tiled")
    for args in ((0, 9, -1, 0.1), (4, 4, -1, 0.1), (0, 8, 3, 0.1), (0, 8, -1, 0.0)):
        with pytest.raises(vb.VespaB200Error) as e:
            _lib.call("vb_grid_set_zwindow", sim.handle, *args)
        assert e.value.status == _lib.VB_EINVAL
    _lib.call("vb_grid_set_zwindow", sim.handle, 2, 6, -1, 1.0 / 8)
    sim.set_kernel("cell")
    with pytest.raises(vb.VespaB200Error) as e:
        vb.step(sim, 1e-4)
    assert e.value.status == _lib.VB_ENOTSUP
    sim.close()
