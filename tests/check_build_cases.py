"""Small parity cases through the check build (libvespa_b200_check.so:
device bounds checks on), run by tests/test_gpu_check_build.py in a process
of their own, since the library is chosen once per process (VESPA_B200_LIB).
Prints one JSON line: per case, whether the device result equals the oracle
bit for bit, and the bounds-check record after it (0: no check failed)."""
import json
import math
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "vespa.jl_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)

import numpy as np  # noqa: E402

import vespa_b200 as vb  # noqa: E402
from vespa_b200 import amr as A  # noqa: E402
from oracle import oracle as O  # noqa: E402


def uniform(dims, bcs, kernel, precision="fp64", nsteps=3, bflux=False):
    prob = vb.smooth_random_problem(dims, seed=11)
    prob.bcs = bcs
    U0 = vb.initial_state(prob)
    sim = vb.Simulation(vb.B200Mesh(prob.dims, prob.domain), prob, precision=precision,
                        initial=U0)
    sim.set_kernel(kernel)
    if bflux:
        sim.bflux_enable(True)
    g = O.grid_from_problem(prob)
    reg = O.BoundaryFluxRegister(g) if bflux else None
    U = U0.copy()
    for _ in range(nsteps):
        dt = O.compute_dt(g, U)
        vb.step(sim, dt)
        if bflux:
            O.step_breg(g, U, dt, reg)
        else:
            O.step(g, U, dt)
    same = precision == "mixed" or bool(np.array_equal(sim.state(), U))
    if bflux:
        same = same and bool(np.array_equal(sim.bflux_read(), reg.dense()))
    finite = bool(np.isfinite(sim.state()).all())
    sim.close()
    return same and finite


def amr(subcycle):
    prob = vb.sod_problem_defaults(n=64)
    dev = A.AmrSimulation(A.AmrMesh(prob.dims, prob.domain), prob)
    ora = O.Amr(O.grid_from_problem(prob))
    ora.set_state(vb.initial_state(prob))
    A.evolve(dev, policy=A.RefinementPolicy(0.05, 3, 3), subcycle=subcycle)
    ora.evolve(prob.tfinal, refine_above=0.05, max_level=3, every=3, subcycle=subcycle)
    same = bool(np.array_equal(dev.state(), ora.state())) and dev.max_level >= 2
    dev.close()
    return same


def main():
    ctx = vb.default_context()
    first = ctx.check_read()
    P = vb.problem
    walls3 = ((P.Outflow, P.Reflecting), (P.Reflecting, P.Outflow), (P.Periodic, P.Periodic))
    walls2 = ((P.Outflow, P.Reflecting), (P.Reflecting, P.Outflow))
    cases = {
        "cell_3d_walls": lambda: uniform((32, 16, 9), walls3, "cell"),
        "tiled_3d_fp64_walls": lambda: uniform((32, 16, 9), walls3, "tiled"),
        "tiled_3d_mixed_walls": lambda: uniform((32, 16, 9), walls3, "tiled", "mixed"),
        "tiled_3d_fp64_bflux": lambda: uniform((32, 16, 9), walls3, "tiled", bflux=True),
        "tiled_2d_fp64_walls": lambda: uniform((256, 9), walls2, "tiled"),
        "amr_single_rate": lambda: amr(False),
        "amr_subcycled": lambda: amr(True),
    }
    out = {"check_build": first >= 0, "cases": {}}
    for name, fn in cases.items():
        same = fn()
        out["cases"][name] = {"same": same, "check": ctx.check_read()}
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
