"""Generate the golden fixtures under tests/golden/ from the CPU oracle.

The reference (Julia) cannot run in this container, so the fixtures are the
oracle's outputs on small seeded cases.  The oracle itself is pinned by the
reference's known-answer tests and by an independent Python restatement
(tests/test_oracle.py); the fixtures freeze those outputs so that drift in
either the oracle or the CUDA path shows up against a committed file.

Run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "vespa.jl_b200")]

from oracle import oracle as O  # noqa: E402
from vespa_b200 import problem as P  # noqa: E402


def random_faces(nf: int, seed: int):
    """Face batch covering every HLLC branch: supersonic left/right, both star
    sides, strong jumps, all three axes."""
    rng = np.random.default_rng(seed)
    WL = np.empty((nf, 5))
    WR = np.empty((nf, 5))
    for W in (WL, WR):
        W[:, 0] = np.exp(rng.uniform(np.log(0.05), np.log(20.0), nf))
        W[:, 1:4] = rng.uniform(-3.0, 3.0, (nf, 3))
        W[:, 4] = np.exp(rng.uniform(np.log(0.01), np.log(10.0), nf))
    # a slice of strongly supersonic faces in both directions
    q = nf // 8
    WL[:q, 1:4] += 20.0
    WR[:q, 1:4] += 20.0
    WL[q:2 * q, 1:4] -= 20.0
    WR[q:2 * q, 1:4] -= 20.0
    axis = rng.integers(1, 4, nf).astype(np.int32)
    return WL, WR, axis


def cases():
    """(name, problem, steps) for the stepped fixtures."""
    out = []
    out.append(("sod64", P.sod_problem_defaults(64), 12))
    out.append(("smooth2d_periodic", P.smooth_random_problem((16, 12), seed=11), 5))
    out.append(("smooth3d_periodic", P.smooth_random_problem((8, 6, 5), seed=12), 3))
    p = P.smooth_random_problem((10, 9), seed=13)
    p.bcs = ((P.Outflow, P.Reflecting), (P.Reflecting, P.Outflow))
    out.append(("mixedbc2d", p, 4))
    p = P.smooth_random_problem((6, 5, 4), seed=14)
    p.bcs = ((P.Reflecting, P.Reflecting), (P.Periodic, P.Periodic), (P.Outflow, P.Outflow))
    out.append(("mixedbc3d", p, 3))
    out.append(("sedov16", P.sedov_problem(16, tfinal=0.02), 6))
    return out


def main():
    O.build()
    WL, WR, axis = random_faces(1024, seed=7)
    F = O.compute_face_fluxes(WL, WR, axis, 1.4)
    np.savez_compressed(os.path.join(HERE, "hllc_faces.npz"), WL=WL, WR=WR, axis=axis, F=F,
                        gamma=np.float64(1.4))
    for name, prob, nsteps in cases():
        U0 = P.initial_state(prob)
        g = O.grid_from_problem(prob)
        U = U0.copy()
        dts = []
        for _ in range(nsteps):
            dt = O.compute_dt(g, U)
            O.step(g, U, dt)
            dts.append(dt)
        lo = [b[0] for b in prob.bc_pairs()]
        hi = [b[1] for b in prob.bc_pairs()]
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), U0=U0, U=U, dts=np.array(dts),
                            dims=np.array(prob.dims), domain=np.array(prob.domain),
                            bc_lo=np.array(lo), bc_hi=np.array(hi), gamma=np.float64(prob.gamma),
                            cfl=np.float64(prob.cfl), nsteps=np.int64(nsteps))
        print(name, prob.dims, nsteps, "steps, final dt", dts[-1])


if __name__ == "__main__":
    main()
