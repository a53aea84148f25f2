"""Self-gravity on a device-resident uniform mesh (src/gravity.jl).

``enable_gravity`` attaches a ``GravityField`` to a ``Simulation``: the
potential phi lives on the device with its own boundary conditions (Periodic
wraps; any other BC is a homogeneous Neumann wall), ``solve_poisson`` runs
matrix-free conjugate gradients on A = -lap * V warm-started from the stored
phi, and while the field is attached ``evolve`` solves once per step and every
stage adds the source (+rho g on momentum, +rho v.g on energy) with g = -grad
phi held over the step; ``compute_dt`` takes the free-fall limiter.  All of it
runs in libvespa_b200.so.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import _lib
from .problem import BC, Periodic, _bc_pairs


class GravityField:
    """enable_gravity!'s GravityField (src/gravity.jl:34-49): phi and the
    solver configuration, bound to one Simulation."""

    PRECONDS = {"none": 0, "mg": 1}

    def __init__(self, sim, G: float, bcs, maxiter: int, tol: float, project_mean: bool,
                 precond: str = "none"):
        if precond not in self.PRECONDS:
            raise ValueError("precond must be 'none' or 'mg'")
        self.sim = sim
        self.precond = precond
        self.G = float(G)
        self.bcs = bcs
        self.maxiter = int(maxiter)
        self.tol = float(tol)
        self.project_mean = bool(project_mean)
        desc = _lib.GravityDesc()
        desc.G = self.G
        desc.tol = self.tol
        desc.maxiter = self.maxiter
        for d, (lo, hi) in enumerate(_bc_pairs(bcs, sim.problem.ndim)):
            desc.bc_lo[d] = lo.code
            desc.bc_hi[d] = hi.code
        desc.project_mean = int(self.project_mean)
        desc.precond = self.PRECONDS[precond]
        desc.flags = 0
        _lib.call("vb_gravity_enable", sim.handle, C.byref(desc))

    @property
    def phi(self) -> np.ndarray:
        out = np.empty(self.sim.ncell)
        _lib.call("vb_gravity_phi", self.sim.handle, _lib.dptr(out))
        return out

    @phi.setter
    def phi(self, values) -> None:
        v = np.ascontiguousarray(values, dtype=np.float64).reshape(-1)
        if v.size != self.sim.ncell:
            raise ValueError(f"phi must have {self.sim.ncell} values")
        _lib.call("vb_gravity_set_phi", self.sim.handle, _lib.dptr(v))

    def accel(self) -> np.ndarray:
        """g = -grad phi as the stages use it, shape (ndim, ncell)."""
        out = np.empty((self.sim.problem.ndim, self.sim.ncell))
        _lib.call("vb_gravity_accel", self.sim.handle, _lib.dptr(out))
        return out


def enable_gravity(sim, *, G: float = 1.0, bcs=Periodic, maxiter: int = 500, tol: float = 1e-8,
                   project_mean: Optional[bool] = None, precond: str = "none") -> GravityField:
    """enable_gravity!(sim; G, bcs, maxiter, tol, project_mean, precond)
    (src/gravity.jl:65-83).  project_mean defaults to bcs being Periodic, as in
    the reference; precond is "none" (plain CG) or "mg" (CG preconditioned by
    one multigrid cycle, ext/mg_pcg.jl; 3D cubic periodic grids)."""
    if project_mean is None:
        project_mean = isinstance(bcs, BC) and bcs == Periodic
    grav = GravityField(sim, G, bcs, maxiter, tol, project_mean, precond)
    sim.grav = grav
    return grav


def disable_gravity(sim) -> None:
    _lib.call("vb_gravity_disable", sim.handle)
    sim.grav = None


def solve_poisson(sim, grav: Optional[GravityField] = None) -> tuple:
    """solve_poisson!(sim, grav) -> (iters, relres) (src/gravity.jl:243-249)."""
    if grav is not None and grav.sim is not sim:
        raise ValueError("the GravityField belongs to another Simulation")
    iters = C.c_int64()
    relres = C.c_double()
    _lib.call("vb_gravity_solve", sim.handle, C.byref(iters), C.byref(relres))
    return int(iters.value), float(relres.value)


def apply_laplacian(sim, grav: GravityField, x) -> np.ndarray:
    """A x with A = -lap * V (apply_laplacian!, src/gravity.jl:96-106)."""
    xv = np.ascontiguousarray(x, dtype=np.float64).reshape(-1)
    if xv.size != sim.ncell:
        raise ValueError(f"x must have {sim.ncell} values")
    out = np.empty(sim.ncell)
    _lib.call("vb_gravity_laplacian", sim.handle, _lib.dptr(xv), _lib.dptr(out))
    return out
