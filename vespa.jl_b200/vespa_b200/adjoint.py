"""Adjoint of the float64 hydro step (host side of vb_adjoint_* in
include/vespa_b200.h).

The reference has no adjoint.  This module gives the reverse-mode
derivative of the map evolve! applies (src/driver.jl:483-508) on a periodic
VB_FP64 grid, with each step's dt held at its forward value and every
limiter / Riemann branch held at its forward choice, computed by the CUDA
library: a checkpointed forward run, then a reverse sweep that recomputes
each segment from its checkpoint.

``evolve_with_adjoint`` plays the role of a ChainRulesCore ``rrule`` for
``evolve!``: it returns the final state and a pullback mapping dJ/dU(t_end) to
dJ/dU(t_0).  ``EvolveFunction`` wraps the same pair as a torch.autograd
Function so a torch objective can be differentiated through the device run.
"""
from __future__ import annotations

import ctypes as C
import math
from typing import Callable, Optional

import numpy as np

from . import _lib
from .simulation import Simulation


class Adjoint:
    """Checkpointed adjoint of up to ``max_steps`` steps of ``sim``
    (vb_adjoint_create); a state copy is kept every ``checkpoint_every``
    steps.  ``checkpoint_every=1`` keeps a tape of both states of every step
    in device memory instead, and the reverse sweep recomputes nothing."""

    def __init__(self, sim: Simulation, max_steps: int, checkpoint_every: int = 20):
        self.sim = sim
        self.max_steps = int(max_steps)
        self.checkpoint_every = int(checkpoint_every)
        h = C.c_void_p()
        _lib.call("vb_adjoint_create", sim.handle, self.max_steps, self.checkpoint_every,
                  C.byref(h))
        self.handle = h
        sim._dependents.add(self)

    def close(self):
        if getattr(self, "handle", None):
            _lib.load().vb_adjoint_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def forward(self, *, tfinal: Optional[float] = None, max_steps: int = -1) -> tuple:
        """Advance the simulation (CFL-limited steps, as evolve!) while
        recording checkpoints and dts; returns (t, nsteps)."""
        tf = math.inf if tfinal is None else float(tfinal)
        t = C.c_double()
        n = C.c_int64()
        _lib.call("vb_adjoint_forward", self.handle, tf, int(max_steps), C.byref(t), C.byref(n))
        return t.value, n.value

    @property
    def nsteps(self) -> int:
        n = C.c_int64()
        _lib.call("vb_adjoint_steps", self.handle, C.byref(n))
        return n.value

    def dts(self) -> np.ndarray:
        n = self.nsteps
        out = np.empty(n)
        _lib.call("vb_adjoint_dts", self.handle, _lib.dptr(out), n)
        return out

    def backward(self, lam_final: np.ndarray) -> np.ndarray:
        """dJ/dU(t_0) from dJ/dU(t_end) (both (5, ncell) float64)."""
        lam = np.ascontiguousarray(lam_final, dtype=np.float64)
        if lam.shape != (5, self.sim.ncell):
            raise ValueError(f"adjoint must have shape (5, {self.sim.ncell})")
        out = np.empty_like(lam)
        _lib.call("vb_adjoint_backward", self.handle, _lib.dptr(lam), _lib.dptr(out))
        return out

    def step(self, dt: float, lam_out: np.ndarray) -> np.ndarray:
        """(dU^{n+1}/dU^n)^T lam_out for one step of size dt from the
        simulation's current state (which is left unchanged)."""
        lam = np.ascontiguousarray(lam_out, dtype=np.float64)
        out = np.empty_like(lam)
        _lib.call("vb_adjoint_step", self.handle, float(dt), _lib.dptr(lam), _lib.dptr(out))
        return out

    def timing(self) -> dict:
        """Device milliseconds of the last forward run and of the last
        reverse sweep's recompute and adjoint stages."""
        ms = np.zeros(3)
        _lib.call("vb_adjoint_timing", self.handle, _lib.dptr(ms))
        return {"forward_ms": ms[0], "recompute_ms": ms[1], "adjoint_ms": ms[2]}


def rho2_integral(sim: Simulation, U: Optional[np.ndarray] = None) -> float:
    """J = sum over cells of rho^2 * V (the integral of rho^2)."""
    U = sim.state() if U is None else U
    return float(np.sum(U[0] * U[0]) * sim.backend.cell_volume())


def rho2_seed(sim: Simulation, U: np.ndarray) -> np.ndarray:
    """dJ/dU of rho2_integral: (2 rho V, 0, 0, 0, 0)."""
    lam = np.zeros_like(U)
    lam[0] = 2.0 * U[0] * sim.backend.cell_volume()
    return lam


def evolve_with_adjoint(sim: Simulation, nsteps: int, checkpoint_every: int = 20):
    """rrule-style evolve!: advance ``sim`` by ``nsteps`` CFL-limited steps and
    return (U_end, pullback, adjoint); pullback(dJ/dU_end) -> dJ/dU_start."""
    adj = Adjoint(sim, nsteps, checkpoint_every)
    adj.forward(max_steps=nsteps)
    return sim.state(), adj.backward, adj


try:  # optional torch.autograd bridge
    import torch

    class EvolveFunction(torch.autograd.Function):
        """U_end = evolve(U_0) on the device; backward runs the adjoint.

        ``apply(U0, sim, nsteps, checkpoint_every)`` with U0 a (5, ncell)
        float64 CPU tensor."""

        @staticmethod
        def forward(ctx, U0, sim, nsteps, checkpoint_every=20):
            sim.upload(U0.detach().cpu().numpy())
            sim.set_time(0.0, 0)
            UT, pullback, adj = evolve_with_adjoint(sim, int(nsteps), int(checkpoint_every))
            ctx.pullback = pullback
            ctx.adj = adj
            return torch.from_numpy(UT)

        @staticmethod
        def backward(ctx, grad_out):
            lam0 = ctx.pullback(grad_out.detach().cpu().numpy().astype(np.float64))
            return torch.from_numpy(lam0), None, None, None

except ImportError:  # pragma: no cover
    EvolveFunction = None
