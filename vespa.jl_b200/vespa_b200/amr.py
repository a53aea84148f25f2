"""Composite AMR mesh on the device (host side of vb_amr_* in
include/vespa_b200.h).

Mirrors the reference's AMR surface: an adaptive mesh backend
(``HGMesh``, lib/HGBackend/src/HGBackend.jl) bound to a Problem by a
``Simulation``, ``RefinementPolicy`` / ``regrid!`` / ``density_gradient_indicator``
(src/driver.jl:400-462), ``evolve!(sim; policy, subcycle)`` and
``step!(sim, dt; level)`` (src/driver.jl:333-359, 483-605) and
``conserved_totals``.  The mesh topology, its face and neighbour tables and
the regrid bookkeeping live in the C++ library; every step runs on the GPU.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import _lib
from .problem import Problem, initial_state
from .simulation import Totals, problem_desc


@dataclass(frozen=True)
class RefinementPolicy:
    """RefinementPolicy(; refine_above, max_level, every=8) with the density
    gradient indicator (src/driver.jl:422-441); refine-only."""
    refine_above: float
    max_level: int
    every: int = 8


class AmrMesh:
    """Adaptive mesh over a base grid of ``dims`` root cells on ``domain``
    (the HGMesh role).  Any base dims are accepted (a forest of roots)."""

    def __init__(self, dims, domain):
        self.dims = tuple(int(n) for n in dims)
        self.domain = tuple((float(a), float(b)) for a, b in domain)

    def rank(self) -> int:
        return len(self.dims)


class AmrSimulation:
    """Simulation(AmrMesh, problem): float64 state on the composite mesh,
    initial conditions evaluated on the base grid (set_initial_conditions!,
    src/driver.jl:101-112); refinement later prolongs cell means."""

    def __init__(self, backend: AmrMesh, problem: Problem, *, ctx: Optional[_lib.Context] = None):
        if tuple(backend.dims) != tuple(problem.dims):
            raise ValueError("mesh dims do not match the problem")
        self.backend = backend
        self.problem = problem
        self.gamma = problem.gamma
        self.ctx = ctx or _lib.default_context()
        desc = problem_desc(problem)
        for d, (lo, hi) in enumerate(backend.domain):
            desc.lo[d] = lo
            desc.hi[d] = hi
        h = C.c_void_p()
        _lib.call("vb_amr_create", self.ctx.handle, C.byref(desc), C.byref(h))
        self.handle = h
        self.upload(initial_state(problem))

    def close(self):
        if getattr(self, "handle", None):
            _lib.load().vb_amr_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- mesh --
    @property
    def nleaf(self) -> int:
        n = C.c_int64()
        _lib.call("vb_amr_nleaf", self.handle, C.byref(n))
        return n.value

    @property
    def nface(self) -> int:
        n = C.c_int64()
        _lib.call("vb_amr_nface", self.handle, C.byref(n))
        return n.value

    @property
    def max_level(self) -> int:
        m = C.c_int32()
        _lib.call("vb_amr_max_level", self.handle, C.byref(m))
        return m.value

    def leaves(self):
        """(level, coords): level per leaf (0 = base) and integer coordinates
        at that level, in leaf order."""
        n = self.nleaf
        lev = np.empty(n, dtype=np.int32)
        cx = np.empty((n, 3), dtype=np.int64)
        _lib.call("vb_amr_leaves", self.handle, _lib.i32ptr(lev),
                  cx.ctypes.data_as(C.POINTER(C.c_int64)))
        return lev, cx

    def cell_centers(self):
        lev, cx = self.leaves()
        out = []
        for d, (lo, hi) in enumerate(self.backend.domain):
            w = (hi - lo) / self.backend.dims[d] * np.ldexp(1.0, -lev)
            out.append(lo + (cx[:, d] + 0.5) * w)
        return out

    def cell_volumes(self):
        lev, _ = self.leaves()
        v = np.ones(len(lev))
        for d, (lo, hi) in enumerate(self.backend.domain):
            v = v * ((hi - lo) / self.backend.dims[d] * np.ldexp(1.0, -lev))
        return v

    # -- state --
    def upload(self, U: np.ndarray) -> None:
        U = np.ascontiguousarray(U, dtype=np.float64)
        if U.shape != (5, self.nleaf):
            raise ValueError(f"state must have shape (5, {self.nleaf})")
        _lib.call("vb_amr_upload", self.handle, _lib.dptr(U))

    def state(self) -> np.ndarray:
        out = np.empty((5, self.nleaf))
        _lib.call("vb_amr_download", self.handle, _lib.dptr(out))
        return out

    @property
    def t(self) -> float:
        t = C.c_double()
        _lib.call("vb_amr_get_time", self.handle, C.byref(t), None)
        return t.value

    @property
    def step(self) -> int:
        n = C.c_int64()
        _lib.call("vb_amr_get_time", self.handle, None, C.byref(n))
        return n.value

    def set_time(self, t: float, step: int = 0) -> None:
        _lib.call("vb_amr_set_time", self.handle, float(t), int(step))

    def refine(self, leaves) -> None:
        """refine!(backend, leaves): the given leaf indices, with 2:1 balance."""
        idx = np.ascontiguousarray(leaves, dtype=np.int64)
        _lib.call("vb_amr_refine", self.handle, idx.ctypes.data_as(C.POINTER(C.c_int64)), len(idx))

    def indicator(self) -> np.ndarray:
        out = np.empty(self.nleaf)
        _lib.call("vb_amr_indicator", self.handle, _lib.dptr(out))
        return out

    def regrid_ms(self) -> float:
        ms = C.c_double()
        _lib.call("vb_amr_regrid_ms", self.handle, C.byref(ms))
        return ms.value


def density_gradient_indicator(sim: AmrSimulation) -> np.ndarray:
    """max |rho_n - rho_c| / max(rho_c, rho_n, eps) over face neighbours."""
    return sim.indicator()


def regrid(sim: AmrSimulation, policy: RefinementPolicy) -> int:
    """regrid!(sim, policy): returns the number of leaves tagged."""
    n = C.c_int64()
    _lib.call("vb_amr_regrid", sim.handle, float(policy.refine_above), int(policy.max_level),
              C.byref(n))
    return n.value


def compute_dt(sim: AmrSimulation, level: Optional[int] = None) -> float:
    dt = C.c_double()
    _lib.call("vb_amr_compute_dt", sim.handle, -1 if level is None else int(level), C.byref(dt))
    return dt.value


def step(sim: AmrSimulation, dt: float, level: Optional[int] = None) -> AmrSimulation:
    if level is None:
        _lib.call("vb_amr_step", sim.handle, float(dt))
    else:
        _lib.call("vb_amr_step_level", sim.handle, float(dt), int(level))
    return sim


def evolve(sim: AmrSimulation, *, tfinal: Optional[float] = None,
           policy: Optional[RefinementPolicy] = None, subcycle: bool = False,
           max_steps: int = -1) -> AmrSimulation:
    """evolve!(sim; policy, subcycle) to ``tfinal`` (default problem.tfinal)."""
    tf = sim.problem.tfinal if tfinal is None else float(tfinal)
    above, lmax, every = (0.0, 0, 0) if policy is None else (
        float(policy.refine_above), int(policy.max_level), int(policy.every))
    t = C.c_double()
    n = C.c_int64()
    _lib.call("vb_amr_evolve", sim.handle, tf, int(max_steps), above, lmax, every,
              int(bool(subcycle)), C.byref(t), C.byref(n))
    return sim


def conserved_totals(sim: AmrSimulation) -> Totals:
    out = np.empty(5)
    _lib.call("vb_amr_conserved_totals", sim.handle, _lib.dptr(out))
    return Totals(*out)
