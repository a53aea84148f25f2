"""lib/PPMKernels' unsplit MUSCL step on the device (muscl_step_3d!,
lib/PPMKernels/src/muscl_grid.jl:314-380; Enzo HydroMethod=3).

``MusclGrid(dims, ng)`` holds the device state and scratch of one grid of
``dims`` cells (ghost zones included, x fastest); ``muscl_step_3d(D, S1, S2,
S3, Tau, dims, ng; dt, gamma, theta, dx, small_rho, bc)`` mirrors the
reference's call on host arrays (copied to the device, stepped, copied back).
``bc`` is ``None`` (ghost zones left as they are, the reference without a bc!
callback) or ``"periodic"``.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import _lib

BCS = {None: 0, "none": 0, "periodic": 1}


def _params(dt, gamma, theta, dx, small_rho, bc) -> _lib.MusclParams:
    if bc not in BCS:
        raise ValueError("bc must be None or 'periodic'")
    p = _lib.MusclParams()
    p.dt, p.gamma, p.theta, p.dx, p.small_rho = float(dt), float(gamma), float(theta), float(dx), float(small_rho)
    p.bc = BCS[bc]
    p.flags = 0
    return p


class MusclGrid:
    def __init__(self, dims, ng: int = 3, ctx: Optional[_lib.Context] = None):
        self.dims = tuple(int(n) for n in dims)
        if len(self.dims) != 3:
            raise ValueError("muscl_step_3d works on 3-D grids")
        self.ng = int(ng)
        self.N = int(np.prod(self.dims))
        self.ctx = ctx or _lib.default_context()
        d = (C.c_int64 * 3)(*self.dims)
        h = C.c_void_p()
        _lib.call("vb_muscl_create", self.ctx.handle, d, self.ng, C.byref(h))
        self.handle = h

    def close(self):
        if getattr(self, "handle", None):
            _lib.load().vb_muscl_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def upload(self, U) -> None:
        U = np.ascontiguousarray(U, dtype=np.float64)
        if U.shape != (5, self.N):
            raise ValueError(f"state must have shape (5, {self.N}): D, S1, S2, S3, Tau")
        _lib.call("vb_muscl_upload", self.handle, _lib.dptr(U))

    def state(self) -> np.ndarray:
        out = np.empty((5, self.N))
        _lib.call("vb_muscl_download", self.handle, _lib.dptr(out))
        return out

    def device_state_ptr(self) -> int:
        p = C.c_void_p()
        _lib.call("vb_muscl_state", self.handle, C.byref(p))
        return int(p.value)

    def step(self, *, dt, gamma, theta=1.5, dx=1.0, small_rho=1e-10, bc=None) -> None:
        p = _params(dt, gamma, theta, dx, small_rho, bc)
        _lib.call("vb_muscl_step", self.handle, C.byref(p))

    def run_async(self, nsteps, *, dt, gamma, theta=1.5, dx=1.0, small_rho=1e-10, bc=None) -> None:
        p = _params(dt, gamma, theta, dx, small_rho, bc)
        _lib.call("vb_muscl_run_async", self.handle, C.byref(p), int(nsteps))

    def step_fields(self, ptrs, *, dt, gamma, theta=1.5, dx=1.0, small_rho=1e-10, bc=None) -> None:
        """One step of five caller-owned device arrays (addresses D, S1, S2, S3, Tau)."""
        p = _params(dt, gamma, theta, dx, small_rho, bc)
        _lib.call("vb_muscl_step_fields", self.handle, *[C.c_void_p(int(a)) for a in ptrs], C.byref(p))


def muscl_step_3d(D, S1, S2, S3, Tau, dims, ng, *, dt, gamma, theta=1.5, dx=1.0, small_rho=1e-10,
                  bc=None, grid: Optional[MusclGrid] = None):
    """muscl_step_3d!(D, S1, S2, S3, Tau, dims, ng; dt, gamma, theta, dx, small_rho)
    on host float64 arrays, in place."""
    g = grid or MusclGrid(dims, ng)
    g.upload(np.array([np.ravel(D), np.ravel(S1), np.ravel(S2), np.ravel(S3), np.ravel(Tau)]))
    g.step(dt=dt, gamma=gamma, theta=theta, dx=dx, small_rho=small_rho, bc=bc)
    out = g.state()
    for a, row in zip((D, S1, S2, S3, Tau), out):
        a.reshape(-1)[...] = row
    return D, S1, S2, S3, Tau
