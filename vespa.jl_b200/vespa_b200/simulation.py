"""Device-resident Simulation API (host side of the drop-in).

Mirrors the reference's driver API on a device-resident uniform mesh:
``Simulation`` (src/driver.jl:27-79), ``step!`` (333-359), ``compute_dt``
(169-199), ``evolve!`` (483-508), ``conserved_totals``
(src/diagnostics.jl:16-31), ``primitive_at`` / ``cell_samples`` /
``dump_fields`` (diagnostics.jl:9-67).  Every call goes through the C ABI of
libvespa_b200.so; the state never leaves the GPU unless the caller reads it.
"""
from __future__ import annotations

import ctypes as C
import weakref
import math
from collections import namedtuple
from typing import Callable, Optional

import numpy as np

from . import _lib
from .problem import IdealHydro, Problem, cons2prim, initial_state

Totals = namedtuple("Totals", "mass momentum_x momentum_y momentum_z energy")

PRECISIONS = {"fp64": _lib.FP64, "mixed": _lib.MIXED}


class B200Mesh:
    """A uniform mesh whose fields live in B200 device memory.

    The device analogue of ``UniformMesh(dims, domain)``
    (lib/RefMesh/src/RefMesh.jl:89-100): same geometry, same column-major
    cell order, same boundary resolution."""

    def __init__(self, dims, domain):
        self.dims = tuple(int(n) for n in dims)
        self.domain = tuple((float(a), float(b)) for a, b in domain)
        if len(self.dims) != len(self.domain) or not 1 <= len(self.dims) <= 3:
            raise ValueError("B200Mesh supports rank 1-3 with one (lo, hi) pair per axis")

    def rank(self) -> int:
        return len(self.dims)

    def n_cells(self) -> int:
        return int(np.prod(self.dims))

    def cell_width(self):
        return tuple((b - a) / n for (a, b), n in zip(self.domain, self.dims))

    def cell_volume(self) -> float:
        w = self.cell_width()
        v = w[0]
        for x in w[1:]:
            v = v * x
        return v


def problem_desc(problem: Problem) -> _lib.ProblemDesc:
    """vb_problem_desc of a Problem on a uniform mesh."""
    desc = _lib.ProblemDesc()
    desc.ndim = problem.ndim
    for d, ((lo, hi), (blo, bhi)) in enumerate(zip(problem.domain, problem.bc_pairs())):
        desc.dims[d] = problem.dims[d]
        desc.lo[d] = lo
        desc.hi[d] = hi
        desc.bc_lo[d] = blo
        desc.bc_hi[d] = bhi
    desc.gamma = problem.gamma
    desc.cfl = problem.cfl
    desc.aexp = 1.0
    desc.flags = 0
    return desc


class Batch:
    """Many independent 3D problems stepped together on one GPU.

    One persistent kernel launch per RK2 stage covers every box's column
    tiles; each box keeps its own clock and CFL dt; runs of steps replay a
    CUDA graph.  Each problem needs nx, ny multiples of 16 and nz >= 2."""

    def __init__(self, problems, *, precision: str = "fp64", ctx: Optional[_lib.Context] = None,
                 initial=None):
        self.problems = list(problems)
        self.ctx = ctx or _lib.default_context()
        descs = (_lib.ProblemDesc * len(self.problems))(*[problem_desc(p) for p in self.problems])
        h = C.c_void_p()
        _lib.call("vb_batch_create", self.ctx.handle, len(self.problems), descs,
                  PRECISIONS[precision], C.byref(h))
        self.handle = h
        self.precision = precision
        for i, p in enumerate(self.problems):
            U = initial[i] if initial is not None else initial_state(p)
            self.upload(i, U)

    def close(self):
        if getattr(self, "handle", None):
            _lib.load().vb_batch_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __len__(self):
        return len(self.problems)

    def ncell(self, box: int = -1) -> int:
        n = C.c_int64()
        _lib.call("vb_batch_ncell", self.handle, int(box), C.byref(n))
        return n.value

    def upload(self, box: int, U) -> None:
        U = np.ascontiguousarray(U, dtype=np.float64)
        if U.shape != (5, self.ncell(box)):
            raise ValueError("state shape does not match the box")
        _lib.call("vb_batch_upload", self.handle, int(box), _lib.dptr(U))

    def state(self, box: int, out: Optional[np.ndarray] = None) -> np.ndarray:
        if out is None:
            out = np.empty((5, self.ncell(box)))
        _lib.call("vb_batch_download", self.handle, int(box), _lib.dptr(out))
        return out

    def run_steps(self, nsteps: int) -> None:
        _lib.call("vb_batch_run_steps", self.handle, int(nsteps))

    def run_steps_async(self, nsteps: int) -> None:
        _lib.call("vb_batch_run_steps_async", self.handle, int(nsteps))

    def autotune(self, nsteps: int = 3) -> tuple:
        """Pick the work items' depth (vb_batch_autotune): returns (cap, ms per
        step); cap 0 = each box's default chunk, else the cap on every box's
        z chunk.  States and clocks are restored."""
        cap, ms = C.c_int64(), C.c_double()
        _lib.call("vb_batch_autotune", self.handle, int(nsteps), C.byref(cap), C.byref(ms))
        return cap.value, ms.value

    def time(self, box: int) -> tuple:
        t, n = C.c_double(), C.c_int64()
        _lib.call("vb_batch_get_time", self.handle, int(box), C.byref(t), C.byref(n))
        return t.value, n.value

    def conserved_totals(self, box: int) -> Totals:
        out = np.empty(5)
        _lib.call("vb_batch_conserved_totals", self.handle, int(box), _lib.dptr(out))
        return Totals(*[float(v) for v in out])


class Simulation:
    """Bind a Problem to a B200Mesh, allocate the device state and set the
    initial conditions (src/driver.jl:62-79).

    ``precision`` is ``"fp64"`` (bit-identical to the reference's float64
    arithmetic) or ``"mixed"`` (float32 reconstruction and HLLC, float64 state,
    pressure recovery, accumulation and reductions)."""

    def __init__(self, backend: B200Mesh, problem: Problem, *, precision: str = "fp64",
                 ctx: Optional[_lib.Context] = None, initial: Optional[np.ndarray] = None):
        if tuple(backend.dims) != tuple(problem.dims):
            raise ValueError("mesh dims do not match the problem")
        self.backend = backend
        self.problem = problem
        self.model = IdealHydro(problem.gamma)
        self.gamma = problem.gamma
        self.precision = precision
        self.ctx = ctx or _lib.default_context()
        desc = problem_desc(problem)
        for d, (lo, hi) in enumerate(backend.domain):
            desc.lo[d] = lo
            desc.hi[d] = hi
        h = C.c_void_p()
        _lib.call("vb_grid_create", self.ctx.handle, C.byref(desc), PRECISIONS[precision],
                  C.byref(h))
        self.handle = h
        self._dependents = weakref.WeakSet()  # adjoints bound to this grid
        self.grav = None  # GravityField while self-gravity is enabled (gravity.py)
        self.ncell = backend.n_cells()
        U = initial if initial is not None else initial_state(problem)
        self.upload(U)

    # -- lifetime --
    def close(self):
        for dep in list(getattr(self, "_dependents", ())):
            dep.close()
        if getattr(self, "handle", None):
            _lib.load().vb_grid_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- state I/O (the `sv` views) --
    def upload(self, U: np.ndarray) -> None:
        U = np.ascontiguousarray(U, dtype=np.float64)
        if U.shape != (5, self.ncell):
            raise ValueError(f"state must have shape (5, {self.ncell})")
        _lib.call("vb_grid_upload", self.handle, _lib.dptr(U))

    def state(self, out: Optional[np.ndarray] = None) -> np.ndarray:
        if out is None:
            out = np.empty((5, self.ncell))
        _lib.call("vb_grid_download", self.handle, _lib.dptr(out))
        return out

    def device_state_ptr(self) -> int:
        p = C.c_void_p()
        _lib.call("vb_grid_device_state", self.handle, C.byref(p))
        return p.value

    # -- clock --
    @property
    def t(self) -> float:
        t = C.c_double()
        _lib.call("vb_grid_get_time", self.handle, C.byref(t), None)
        return t.value

    @property
    def step(self) -> int:
        n = C.c_int64()
        _lib.call("vb_grid_get_time", self.handle, None, C.byref(n))
        return n.value

    def set_time(self, t: float, step: int = 0) -> None:
        _lib.call("vb_grid_set_time", self.handle, float(t), int(step))

    # -- kernel selection / tuning (results do not depend on these) --
    def set_kernel(self, kind: str = "auto", kz: Optional[int] = None,
                   taper: Optional[bool] = None) -> None:
        """kind: "auto", "cell" (cell-centric kernel) or "tiled" (tiled 3D kernel).
        kz: z planes per tiled work item.  taper: tapered (True) or uniform
        (False) z chunks in the 3D work queue; None restores the default
        (tapered for VB_MIXED grids)."""
        _lib.call("vb_grid_set_option", self.handle, _lib.OPT_KERNEL, _lib.KERNELS[kind])
        if kz is not None:
            _lib.call("vb_grid_set_option", self.handle, _lib.OPT_TILE_KZ, int(kz))
        _lib.call("vb_grid_set_option", self.handle, _lib.OPT_TILE_TAPER,
                  -1 if taper is None else int(bool(taper)))

    @property
    def taper(self) -> bool:
        v = C.c_int64()
        _lib.call("vb_grid_get_option", self.handle, _lib.OPT_TILE_TAPER, C.byref(v))
        return bool(v.value)

    def autotune(self, nsteps: int = 3) -> tuple:
        """Pick the fastest z-chunk for the tiled kernel on this grid (state and
        clock are restored).  Returns (kz, ms_per_step)."""
        kz, ms = C.c_int64(), C.c_double()
        _lib.call("vb_grid_autotune", self.handle, int(nsteps), C.byref(kz), C.byref(ms))
        return kz.value, ms.value

    @property
    def kz(self) -> int:
        v = C.c_int64()
        _lib.call("vb_grid_get_option", self.handle, _lib.OPT_TILE_KZ, C.byref(v))
        return v.value

    @property
    def kernel(self) -> str:
        v = C.c_int64()
        _lib.call("vb_grid_get_option", self.handle, _lib.OPT_KERNEL, C.byref(v))
        return {1: "cell", 2: "tiled"}[v.value]

    def profile_step(self, nsteps: int = 5) -> dict:
        """Mean device milliseconds of each kernel of a CFL step (advances the state)."""
        fin, s1, s2 = C.c_double(), C.c_double(), C.c_double()
        _lib.call("vb_grid_profile_step", self.handle, int(nsteps), C.byref(fin), C.byref(s1),
                  C.byref(s2))
        return {"ms_finalize": fin.value, "ms_stage1": s1.value, "ms_stage2": s2.value}

    # -- boundary-flux register --
    def bflux_enable(self, on=True) -> None:
        """on: False / True (outer faces) or "interior" (outer and interior faces,
        BoundaryFluxRegister(record_interior = true))."""
        mode = _lib.BFLUX_INTERIOR if on == "interior" else (_lib.BFLUX_OUTER if on else _lib.BFLUX_OFF)
        _lib.call("vb_bflux_enable", self.handle, mode)

    def bflux_plane(self, dim: int, source: str, start, stop, g0, flux_off: int, comp: int,
                    vcell: float) -> np.ndarray:
        """bflux_plane (src/reflux.jl:171-191) on the device: `source` "lo", "hi"
        or "interior" picks the register keys the reference's lookup reads."""
        R = len(start)
        st = np.ascontiguousarray(start, dtype=np.int64)
        sp = np.ascontiguousarray(stop, dtype=np.int64)
        g0a = np.ascontiguousarray(g0, dtype=np.int64)
        n = int(np.prod(sp - st + 1)) if R else 0
        out = np.empty(n)
        src = {"lo": _lib.BFLUX_PLANE_LO, "hi": _lib.BFLUX_PLANE_HI,
               "interior": _lib.BFLUX_PLANE_INTERIOR}[source]
        _lib.call("vb_bflux_plane", self.handle, int(dim), src, _lib.i64ptr(st), _lib.i64ptr(sp),
                  _lib.i64ptr(g0a), int(flux_off), int(comp), float(vcell), _lib.dptr(out), n)
        return out

    def bflux_clear(self) -> None:
        _lib.call("vb_bflux_clear", self.handle)

    def bflux_read(self) -> np.ndarray:
        n = C.c_int64()
        _lib.call("vb_bflux_size", self.handle, C.byref(n))
        out = np.empty(n.value)
        _lib.call("vb_bflux_read", self.handle, _lib.dptr(out), n.value)
        return out


def compute_dt(sim: Simulation) -> float:
    """compute_dt(sim) (src/driver.jl:169-199)."""
    dt = C.c_double()
    _lib.call("vb_compute_dt", sim.handle, C.byref(dt))
    return dt.value


def step(sim: Simulation, dt: float) -> Simulation:
    """step!(sim, dt) (src/driver.jl:333-359): one SSP-RK2 step."""
    _lib.call("vb_step", sim.handle, float(dt))
    return sim


def evolve(sim: Simulation, *, tfinal: Optional[float] = None, max_steps: int = -1,
           callback: Optional[Callable] = None, callback_every: int = 1) -> Simulation:
    """evolve!(sim) (src/driver.jl:483-508): integrate to problem.tfinal.

    The dt loop runs on the device.  ``callback(sim, stage)`` is called with
    ``"init"`` before the first step and ``"step"`` after every
    ``callback_every`` steps, as in the reference."""
    tf = sim.problem.tfinal if tfinal is None else float(tfinal)
    t = C.c_double()
    n = C.c_int64()
    if callback is None:
        _lib.call("vb_evolve", sim.handle, tf, int(max_steps), C.byref(t), C.byref(n))
        return sim
    callback(sim, "init")
    done = 0
    every = max(1, int(callback_every))
    while max_steps < 0 or done < max_steps:
        chunk = every if max_steps < 0 else min(every, max_steps - done)
        _lib.call("vb_evolve", sim.handle, tf, chunk, C.byref(t), C.byref(n))
        done += n.value
        if n.value == 0:
            break
        if n.value == chunk and callback_every > 0:
            callback(sim, "step")
        if n.value < chunk:
            break
    return sim


def run_steps_async(sim: Simulation, nsteps: int) -> None:
    """Queue `nsteps` CFL-limited RK2 steps on the context stream (no final time)."""
    _lib.call("vb_run_steps_async", sim.handle, int(nsteps))


def conserved_totals(sim: Simulation) -> Totals:
    """conserved_totals(sim) (src/diagnostics.jl:16-31)."""
    out = np.empty(5)
    _lib.call("vb_conserved_totals", sim.handle, _lib.dptr(out))
    return Totals(*[float(v) for v in out])


def primitive_state(sim: Simulation) -> np.ndarray:
    return cons2prim(sim.state(), sim.gamma)


def primitive_at(sim: Simulation, cell: int) -> tuple:
    """primitive_at(sim, cell) (src/diagnostics.jl:9)."""
    return tuple(float(v) for v in primitive_state(sim)[:, int(cell)])


def cell_samples(sim: Simulation):
    """cell_samples(sim) (src/diagnostics.jl:40-48): (centres, primitives)."""
    return sim.problem.cell_centers(), primitive_state(sim)


def dump_fields(sim: Simulation) -> dict:
    """dump_fields(sim) (src/diagnostics.jl:57-67), 1D only."""
    if sim.backend.rank() != 1:
        raise ValueError("dump_fields currently supports 1D; use cell_samples for ND")
    (x,), W = cell_samples(sim)
    return {"x": x, "density": W[0], "velocity_x": W[1], "pressure": W[4]}
