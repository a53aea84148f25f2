"""Problem specifications and initial conditions (host side).

Mirrors ``Problem`` (src/problem.jl:20-50), ``sod_problem_defaults``
(src/problem.jl:61-71), ``sedov_problem`` (problems/sedov_blast.jl:24-45) and
``set_initial_conditions!`` (src/driver.jl:101-112), plus the seeded synthetic
workloads the benchmarks and parity tests use.  Initial conditions are
evaluated with numpy in the reference's operation order, so the conserved
state handed to the device is bit-identical to the reference's.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Callable, Optional, Sequence

import numpy as np

from ._lib import BC_OUTFLOW, BC_PERIODIC, BC_REFLECTING


@dataclass(frozen=True)
class BC:
    """A boundary condition (lib/MeshInterface/src/MeshInterface.jl:74-83)."""
    name: str
    code: int

    def __repr__(self):
        return f"{self.name}()"


Outflow = BC("Outflow", BC_OUTFLOW)
Periodic = BC("Periodic", BC_PERIODIC)
Reflecting = BC("Reflecting", BC_REFLECTING)


@dataclass(frozen=True)
class IdealHydro:
    """IdealHydro(γ) equation set (src/equationset.jl:31-60)."""
    gamma: float
    nvars: int = 5
    conserved_names: tuple = ("density", "momentum_x", "momentum_y", "momentum_z", "total_energy")
    density_index: int = 1
    momentum_indices: tuple = (2, 3, 4)
    energy_index: int = 5

    def adiabatic_index(self) -> float:
        return self.gamma


def _bc_pairs(bcs, ndim):
    if isinstance(bcs, BC):
        return tuple((bcs, bcs) for _ in range(ndim))
    pairs = tuple(tuple(p) for p in bcs)
    if len(pairs) != ndim or any(len(p) != 2 for p in pairs):
        raise ValueError("bcs must be one BC or a (lo, hi) pair per axis")
    return pairs


@dataclass
class Problem:
    """Self-contained hydro problem (src/problem.jl:20-50).

    ``init(x, y, z)`` receives numpy arrays of cell-centre coordinates (padded
    with zeros to rank 3) and returns the primitive tuple
    ``(rho, vx, vy, vz, p)`` as arrays or scalars.  Generators whose state is
    defined per cell instead of per coordinate set ``init_prim(problem)``,
    returning a ``(5, ncell)`` primitive array in column-major cell order.
    """
    name: str
    dims: tuple
    domain: tuple
    gamma: float
    bcs: object
    init: Optional[Callable] = None
    tfinal: float = math.inf
    cfl: float = 0.4
    init_prim: Optional[Callable] = None
    meta: dict = field(default_factory=dict)

    def __post_init__(self):
        self.dims = tuple(int(n) for n in self.dims)
        self.domain = tuple((float(a), float(b)) for a, b in self.domain)
        self.gamma = float(self.gamma)
        self.tfinal = float(self.tfinal)
        self.cfl = float(self.cfl)
        # validation as in src/problem.jl:39-46
        if not self.gamma > 1:
            raise ValueError(f"γ must exceed 1 (got {self.gamma})")
        if not self.tfinal > 0:
            raise ValueError(f"tfinal must be positive (got {self.tfinal})")
        if not (0 < self.cfl <= 1):
            raise ValueError(f"cfl must be in (0, 1] (got {self.cfl})")
        if not all(n > 0 for n in self.dims):
            raise ValueError("all dims must be positive")
        if len(self.domain) != len(self.dims):
            raise ValueError("domain needs one (lo, hi) pair per axis")
        for d, (a, b) in enumerate(self.domain):
            if not b > a:
                raise ValueError(f"domain[{d + 1}] must have hi > lo (got {(a, b)})")
        _bc_pairs(self.bcs, self.ndim)
        if self.init is None and self.init_prim is None:
            raise ValueError("a problem needs init or init_prim")

    @property
    def ndim(self) -> int:
        return len(self.dims)

    @property
    def ncell(self) -> int:
        return int(np.prod(self.dims))

    def bc_pairs(self):
        """Per-axis (lo, hi) boundary codes."""
        return tuple((lo.code, hi.code) for lo, hi in _bc_pairs(self.bcs, self.ndim))

    def cell_width(self):
        # _width, lib/RefMesh/src/RefMesh.jl:122-123
        return tuple((b - a) / n for (a, b), n in zip(self.domain, self.dims))

    def cell_volume(self) -> float:
        w = self.cell_width()
        v = w[0]
        for x in w[1:]:
            v = v * x
        return v

    def cell_centers(self):
        """Cell-centre coordinate arrays (ncell each, column-major, x fastest).

        cell_center, lib/RefMesh/src/RefMesh.jl:129-132: lo + (I - 0.5) * w."""
        w = self.cell_width()
        axes = [self.domain[d][0] + ((np.arange(self.dims[d], dtype=np.float64) + 1.0) - 0.5) * w[d]
                for d in range(self.ndim)]
        grids = np.meshgrid(*axes, indexing="ij")
        return [g.reshape(-1, order="F") for g in grids]


def prim2cons(W: np.ndarray, gamma: float) -> np.ndarray:
    """Vectorised prim2cons (src/eos.jl:28-32), reference operation order."""
    rho, vx, vy, vz, p = W
    E = p / (gamma - 1.0) + 0.5 * rho * (vx * vx + vy * vy + vz * vz)
    return np.stack([rho, rho * vx, rho * vy, rho * vz, E])


def cons2prim(U: np.ndarray, gamma: float) -> np.ndarray:
    """Vectorised cons2prim (src/eos.jl:8-25), reference operation order."""
    rho = U[0]
    inv = 1.0 / rho
    vx, vy, vz = U[1] * inv, U[2] * inv, U[3] * inv
    kinetic = 0.5 * rho * (vx * vx + vy * vy + vz * vz)
    p = (gamma - 1.0) * (U[4] - kinetic)
    return np.stack([rho, vx, vy, vz, np.maximum(p, 1e-12 * kinetic)])


def initial_primitive(prob: Problem) -> np.ndarray:
    if prob.init_prim is not None:
        W = np.asarray(prob.init_prim(prob), dtype=np.float64)
        if W.shape != (5, prob.ncell):
            raise ValueError(f"init_prim must return shape (5, {prob.ncell})")
        return W
    c = prob.cell_centers()
    while len(c) < 3:
        c.append(np.zeros(prob.ncell))
    out = prob.init(*c)
    return np.stack([np.broadcast_to(np.asarray(v, dtype=np.float64), (prob.ncell,)) for v in out])


def initial_state(prob: Problem) -> np.ndarray:
    """set_initial_conditions! (src/driver.jl:101-112): (5, ncell) conserved state."""
    return np.ascontiguousarray(prim2cons(initial_primitive(prob), prob.gamma))


# --------------------------------------------------------------- seeded PRNG
# splitmix64 on (seed, stream, index) -> uniform double in [0, 1).  One counter
# per (stream, cell) so any subset of cells can be regenerated independently.
_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_STREAM = np.uint64(0xD1B54A32D192ED03)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def uniform01(seed: int, stream: int, index) -> np.ndarray:
    idx = np.asarray(index, dtype=np.uint64)
    with np.errstate(over="ignore"):
        x = np.uint64(seed & 0xFFFFFFFFFFFFFFFF) + np.uint64(stream) * _STREAM + (idx + np.uint64(1)) * _GOLDEN
        z = x
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


DEFAULT_SEED = 20261203


# ------------------------------------------------------------- the problems
def sod_problem_defaults(n: int = 128, cfl: float = 0.4) -> Problem:
    """The Sod shock tube (src/problem.jl:61-71)."""
    def init(x, y, z):
        left = x < 0.5
        return (np.where(left, 1.0, 0.125), 0.0, 0.0, 0.0, np.where(left, 1.0, 0.1))
    return Problem(name="SodShockTube", dims=(int(n),), domain=((0.0, 1.0),), gamma=1.4,
                   bcs=Outflow, init=init, tfinal=0.2, cfl=cfl)


def sedov_problem(n: int = 64, E0: float = 1.0, rho0: float = 1.0, p0: float = 1e-5,
                  gamma: float = 1.4, r0: Optional[float] = None, tfinal: float = 0.05) -> Problem:
    """2D Sedov blast on [0,1]^2 (problems/sedov_blast.jl:24-45)."""
    dx = 1.0 / n
    rhot = 2.0 * dx if r0 is None else float(r0)
    area = math.pi * rhot ** 2
    p_hot = (gamma - 1) * E0 / area

    def init(x, y, z):
        r = np.hypot(x - 0.5, y - 0.5)
        return (float(rho0), 0.0, 0.0, 0.0, np.where(r <= rhot, p_hot, float(p0)))
    return Problem(name="Sedov2D", dims=(int(n), int(n)), domain=((0.0, 1.0), (0.0, 1.0)),
                   gamma=float(gamma), bcs=Reflecting, init=init, tfinal=float(tfinal), cfl=0.3)


def smooth_random_problem(dims: Sequence[int], seed: int = DEFAULT_SEED, gamma: float = 5.0 / 3.0,
                          cfl: float = 0.4, tfinal: float = math.inf) -> Problem:
    """Seeded smooth random periodic state on [0,1]^d.

    rho = 1 + 0.3 * (1/8) * sum_m sin(2 pi k_m . x + phi_m) with integer
    k_m in [-4,4]^d minus 0 and phi_m in [0, 2 pi); each velocity component
    uniform in [-0.5, 0.5] per cell on the active axes (0 on the others);
    p = 1 + 0.2 * uniform[-1, 1] per cell."""
    dims = tuple(int(n) for n in dims)
    nd = len(dims)

    def modes():
        ks, phis = [], []
        ctr = 0
        while len(ks) < 8:
            u = uniform01(seed, 0, np.arange(ctr, ctr + nd + 1))
            ctr += nd + 1
            k = tuple(int(math.floor(v * 9.0)) - 4 for v in u[:nd])
            if all(c == 0 for c in k):
                continue
            ks.append(k)
            phis.append(2.0 * math.pi * float(u[nd]))
        return ks, phis

    def init_prim(prob):
        n = prob.ncell
        xs = prob.cell_centers()
        ks, phis = modes()
        s = np.zeros(n)
        for k, phi in zip(ks, phis):
            arg = np.zeros(n)
            for d in range(nd):
                if k[d]:
                    arg += float(k[d]) * xs[d]
            s += np.sin(2.0 * math.pi * arg + phi)
        del xs
        W = np.empty((5, n))
        W[0] = 1.0 + 0.3 * (s / 8.0)
        idx = np.arange(n, dtype=np.uint64)
        for d in range(3):
            W[1 + d] = uniform01(seed, 1 + d, idx) - 0.5 if d < nd else 0.0
        W[4] = 1.0 + 0.2 * (2.0 * uniform01(seed, 4, idx) - 1.0)
        return W
    return Problem(name=f"SmoothRandom{nd}D", dims=dims, domain=tuple((0.0, 1.0) for _ in dims),
                   gamma=gamma, bcs=Periodic, init_prim=init_prim, tfinal=tfinal, cfl=cfl,
                   meta={"seed": seed})


def kelvin_helmholtz_problem(n: int = 512, seed: int = DEFAULT_SEED, tfinal: float = math.inf,
                             cfl: float = 0.4, texture: float = 0.0) -> Problem:
    """2D Kelvin-Helmholtz: rho=2, u_x=+0.5 in |y-0.5|<0.25, else rho=1,
    u_x=-0.5; p=2.5; u_y = 0.01 sin(4 pi x) + 1e-3 * uniform[-1,1]; periodic.

    ``texture`` > 0 multiplies rho and p by (1 + texture*uniform[-1,1]) and
    adds texture*uniform[-1,1] to u_x, cell by cell (seeded).  Without it the
    bands are exactly uniform in rho, u_x and p, so the minmod limiter sits on
    its kinks there and the step map has no derivative at that state; a
    texture makes the state generic for finite-difference checks."""
    def init_prim(prob):
        x, y = prob.cell_centers()
        band = np.abs(y - 0.5) < 0.25
        W = np.empty((5, prob.ncell))
        W[0] = np.where(band, 2.0, 1.0)
        W[1] = np.where(band, 0.5, -0.5)
        cells = np.arange(prob.ncell, dtype=np.uint64)
        noise = 2.0 * uniform01(seed, 7, cells) - 1.0
        W[2] = 0.01 * np.sin(4.0 * math.pi * x) + 1e-3 * noise
        W[3] = 0.0
        W[4] = 2.5
        if texture > 0.0:
            W[0] = W[0] * (1.0 + texture * (2.0 * uniform01(seed, 8, cells) - 1.0))
            W[1] = W[1] + texture * (2.0 * uniform01(seed, 9, cells) - 1.0)
            W[4] = W[4] * (1.0 + texture * (2.0 * uniform01(seed, 10, cells) - 1.0))
        return W
    return Problem(name="KelvinHelmholtz2D", dims=(n, n), domain=((0.0, 1.0), (0.0, 1.0)),
                   gamma=1.4, bcs=Periodic, init_prim=init_prim, tfinal=tfinal, cfl=cfl,
                   meta={"seed": seed, "texture": texture})


BOX_SIDES = (32, 48, 64, 96, 128, 192, 256)


def riemann_box_problem(index: int, seed: int = DEFAULT_SEED, sides=BOX_SIDES,
                        side: Optional[int] = None, cfl: float = 0.4) -> Problem:
    """One of the batched 3D Riemann-problem boxes: a cube on [0,1]^3 whose
    side is drawn from `sides`, split by a random plane into two states with
    rho in [0.1, 10], |u| <= 2, p in [0.01, 10]; gamma = 1.4; outflow."""
    u = uniform01(seed, 100 + index, np.arange(16))
    n = int(side) if side is not None else int(sides[min(int(u[0] * len(sides)), len(sides) - 1)])
    normal = np.array([2.0 * u[1] - 1.0, 2.0 * u[2] - 1.0, 2.0 * u[3] - 1.0])
    nn = float(np.linalg.norm(normal))
    normal = normal / nn if nn > 1e-6 else np.array([1.0, 0.0, 0.0])
    point = 0.5 + 0.2 * (2.0 * u[4:7] - 1.0)
    states = []
    for s in range(2):
        v = uniform01(seed, 200 + 2 * index + s, np.arange(6))
        rho = 0.1 + 9.9 * v[0]
        d = np.array([2.0 * v[1] - 1.0, 2.0 * v[2] - 1.0, 2.0 * v[3] - 1.0])
        dn = float(np.linalg.norm(d))
        d = d / dn if dn > 1e-6 else np.zeros(3)
        vel = 2.0 * v[4] * d
        p = 0.01 + 9.99 * v[5]
        states.append((rho, vel[0], vel[1], vel[2], p))
    off = float(np.dot(normal, point))

    def init(x, y, z):
        left = (normal[0] * x + normal[1] * y + normal[2] * z) < off
        return tuple(np.where(left, states[0][k], states[1][k]) for k in range(5))
    return Problem(name=f"RiemannBox{index}", dims=(n, n, n),
                   domain=((0.0, 1.0), (0.0, 1.0), (0.0, 1.0)), gamma=1.4, bcs=Outflow,
                   init=init, cfl=cfl, meta={"seed": seed, "index": index})
