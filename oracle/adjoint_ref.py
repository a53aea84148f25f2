"""Reference gradient of the float64 SSP-RK2 hydro step: a PyTorch float64
restatement of the step on periodic meshes, differentiated by autograd.

TEST INFRASTRUCTURE ONLY: imported by tests/ and by ``bench.py``'s checks; the
product package never imports it.

The reference has no adjoint, so there is no reference gradient to compare
with.  This module restates the forward step with torch tensor operations so
torch.autograd can supply one, on grids small enough for the CPU:

  - cons2prim with the pressure floor        src/eos.jl:8-25
  - minmod / limited_slope                   src/reconstruct.jl:6-16
  - PLM face values w +- s/2                 src/driver.jl:227-233
  - HLLC with Davis speeds and the star flux src/riemann.jl:9-88
  - flux divergence and the SSP-RK2 stages   src/driver.jl:236-321

Branches (minmod's choice, the pressure floor, fmin/fmax of the wave speeds,
the HLLC region and star side) are written as ``torch.where`` on the forward
values, so the gradient flows through the branch the forward takes -- the same
frozen-branch convention as the CUDA adjoint.  Unselected branches get safe
denominators so no inf/NaN reaches the backward pass.

Values are bit-identical to the C oracle's (the per-cell summation order of
the flux divergence is reproduced), which the tests check.  That matters at
rounding-level ties -- e.g. u_x inside a uniform Kelvin-Helmholtz band, whose
cell differences are pure rounding noise -- where any other order would flip
minmod choices and hence the frozen-branch gradient.

Layout: the state is a ``(5, ncell)`` float64 tensor, cells column-major with
x fastest (``vespa_oracle.h``).  Internally it is viewed as
``(5, n_{nd-1}, ..., n_0)`` so axis d is tensor dimension ``nd - d``.

Frozen map.  With a ``Tape`` every branch condition above is recorded in
evaluation order during one run (``Tape(record=True)``) and replayed in a
later run: that run then evaluates the step map with the recorded branch
choices at any nearby input, a smooth map whose derivative is exactly what
a frozen-branch adjoint computes.  Central differences of it check such an
adjoint even where the unfrozen map has kinks (minmod ties in a uniform
state).  Tensors may live on a GPU: there torch's float64 square root and
division are correctly rounded, so the values stay bit-identical to the C
oracle's.
"""
from __future__ import annotations

import math

import numpy as np
import torch


class _Sqrt(torch.autograd.Function):
    """Correctly rounded sqrt (numpy's), as the C oracle and the CUDA kernels
    use; torch's vectorised CPU sqrt is not always correctly rounded."""

    @staticmethod
    def forward(ctx, x):
        out = torch.from_numpy(np.sqrt(x.detach().numpy()))
        ctx.save_for_backward(out)
        return out

    @staticmethod
    def backward(ctx, g):
        (out,) = ctx.saved_tensors
        return g * (0.5 / out)


def _sqrt(x):
    if x.is_cuda:
        return torch.sqrt(x)
    return _Sqrt.apply(x)


class Tape:
    """Branch conditions of one run, in evaluation order: recorded when
    `record` is true, else replayed (the conditions computed from the current
    values are ignored)."""

    def __init__(self, record: bool = True):
        self.record = record
        self.masks = []
        self.pos = 0

    def replay(self):
        self.record = False
        self.pos = 0
        return self

    def __call__(self, cond):
        if self.record:
            self.masks.append(cond)
            return cond
        m = self.masks[self.pos]
        self.pos += 1
        return m


_TAPE = None  # the active tape (set by evolve/rk2_step callers), or None


def _br(cond):
    return cond if _TAPE is None else _TAPE(cond)


def cons2prim(U, g):
    rho = U[0]
    inv = 1.0 / rho
    vx = U[1] * inv
    vy = U[2] * inv
    vz = U[3] * inv
    ke = 0.5 * rho * (vx * vx + vy * vy + vz * vz)
    p = (g - 1.0) * (U[4] - ke)
    floor = 1e-12 * ke
    p = torch.where(_br(p >= floor), p, floor)
    return [rho, vx, vy, vz, p]


def minmod(a, b):
    z = torch.zeros_like(a)
    return torch.where(_br(a * b <= 0), z, torch.where(_br(a.abs() < b.abs()), a, b))


def hllc(WL, WR, g, dim):
    """HLLC flux through faces with normal axis ``dim`` (1..3); WL/WR are
    lists of five tensors (rho, vx, vy, vz, p)."""
    rhoL, rhoR = WL[0], WR[0]
    pL, pR = WL[4], WR[4]
    unL, unR = WL[dim], WR[dim]
    cL = _sqrt(g * pL / rhoL)
    cR = _sqrt(g * pR / rhoR)
    aL, aR = unL - cL, unR - cR
    SL = torch.where(_br(aL <= aR), aL, aR)
    bL, bR = unL + cL, unR + cR
    SR = torch.where(_br(bL >= bR), bL, bR)
    one = torch.ones_like(SL)
    zero = torch.zeros_like(SL)
    supL = _br(SL >= 0)
    supR = (~supL) & _br(SR <= 0)
    star = ~(supL | supR)
    N = pR - pL + rhoL * unL * (SL - unL) - rhoR * unR * (SR - unR)
    D = rhoL * (SL - unL) - rhoR * (SR - unR)
    Sstar = torch.where(star, N / torch.where(star, D, one), zero)
    left = supL | (star & _br(Sstar >= 0))
    SK = torch.where(left, SL, SR)
    rho = torch.where(left, rhoL, rhoR)
    v = [torch.where(left, WL[1 + j], WR[1 + j]) for j in range(3)]
    p = torch.where(left, pL, pR)
    un = v[dim - 1]
    # a tensor divisor: torch divides a CUDA tensor by a Python scalar as a
    # multiplication by its reciprocal, which rounds differently
    E = p / torch.full_like(p, g - 1.0) + 0.5 * rho * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2])
    Fk = [rho * un, (rho * v[0]) * un, (rho * v[1]) * un, (rho * v[2]) * un, (E + p) * un]
    Fk[dim] = Fk[dim] + p
    q = torch.where(star, rho * (SK - un), one)
    d = torch.where(star, SK - Sstar, one)
    factor = q / d
    Estar = E / rho + (Sstar - un) * (Sstar + p / q)
    vstar = list(v)
    vstar[dim - 1] = Sstar
    Us = [factor, factor * vstar[0], factor * vstar[1], factor * vstar[2], factor * Estar]
    Uk = [rho, rho * v[0], rho * v[1], rho * v[2], E]
    return [torch.where(star, Fk[k] + SK * (Us[k] - Uk[k]), Fk[k]) for k in range(5)]


class PeriodicGrid:
    """Geometry of a periodic uniform mesh (lib/RefMesh/src/RefMesh.jl:111-132)."""

    def __init__(self, dims, domain, gamma, aexp=1.0):
        self.dims = tuple(int(n) for n in dims)
        self.nd = len(self.dims)
        self.gamma = float(gamma)
        self.aexp = float(aexp)
        self.w = [(b - a) / n for (a, b), n in zip(domain, self.dims)]
        vol = self.w[0]
        for x in self.w[1:]:
            vol = vol * x
        self.vol = vol
        self.area = []
        for d in range(self.nd):
            a = 1.0
            for e in range(self.nd):
                if e != d:
                    a = a * self.w[e]
            self.area.append(a)

    @property
    def ncell(self):
        return math.prod(self.dims)

    def view(self, U):
        return U.reshape((5,) + self.dims[::-1])

    def flat(self, V):
        return V.reshape(5, -1)


def flux_divergence(grid: PeriodicGrid, U):
    """acc = sum over faces of +-area*F (src/driver.jl:236-281), periodic.

    Each cell adds its face contributions in the order the reference's
    column-major face enumeration (lib/RefMesh/src/RefMesh.jl:187-197) adds
    them into that cell: lo faces emitted by a lower-index neighbour (axes in
    reverse order), then per axis the hi face and, on a 1-cell axis, the lo
    face, then lo faces emitted by a periodic partner on the far edge.  So the
    values are bit-identical to the C oracle's."""
    V = grid.view(U)
    W = cons2prim(V, grid.gamma)
    shape = W[0].shape
    coords = []
    for d in range(grid.nd):
        td = grid.nd - d - 1
        idx = torch.arange(grid.dims[d], device=U.device)
        idx = idx.reshape([-1 if e == td else 1 for e in range(grid.nd)])
        coords.append(idx.expand(shape))
    Fhi, Flo = [], []
    for d in range(grid.nd):
        td = grid.nd - d - 1  # tensor dim of axis d within one field
        s = [minmod(w - torch.roll(w, 1, td), torch.roll(w, -1, td) - w) for w in W]
        WL = [W[k] + 0.5 * s[k] for k in range(5)]
        WR = [torch.roll(W[k], -1, td) + (-0.5) * torch.roll(s[k], -1, td) for k in range(5)]
        F = hllc(WL, WR, grid.gamma, d + 1)
        Fhi.append(F)
        Flo.append([torch.roll(F[k], 1, td) for k in range(5)])
    acc = []
    for k in range(5):
        a = torch.zeros(shape, dtype=W[0].dtype, device=U.device)
        for d in reversed(range(grid.nd)):
            before = (coords[d] > 0) if grid.dims[d] > 1 else torch.zeros(shape, dtype=torch.bool,
                                                                          device=U.device)
            a = torch.where(before, a + (-grid.area[d]) * Flo[d][k], a)
        for d in range(grid.nd):
            a = a + grid.area[d] * Fhi[d][k]
            if grid.dims[d] == 1:
                a = a + (-grid.area[d]) * Flo[d][k]
        for d in range(grid.nd):
            if grid.dims[d] > 1:
                a = torch.where(coords[d] == 0, a + (-grid.area[d]) * Flo[d][k], a)
        acc.append(a)
    return grid.flat(torch.stack(acc))


def rk2_step(grid: PeriodicGrid, U, dt):
    """step!(sim, dt) (src/driver.jl:339-359): two SSP-RK2 stages."""
    invV = dt / (grid.aexp * grid.vol)
    U1 = U - invV * flux_divergence(grid, U)
    return 0.5 * U + 0.5 * (U1 - invV * flux_divergence(grid, U1))


def evolve(grid: PeriodicGrid, U, dts, tape: Tape = None):
    """The run with the given dt sequence; with a tape, its branches are
    recorded (tape.record) or replayed."""
    global _TAPE
    _TAPE = tape
    try:
        for dt in dts:
            U = rk2_step(grid, U, float(dt))
    finally:
        _TAPE = None
    return U


def vjp(grid: PeriodicGrid, U0, dts, lam):
    """(dU_T/dU_0)^T lam for the run with the given dt sequence; returns
    (U_T, lam_0) as numpy arrays."""
    U = torch.tensor(U0, dtype=torch.float64, requires_grad=True)
    UT = evolve(grid, U, dts)
    (g,) = torch.autograd.grad(UT, U, grad_outputs=torch.tensor(lam, dtype=torch.float64))
    return UT.detach().numpy(), g.numpy()
