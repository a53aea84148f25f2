"""Independent pure-Python restatement of the reference's uniform-grid step.

TEST INFRASTRUCTURE ONLY.  A second, line-by-line transcription of the Julia
source (written separately from vespa_oracle.c) used on tiny grids to check
that the C oracle follows the reference's operation order: both must agree bit
for bit.  Python floats are IEEE doubles and Python never fuses a multiply-add,
so the arithmetic matches Julia's.  Pure-Python loops: small cases only.
"""
from __future__ import annotations

import math


def jl_min(x, y):  # Base.min for floats (sign of x - y decides, NaN propagates)
    d = x - y
    if math.isnan(x) or math.isnan(y):
        return d
    return x if math.copysign(1.0, d) < 0 else y


def jl_max(x, y):
    d = x - y
    if math.isnan(x) or math.isnan(y):
        return d
    return y if math.copysign(1.0, d) < 0 else x


# src/eos.jl:8-25
def cons2prim(U, g):
    rho = U[0]
    inv = 1.0 / rho
    vx = U[1] * inv
    vy = U[2] * inv
    vz = U[3] * inv
    kinetic = 0.5 * rho * (vx * vx + vy * vy + vz * vz)
    p = (g - 1.0) * (U[4] - kinetic)
    return (rho, vx, vy, vz, jl_max(p, 1e-12 * kinetic))


# src/eos.jl:28-32
def prim2cons(W, g):
    rho, vx, vy, vz, p = W
    E = p / (g - 1.0) + 0.5 * rho * (vx * vx + vy * vy + vz * vz)
    return (rho, rho * vx, rho * vy, rho * vz, E)


# src/reconstruct.jl:6-16
def minmod(a, b):
    if a * b <= 0:
        return 0.0
    return a if abs(a) < abs(b) else b


def limited_slope(l, c, r):
    return minmod(c - l, r - c)


# src/riemann.jl:9-20
def euler_flux(W, g, dim):
    rho, vx, vy, vz, p = W
    un = (vx, vy, vz)[dim - 1]
    E = p / (g - 1.0) + 0.5 * rho * (vx * vx + vy * vy + vz * vz)
    m = (rho * vx, rho * vy, rho * vz)
    pf = tuple(p if dim == d else 0.0 for d in (1, 2, 3))
    return (rho * un, m[0] * un + pf[0], m[1] * un + pf[1], m[2] * un + pf[2], (E + p) * un)


# src/riemann.jl:69-88
def hllc_star(W, U, F, SK, Sstar, dim, g):
    rho = W[0]
    un = W[dim]
    p = W[4]
    E = U[4]
    factor = rho * (SK - un) / (SK - Sstar)
    v = [W[1], W[2], W[3]]
    v[dim - 1] = Sstar
    Estar = E / rho + (Sstar - un) * (Sstar + p / (rho * (SK - un)))
    Ustar = (factor, factor * v[0], factor * v[1], factor * v[2], factor * Estar)
    return tuple(F[k] + SK * (Ustar[k] - U[k]) for k in range(5))


# src/riemann.jl:33-66
def hllc_flux(WL, WR, g, dim):
    rhoL, rhoR = WL[0], WR[0]
    pL, pR = WL[4], WR[4]
    unL, unR = WL[dim], WR[dim]
    cL = math.sqrt(g * pL / rhoL)
    cR = math.sqrt(g * pR / rhoR)
    SL = jl_min(unL - cL, unR - cR)
    SR = jl_max(unL + cL, unR + cR)
    UL, UR = prim2cons(WL, g), prim2cons(WR, g)
    FL, FR = euler_flux(WL, g, dim), euler_flux(WR, g, dim)
    if SL >= 0:
        return FL
    elif SR <= 0:
        return FR
    Sstar = (pR - pL + rhoL * unL * (SL - unL) - rhoR * unR * (SR - unR)) / \
            (rhoL * (SL - unL) - rhoR * (SR - unR))
    if Sstar >= 0:
        return hllc_star(WL, UL, FL, SL, Sstar, dim, g)
    return hllc_star(WR, UR, FR, SR, Sstar, dim, g)


class UniformGrid:
    """lib/RefMesh/src/RefMesh.jl:89-197 (0-based coordinates here)."""

    def __init__(self, dims, lo, hi, bc_lo, bc_hi, gamma, cfl):
        self.dims = tuple(int(n) for n in dims)
        self.N = len(self.dims)
        self.w = tuple((hi[d] - lo[d]) / self.dims[d] for d in range(self.N))
        self.bc_lo, self.bc_hi = tuple(bc_lo), tuple(bc_hi)
        self.g, self.cfl = gamma, cfl
        v = self.w[0]
        for d in range(1, self.N):
            v = v * self.w[d]
        self.vol = v

    def cells(self):
        # column-major: axis 0 fastest
        idx = [0] * self.N
        total = 1
        for n in self.dims:
            total *= n
        for lin in range(total):
            r = lin
            for d in range(self.N):
                idx[d] = r % self.dims[d]
                r //= self.dims[d]
            yield tuple(idx)

    def face_area(self, axis):
        a = 1.0
        for d in range(self.N):
            if d != axis:
                a *= self.w[d]
        return a

    def neighbor(self, I, axis, hi):  # None = domain boundary
        j = I[axis] + (1 if hi else -1)
        n = self.dims[axis]
        if 0 <= j < n:
            return I[:axis] + (j,) + I[axis + 1:]
        bc = self.bc_hi[axis] if hi else self.bc_lo[axis]
        if bc == 1:  # Periodic
            jw = n - 1 if j < 0 else 0
            return I[:axis] + (jw,) + I[axis + 1:]
        return None


def _ghost(W, bc, axis):  # src/driver.jl:117-122
    if bc == 2:
        return tuple(-W[k] if k == axis + 1 else W[k] for k in range(5))
    return tuple(W)


def accumulate_flux(m: UniformGrid, U):
    """src/driver.jl:209-281; U maps cell tuple -> conserved 5-tuple."""
    acc = {I: [0.0] * 5 for I in m.cells()}
    W = {I: cons2prim(U[I], m.g) for I in m.cells()}

    def slope(I, axis):
        nlo, nhi = m.neighbor(I, axis, False), m.neighbor(I, axis, True)
        Wc = W[I]
        WL = _ghost(Wc, m.bc_lo[axis], axis) if nlo is None else W[nlo]
        WR = _ghost(Wc, m.bc_hi[axis], axis) if nhi is None else W[nhi]
        return tuple(limited_slope(WL[k], Wc[k], WR[k]) for k in range(5))

    def face_value(I, axis, hi):
        s = slope(I, axis)
        h = 0.5 if hi else -0.5
        return tuple(W[I][k] + h * s[k] for k in range(5))

    def add(I, F, s):
        a = acc[I]
        for k in range(5):
            a[k] += s * F[k]

    for I in m.cells():
        for d in range(m.N):
            a = m.face_area(d)
            nhi = m.neighbor(I, d, True)
            if nhi is not None:
                F = hllc_flux(face_value(I, d, True), face_value(nhi, d, False), m.g, d + 1)
                add(I, F, a)
                add(nhi, F, -a)
            else:
                WL = face_value(I, d, True)
                F = hllc_flux(WL, _ghost(WL, m.bc_hi[d], d), m.g, d + 1)
                add(I, F, a)
            if m.neighbor(I, d, False) is None:
                WR = face_value(I, d, False)
                F = hllc_flux(_ghost(WR, m.bc_lo[d], d), WR, m.g, d + 1)
                add(I, F, -a)
    return acc


def compute_dt(m: UniformGrid, U):  # src/driver.jl:169-199
    invdt = 0.0
    for I in m.cells():
        Wc = cons2prim(U[I], m.g)
        c = math.sqrt(m.g * Wc[4] / Wc[0])
        for d in range(m.N):
            invdt = jl_max(invdt, (abs(Wc[1 + d]) + c) / m.w[d])
    invdt = jl_max(invdt, 0.0)
    return math.inf if invdt == 0 else m.cfl / invdt


def step(m: UniformGrid, U, dt):  # src/driver.jl:333-359
    u0 = {I: tuple(U[I]) for I in m.cells()}
    acc = accumulate_flux(m, U)
    invV = dt / (1.0 * m.vol)
    U1 = {I: tuple(u0[I][k] - invV * acc[I][k] for k in range(5)) for I in m.cells()}
    acc = accumulate_flux(m, U1)
    return {I: tuple(0.5 * u0[I][k] + 0.5 * (U1[I][k] - invV * acc[I][k]) for k in range(5))
            for I in m.cells()}
