"""ctypes binding of the CPU oracle (oracle/vespa_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of ``bench.py``; the product package never imports it.

Arrays follow the conventions of ``vespa_oracle.h``: the state is a
``(5, ncell)`` float64 array (structure of arrays, x fastest) and face batches
are ``(nf, 5)`` float64 arrays (five components contiguous per face).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libvespa_oracle.so")

BC_OUTFLOW, BC_PERIODIC, BC_REFLECTING = 0, 1, 2


class VoGrid(C.Structure):
    _fields_ = [
        ("ndim", C.c_int32),
        ("bc_lo", C.c_int32 * 3),
        ("bc_hi", C.c_int32 * 3),
        ("reserved", C.c_int32),
        ("dims", C.c_int64 * 3),
        ("lo", C.c_double * 3),
        ("hi", C.c_double * 3),
        ("gamma", C.c_double),
        ("cfl", C.c_double),
        ("aexp", C.c_double),
    ]


class VoGravity(C.Structure):
    _fields_ = [
        ("G", C.c_double),
        ("tol", C.c_double),
        ("bc_lo", C.c_int32 * 3),
        ("bc_hi", C.c_int32 * 3),
        ("maxiter", C.c_int32),
        ("project_mean", C.c_int32),
    ]


def build() -> str:
    """Compile the oracle with its Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        dp = C.POINTER(C.c_double)
        gp = C.POINTER(VoGrid)
        L.vo_cons2prim.argtypes = [dp, C.c_double, dp]
        L.vo_prim2cons.argtypes = [dp, C.c_double, dp]
        L.vo_minmod.argtypes = [C.c_double, C.c_double]
        L.vo_minmod.restype = C.c_double
        L.vo_hllc_flux.argtypes = [dp, dp, C.c_double, C.c_int, dp]
        L.vo_compute_face_fluxes.argtypes = [C.c_int64, dp, dp, C.POINTER(C.c_int32),
                                             C.c_double, dp]
        L.vo_ncell.argtypes = [gp]
        L.vo_ncell.restype = C.c_int64
        L.vo_compute_dt.argtypes = [gp, dp]
        L.vo_compute_dt.restype = C.c_double
        L.vo_accumulate_flux.argtypes = [gp, dp, dp, dp, C.c_double]
        L.vo_accumulate_flux_gather.argtypes = [gp, dp, dp, C.c_int]
        L.vo_accumulate_flux_gather_range.argtypes = [gp, dp, dp, C.c_int64, C.c_int64, C.c_int]
        L.vo_invdt_range.argtypes = [gp, dp, C.c_int64, C.c_int64]
        L.vo_invdt_range.restype = C.c_double
        L.vo_step.argtypes = [gp, dp, dp, dp, C.c_double, dp, C.c_int, C.c_int]
        L.vo_evolve.argtypes = [gp, dp, dp, dp, C.c_double, C.c_int64, dp, C.c_int, C.c_int]
        L.vo_evolve.restype = C.c_int64
        L.vo_conserved_totals.argtypes = [gp, dp, dp]
        L.vo_bflux_size.argtypes = [gp]
        L.vo_bflux_size.restype = C.c_int64
        u8p = C.POINTER(C.c_uint8)
        i64p = C.POINTER(C.c_int64)
        L.vo_step_breg.argtypes = [gp, dp, dp, dp, C.c_double, dp, u8p, dp, u8p]
        L.vo_bflux_plane.argtypes = [gp, dp, u8p, dp, u8p, C.c_int, C.c_int, i64p, i64p, i64p,
                                     C.c_int64, C.c_int, C.c_double, dp]
        L.vo_exact_riemann_star.argtypes = [dp, dp, C.c_double, dp]
        L.vo_exact_riemann_sample.argtypes = [dp, dp, C.c_double, C.c_double, dp]
        vp = C.c_void_p
        i64 = C.c_int64
        L.vo_amr_create.argtypes = [gp]
        L.vo_amr_create.restype = vp
        L.vo_amr_destroy.argtypes = [vp]
        L.vo_amr_nleaf.argtypes = [vp]
        L.vo_amr_nleaf.restype = i64
        L.vo_amr_leaves.argtypes = [vp, C.POINTER(C.c_int32), C.POINTER(C.c_int64)]
        L.vo_amr_set_state.argtypes = [vp, dp]
        L.vo_amr_get_state.argtypes = [vp, dp]
        L.vo_amr_set_time.argtypes = [vp, C.c_double, i64]
        L.vo_amr_time.argtypes = [vp]
        L.vo_amr_time.restype = C.c_double
        L.vo_amr_steps.argtypes = [vp]
        L.vo_amr_steps.restype = i64
        L.vo_amr_max_level.argtypes = [vp]
        L.vo_amr_refine.argtypes = [vp, C.POINTER(C.c_int64), i64]
        L.vo_amr_refine.restype = i64
        L.vo_amr_indicator.argtypes = [vp, dp]
        L.vo_amr_regrid.argtypes = [vp, C.c_double, C.c_int]
        L.vo_amr_regrid.restype = i64
        L.vo_amr_compute_dt.argtypes = [vp, C.c_int]
        L.vo_amr_compute_dt.restype = C.c_double
        L.vo_amr_step.argtypes = [vp, C.c_double, C.c_int]
        L.vo_amr_evolve.argtypes = [vp, C.c_double, i64, C.c_double, C.c_int, C.c_int, C.c_int]
        L.vo_amr_evolve.restype = i64
        L.vo_amr_totals.argtypes = [vp, dp]
        gvp = C.POINTER(VoGravity)
        L.vo_grav_laplacian.argtypes = [gp, gvp, dp, dp]
        L.vo_grav_solve.argtypes = [gp, gvp, dp, dp, dp]
        L.vo_grav_solve.restype = i64
        L.vo_grav_accel.argtypes = [gp, gvp, dp, dp]
        L.vo_compute_dt_gravity.argtypes = [gp, C.c_double, dp]
        L.vo_compute_dt_gravity.restype = C.c_double
        L.vo_step_gravity.argtypes = [gp, dp, dp, dp, dp, C.c_double]
        i64p = C.POINTER(C.c_int64)
        L.vo_muscl_step.argtypes = [i64p, C.c_int, C.c_double, C.c_double, C.c_double,
                                    C.c_double, C.c_double, C.c_int, dp]
        L.vo_muscl_flux_line.argtypes = [i64, C.c_int, dp, C.c_double, C.c_double, C.c_double, dp]
        _lib = L
    return _lib


def _dp(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_double))


def make_grid(dims, lo, hi, bc_lo, bc_hi, gamma, cfl=0.4, aexp=1.0) -> VoGrid:
    """Grid descriptor; ``dims/lo/hi/bc_*`` are per-axis sequences (length 1-3)."""
    nd = len(dims)
    g = VoGrid()
    g.ndim = nd
    for d in range(3):
        g.dims[d] = int(dims[d]) if d < nd else 1
        g.lo[d] = float(lo[d]) if d < nd else 0.0
        g.hi[d] = float(hi[d]) if d < nd else 1.0
        g.bc_lo[d] = int(bc_lo[d]) if d < nd else BC_PERIODIC
        g.bc_hi[d] = int(bc_hi[d]) if d < nd else BC_PERIODIC
    g.gamma = float(gamma)
    g.cfl = float(cfl)
    g.aexp = float(aexp)
    return g


def grid_from_problem(prob) -> VoGrid:
    """Oracle grid for a product ``Problem`` (duck-typed: dims/domain/bcs/gamma/cfl)."""
    lo = [d[0] for d in prob.domain]
    hi = [d[1] for d in prob.domain]
    bc_lo = [b[0] for b in prob.bc_pairs()]
    bc_hi = [b[1] for b in prob.bc_pairs()]
    return make_grid(prob.dims, lo, hi, bc_lo, bc_hi, prob.gamma, prob.cfl)


def ncell(g: VoGrid) -> int:
    return int(lib().vo_ncell(C.byref(g)))


def cons2prim(U, gamma):
    U = np.ascontiguousarray(U, dtype=np.float64)
    W = np.empty(5)
    lib().vo_cons2prim(_dp(U), gamma, _dp(W))
    return W


def prim2cons(W, gamma):
    W = np.ascontiguousarray(W, dtype=np.float64)
    U = np.empty(5)
    lib().vo_prim2cons(_dp(W), gamma, _dp(U))
    return U


def hllc_flux(WL, WR, gamma, dim):
    WL = np.ascontiguousarray(WL, dtype=np.float64)
    WR = np.ascontiguousarray(WR, dtype=np.float64)
    F = np.empty(5)
    lib().vo_hllc_flux(_dp(WL), _dp(WR), gamma, int(dim), _dp(F))
    return F


def compute_face_fluxes(WL, WR, axis, gamma):
    WL = np.ascontiguousarray(WL, dtype=np.float64)
    WR = np.ascontiguousarray(WR, dtype=np.float64)
    ax = np.ascontiguousarray(axis, dtype=np.int32)
    nf = ax.shape[0]
    F = np.empty((nf, 5))
    lib().vo_compute_face_fluxes(nf, _dp(WL), _dp(WR), ax.ctypes.data_as(C.POINTER(C.c_int32)),
                                 gamma, _dp(F))
    return F


def compute_dt(g: VoGrid, U) -> float:
    U = np.ascontiguousarray(U, dtype=np.float64)
    return float(lib().vo_compute_dt(C.byref(g), _dp(U)))


def accumulate_flux(g: VoGrid, U, gather=False, nthreads=0):
    U = np.ascontiguousarray(U, dtype=np.float64)
    acc = np.empty_like(U)
    if gather:
        lib().vo_accumulate_flux_gather(C.byref(g), _dp(U), _dp(acc), int(nthreads))
    else:
        lib().vo_accumulate_flux(C.byref(g), _dp(U), _dp(acc), None, 0.0)
    return acc


def accumulate_flux_range(g: VoGrid, U, acc, lin0, lin1, nthreads=0):
    """The per-cell gather for the cells lin0 <= lin < lin1 into acc (in place)."""
    assert U.dtype == np.float64 and U.flags.c_contiguous and acc.flags.c_contiguous
    lib().vo_accumulate_flux_gather_range(C.byref(g), _dp(U), _dp(acc), int(lin0), int(lin1),
                                          int(nthreads))
    return acc


def invdt_range(g: VoGrid, U, lin0, lin1) -> float:
    """compute_dt's CFL maximum over the cells lin0 <= lin < lin1."""
    U = np.ascontiguousarray(U, dtype=np.float64)
    return float(lib().vo_invdt_range(C.byref(g), _dp(U), int(lin0), int(lin1)))


def step(g: VoGrid, U, dt, mode=0, nthreads=0, bflux=None):
    """One SSP-RK2 step in place on ``U`` (a (5, ncell) float64 array)."""
    assert U.dtype == np.float64 and U.flags.c_contiguous
    u0 = np.empty_like(U)
    acc = np.empty_like(U)
    bp = _dp(bflux) if bflux is not None else None
    lib().vo_step(C.byref(g), _dp(U), _dp(u0), _dp(acc), float(dt), bp, int(mode), int(nthreads))
    return U


def evolve(g: VoGrid, U, tfinal, max_steps=-1, t0=0.0, mode=0, nthreads=0):
    """evolve! in place; returns (t, nsteps)."""
    assert U.dtype == np.float64 and U.flags.c_contiguous
    u0 = np.empty_like(U)
    acc = np.empty_like(U)
    t = C.c_double(t0)
    n = lib().vo_evolve(C.byref(g), _dp(U), _dp(u0), _dp(acc), float(tfinal), int(max_steps),
                        C.byref(t), int(mode), int(nthreads))
    return t.value, int(n)


def conserved_totals(g: VoGrid, U):
    U = np.ascontiguousarray(U, dtype=np.float64)
    out = np.empty(5)
    lib().vo_conserved_totals(C.byref(g), _dp(U), _dp(out))
    return out


def bflux_size(g: VoGrid) -> int:
    return int(lib().vo_bflux_size(C.byref(g)))


class BoundaryFluxRegister:
    """BoundaryFluxRegister (src/reflux.jl:113-118) in dense form: the outer
    values in the vb_bflux_read plane layout plus a mask of the keys the Dict
    would hold; with record_interior, the interior values [axis][5][ncell] and
    their mask."""

    def __init__(self, g: VoGrid, record_interior: bool = False):
        self.g = g
        n = bflux_size(g)
        nc = ncell(g)
        self.vals = np.zeros(n)
        self.seen = np.zeros(n, dtype=np.uint8)
        self.ivals = np.zeros(g.ndim * 5 * nc) if record_interior else None
        self.iseen = np.zeros(g.ndim * nc, dtype=np.uint8) if record_interior else None

    def empty(self):
        self.vals[:] = 0.0
        self.seen[:] = 0
        if self.ivals is not None:
            self.ivals[:] = 0.0
            self.iseen[:] = 0

    def dense(self) -> np.ndarray:
        """The register in vb_bflux_read's layout (outer planes, then interior)."""
        return self.vals if self.ivals is None else np.concatenate([self.vals, self.ivals])


def _u8p(a):
    return a.ctypes.data_as(C.POINTER(C.c_uint8)) if a is not None else None


def step_breg(g: VoGrid, U, dt, reg: BoundaryFluxRegister):
    """step!(sim, dt; bflux = reg), serial face enumeration, in place on U."""
    assert U.dtype == np.float64 and U.flags.c_contiguous
    u0 = np.empty_like(U)
    acc = np.empty_like(U)
    lib().vo_step_breg(C.byref(g), _dp(U), _dp(u0), _dp(acc), float(dt), _dp(reg.vals),
                       _u8p(reg.seen), _dp(reg.ivals) if reg.ivals is not None else None,
                       _u8p(reg.iseen))
    return U


def bflux_plane(g: VoGrid, reg: BoundaryFluxRegister, dim, source, start, stop, g0, flux_off,
                comp, vcell):
    """bflux_plane (src/reflux.jl:171-191); source 0 / 1 / 2 = the outer lo /
    hi keys or the interior keys stand for the caller's lookup."""
    st = np.ascontiguousarray(start, dtype=np.int64)
    sp = np.ascontiguousarray(stop, dtype=np.int64)
    g0a = np.ascontiguousarray(g0, dtype=np.int64)
    out = np.empty(int(np.prod(sp - st + 1)))
    i64p = C.POINTER(C.c_int64)
    lib().vo_bflux_plane(C.byref(g), _dp(reg.vals), _u8p(reg.seen),
                         _dp(reg.ivals) if reg.ivals is not None else None, _u8p(reg.iseen),
                         int(dim), int(source), st.ctypes.data_as(i64p), sp.ctypes.data_as(i64p),
                         g0a.ctypes.data_as(i64p), int(flux_off), int(comp), float(vcell),
                         _dp(out))
    return out


def exact_riemann_star(WL, WR, gamma):
    WL = np.ascontiguousarray(WL, dtype=np.float64)
    WR = np.ascontiguousarray(WR, dtype=np.float64)
    out = np.empty(2)
    lib().vo_exact_riemann_star(_dp(WL), _dp(WR), gamma, _dp(out))
    return out


def exact_riemann_sample(WL, WR, gamma, s):
    WL = np.ascontiguousarray(WL, dtype=np.float64)
    WR = np.ascontiguousarray(WR, dtype=np.float64)
    out = np.empty(3)
    lib().vo_exact_riemann_sample(_dp(WL), _dp(WR), gamma, float(s), _dp(out))
    return out


class Amr:
    """The AMR restatement (vespa_oracle_amr.c): a composite leaf-only mesh
    over a base grid, with the reference's face rules, regrid and drivers.
    The state is a (5, nleaf) float64 array in leaf order."""

    def __init__(self, g: VoGrid):
        self.h = lib().vo_amr_create(C.byref(g))

    def close(self):
        if self.h:
            lib().vo_amr_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def nleaf(self) -> int:
        return int(lib().vo_amr_nleaf(self.h))

    def leaves(self):
        n = self.nleaf
        lev = np.empty(n, dtype=np.int32)
        cx = np.empty((n, 3), dtype=np.int64)
        lib().vo_amr_leaves(self.h, lev.ctypes.data_as(C.POINTER(C.c_int32)),
                            cx.ctypes.data_as(C.POINTER(C.c_int64)))
        return lev, cx

    def set_state(self, U):
        U = np.ascontiguousarray(U, dtype=np.float64)
        assert U.shape == (5, self.nleaf)
        lib().vo_amr_set_state(self.h, _dp(U))

    def state(self):
        U = np.empty((5, self.nleaf))
        lib().vo_amr_get_state(self.h, _dp(U))
        return U

    def set_time(self, t, step=0):
        lib().vo_amr_set_time(self.h, float(t), int(step))

    @property
    def t(self):
        return float(lib().vo_amr_time(self.h))

    @property
    def step_count(self):
        return int(lib().vo_amr_steps(self.h))

    @property
    def max_level(self):
        return int(lib().vo_amr_max_level(self.h))

    def refine(self, leaves):
        idx = np.ascontiguousarray(leaves, dtype=np.int64)
        return int(lib().vo_amr_refine(self.h, idx.ctypes.data_as(C.POINTER(C.c_int64)), len(idx)))

    def indicator(self):
        out = np.empty(self.nleaf)
        lib().vo_amr_indicator(self.h, _dp(out))
        return out

    def regrid(self, refine_above, max_level):
        return int(lib().vo_amr_regrid(self.h, float(refine_above), int(max_level)))

    def compute_dt(self, level=-1):
        return float(lib().vo_amr_compute_dt(self.h, int(level)))

    def step(self, dt, level=-1):
        lib().vo_amr_step(self.h, float(dt), int(level))

    def evolve(self, tfinal, max_steps=-1, refine_above=0.0, max_level=0, every=0, subcycle=False):
        return int(lib().vo_amr_evolve(self.h, float(tfinal), int(max_steps), float(refine_above),
                                       int(max_level), int(every), int(bool(subcycle))))

    def totals(self):
        out = np.empty(5)
        lib().vo_amr_totals(self.h, _dp(out))
        return out


# ------------------------------------------------------------ self-gravity
def make_gravity(G, bc_lo, bc_hi, maxiter=500, tol=1e-8, project_mean=True) -> VoGravity:
    """Gravity descriptor; ``bc_lo/bc_hi`` are phi's per-axis codes (length 1-3)."""
    P = VoGravity()
    P.G = float(G)
    P.tol = float(tol)
    for d in range(3):
        P.bc_lo[d] = int(bc_lo[d]) if d < len(bc_lo) else BC_PERIODIC
        P.bc_hi[d] = int(bc_hi[d]) if d < len(bc_hi) else BC_PERIODIC
    P.maxiter = int(maxiter)
    P.project_mean = int(bool(project_mean))
    return P


def grav_laplacian(g: VoGrid, P: VoGravity, x):
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.empty_like(x)
    lib().vo_grav_laplacian(C.byref(g), C.byref(P), _dp(x), _dp(out))
    return out


def grav_solve(g: VoGrid, P: VoGravity, U, phi):
    """solve_poisson! in place on ``phi`` (warm start); returns (iters, relres)."""
    U = np.ascontiguousarray(U, dtype=np.float64)
    assert phi.dtype == np.float64 and phi.flags.c_contiguous
    rr = np.zeros(1)
    it = lib().vo_grav_solve(C.byref(g), C.byref(P), _dp(U), _dp(phi), _dp(rr))
    return int(it), float(rr[0])


def grav_accel(g: VoGrid, P: VoGravity, phi):
    phi = np.ascontiguousarray(phi, dtype=np.float64)
    out = np.empty((g.ndim, phi.size))
    lib().vo_grav_accel(C.byref(g), C.byref(P), _dp(phi), _dp(out))
    return out


def compute_dt_gravity(g: VoGrid, G, U) -> float:
    U = np.ascontiguousarray(U, dtype=np.float64)
    return float(lib().vo_compute_dt_gravity(C.byref(g), float(G), _dp(U)))


def step_gravity(g: VoGrid, gacc, U, dt):
    """One SSP-RK2 step with the gravity source (field gacc held), in place on U."""
    assert U.dtype == np.float64 and U.flags.c_contiguous
    gacc = np.ascontiguousarray(gacc, dtype=np.float64)
    u0 = np.empty_like(U)
    acc = np.empty_like(U)
    lib().vo_step_gravity(C.byref(g), _dp(gacc), _dp(U), _dp(u0), _dp(acc), float(dt))
    return U


# ------------------------------------------------- PPMKernels unsplit MUSCL
def muscl_step(dims, ng, U, dt, gamma, theta=1.5, dx=1.0, small_rho=1e-10, bc=0):
    """muscl_step_3d! in place on U, a (5, N) float64 array (D, S1, S2, S3, Tau)."""
    assert U.dtype == np.float64 and U.flags.c_contiguous
    d = (C.c_int64 * 3)(*[int(x) for x in dims])
    lib().vo_muscl_step(d, int(ng), float(dt), float(gamma), float(theta), float(dx),
                        float(small_rho), int(bc), _dp(U))
    return U


def muscl_flux_line(prim, ng, gamma, theta=1.5, small_rho=1e-10):
    """muscl_flux_line! on one pencil: prim (5, na) -> F (5, na - 2 ng + 1)."""
    prim = np.ascontiguousarray(prim, dtype=np.float64)
    na = prim.shape[1]
    F = np.empty((5, na - 2 * ng + 1))
    lib().vo_muscl_flux_line(na, int(ng), _dp(prim), float(gamma), float(theta),
                             float(small_rho), _dp(F))
    return F
