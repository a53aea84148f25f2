/*
 * vespa_oracle.c -- CPU oracle for the Vespa.jl finite-volume hydro step.
 *
 * TEST INFRASTRUCTURE ONLY (see vespa_oracle.h): the checker for the CUDA
 * library and the timed CPU baseline, never part of the product path.
 *
 * Every expression below is written in the reference's operation order so a
 * correctly rounded evaluation of the same expression tree agrees bit for bit.
 * Build with -ffp-contract=off and without -ffast-math (oracle/Makefile does):
 * Julia never fuses a multiply-add in these kernels, so neither may we.
 *
 * Parity status: pinned against the reference's known-answer tests (Sod vs the
 * exact Riemann solution and conservation, test/test_sod.jl:32-43; boundary-flux
 * identity, test/test_boundary_flux.jl:35) and Toro's published Sod star state;
 * bit-level agreement with the reference's own outputs is unpinned because the
 * reference (Julia) cannot run here.
 */
#include "vespa_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* Julia's Base.min / Base.max for IEEE floats: the sign of x - y picks the
 * result, NaN propagates (base/math.jl). */
static inline double jl_min(double x, double y)
{
    double diff = x - y;
    if (isnan(x) || isnan(y)) return diff;
    return signbit(diff) ? x : y;
}
static inline double jl_max(double x, double y)
{
    double diff = x - y;
    if (isnan(x) || isnan(y)) return diff;
    return signbit(diff) ? y : x;
}

/* ---------------------------------------------------------------- eos.jl */

/* cons2prim, src/eos.jl:8-25 (pressure floor max(p, 1e-12 * kinetic) at :24) */
void vo_cons2prim(const double *U, double gamma, double *W)
{
    double g = gamma;
    double rho = U[0];
    double inv = 1.0 / rho;
    double vx = U[1] * inv;
    double vy = U[2] * inv;
    double vz = U[3] * inv;
    double kinetic = 0.5 * rho * (vx * vx + vy * vy + vz * vz);
    double p = (g - 1.0) * (U[4] - kinetic);
    W[0] = rho;
    W[1] = vx;
    W[2] = vy;
    W[3] = vz;
    W[4] = jl_max(p, 1e-12 * kinetic);
}

/* prim2cons, src/eos.jl:28-32 */
void vo_prim2cons(const double *W, double gamma, double *U)
{
    double rho = W[0], vx = W[1], vy = W[2], vz = W[3], p = W[4];
    double E = p / (gamma - 1.0) + 0.5 * rho * (vx * vx + vy * vy + vz * vz);
    U[0] = rho;
    U[1] = rho * vx;
    U[2] = rho * vy;
    U[3] = rho * vz;
    U[4] = E;
}

/* ---------------------------------------------------------- reconstruct.jl */

/* minmod, src/reconstruct.jl:6-12 */
double vo_minmod(double a, double b)
{
    if (a * b <= 0.0) return 0.0;
    return fabs(a) < fabs(b) ? a : b;
}

/* limited_slope, src/reconstruct.jl:15-16 */
static inline double limited_slope(double l, double c, double r)
{
    return vo_minmod(c - l, r - c);
}

/* ---------------------------------------------------------------- riemann.jl */

/* euler_flux, src/riemann.jl:9-20; dim is 1-based */
static void euler_flux(const double *W, double gamma, int dim, double *F)
{
    double rho = W[0], vx = W[1], vy = W[2], vz = W[3], p = W[4];
    double un = W[dim];
    double E = p / (gamma - 1.0) + 0.5 * rho * (vx * vx + vy * vy + vz * vz);
    double m1 = rho * vx, m2 = rho * vy, m3 = rho * vz;
    F[0] = rho * un;
    F[1] = m1 * un + (dim == 1 ? p : 0.0);
    F[2] = m2 * un + (dim == 2 ? p : 0.0);
    F[3] = m3 * un + (dim == 3 ? p : 0.0);
    F[4] = (E + p) * un;
}

/* _hllc_star, src/riemann.jl:69-88 */
static void hllc_star(const double *W, const double *U, const double *F, double SK,
                      double Sstar, int dim, double *out)
{
    double rho = W[0];
    double un = W[dim];
    double p = W[4];
    double E = U[4];
    double factor = rho * (SK - un) / (SK - Sstar);
    double vstar[3] = {W[1], W[2], W[3]};
    vstar[dim - 1] = Sstar;
    double Estar = E / rho + (Sstar - un) * (Sstar + p / (rho * (SK - un)));
    double Ustar[5] = {factor, factor * vstar[0], factor * vstar[1], factor * vstar[2],
                       factor * Estar};
    for (int k = 0; k < 5; ++k) out[k] = F[k] + SK * (Ustar[k] - U[k]);
}

/* hllc_flux, src/riemann.jl:33-66 (Davis wave speeds, no HLL fallback) */
void vo_hllc_flux(const double *WL, const double *WR, double gamma, int dim, double *F)
{
    double rhoL = WL[0], rhoR = WR[0];
    double pL = WL[4], pR = WR[4];
    double unL = WL[dim], unR = WR[dim];
    double g = gamma;
    double cL = sqrt(g * pL / rhoL);
    double cR = sqrt(g * pR / rhoR);
    double SL = jl_min(unL - cL, unR - cR);
    double SR = jl_max(unL + cL, unR + cR);
    double UL[5], UR[5], FL[5], FR[5];
    vo_prim2cons(WL, gamma, UL);
    vo_prim2cons(WR, gamma, UR);
    euler_flux(WL, gamma, dim, FL);
    euler_flux(WR, gamma, dim, FR);
    if (SL >= 0.0) {
        memcpy(F, FL, sizeof FL);
        return;
    } else if (SR <= 0.0) {
        memcpy(F, FR, sizeof FR);
        return;
    }
    double Sstar = (pR - pL + rhoL * unL * (SL - unL) - rhoR * unR * (SR - unR)) /
                   (rhoL * (SL - unL) - rhoR * (SR - unR));
    if (Sstar >= 0.0)
        hllc_star(WL, UL, FL, SL, Sstar, dim, F);
    else
        hllc_star(WR, UR, FR, SR, Sstar, dim, F);
}

/* compute_face_fluxes!(::HostBatchedFlux, ...), src/ka_flux.jl:48-53 */
void vo_compute_face_fluxes(int64_t nf, const double *WL, const double *WR,
                            const int32_t *axis, double gamma, double *F)
{
    for (int64_t f = 0; f < nf; ++f)
        vo_hllc_flux(WL + 5 * f, WR + 5 * f, gamma, (int)axis[f], F + 5 * f);
}

/* ------------------------------------------------ RefMesh geometry/topology */

typedef struct {
    int nd;
    int64_t n[3];
    int64_t stride[3];
    int64_t ncell;
    double w[3];
    double area[3];
    double vol;
} geom_t;

static void make_geom(const vo_grid *g, geom_t *G)
{
    G->nd = g->ndim;
    int64_t s = 1;
    for (int d = 0; d < 3; ++d) {
        G->n[d] = d < g->ndim ? g->dims[d] : 1;
        G->stride[d] = s;
        s *= G->n[d];
    }
    G->ncell = s;
    /* _width, lib/RefMesh/src/RefMesh.jl:122-123 */
    for (int d = 0; d < g->ndim; ++d) G->w[d] = (g->hi[d] - g->lo[d]) / (double)g->dims[d];
    /* face_area, RefMesh.jl:135-142 */
    for (int d = 0; d < g->ndim; ++d) {
        double a = 1.0;
        for (int e = 0; e < g->ndim; ++e)
            if (e != d) a *= G->w[e];
        G->area[d] = a;
    }
    /* cell_volume = prod(_width), RefMesh.jl:127 (left fold) */
    double v = G->w[0];
    for (int d = 1; d < g->ndim; ++d) v = v * G->w[d];
    G->vol = v;
}

int64_t vo_ncell(const vo_grid *g)
{
    geom_t G;
    make_geom(g, &G);
    return G.ncell;
}

static inline int64_t coord_of(const geom_t *G, int64_t lin, int d)
{
    return (lin / G->stride[d]) % G->n[d];
}

/* neighbor, RefMesh.jl:147-161: linear index of the neighbour, or -1 for a
 * domain boundary; periodic wraps to the opposite edge. d is 0-based. */
static inline int64_t neighbor(const vo_grid *g, const geom_t *G, int64_t lin, int d, int hi)
{
    int64_t c = coord_of(G, lin, d);
    int64_t n = G->n[d];
    int64_t j = c + (hi ? 1 : -1);
    if (j >= 0 && j < n) return lin + (j - c) * G->stride[d];
    int bc = hi ? g->bc_hi[d] : g->bc_lo[d];
    if (bc == VO_BC_PERIODIC) {
        int64_t jw = j < 0 ? n - 1 : 0;
        return lin + (jw - c) * G->stride[d];
    }
    return -1;
}

static inline void load_U(const geom_t *G, const double *U, int64_t lin, double *u)
{
    for (int k = 0; k < 5; ++k) u[k] = U[k * G->ncell + lin];
}

/* _W, src/driver.jl:137 */
static inline void prim_at(const vo_grid *g, const geom_t *G, const double *U, int64_t lin,
                           double *W)
{
    double u[5];
    load_U(G, U, lin, u);
    vo_cons2prim(u, g->gamma, W);
}

/* ghost_state, src/driver.jl:117-122 (Outflow copy; Reflecting negates the
 * normal velocity, momentum_indices(model)[axis]); d is 0-based. */
static inline void ghost_state(const double *W, int bc, int d, double *out)
{
    for (int k = 0; k < 5; ++k) out[k] = W[k];
    if (bc == VO_BC_REFLECTING) out[1 + d] = -W[1 + d];
}

/* _plm_slope, src/driver.jl:145-159 */
static void plm_slope(const vo_grid *g, const geom_t *G, const double *U, int64_t lin,
                      const double *Wc, int d, double *s)
{
    double WL[5], WR[5];
    int64_t nlo = neighbor(g, G, lin, d, 0);
    int64_t nhi = neighbor(g, G, lin, d, 1);
    if (nlo < 0)
        ghost_state(Wc, g->bc_lo[d], d, WL);
    else
        prim_at(g, G, U, nlo, WL);
    if (nhi < 0)
        ghost_state(Wc, g->bc_hi[d], d, WR);
    else
        prim_at(g, G, U, nhi, WR);
    for (int k = 0; k < 5; ++k) s[k] = limited_slope(WL[k], Wc[k], WR[k]);
}

/* _face_value, src/driver.jl:227-233 */
static void face_value(const vo_grid *g, const geom_t *G, const double *U, int64_t lin, int d,
                       int hi, double *out)
{
    double Wi[5], s[5];
    prim_at(g, G, U, lin, Wi);
    plm_slope(g, G, U, lin, Wi, d, s);
    double h = hi ? 0.5 : -0.5;
    for (int k = 0; k < 5; ++k) out[k] = Wi[k] + h * s[k];
}

/* _acc_add!, src/driver.jl:98-99: acc[cell] += s * F */
static inline void acc_add(const geom_t *G, double *acc, int64_t lin, const double *F, double s)
{
    for (int k = 0; k < 5; ++k) acc[k * G->ncell + lin] += s * F[k];
}

/* bflux plane offset for (axis d, side, component k): dense planes with the
 * flux axis collapsed, remaining axes column-major, dim-0 fastest
 * (src/reflux.jl:148-166 plane raster order). */
static int64_t bflux_plane_index(const geom_t *G, int64_t lin, int d)
{
    int64_t idx = 0, mul = 1;
    for (int e = 0; e < G->nd; ++e) {
        if (e == d) continue;
        idx += coord_of(G, lin, e) * mul;
        mul *= G->n[e];
    }
    return idx;
}
static int64_t bflux_base(const geom_t *G, int d, int side)
{
    int64_t off = 0;
    for (int e = 0; e < d; ++e) off += 2 * 5 * (G->ncell / G->n[e]);
    return off + (int64_t)side * 5 * (G->ncell / G->n[d]);
}

int64_t vo_bflux_size(const vo_grid *g)
{
    geom_t G;
    make_geom(g, &G);
    return bflux_base(&G, G.nd, 0);
}

/* _bflux_capture!, src/reflux.jl:125-132: reg += (scale * f) * area */
static void bflux_capture(const geom_t *G, double *bflux, double scale, int d, int side,
                          int64_t lin, const double *F, double area)
{
    if (!bflux) return;
    int64_t P = G->ncell / G->n[d];
    int64_t base = bflux_base(G, d, side) + bflux_plane_index(G, lin, d);
    for (int k = 0; k < 5; ++k) bflux[base + k * P] += scale * F[k] * area;
}

/* The boundary-flux register as a dense restatement of its Dicts
 * (src/reflux.jl:113-118): `vals` holds the values, `seen` marks the keys the
 * Dict would contain (captured at least once).  Outer keys (axis, side, cell)
 * map to the plane layout above; interior keys (axis, lo cell) to
 * [axis][5][ncell]. */
typedef struct {
    double *vals, *ivals;
    unsigned char *seen, *iseen;
} breg_t;

/* _bflux_capture!, keyed (axis d, side, cell lin) */
static void breg_outer(const geom_t *G, const breg_t *r, double scale, int d, int side,
                       int64_t lin, const double *F, double area)
{
    if (!r || !r->vals) return;
    bflux_capture(G, r->vals, scale, d, side, lin, F, area);
    if (r->seen) r->seen[bflux_base(G, d, side) + bflux_plane_index(G, lin, d)] = 1;
}

/* _bflux_capture_interior!, src/reflux.jl:138-146: keyed (axis d, lo cell lin),
 * reg += (scale * f) * area, only when the register records interior faces */
static void breg_interior(const geom_t *G, const breg_t *r, double scale, int d, int64_t lin,
                          const double *F, double area)
{
    if (!r || !r->ivals) return;
    for (int k = 0; k < 5; ++k) r->ivals[((int64_t)d * 5 + k) * G->ncell + lin] += scale * F[k] * area;
    if (r->iseen) r->iseen[(int64_t)d * G->ncell + lin] = 1;
}

static void accumulate_flux_reg(const vo_grid *g, const double *U, double *acc, const breg_t *reg,
                                double bscale);

/* accumulate_flux! + for_each_face (src/driver.jl:209-281,
 * lib/RefMesh/src/RefMesh.jl:187-197): cells column-major; per cell and axis,
 * the hi face, then the lo face only when it is a domain boundary. */
void vo_accumulate_flux(const vo_grid *g, const double *U, double *acc, double *bflux,
                        double bscale)
{
    breg_t r = {bflux, NULL, NULL, NULL};
    accumulate_flux_reg(g, U, acc, bflux ? &r : NULL, bscale);
}

static void accumulate_flux_reg(const vo_grid *g, const double *U, double *acc, const breg_t *reg,
                                double bscale)
{
    geom_t G;
    make_geom(g, &G);
    memset(acc, 0, sizeof(double) * 5 * G.ncell);
    double WL[5], WR[5], Wg[5], F[5];
    for (int64_t lin = 0; lin < G.ncell; ++lin) {
        for (int d = 0; d < G.nd; ++d) {
            double a = G.area[d];
            int64_t nhi = neighbor(g, &G, lin, d, 1);
            if (nhi >= 0) {
                /* interior <-> interior, driver.jl:236-253 */
                face_value(g, &G, U, lin, d, 1, WL);
                face_value(g, &G, U, nhi, d, 0, WR);
                vo_hllc_flux(WL, WR, g->gamma, d + 1, F);
                acc_add(&G, acc, lin, F, a);
                acc_add(&G, acc, nhi, F, -a);
                breg_interior(&G, reg, bscale, d, lin, F, a);  /* +axis lo cell = lin */
            } else {
                /* hi-side domain boundary, driver.jl:256-267 */
                face_value(g, &G, U, lin, d, 1, WL);
                ghost_state(WL, g->bc_hi[d], d, Wg);
                vo_hllc_flux(WL, Wg, g->gamma, d + 1, F);
                acc_add(&G, acc, lin, F, a);
                breg_outer(&G, reg, bscale, d, 1, lin, F, a);
            }
            int64_t nlo = neighbor(g, &G, lin, d, 0);
            if (nlo < 0) {
                /* lo-side domain boundary, driver.jl:270-281 */
                face_value(g, &G, U, lin, d, 0, WR);
                ghost_state(WR, g->bc_lo[d], d, Wg);
                vo_hllc_flux(Wg, WR, g->gamma, d + 1, F);
                breg_outer(&G, reg, bscale, d, 0, lin, F, a);
                acc_add(&G, acc, lin, F, -a);
            }
        }
    }
}

/* Per-cell gather with the same per-cell summation order as the enumeration
 * above: each contribution is keyed by (emitting cell, axis, sub-order) and the
 * keys are sorted, so the result is bit-identical to vo_accumulate_flux while
 * cells can be processed in parallel.  The face flux itself is a pure function
 * of the state, so recomputing it per adjacent cell changes nothing. */
typedef struct {
    int64_t owner;
    int d;
    int sub;
    double s;
    double F[5];
} contrib_t;

static void gather_cell(const vo_grid *g, const geom_t *G, const double *U, int64_t lin,
                        double *accv)
{
    contrib_t c[6];
    int nc = 0;
    double WL[5], WR[5], Wg[5];
    for (int d = 0; d < G->nd; ++d) {
        double a = G->area[d];
        int64_t nhi = neighbor(g, G, lin, d, 1);
        contrib_t *h = &c[nc++];
        h->owner = lin;
        h->d = d;
        h->sub = 0;
        h->s = a;
        face_value(g, G, U, lin, d, 1, WL);
        if (nhi >= 0) {
            face_value(g, G, U, nhi, d, 0, WR);
            vo_hllc_flux(WL, WR, g->gamma, d + 1, h->F);
        } else {
            ghost_state(WL, g->bc_hi[d], d, Wg);
            vo_hllc_flux(WL, Wg, g->gamma, d + 1, h->F);
        }
        int64_t nlo = neighbor(g, G, lin, d, 0);
        contrib_t *l = &c[nc++];
        l->d = d;
        l->s = -a;
        face_value(g, G, U, lin, d, 0, WR);
        if (nlo >= 0) {
            /* emitted by nlo's hi query: interior face (nlo, lin) */
            l->owner = nlo;
            l->sub = 1;
            face_value(g, G, U, nlo, d, 1, WL);
            vo_hllc_flux(WL, WR, g->gamma, d + 1, l->F);
        } else {
            l->owner = lin;
            l->sub = 2;
            ghost_state(WR, g->bc_lo[d], d, Wg);
            vo_hllc_flux(Wg, WR, g->gamma, d + 1, l->F);
        }
    }
    /* insertion sort on (owner, d, sub) */
    for (int i = 1; i < nc; ++i) {
        contrib_t t = c[i];
        int j = i - 1;
        while (j >= 0 && (c[j].owner > t.owner ||
                          (c[j].owner == t.owner &&
                           (c[j].d > t.d || (c[j].d == t.d && c[j].sub > t.sub))))) {
            c[j + 1] = c[j];
            --j;
        }
        c[j + 1] = t;
    }
    for (int k = 0; k < 5; ++k) {
        double acc = 0.0;
        for (int i = 0; i < nc; ++i) acc += c[i].s * c[i].F[k];
        accv[k * G->ncell + lin] = acc;
    }
}

void vo_accumulate_flux_gather(const vo_grid *g, const double *U, double *acc, int nthreads)
{
    geom_t G;
    make_geom(g, &G);
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(static) num_threads(nthreads)
#endif
    for (int64_t lin = 0; lin < G.ncell; ++lin) gather_cell(g, &G, U, lin, acc);
    (void)nthreads;
}

/* The per-cell gather for the cells lin0 <= lin < lin1 only (a slab of whole
 * planes of a domain split along its last axis).  The state must be valid on
 * the cells the stencils reach: the slab and two planes on each side. */
void vo_accumulate_flux_gather_range(const vo_grid *g, const double *U, double *acc, int64_t lin0,
                                     int64_t lin1, int nthreads)
{
    geom_t G;
    make_geom(g, &G);
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(static) num_threads(nthreads)
#endif
    for (int64_t lin = lin0; lin < lin1; ++lin) gather_cell(g, &G, U, lin, acc);
    (void)nthreads;
}

/* compute_dt's maximum of (|v_d| + c) / w_d (src/driver.jl:176-187) over the
 * cells lin0 <= lin < lin1: a slab's share of the global reduction (the
 * maximum of the shares, then cfl / max, is compute_dt of the whole domain). */
double vo_invdt_range(const vo_grid *g, const double *U, int64_t lin0, int64_t lin1)
{
    geom_t G;
    make_geom(g, &G);
    double invdt = 0.0;
    double W[5];
    for (int64_t lin = lin0; lin < lin1; ++lin) {
        prim_at(g, &G, U, lin, W);
        double c = sqrt(g->gamma * W[4] / W[0]);
        for (int d = 0; d < G.nd; ++d) invdt = jl_max(invdt, (fabs(W[1 + d]) + c) / G.w[d]);
    }
    return jl_max(invdt, 0.0);
}

/* compute_dt, src/driver.jl:169-199 (no gravity, no cosmology) */
double vo_compute_dt(const vo_grid *g, const double *U)
{
    geom_t G;
    make_geom(g, &G);
    double invdt = 0.0;
    double W[5];
    for (int64_t lin = 0; lin < G.ncell; ++lin) {
        prim_at(g, &G, U, lin, W);
        double c = sqrt(g->gamma * W[4] / W[0]); /* sound_speed, src/eos.jl:35 */
        for (int d = 0; d < G.nd; ++d) {
            double vd = W[1 + d];
            invdt = jl_max(invdt, (fabs(vd) + c) / G.w[d]);
        }
    }
    invdt = jl_max(invdt, 0.0);
    if (invdt == 0.0) return INFINITY;
    return g->cfl / invdt;
}

/* step!, src/driver.jl:333-359 with _copy_state! (285-290), _euler_apply!
 * (297-307) and _rk2_combine! (310-321).  mode 0 = faithful serial face
 * enumeration, mode 1 = per-cell gather (OpenMP). */
void vo_step(const vo_grid *g, double *U, double *u0, double *acc, double dt, double *bflux,
             int mode, int nthreads)
{
    geom_t G;
    make_geom(g, &G);
    int64_t n5 = 5 * G.ncell;
    double bscale = 0.5 * dt;
    memcpy(u0, U, sizeof(double) * n5);
    if (mode == 0)
        vo_accumulate_flux(g, U, acc, bflux, bscale);
    else
        vo_accumulate_flux_gather(g, U, acc, nthreads);
    double invV = dt / (g->aexp * G.vol);
#ifdef _OPENMP
#pragma omp parallel for schedule(static) num_threads(nthreads > 0 ? nthreads : omp_get_max_threads()) if (mode == 1)
#endif
    for (int64_t i = 0; i < n5; ++i) U[i] = u0[i] - invV * acc[i];
    if (mode == 0)
        vo_accumulate_flux(g, U, acc, bflux, bscale);
    else
        vo_accumulate_flux_gather(g, U, acc, nthreads);
#ifdef _OPENMP
#pragma omp parallel for schedule(static) num_threads(nthreads > 0 ? nthreads : omp_get_max_threads()) if (mode == 1)
#endif
    for (int64_t i = 0; i < n5; ++i) U[i] = 0.5 * u0[i] + 0.5 * (U[i] - invV * acc[i]);
}

/* step!(sim, dt; bflux = reg) with a register that may record interior
 * faces (src/driver.jl:333-359, src/reflux.jl:113-146): serial face
 * enumeration, the register's scale set to 0.5*dt for both stages.  ivals and
 * the masks may be NULL. */
void vo_step_breg(const vo_grid *g, double *U, double *u0, double *acc, double dt, double *vals,
                  unsigned char *seen, double *ivals, unsigned char *iseen)
{
    geom_t G;
    make_geom(g, &G);
    int64_t n5 = 5 * G.ncell;
    breg_t r = {vals, ivals, seen, iseen};
    double bscale = 0.5 * dt;
    memcpy(u0, U, sizeof(double) * n5);
    accumulate_flux_reg(g, U, acc, &r, bscale);
    double invV = dt / (g->aexp * G.vol);
    for (int64_t i = 0; i < n5; ++i) U[i] = u0[i] - invV * acc[i];
    accumulate_flux_reg(g, U, acc, &r, bscale);
    for (int64_t i = 0; i < n5; ++i) U[i] = 0.5 * u0[i] + 0.5 * (U[i] - invV * acc[i]);
}

/* bflux_plane, src/reflux.jl:171-191.  The lookup closure of the reference's
 * callers (lib/EnzoLib/test/reflux_common.jl:104-133) becomes `source`: 0 / 1
 * the outer register's (dim+1, :lo / :hi, I) keys, 2 the interior register's
 * (dim+1, I) keys; a key the register never captured reads as `nothing`.  R =
 * ndim; dim is 0-based; start, stop, g0 hold R global indices; out gets
 * prod(stop - start + 1) values. */
void vo_bflux_plane(const vo_grid *g, const double *vals, const unsigned char *seen,
                    const double *ivals, const unsigned char *iseen, int dim, int source,
                    const int64_t *start, const int64_t *stop, const int64_t *g0, int64_t flux_off,
                    int comp, double vcell, double *out)
{
    geom_t G;
    make_geom(g, &G);
    const int R = G.nd;
    int64_t Dim[3] = {1, 1, 1}, n = 1;
    for (int d = 0; d < R; ++d) {
        Dim[d] = stop[d] - start[d] + 1;
        n *= Dim[d];
    }
    for (int64_t lin = 0; lin < n; ++lin) {
        /* decode column-major (dim-0 fastest) plane offset -> active index */
        int64_t rem = lin, act[3] = {1, 1, 1};
        for (int d = 0; d < R; ++d) {
            int64_t od = rem % Dim[d];
            rem /= Dim[d];
            int64_t gi = start[d] + od;
            act[d] = d == dim ? flux_off : (gi - g0[d] + 1);
        }
        /* lookup(I): a captured key of a cell of this grid, else nothing */
        const double *F = NULL;
        double Fv[5];
        int inside = 1;
        for (int d = 0; d < R; ++d) inside = inside && act[d] >= 1 && act[d] <= G.n[d];
        if (inside) {
            int64_t cell = 0, mul = 1;
            for (int d = 0; d < R; ++d) {
                cell += (act[d] - 1) * mul;
                mul *= G.n[d];
            }
            if (source == 2) {
                if (iseen[(int64_t)dim * G.ncell + cell]) {
                    for (int k = 0; k < 5; ++k) Fv[k] = ivals[((int64_t)dim * 5 + k) * G.ncell + cell];
                    F = Fv;
                }
            } else {
                int64_t base = bflux_base(&G, dim, source) + bflux_plane_index(&G, cell, dim);
                /* the key holds the cell itself: only its own side's face */
                int on_side = act[dim] == (source ? G.n[dim] : 1);
                if (on_side && seen[base]) {
                    int64_t P = G.ncell / G.n[dim];
                    for (int k = 0; k < 5; ++k) Fv[k] = vals[base + k * P];
                    F = Fv;
                }
            }
        }
        out[lin] = (F != NULL && comp > 0) ? F[comp - 1] / vcell : 0.0;
    }
}

/* evolve!, src/driver.jl:483-508 (single-rate path, no regrid/callback) */
int64_t vo_evolve(const vo_grid *g, double *U, double *u0, double *acc, double tfinal,
                  int64_t max_steps, double *t, int mode, int nthreads)
{
    int64_t n = 0;
    while (*t < tfinal * (1.0 - 1e-12)) {
        if (max_steps >= 0 && n >= max_steps) break;
        double dt = jl_min(vo_compute_dt(g, U), tfinal - *t);
        vo_step(g, U, u0, acc, dt, NULL, mode, nthreads);
        *t += dt;
        ++n;
    }
    return n;
}

/* conserved_totals, src/diagnostics.jl:16-31 (serial column-major sum) */
void vo_conserved_totals(const vo_grid *g, const double *U, double *out)
{
    geom_t G;
    make_geom(g, &G);
    double tot[5] = {0, 0, 0, 0, 0};
    for (int64_t lin = 0; lin < G.ncell; ++lin)
        for (int k = 0; k < 5; ++k) tot[k] += U[k * G.ncell + lin] * G.vol;
    memcpy(out, tot, sizeof tot);
}

/* ---------------------------------------------------------- exact_riemann.jl */

static inline double snd(double rho, double p, double g) { return sqrt(g * p / rho); }

/* _pressure_fn, src/exact_riemann.jl:11-23 */
static void pressure_fn(double p, double rhoK, double pK, double cK, double g, double *f,
                        double *df)
{
    if (p > pK) {
        double AK = 2.0 / ((g + 1.0) * rhoK);
        double BK = (g - 1.0) / (g + 1.0) * pK;
        *f = (p - pK) * sqrt(AK / (p + BK));
        *df = sqrt(AK / (BK + p)) * (1.0 - (p - pK) / (2.0 * (BK + p)));
    } else {
        *f = 2.0 * cK / (g - 1.0) * (pow(p / pK, (g - 1.0) / (2.0 * g)) - 1.0);
        *df = 1.0 / (rhoK * cK) * pow(p / pK, -(g + 1.0) / (2.0 * g));
    }
}

/* _star_state, src/exact_riemann.jl:25-48; WL/WR are (rho, u, p) */
void vo_exact_riemann_star(const double *WL, const double *WR, double g, double *pu)
{
    const double tol = 1e-12;
    double rhoL = WL[0], uL = WL[1], pL = WL[2];
    double rhoR = WR[0], uR = WR[1], pR = WR[2];
    double cL = snd(rhoL, pL, g), cR = snd(rhoR, pR, g);
    double p = fmax(tol, 0.5 * (pL + pR));
    for (int it = 0; it < 100; ++it) {
        double fL, dfL, fR, dfR;
        pressure_fn(p, rhoL, pL, cL, g, &fL, &dfL);
        pressure_fn(p, rhoR, pR, cR, g, &fR, &dfR);
        double f = fL + fR + (uR - uL);
        double p_new = fmax(tol, p - f / (dfL + dfR));
        if (fabs(p_new - p) / (0.5 * (p_new + p)) < tol) {
            p = p_new;
            break;
        }
        p = p_new;
    }
    double fL, fR, dummy;
    pressure_fn(p, rhoL, pL, cL, g, &fL, &dummy);
    pressure_fn(p, rhoR, pR, cR, g, &fR, &dummy);
    pu[0] = p;
    pu[1] = 0.5 * (uL + uR) + 0.5 * (fR - fL);
}

/* exact_riemann_sample, src/exact_riemann.jl:56-120 */
void vo_exact_riemann_sample(const double *WL, const double *WR, double g, double s,
                             double *out)
{
    double rhoL = WL[0], uL = WL[1], pL = WL[2];
    double rhoR = WR[0], uR = WR[1], pR = WR[2];
    double cL = snd(rhoL, pL, g), cR = snd(rhoR, pR, g);
    double pu[2];
    vo_exact_riemann_star(WL, WR, g, pu);
    double pstar = pu[0], ustar = pu[1];
    double gm = (g - 1.0) / (g + 1.0);
    if (s <= ustar) {
        if (pstar > pL) {
            double SL = uL - cL * sqrt((g + 1.0) / (2.0 * g) * pstar / pL + (g - 1.0) / (2.0 * g));
            if (s <= SL) {
                out[0] = rhoL; out[1] = uL; out[2] = pL;
            } else {
                out[0] = rhoL * (pstar / pL + gm) / (gm * pstar / pL + 1.0);
                out[1] = ustar; out[2] = pstar;
            }
        } else {
            double SHL = uL - cL;
            double cstar = cL * pow(pstar / pL, (g - 1.0) / (2.0 * g));
            double STL = ustar - cstar;
            if (s <= SHL) {
                out[0] = rhoL; out[1] = uL; out[2] = pL;
            } else if (s >= STL) {
                out[0] = rhoL * pow(pstar / pL, 1.0 / g);
                out[1] = ustar; out[2] = pstar;
            } else {
                double u = 2.0 / (g + 1.0) * (cL + (g - 1.0) / 2.0 * uL + s);
                double c = 2.0 / (g + 1.0) * (cL + (g - 1.0) / 2.0 * (uL - s));
                out[0] = rhoL * pow(c / cL, 2.0 / (g - 1.0));
                out[1] = u;
                out[2] = pL * pow(c / cL, 2.0 * g / (g - 1.0));
            }
        }
    } else {
        if (pstar > pR) {
            double SR = uR + cR * sqrt((g + 1.0) / (2.0 * g) * pstar / pR + (g - 1.0) / (2.0 * g));
            if (s >= SR) {
                out[0] = rhoR; out[1] = uR; out[2] = pR;
            } else {
                out[0] = rhoR * (pstar / pR + gm) / (gm * pstar / pR + 1.0);
                out[1] = ustar; out[2] = pstar;
            }
        } else {
            double SHR = uR + cR;
            double cstar = cR * pow(pstar / pR, (g - 1.0) / (2.0 * g));
            double STR = ustar + cstar;
            if (s >= SHR) {
                out[0] = rhoR; out[1] = uR; out[2] = pR;
            } else if (s <= STR) {
                out[0] = rhoR * pow(pstar / pR, 1.0 / g);
                out[1] = ustar; out[2] = pstar;
            } else {
                double u = 2.0 / (g + 1.0) * (-cR + (g - 1.0) / 2.0 * uR + s);
                double c = 2.0 / (g + 1.0) * (cR - (g - 1.0) / 2.0 * (uR - s));
                out[0] = rhoR * pow(c / cR, 2.0 / (g - 1.0));
                out[1] = u;
                out[2] = pR * pow(c / cR, 2.0 * g / (g - 1.0));
            }
        }
    }
}

/* ----------------------------------------------------------- src/gravity.jl */
/* Self-gravity on the uniform mesh.  The potential phi carries its own
 * boundary codes (periodic wraps; any other code is the homogeneous Neumann
 * wall of _lap_face!, src/gravity.jl:126-127). */

#define VO_FOURPI (4.0 * 3.14159265358979323846) /* FOURPI, src/gravity.jl:21 */

/* neighbour of `lin` across (d, hi) under phi's boundary codes, -1 at a wall */
static inline int64_t grav_nb(const vo_gravity *P, const geom_t *G, int64_t lin, int d, int hi)
{
    int64_t c = coord_of(G, lin, d);
    int64_t n = G->n[d];
    int64_t j = c + (hi ? 1 : -1);
    if (j >= 0 && j < n) return lin + (j - c) * G->stride[d];
    int bc = hi ? P->bc_hi[d] : P->bc_lo[d];
    if (bc == VO_BC_PERIODIC) return lin + ((j < 0 ? n - 1 : 0) - c) * G->stride[d];
    return -1;
}

/* (A x)[lin] with A = -lap * V, src/gravity.jl:325-334 (_lap_csr_cpu!):
 * s = sum_k coef_k * (x_c - x_nb(k)) over the row of the CSR adjacency that
 * _assemble_poisson_struct (src/gravity.jl:514-545) builds from for_each_face.
 * A row lists its faces in emission order: lo faces emitted by a lower cell
 * (z, y, x: ascending emitter index), then the cell's own hi faces (x, y, z),
 * then lo faces emitted by a periodic partner above it (x, y, z).  A 1-cell
 * periodic axis yields the self face (c, c) twice, at its hi position.
 * coef = area / face distance = area_d / (0.5 * (w_d + w_d)). */
static double grav_row(const vo_gravity *P, const geom_t *G, const double *x, int64_t lin)
{
    const double xc = x[lin];
    double s = 0.0;
    double coef[3];
    for (int d = 0; d < G->nd; ++d) coef[d] = G->area[d] / (0.5 * (G->w[d] + G->w[d]));
    for (int d = G->nd - 1; d >= 0; --d) {
        int64_t nb = grav_nb(P, G, lin, d, 0);
        if (nb >= 0 && nb < lin) s += coef[d] * (xc - x[nb]);
    }
    for (int d = 0; d < G->nd; ++d) {
        int64_t nb = grav_nb(P, G, lin, d, 1);
        if (nb < 0) continue;
        s += coef[d] * (xc - x[nb]);
        if (nb == lin) s += coef[d] * (xc - x[nb]); /* 1-cell periodic axis: the self face's second entry */
    }
    for (int d = 0; d < G->nd; ++d) {
        int64_t nb = grav_nb(P, G, lin, d, 0);
        if (nb > lin) s += coef[d] * (xc - x[nb]);
    }
    return s;
}

void vo_grav_laplacian(const vo_grid *g, const vo_gravity *P, const double *x, double *out)
{
    geom_t G;
    make_geom(g, &G);
    for (int64_t lin = 0; lin < G.ncell; ++lin) out[lin] = grav_row(P, &G, x, lin);
}

static double dot64(const double *a, const double *b, int64_t n)
{
    double s = 0.0;
    for (int64_t i = 0; i < n; ++i) s += a[i] * b[i];
    return s;
}

/* _rhs_flat_kernel!, src/gravity.jl:215-231 (no particles, no cosmology):
 * b = -4 pi G (rho - rhobar) V, rhobar the volume-weighted mean when the
 * constant null mode is projected out. */
static void grav_rhs(const vo_gravity *P, const geom_t *G, const double *U, double *b)
{
    double rhobar = 0.0;
    if (P->project_mean) {
        double s = 0.0, vsum = 0.0;
        for (int64_t i = 0; i < G->ncell; ++i) {
            s += U[i] * G->vol;
            vsum += G->vol;
        }
        rhobar = s / vsum;
    }
    for (int64_t i = 0; i < G->ncell; ++i)
        b[i] = -VO_FOURPI * P->G * (U[i] - rhobar) * G->vol * 1.0;
}

/* solve_poisson! on the CPU path, src/gravity.jl:251-300 (_cg_csr_run!):
 * warm start from phi, plain CG on A = -lap * V, then the volume-weighted
 * mean removed when project_mean.  Returns the iteration count. */
int64_t vo_grav_solve(const vo_grid *g, const vo_gravity *P, const double *U, double *phi,
                      double *relres_out)
{
    geom_t G;
    make_geom(g, &G);
    const int64_t n = G.ncell;
    double *b = calloc((size_t)n + 1, sizeof(double)), *r = calloc((size_t)n + 1, sizeof(double));
    double *p = calloc((size_t)n + 1, sizeof(double)), *Ap = calloc((size_t)n + 1, sizeof(double));
    grav_rhs(P, &G, U, b);
    vo_grav_laplacian(g, P, phi, Ap);
    for (int64_t i = 0; i < n; ++i) r[i] = b[i] - Ap[i];
    memcpy(p, r, sizeof(double) * n);
    double rsold = dot64(r, r, n);
    double bnorm = sqrt(dot64(b, b, n));
    if (bnorm == 0.0) bnorm = 1.0;
    int64_t iters = 0;
    double relres = sqrt(rsold) / bnorm;
    for (int64_t k = 1; k <= P->maxiter; ++k) {
        iters = k;
        vo_grav_laplacian(g, P, p, Ap);
        double pAp = dot64(p, Ap, n);
        if (pAp <= 0.0) break;
        double alpha = rsold / pAp;
        for (int64_t i = 0; i < n; ++i) {
            phi[i] += alpha * p[i];
            r[i] -= alpha * Ap[i];
        }
        double rsnew = dot64(r, r, n);
        relres = sqrt(rsnew) / bnorm;
        if (relres <= P->tol) break;
        double beta = rsnew / rsold;
        for (int64_t i = 0; i < n; ++i) p[i] = r[i] + beta * p[i];
        rsold = rsnew;
    }
    if (P->project_mean) {
        double s = 0.0, vsum = 0.0;
        for (int64_t i = 0; i < n; ++i) {
            s += G.vol * phi[i];
            vsum += G.vol;
        }
        double mu = s / vsum;
        for (int64_t i = 0; i < n; ++i) phi[i] -= mu;
    }
    free(b); free(r); free(p); free(Ap);
    if (relres_out) *relres_out = relres;
    return iters;
}

/* g = -grad phi per cell, _gax (src/gravity.jl:387-394): central difference
 * over the two face distances; across a wall the neighbour value is the
 * cell's own and the distance half a width.  gacc[d * ncell + lin], d < nd. */
void vo_grav_accel(const vo_grid *g, const vo_gravity *P, const double *phi, double *gacc)
{
    geom_t G;
    make_geom(g, &G);
    for (int64_t lin = 0; lin < G.ncell; ++lin) {
        const double pc = phi[lin];
        for (int d = 0; d < G.nd; ++d) {
            int64_t lo = grav_nb(P, &G, lin, d, 0), hi = grav_nb(P, &G, lin, d, 1);
            double wlo = lo < 0 ? pc : phi[lo], whi = hi < 0 ? pc : phi[hi];
            double fd = 0.5 * (G.w[d] + G.w[d]); /* _face_distance */
            double dlo = lo < 0 ? 0.5 * G.w[d] : fd, dhi = hi < 0 ? 0.5 * G.w[d] : fd;
            gacc[(int64_t)d * G.ncell + lin] = -(whi - wlo) / (dlo + dhi);
        }
    }
}

/* apply_gravity_source! (src/gravity.jl:419-437) into acc, from the stage
 * state U: +rho g on momentum and +rho v.g on energy, pushed with a minus
 * sign because the stage update subtracts acc (_grav_src_tuple, 371-382). */
static void grav_source(const geom_t *G, const double *U, const double *gacc, double *acc)
{
    const int64_t n = G->ncell;
    const double V = G->vol;
    for (int64_t lin = 0; lin < n; ++lin) {
        double gv[3] = {0.0, 0.0, 0.0};
        for (int d = 0; d < G->nd; ++d) gv[d] = gacc[(int64_t)d * n + lin];
        const double rho = U[lin];
        double es = 0.0;
        for (int d = 0; d < 3; ++d) es += U[(int64_t)(1 + d) * n + lin] * gv[d];
        const double esV = es * V;
        acc[lin] += 0.0;
        for (int d = 0; d < 3; ++d) acc[(int64_t)(1 + d) * n + lin] += -(rho * gv[d] * V);
        acc[4 * n + lin] += -esV;
    }
}

/* compute_dt with the free-fall limiter (src/driver.jl:169-199 with
 * _gravity_invdt, src/gravity.jl:439-441): invdt also takes
 * sqrt(4 pi G rho) / 0.5 over cells with rho > 0. */
double vo_compute_dt_gravity(const vo_grid *g, double Ggrav, const double *U)
{
    geom_t G;
    make_geom(g, &G);
    double invdt = 0.0, ginv = 0.0;
    double W[5];
    for (int64_t lin = 0; lin < G.ncell; ++lin) {
        prim_at(g, &G, U, lin, W);
        double c = sqrt(g->gamma * W[4] / W[0]);
        for (int d = 0; d < G.nd; ++d) invdt = jl_max(invdt, (fabs(W[1 + d]) + c) / G.w[d]);
        double gi = W[0] > 0.0 ? sqrt(VO_FOURPI * Ggrav * W[0]) / 0.5 : 0.0;
        ginv = jl_max(ginv, gi);
    }
    invdt = jl_max(invdt, ginv);
    if (invdt == 0.0) return INFINITY;
    return g->cfl / invdt;
}

/* step! with self-gravity (src/driver.jl:333-359): the source follows each
 * accumulate_flux! with the gravity field held over the step.  Serial face
 * enumeration (mode 0 of vo_step). */
void vo_step_gravity(const vo_grid *g, const double *gacc, double *U, double *u0, double *acc,
                     double dt)
{
    geom_t G;
    make_geom(g, &G);
    int64_t n5 = 5 * G.ncell;
    memcpy(u0, U, sizeof(double) * n5);
    vo_accumulate_flux(g, U, acc, NULL, 0.0);
    grav_source(&G, U, gacc, acc);
    double invV = dt / (g->aexp * G.vol);
    for (int64_t i = 0; i < n5; ++i) U[i] = u0[i] - invV * acc[i];
    vo_accumulate_flux(g, U, acc, NULL, 0.0);
    grav_source(&G, U, gacc, acc);
    for (int64_t i = 0; i < n5; ++i) U[i] = 0.5 * u0[i] + 0.5 * (U[i] - invV * acc[i]);
}

/* ------------------------------------- lib/PPMKernels: unsplit MUSCL (RK2) */
/* muscl_step_3d! (lib/PPMKernels/src/muscl_grid.jl:314-380): Enzo's
 * HydroMethod=3 step on five conserved arrays D, S1, S2, S3, Tau (Tau = rho *
 * specific total energy) of dims (nx, ny, nz) flat column-major with ng ghost
 * zones each side.  Restated in the reference's structure: per stage the
 * primitives (_cons2prim_k!, 23-34), then per axis the PLM + HLL flux line over
 * every pencil (ghost pencils included) and the flux divergence added into one
 * zeroed dU (x in place, y and z through zero-filled slabs that are added over
 * the whole grid), then the SSP-RK2 update of every cell. */

static inline double msign(double x) { return x > 0.0 ? 1.0 : -1.0; } /* _msign, muscl.jl:13 */

/* _minmod3, muscl.jl:16-19 */
static inline double minmod3(double a, double b, double c)
{
    double sa = msign(a), sb = msign(b), sc = msign(c);
    return 0.25 * (sa + sb) * fabs(sa + sc) * jl_min(fabs(a), jl_min(fabs(b), fabs(c)));
}

/* _plm_pt, muscl.jl:24-26: v + 0.5 * minmod3((v - vm1) th, (vp1 - v) th, 0.5 (vp1 - vm1)) */
static inline double plm_pt(double vm1, double v, double vp1, double th)
{
    return v + 0.5 * minmod3((v - vm1) * th, (vp1 - v) * th, 0.5 * (vp1 - vm1));
}

/* _hll, muscl.jl:29-30 */
static inline double hll1(double ap, double am, double fl, double fr, double ul, double ur)
{
    return (ap * fl + am * fr - ap * am * (ur - ul)) / (ap + am);
}

/* _hll5 / the first five of _hll6, muscl.jl:35-78: primitive L/R states
 * (rho, eint, u_normal, v, w) -> (F_rho, F_normal, F_t1, F_t2, F_E) */
static void hll5(double rl, double el, double ul, double vl, double wl, double rr, double er,
                 double ur, double vr, double wr, double g, double gm1, double F[5])
{
    const double h = 0.5;
    double v2l = ul * ul + vl * vl + wl * wl, pl = gm1 * rl * el, csl = sqrt(g * pl / rl);
    double etl = el + h * v2l;
    double UlD = rl, UlS1 = rl * ul, UlS2 = rl * vl, UlS3 = rl * wl, UlE = rl * etl;
    double FlD = rl * ul, FlS1 = UlS1 * ul + pl, FlS2 = UlS2 * ul, FlS3 = UlS3 * ul, FlE = (UlE + pl) * ul;
    double lpl = ul + csl, lml = ul - csl;
    double v2r = ur * ur + vr * vr + wr * wr, pr = gm1 * rr * er, csr = sqrt(g * pr / rr);
    double etr = er + h * v2r;
    double UrD = rr, UrS1 = rr * ur, UrS2 = rr * vr, UrS3 = rr * wr, UrE = rr * etr;
    double FrD = rr * ur, FrS1 = UrS1 * ur + pr, FrS2 = UrS2 * ur, FrS3 = UrS3 * ur, FrE = (UrE + pr) * ur;
    double lpr = ur + csr, lmr = ur - csr;
    double ap = jl_max(0.0, jl_max(lpl, lpr)), am = jl_max(0.0, jl_max(-lml, -lmr));
    F[0] = hll1(ap, am, FlD, FrD, UlD, UrD);
    F[1] = hll1(ap, am, FlS1, FrS1, UlS1, UrS1);
    F[2] = hll1(ap, am, FlS2, FrS2, UlS2, UrS2);
    F[3] = hll1(ap, am, FlS3, FrS3, UlS3, UrS3);
    F[4] = hll1(ap, am, FlE, FrE, UlE, UrE);
}

/* _muscl_hll_kernel! (muscl.jl:181-215) for one pencil of primitives q[5][na]
 * (rho, eint, u_normal, v_t1, v_t2) with stride `st`: fluxes at the nfi = na -
 * 2 ng + 1 interfaces, F[5][nfi]. */
static void flux_line(const double *const q[5], int64_t base, int64_t st, int64_t na, int ng,
                      double g, double th, double small_rho, double *F)
{
    const int64_t nfi = na - 2 * ng + 1;
    const double gm1 = g - 1.0;
    for (int64_t gi = 0; gi < nfi; ++gi) {
        const int64_t cl = ng + gi - 1; /* left cell of the interface, 0-based */
#define Q(f, m) q[f][base + (m) * st]
        double L[5], R[5];
        for (int f = 0; f < 5; ++f) {
            L[f] = plm_pt(Q(f, cl - 1), Q(f, cl), Q(f, cl + 1), th);
            R[f] = plm_pt(Q(f, cl + 2), Q(f, cl + 1), Q(f, cl), th);
        }
#undef Q
        L[0] = jl_max(L[0], small_rho);
        R[0] = jl_max(R[0], small_rho);
        double Fi[5];
        hll5(L[0], L[1], L[2], L[3], L[4], R[0], R[1], R[2], R[3], R[4], g, gm1, Fi);
        for (int f = 0; f < 5; ++f) F[f * nfi + gi] = Fi[f];
    }
}

/* dU of one stage: prim = cons2prim(U) everywhere, dU = 0 + axis sweeps */
static void muscl_L(const int64_t dims[3], int ng, double dt, double g, double th, double dx,
                    double small_rho, double *const U[5], double *prim, double *dU, double *slab)
{
    const int64_t N = dims[0] * dims[1] * dims[2];
    double *rho = prim, *eint = prim + N, *vx = prim + 2 * N, *vy = prim + 3 * N, *vz = prim + 4 * N;
    for (int64_t i = 0; i < N; ++i) { /* _cons2prim_k! */
        double d = U[0][i], u = U[1][i] / d, v = U[2][i] / d, w = U[3][i] / d;
        rho[i] = d; vx[i] = u; vy[i] = v; vz[i] = w;
        eint[i] = jl_max(U[4][i] / d - 0.5 * (u * u + v * v + w * w), small_rho);
    }
    memset(dU, 0, sizeof(double) * 5 * N);
    const double dtdx = dt / dx;
    const int64_t stride[3] = {1, dims[0], dims[0] * dims[1]};
    for (int axis = 0; axis < 3; ++axis) {
        const int64_t na = dims[axis], nfi = na - 2 * ng + 1, st = stride[axis];
        /* cyclic roles (normal, t1, t2), muscl_grid.jl:236 */
        const double *vu = axis == 0 ? vx : axis == 1 ? vy : vz;
        const double *vv = axis == 0 ? vy : axis == 1 ? vz : vx;
        const double *vw = axis == 0 ? vz : axis == 1 ? vx : vy;
        const double *q[5] = {rho, eint, vu, vv, vw};
        /* momentum slots receiving (normal, t1, t2) */
        const int sn = 1 + axis, s1 = 1 + (axis + 1) % 3, s2 = 1 + (axis + 2) % 3;
        const int slot[5] = {0, sn, s1, s2, 4};
        double *F = malloc(sizeof(double) * 5 * nfi);
        if (axis > 0) memset(slab, 0, sizeof(double) * 5 * N);
        /* every pencil: the other two coordinates over their full (ghosted) range */
        const int64_t o1 = axis == 0 ? 1 : 0, o2 = axis == 2 ? 1 : 2;
        for (int64_t b = 0; b < dims[o2]; ++b)
            for (int64_t a = 0; a < dims[o1]; ++a) {
                const int64_t base = a * stride[o1] + b * stride[o2];
                flux_line(q, base, st, na, ng, g, th, small_rho, F);
                for (int64_t m = 0; m < na - 2 * ng; ++m) {
                    const int64_t c = base + (ng + m) * st;
                    for (int f = 0; f < 5; ++f) {
                        const double du = -(F[f * nfi + m + 1] - F[f * nfi + m]) * dtdx;
                        if (axis == 0) dU[slot[f] * N + c] += du;
                        else slab[slot[f] * N + c] = du;
                    }
                }
            }
        if (axis > 0)
            for (int64_t i = 0; i < 5 * N; ++i) dU[i] += slab[i];
        free(F);
    }
}

/* periodic ghost fill along x, then y, then z (ghost p < ng takes p + active,
 * p >= ng + active takes p - active) */
static void muscl_fill_periodic(const int64_t dims[3], int ng, double *const U[5])
{
    const int64_t stride[3] = {1, dims[0], dims[0] * dims[1]};
    const int64_t N = dims[0] * dims[1] * dims[2];
    for (int axis = 0; axis < 3; ++axis) {
        const int64_t na = dims[axis], act = na - 2 * ng, st = stride[axis];
        for (int64_t i = 0; i < N; ++i) {
            const int64_t p = (i / st) % na;
            int64_t src = -1;
            if (p < ng) src = i + act * st;
            else if (p >= ng + act) src = i - act * st;
            if (src >= 0)
                for (int f = 0; f < 5; ++f) U[f][i] = U[f][src];
        }
    }
}

/* One muscl_step_3d! on U = (D, S1, S2, S3, Tau), 5 x N field-major; bc 0:
 * ghosts untouched (no bc! callback), 1: periodic fill before each stage. */
void vo_muscl_step(const int64_t dims[3], int ng, double dt, double gamma, double theta,
                   double dx, double small_rho, int bc, double *U)
{
    const int64_t N = dims[0] * dims[1] * dims[2];
    double *U0 = malloc(sizeof(double) * 5 * N), *prim = malloc(sizeof(double) * 5 * N);
    double *dU = malloc(sizeof(double) * 5 * N), *slab = malloc(sizeof(double) * 5 * N);
    double *Uf[5];
    for (int f = 0; f < 5; ++f) Uf[f] = U + f * N;
    memcpy(U0, U, sizeof(double) * 5 * N);
    if (bc == 1) muscl_fill_periodic(dims, ng, Uf);
    muscl_L(dims, ng, dt, gamma, theta, dx, small_rho, Uf, prim, dU, slab);
    for (int64_t i = 0; i < 5 * N; ++i) U[i] = U0[i] + dU[i];
    if (bc == 1) muscl_fill_periodic(dims, ng, Uf);
    muscl_L(dims, ng, dt, gamma, theta, dx, small_rho, Uf, prim, dU, slab);
    for (int64_t i = 0; i < 5 * N; ++i) U[i] = 0.5 * (U0[i] + U[i] + dU[i]);
    free(U0); free(prim); free(dU); free(slab);
}

/* The reference's certified 1-D flux line (muscl_flux_line!, muscl.jl:223-240)
 * on one pencil of na primitives (rho, eint, vx, vy, vz), for tests. */
void vo_muscl_flux_line(int64_t na, int ng, const double *prim, double gamma, double theta,
                        double small_rho, double *F)
{
    const double *q[5] = {prim, prim + na, prim + 2 * na, prim + 3 * na, prim + 4 * na};
    flux_line(q, 0, 1, na, ng, gamma, theta, small_rho, F);
}
