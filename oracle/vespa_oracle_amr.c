/* vespa_oracle_amr.c -- CPU restatement of Vespa.jl's AMR hydro path.
 *
 * TEST INFRASTRUCTURE ONLY (the oracle); the product library never links it.
 *
 * What it restates:
 *   - the composite leaf-only AMR mesh of lib/HGBackend/src/HGBackend.jl
 *     (2:1 face-balanced cell tree, leaves are the cells; 1 <= rank <= 3)
 *   - face enumeration with hanging nodes, HGBackend.jl:220-276: conforming
 *     faces once from the hi side, coarse<->fine sub-faces once from the fine
 *     side with the fine cell's area, boundary faces from their cell
 *   - PLM slopes from the representative face neighbour (HGBackend.jl:182-200
 *     via src/driver.jl:152-159), face values, HLLC, +F/-F scatter
 *     (src/driver.jl:209-281)
 *   - per-cell volumes in _euler_apply! / _rk2_combine! (src/driver.jl:297-321)
 *   - compute_dt(level) (src/driver.jl:169-199), step!(level) (333-359)
 *   - density_gradient_indicator, regrid! (src/driver.jl:400-462), refine-only,
 *     piecewise-constant conservative prolongation of the cell means
 *   - single-rate evolve! with a RefinementPolicy (src/driver.jl:483-508)
 *   - subcycled evolve_level! / step_level! with FluxRegisters
 *     (src/driver.jl:367-385, 523-605; src/reflux.jl:51-103)
 *   - conserved_totals (src/diagnostics.jl:16-31)
 *
 * HierarchicalGrids.jl (the reference's mesh substrate, an un-vendored
 * sibling package with no version pin) is absent, so three of its choices are
 * made here and documented as such (parity with HG itself is unpinned):
 *   1. the base grid is a forest of root cells (any dims, not only one
 *      power-of-two root); leaves are ordered by root in column-major order,
 *      then depth-first with children in x-fastest order (child index
 *      x + 2y + 4z).  With no refinement this is RefMesh's cell order, so an
 *      unrefined AMR mesh reproduces the uniform path bit for bit.
 *   2. the representative neighbour across a face with finer leaves (used by
 *      PLM and the indicator) is the adjacent fine leaf that comes first in
 *      that order.
 *   3. 2:1 balance is across faces: refining a leaf first refines any
 *      face neighbour one level coarser (recursively).
 * Periodic axes wrap like interior faces (the reference leaves periodic
 * coarse<->fine faces as a follow-up; with no refinement at the wrap the
 * emission is identical).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "vespa_oracle.h"

#define VA_MAXLEV 15
#define VA_CBITS 20

struct vo_amr {
    vo_grid g;
    int nd;
    double w0[3];
    int64_t n, cap;
    int32_t *lev;
    int64_t *cx;   /* 3 per leaf */
    double *U;     /* 5 per leaf, AoS */
    double *u0, *acc, *reg;
    /* hash of (level, coords) -> leaf slot, -1 for a refined (dead) cell */
    int64_t hcap;
    uint64_t *hkey;
    int64_t *hval;
    double t;
    int64_t step;
};

/* Julia's min/max on Float64 (NaN-propagating) */
static inline double jmin(double x, double y)
{
    if (x != x || y != y) return x + y;
    return y < x ? y : x;
}
static inline double jmax(double x, double y)
{
    if (x != x || y != y) return x + y;
    return y > x ? y : x;
}

static uint64_t key_of(int32_t l, const int64_t *c)
{
    return ((uint64_t)l << 60) | ((uint64_t)c[0] << 40) | ((uint64_t)c[1] << 20) | (uint64_t)c[2];
}

static uint64_t hmix(uint64_t k)
{
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdULL;
    k ^= k >> 33;
    k *= 0xc4ceb9fe1a85ec53ULL;
    k ^= k >> 33;
    return k;
}

static void h_put(vo_amr *a, uint64_t k, int64_t v)
{
    uint64_t m = (uint64_t)a->hcap - 1, i = hmix(k) & m;
    while (a->hkey[i] != UINT64_MAX && a->hkey[i] != k) i = (i + 1) & m;
    a->hkey[i] = k;
    a->hval[i] = v;
}

static int64_t h_get(const vo_amr *a, uint64_t k)
{
    uint64_t m = (uint64_t)a->hcap - 1, i = hmix(k) & m;
    while (a->hkey[i] != UINT64_MAX) {
        if (a->hkey[i] == k) return a->hval[i];
        i = (i + 1) & m;
    }
    return -1;
}

static void h_rebuild(vo_amr *a, int64_t extra)
{
    int64_t need = 4 * (a->n + extra) + 64, cap = 64;
    while (cap < need) cap <<= 1;
    if (cap != a->hcap) {
        free(a->hkey);
        free(a->hval);
        a->hkey = malloc(sizeof(uint64_t) * cap);
        a->hval = malloc(sizeof(int64_t) * cap);
        a->hcap = cap;
    }
    memset(a->hkey, 0xff, sizeof(uint64_t) * a->hcap);
    for (int64_t i = 0; i < a->n; ++i)
        if (a->lev[i] >= 0) h_put(a, key_of(a->lev[i], a->cx + 3 * i), i);
}

static void grow(vo_amr *a, int64_t need)
{
    if (need <= a->cap) return;
    int64_t cap = a->cap ? a->cap : 64;
    while (cap < need) cap *= 2;
    a->lev = realloc(a->lev, sizeof(int32_t) * cap);
    a->cx = realloc(a->cx, sizeof(int64_t) * 3 * cap);
    a->U = realloc(a->U, sizeof(double) * 5 * cap);
    a->u0 = realloc(a->u0, sizeof(double) * 5 * cap);
    a->acc = realloc(a->acc, sizeof(double) * 5 * cap);
    a->reg = realloc(a->reg, sizeof(double) * 5 * cap);
    a->cap = cap;
}

static double width(const vo_amr *a, int32_t l, int d) { return a->w0[d] * ldexp(1.0, -l); }

static double cell_volume(const vo_amr *a, int32_t l)
{
    double v = 1.0;
    for (int d = 0; d < a->nd; ++d) v = v * width(a, l, d);
    return v;
}

static double face_area(const vo_amr *a, int32_t l, int axis)
{
    double s = 1.0;
    for (int d = 0; d < a->nd; ++d)
        if (d != axis) s = s * width(a, l, d);
    return s;
}

/* depth-first order key: root (column-major), then the child path */
static uint64_t dfs_key(const vo_amr *a, int32_t l, const int64_t *c)
{
    uint64_t root = 0, mul = 1;
    for (int d = 0; d < a->nd; ++d) {
        root += (uint64_t)(c[d] >> l) * mul;
        mul *= (uint64_t)a->g.dims[d];
    }
    uint64_t path = 0;
    for (int k = VA_MAXLEV - 1; k >= 0; --k) {
        uint64_t digit = 0;
        for (int d = 0; d < a->nd; ++d) {
            uint64_t s = (uint64_t)(c[d] & ((1LL << l) - 1)) << (VA_MAXLEV - l);
            digit |= ((s >> k) & 1u) << d;
        }
        path = (path << a->nd) | digit;
    }
    return (root << (a->nd * VA_MAXLEV)) | path;
}

/* Face neighbour of leaf i across (axis d, side hi): 0 domain boundary,
 * 1 same level, 2 coarser, 3 finer; *rep = representative leaf. */
static int nb_query(const vo_amr *a, int64_t i, int d, int hi, int64_t *rep)
{
    int32_t l = a->lev[i];
    int64_t cc[3] = {a->cx[3 * i], a->cx[3 * i + 1], a->cx[3 * i + 2]};
    int64_t nd = a->g.dims[d] << l;
    cc[d] += hi ? 1 : -1;
    if (cc[d] < 0 || cc[d] >= nd) {
        int bc = hi ? a->g.bc_hi[d] : a->g.bc_lo[d];
        if (bc != VO_BC_PERIODIC) return 0;
        cc[d] = (cc[d] + nd) % nd;
    }
    int64_t j = h_get(a, key_of(l, cc));
    if (j >= 0) { *rep = j; return 1; }
    if (l > 0) {
        int64_t cp[3] = {cc[0] >> 1, cc[1] >> 1, cc[2] >> 1};
        j = h_get(a, key_of(l - 1, cp));
        if (j >= 0) { *rep = j; return 2; }
    }
    int64_t cf[3] = {2 * cc[0], 2 * cc[1], 2 * cc[2]};
    for (int e = a->nd; e < 3; ++e) cf[e] = 0;
    if (!hi) cf[d] += 1;
    j = h_get(a, key_of(l + 1, cf));
    *rep = j;
    return 3;
}

static void prim(const vo_amr *a, const double *U, int64_t i, double *W)
{
    vo_cons2prim(U + 5 * i, a->g.gamma, W);
}

static void ghost(const double *W, int bc, int d, double *out)
{
    for (int k = 0; k < 5; ++k) out[k] = W[k];
    if (bc == VO_BC_REFLECTING) out[1 + d] = -W[1 + d];
}

/* _face_value(sim, i, axis, side) with _plm_slope over representatives */
static void face_value(const vo_amr *a, const double *U, int64_t i, int d, int hi, double *out)
{
    double Wc[5], Wl[5], Wr[5];
    int64_t j;
    prim(a, U, i, Wc);
    if (nb_query(a, i, d, 0, &j)) prim(a, U, j, Wl); else ghost(Wc, a->g.bc_lo[d], d, Wl);
    if (nb_query(a, i, d, 1, &j)) prim(a, U, j, Wr); else ghost(Wc, a->g.bc_hi[d], d, Wr);
    double h = hi ? 0.5 : -0.5;
    for (int k = 0; k < 5; ++k) {
        double s = vo_minmod(Wc[k] - Wl[k], Wr[k] - Wc[k]);
        out[k] = Wc[k] + h * s;
    }
}

static void acc_add(double *acc, int64_t i, const double *F, double s)
{
    for (int k = 0; k < 5; ++k) acc[5 * i + k] += s * F[k];
}

/* active flux registers of one capture pass: coarse level and scale */
typedef struct {
    int n;
    int32_t cl[2];
    double scale[2];
} regset;

/* _reflux_capture!, src/reflux.jl:67-86 */
static void capture(vo_amr *a, const regset *rs, int64_t i, int64_t j, const double *F, double area)
{
    int32_t li = a->lev[i], lj = a->lev[j];
    if (li == lj) return;
    for (int r = 0; r < rs->n; ++r) {
        int32_t cl = rs->cl[r];
        double s = rs->scale[r];
        if (li == cl && lj == cl + 1) {
            for (int k = 0; k < 5; ++k) a->reg[5 * i + k] += s * F[k] * area;
        } else if (lj == cl && li == cl + 1) {
            for (int k = 0; k < 5; ++k) a->reg[5 * j + k] += -s * F[k] * area;
        }
    }
}

/* accumulate_flux! over the composite mesh, in HGBackend's emission order */
static void accumulate(vo_amr *a, const regset *rs)
{
    const double *U = a->U;
    double *acc = a->acc;
    memset(acc, 0, sizeof(double) * 5 * a->n);
    double WL[5], WR[5], Wg[5], F[5];
    for (int64_t i = 0; i < a->n; ++i) {
        int32_t li = a->lev[i];
        for (int d = 0; d < a->nd; ++d) {
            double area = face_area(a, li, d);
            int64_t j;
            int kind = nb_query(a, i, d, 1, &j);
            if (kind == 0) {
                face_value(a, U, i, d, 1, WL);
                ghost(WL, a->g.bc_hi[d], d, Wg);
                vo_hllc_flux(WL, Wg, a->g.gamma, d + 1, F);
                acc_add(acc, i, F, area);
            } else if (kind != 3) {
                face_value(a, U, i, d, 1, WL);
                face_value(a, U, j, d, 0, WR);
                vo_hllc_flux(WL, WR, a->g.gamma, d + 1, F);
                acc_add(acc, i, F, area);
                acc_add(acc, j, F, -area);
                if (rs) capture(a, rs, i, j, F, area);
            }
            kind = nb_query(a, i, d, 0, &j);
            if (kind == 0) {
                face_value(a, U, i, d, 0, WR);
                ghost(WR, a->g.bc_lo[d], d, Wg);
                vo_hllc_flux(Wg, WR, a->g.gamma, d + 1, F);
                acc_add(acc, i, F, -area);
            } else if (kind == 2) {
                face_value(a, U, j, d, 1, WL);
                face_value(a, U, i, d, 0, WR);
                vo_hllc_flux(WL, WR, a->g.gamma, d + 1, F);
                acc_add(acc, j, F, area);
                acc_add(acc, i, F, -area);
                if (rs) capture(a, rs, j, i, F, area);
            }
        }
    }
}

static void step_impl(vo_amr *a, double dt, int level, const regset *rs1, const regset *rs2)
{
    const double aexp = a->g.aexp;
    for (int64_t i = 0; i < a->n; ++i)
        if (level < 0 || a->lev[i] == level) memcpy(a->u0 + 5 * i, a->U + 5 * i, 5 * sizeof(double));
    accumulate(a, rs1);
    for (int64_t i = 0; i < a->n; ++i) {
        if (level >= 0 && a->lev[i] != level) continue;
        double invV = dt / (aexp * cell_volume(a, a->lev[i]));
        for (int k = 0; k < 5; ++k) a->U[5 * i + k] = a->u0[5 * i + k] - invV * a->acc[5 * i + k];
    }
    accumulate(a, rs2);
    for (int64_t i = 0; i < a->n; ++i) {
        if (level >= 0 && a->lev[i] != level) continue;
        double invV = dt / (aexp * cell_volume(a, a->lev[i]));
        for (int k = 0; k < 5; ++k)
            a->U[5 * i + k] =
                0.5 * a->u0[5 * i + k] + 0.5 * (a->U[5 * i + k] - invV * a->acc[5 * i + k]);
    }
}

/* ---------------------------------------------------------------- refine */

/* Replace leaf (l, c) by its 2^nd children, first refining face neighbours
 * one level coarser (2:1 balance).  Children inherit the parent's cell mean. */
static void refine_at(vo_amr *a, int32_t l, const int64_t *c)
{
    int64_t i = h_get(a, key_of(l, c));
    if (i < 0) return;  /* not a leaf (already refined) */
    for (int d = 0; d < a->nd; ++d) {
        for (int hi = 0; hi < 2; ++hi) {
            int64_t cc[3] = {c[0], c[1], c[2]};
            int64_t nd = a->g.dims[d] << l;
            cc[d] += hi ? 1 : -1;
            if (cc[d] < 0 || cc[d] >= nd) {
                int bc = hi ? a->g.bc_hi[d] : a->g.bc_lo[d];
                if (bc != VO_BC_PERIODIC) continue;
                cc[d] = (cc[d] + nd) % nd;
            }
            if (l == 0 || h_get(a, key_of(l, cc)) >= 0) continue;
            int64_t cp[3] = {cc[0] >> 1, cc[1] >> 1, cc[2] >> 1};
            if (h_get(a, key_of(l - 1, cp)) >= 0) refine_at(a, l - 1, cp);
        }
    }
    i = h_get(a, key_of(l, c));
    if (i < 0) return;
    int nch = 1 << a->nd;
    grow(a, a->n + nch);
    if (4 * (a->n + nch) + 64 > a->hcap) h_rebuild(a, 2 * nch + a->n);
    h_put(a, key_of(l, c), -1);
    for (int ch = 0; ch < nch; ++ch) {
        int64_t s = a->n++;
        a->lev[s] = l + 1;
        for (int d = 0; d < 3; ++d)
            a->cx[3 * s + d] = d < a->nd ? 2 * c[d] + ((ch >> d) & 1) : 0;
        memcpy(a->U + 5 * s, a->U + 5 * i, 5 * sizeof(double));
        h_put(a, key_of(l + 1, a->cx + 3 * s), s);
    }
    a->lev[i] = -1;  /* dead slot, compacted after the batch */
}

typedef struct {
    uint64_t key;
    int64_t slot;
} sortent;

static int cmp_ent(const void *x, const void *y)
{
    uint64_t a = ((const sortent *)x)->key, b = ((const sortent *)y)->key;
    return a < b ? -1 : (a > b);
}

/* drop dead slots and restore depth-first leaf order */
static void compact(vo_amr *a)
{
    sortent *e = malloc(sizeof(sortent) * (a->n ? a->n : 1));
    int64_t m = 0;
    for (int64_t i = 0; i < a->n; ++i)
        if (a->lev[i] >= 0) {
            e[m].key = dfs_key(a, a->lev[i], a->cx + 3 * i);
            e[m].slot = i;
            ++m;
        }
    qsort(e, m, sizeof(sortent), cmp_ent);
    int32_t *lev = malloc(sizeof(int32_t) * a->cap);
    int64_t *cx = malloc(sizeof(int64_t) * 3 * a->cap);
    double *U = malloc(sizeof(double) * 5 * a->cap);
    for (int64_t k = 0; k < m; ++k) {
        int64_t s = e[k].slot;
        lev[k] = a->lev[s];
        memcpy(cx + 3 * k, a->cx + 3 * s, 3 * sizeof(int64_t));
        memcpy(U + 5 * k, a->U + 5 * s, 5 * sizeof(double));
    }
    free(a->lev);
    free(a->cx);
    free(a->U);
    a->lev = lev;
    a->cx = cx;
    a->U = U;
    a->n = m;
    free(e);
    h_rebuild(a, 0);
}

/* ---------------------------------------------------------------- API */

vo_amr *vo_amr_create(const vo_grid *g)
{
    vo_amr *a = calloc(1, sizeof(vo_amr));
    a->g = *g;
    a->nd = g->ndim;
    for (int d = 0; d < 3; ++d) {
        if (d >= a->nd) a->g.dims[d] = 1;
        a->w0[d] = d < a->nd ? (g->hi[d] - g->lo[d]) / (double)g->dims[d] : 1.0;
    }
    int64_t n = a->g.dims[0] * a->g.dims[1] * a->g.dims[2];
    grow(a, n);
    for (int64_t i = 0; i < n; ++i) {
        a->lev[i] = 0;
        a->cx[3 * i] = i % a->g.dims[0];
        a->cx[3 * i + 1] = (i / a->g.dims[0]) % a->g.dims[1];
        a->cx[3 * i + 2] = i / (a->g.dims[0] * a->g.dims[1]);
    }
    a->n = n;
    memset(a->U, 0, sizeof(double) * 5 * n);
    h_rebuild(a, 0);
    return a;
}

void vo_amr_destroy(vo_amr *a)
{
    if (!a) return;
    free(a->lev);
    free(a->cx);
    free(a->U);
    free(a->u0);
    free(a->acc);
    free(a->reg);
    free(a->hkey);
    free(a->hval);
    free(a);
}

int64_t vo_amr_nleaf(const vo_amr *a) { return a->n; }

void vo_amr_leaves(const vo_amr *a, int32_t *level, int64_t *coords)
{
    for (int64_t i = 0; i < a->n; ++i) {
        if (level) level[i] = a->lev[i];
        if (coords) memcpy(coords + 3 * i, a->cx + 3 * i, 3 * sizeof(int64_t));
    }
}

void vo_amr_set_state(vo_amr *a, const double *U)
{
    for (int64_t i = 0; i < a->n; ++i)
        for (int k = 0; k < 5; ++k) a->U[5 * i + k] = U[k * a->n + i];
}

void vo_amr_get_state(const vo_amr *a, double *U)
{
    for (int64_t i = 0; i < a->n; ++i)
        for (int k = 0; k < 5; ++k) U[k * a->n + i] = a->U[5 * i + k];
}

void vo_amr_set_time(vo_amr *a, double t, int64_t step)
{
    a->t = t;
    a->step = step;
}

double vo_amr_time(const vo_amr *a) { return a->t; }
int64_t vo_amr_steps(const vo_amr *a) { return a->step; }

int vo_amr_max_level(const vo_amr *a)
{
    int m = 0;
    for (int64_t i = 0; i < a->n; ++i) m = a->lev[i] > m ? a->lev[i] : m;
    return m;
}

int64_t vo_amr_refine(vo_amr *a, const int64_t *leaves, int64_t n)
{
    int32_t *l = malloc(sizeof(int32_t) * (n ? n : 1));
    int64_t *c = malloc(sizeof(int64_t) * 3 * (n ? n : 1));
    for (int64_t k = 0; k < n; ++k) {
        l[k] = a->lev[leaves[k]];
        memcpy(c + 3 * k, a->cx + 3 * leaves[k], 3 * sizeof(int64_t));
    }
    for (int64_t k = 0; k < n; ++k) refine_at(a, l[k], c + 3 * k);
    free(l);
    free(c);
    compact(a);
    return n;
}

/* density_gradient_indicator, src/driver.jl:406-420 */
static double indicator(const vo_amr *a, int64_t i)
{
    double W[5], Wn[5];
    prim(a, a->U, i, W);
    double rc = W[0], g = 0.0;
    for (int d = 0; d < a->nd; ++d)
        for (int hi = 0; hi < 2; ++hi) {
            int64_t j;
            if (!nb_query(a, i, d, hi, &j)) continue;
            prim(a, a->U, j, Wn);
            double rn = Wn[0];
            g = jmax(g, fabs(rn - rc) / jmax(jmax(rc, rn), 2.220446049250313e-16));
        }
    return g;
}

void vo_amr_indicator(const vo_amr *a, double *out)
{
    for (int64_t i = 0; i < a->n; ++i) out[i] = indicator(a, i);
}

int64_t vo_amr_regrid(vo_amr *a, double refine_above, int max_level)
{
    int64_t *tag = malloc(sizeof(int64_t) * (a->n ? a->n : 1)), m = 0;
    for (int64_t i = 0; i < a->n; ++i)
        if (a->lev[i] < max_level && indicator(a, i) > refine_above) tag[m++] = i;
    if (m) vo_amr_refine(a, tag, m);
    free(tag);
    return m;
}

double vo_amr_compute_dt(const vo_amr *a, int level)
{
    double invdt = 0.0, W[5];
    for (int64_t i = 0; i < a->n; ++i) {
        if (level >= 0 && a->lev[i] != level) continue;
        prim(a, a->U, i, W);
        double c = sqrt(a->g.gamma * W[4] / W[0]);
        for (int d = 0; d < a->nd; ++d)
            invdt = jmax(invdt, (fabs(W[1 + d]) + c) / width(a, a->lev[i], d));
    }
    if (invdt == 0.0) return INFINITY;
    return a->g.cfl / invdt;
}

void vo_amr_step(vo_amr *a, double dt, int level)
{
    step_impl(a, dt, level, NULL, NULL);
    if (level < 0) {
        a->t += dt;
        a->step += 1;
    }
}

/* evolve_level!, src/driver.jl:553-578 */
static double evolve_level(vo_amr *a, int level, double dt_target, int has_parent)
{
    double dt_stable = vo_amr_compute_dt(a, level);
    if (!isfinite(dt_stable)) return dt_target;
    double q = ceil(dt_target / dt_stable * (1 - 1e-12));
    int64_t n = q < 1.0 ? 1 : (int64_t)q;
    double dt_sub = dt_target / (double)n;
    int has_finer = level < vo_amr_max_level(a);
    regset rs = {0, {0, 0}, {0, 0}};
    for (int64_t s = 0; s < n; ++s) {
        if (has_finer)
            for (int64_t i = 0; i < a->n; ++i)
                if (a->lev[i] == level) memset(a->reg + 5 * i, 0, 5 * sizeof(double));
        rs.n = 0;
        if (has_parent) { rs.cl[rs.n] = level - 1; rs.scale[rs.n] = 1.0 * (0.5 * dt_sub); rs.n++; }
        if (has_finer) { rs.cl[rs.n] = level; rs.scale[rs.n] = -1.0 * (0.5 * dt_sub); rs.n++; }
        step_impl(a, dt_sub, level, rs.n ? &rs : NULL, rs.n ? &rs : NULL);
        if (has_finer) {
            evolve_level(a, level + 1, dt_sub, 1);
            /* _reflux_apply!, src/reflux.jl:91-101 */
            for (int64_t i = 0; i < a->n; ++i) {
                if (a->lev[i] != level) continue;
                double invV = 1.0 / cell_volume(a, level);
                for (int k = 0; k < 5; ++k) {
                    a->U[5 * i + k] = a->U[5 * i + k] - invV * a->reg[5 * i + k];
                    a->reg[5 * i + k] = 0.0;
                }
            }
        }
    }
    return dt_sub;
}

int64_t vo_amr_evolve(vo_amr *a, double tfinal, int64_t max_steps, double refine_above,
                      int max_level, int every, int subcycle)
{
    int64_t n = 0;
    while (a->t < tfinal * (1 - 1e-12)) {
        if (max_steps >= 0 && n >= max_steps) break;
        if (every > 0 && a->step % every == 0) vo_amr_regrid(a, refine_above, max_level);
        if (subcycle) {
            double dt_root = jmin(vo_amr_compute_dt(a, 0), tfinal - a->t);
            evolve_level(a, 0, dt_root, 0);
            a->t += dt_root;
            a->step += 1;
        } else {
            double dt = jmin(vo_amr_compute_dt(a, -1), tfinal - a->t);
            vo_amr_step(a, dt, -1);
        }
        ++n;
    }
    return n;
}

/* conserved_totals, src/diagnostics.jl:16-31 */
void vo_amr_totals(const vo_amr *a, double *out)
{
    for (int k = 0; k < 5; ++k) out[k] = 0.0;
    for (int64_t i = 0; i < a->n; ++i) {
        double v = cell_volume(a, a->lev[i]);
        for (int k = 0; k < 5; ++k) out[k] += a->U[5 * i + k] * v;
    }
}
