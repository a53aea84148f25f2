/*
 * vespa_oracle.h -- CPU oracle for the Vespa.jl finite-volume hydro step.
 *
 * TEST INFRASTRUCTURE ONLY.  The oracle is the checker: tests/, the smoke()
 * hook and bench.py's CPU-baseline leg may call it; the product library
 * (libvespa_b200.so) never links, loads or calls it.
 *
 * Parity status: the restatement is pinned against the known-answer tests the
 * reference keeps for this path (test/test_sod.jl:32-43 Sod vs the exact
 * Riemann solution and conservation; test/test_boundary_flux.jl:35 boundary
 * flux identity) and against Toro's published star state for the Sod problem.
 * The reference itself (Julia) cannot run in this container, so bit-level
 * agreement with the reference's own outputs is unpinned.
 *
 * Layout conventions shared with the product library:
 *   - state: structure of arrays, U[k * ncell + lin], k = 0..4 for
 *     (rho, mx, my, mz, E), lin = i + n0*(j + n1*kz) (x fastest, column-major
 *     like Julia's CartesianIndices);
 *   - face batches: 5 doubles per face contiguous (Julia's Vector{NTuple{5}}
 *     reinterpreted as a 5 x nf column-major matrix);
 *   - axes are 1-based (1=x, 2=y, 3=z) as in the reference.
 */
#ifndef VESPA_ORACLE_H
#define VESPA_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { VO_BC_OUTFLOW = 0, VO_BC_PERIODIC = 1, VO_BC_REFLECTING = 2 };

typedef struct {
    int32_t ndim;
    int32_t bc_lo[3];
    int32_t bc_hi[3];
    int32_t reserved;
    int64_t dims[3];
    double lo[3];
    double hi[3];
    double gamma;
    double cfl;
    double aexp;
} vo_grid;

/* per-cell / per-face kernels (src/eos.jl, src/reconstruct.jl, src/riemann.jl) */
void vo_cons2prim(const double *U, double gamma, double *W);
void vo_prim2cons(const double *W, double gamma, double *U);
double vo_minmod(double a, double b);
void vo_hllc_flux(const double *WL, const double *WR, double gamma, int dim, double *F);
void vo_compute_face_fluxes(int64_t nf, const double *WL, const double *WR,
                            const int32_t *axis, double gamma, double *F);

/* uniform-grid driver (src/driver.jl + lib/RefMesh/src/RefMesh.jl) */
int64_t vo_ncell(const vo_grid *g);
double vo_compute_dt(const vo_grid *g, const double *U);
void vo_accumulate_flux(const vo_grid *g, const double *U, double *acc,
                        double *bflux, double bscale);
void vo_accumulate_flux_gather(const vo_grid *g, const double *U, double *acc, int nthreads);
void vo_accumulate_flux_gather_range(const vo_grid *g, const double *U, double *acc, int64_t lin0,
                                     int64_t lin1, int nthreads);
double vo_invdt_range(const vo_grid *g, const double *U, int64_t lin0, int64_t lin1);
void vo_step(const vo_grid *g, double *U, double *u0, double *acc, double dt,
             double *bflux, int mode, int nthreads);
void vo_step_breg(const vo_grid *g, double *U, double *u0, double *acc, double dt, double *vals,
                  unsigned char *seen, double *ivals, unsigned char *iseen);
void vo_bflux_plane(const vo_grid *g, const double *vals, const unsigned char *seen,
                    const double *ivals, const unsigned char *iseen, int dim, int source,
                    const int64_t *start, const int64_t *stop, const int64_t *g0, int64_t flux_off,
                    int comp, double vcell, double *out);
int64_t vo_evolve(const vo_grid *g, double *U, double *u0, double *acc, double tfinal,
                  int64_t max_steps, double *t, int mode, int nthreads);
void vo_conserved_totals(const vo_grid *g, const double *U, double *out);
int64_t vo_bflux_size(const vo_grid *g);

/* self-gravity on the uniform mesh (src/gravity.jl): phi's own boundary codes
 * (VO_BC_PERIODIC wraps, anything else is a homogeneous Neumann wall) */
typedef struct {
    double G;
    double tol;
    int32_t bc_lo[3];
    int32_t bc_hi[3];
    int32_t maxiter;
    int32_t project_mean;
} vo_gravity;
void vo_grav_laplacian(const vo_grid *g, const vo_gravity *P, const double *x, double *out);
int64_t vo_grav_solve(const vo_grid *g, const vo_gravity *P, const double *U, double *phi,
                      double *relres);
void vo_grav_accel(const vo_grid *g, const vo_gravity *P, const double *phi, double *gacc);
double vo_compute_dt_gravity(const vo_grid *g, double G, const double *U);
void vo_step_gravity(const vo_grid *g, const double *gacc, double *U, double *u0, double *acc,
                     double dt);

/* lib/PPMKernels unsplit MUSCL step (muscl_step_3d!): U is 5 x N (D, S1, S2,
 * S3, Tau) over dims[3] with ng ghost zones; bc 0 leaves ghosts untouched, 1
 * fills them periodically before each stage. */
void vo_muscl_step(const int64_t dims[3], int ng, double dt, double gamma, double theta,
                   double dx, double small_rho, int bc, double *U);
/* muscl_flux_line! on one pencil: prim is 5 x na (rho, eint, vx, vy, vz); F is
 * 5 x (na - 2 ng + 1). */
void vo_muscl_flux_line(int64_t na, int ng, const double *prim, double gamma, double theta,
                        double small_rho, double *F);

/* exact Riemann solver (src/exact_riemann.jl) */
void vo_exact_riemann_star(const double *WL, const double *WR, double gamma, double *pu);
void vo_exact_riemann_sample(const double *WL, const double *WR, double gamma, double s,
                             double *out);


/* AMR (vespa_oracle_amr.c): composite leaf-only mesh over a base grid. */
typedef struct vo_amr vo_amr;
vo_amr *vo_amr_create(const vo_grid *g);
void vo_amr_destroy(vo_amr *a);
int64_t vo_amr_nleaf(const vo_amr *a);
void vo_amr_leaves(const vo_amr *a, int32_t *level, int64_t *coords);
void vo_amr_set_state(vo_amr *a, const double *U);
void vo_amr_get_state(const vo_amr *a, double *U);
void vo_amr_set_time(vo_amr *a, double t, int64_t step);
double vo_amr_time(const vo_amr *a);
int64_t vo_amr_steps(const vo_amr *a);
int vo_amr_max_level(const vo_amr *a);
int64_t vo_amr_refine(vo_amr *a, const int64_t *leaves, int64_t n);
void vo_amr_indicator(const vo_amr *a, double *out);
int64_t vo_amr_regrid(vo_amr *a, double refine_above, int max_level);
double vo_amr_compute_dt(const vo_amr *a, int level);
void vo_amr_step(vo_amr *a, double dt, int level);
int64_t vo_amr_evolve(vo_amr *a, double tfinal, int64_t max_steps, double refine_above,
                      int max_level, int every, int subcycle);
void vo_amr_totals(const vo_amr *a, double *out);

#ifdef __cplusplus
}
#endif
#endif
