/*
 * vespa_b200.h -- C ABI of libvespa_b200.so, the B200 (sm_100a) implementation
 * of Vespa.jl's finite-volume hydro step: PLM/minmod reconstruction, the HLLC
 * Riemann solver, the ideal-gas EOS, SSP-RK2 stages, the CFL reduction and the
 * conserved totals, with the state resident in device memory.
 *
 * Conventions (all entry points):
 *   - every function returns an int status (vb_status); 0 is success and no
 *     C++ exception crosses the ABI.  vb_last_error() returns the calling
 *     thread's last error message.
 *   - host pointers are borrowed for the duration of the call only; device
 *     buffers are owned by the opaque vb_ctx / vb_grid handles.
 *   - the conserved state is structure-of-arrays float64, five fields
 *     (rho, rho*vx, rho*vy, rho*vz, E), each ncell long, cells column-major
 *     with x fastest (Julia's CartesianIndices order, RefMesh field views).
 *   - face batches are 5 float64 per face, contiguous (Julia's
 *     Vector{NTuple{5,Float64}} reinterpreted as a 5 x nf matrix).
 *   - axes are 1-based (1 = x, 2 = y, 3 = z) as in the reference.
 *   - calls are ordered on the context's CUDA stream and return after the
 *     stream has drained unless the name ends in _async.
 *   - one context per host thread; a context is not thread-safe.
 */
#ifndef VESPA_B200_H
#define VESPA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VB_ABI_VERSION 1

typedef enum {
    VB_OK = 0,
    VB_EINVAL = 1,      /* bad argument */
    VB_ECUDA = 2,       /* CUDA runtime error (message in vb_last_error) */
    VB_ENOMEM = 3,      /* device or pinned allocation failed */
    VB_ENONFINITE = 4,  /* a non-finite or negative density/pressure reached the CFL reduction */
    VB_ETIMEOUT = 5,    /* a bounded device wait gave up */
    VB_ENOTSUP = 6      /* configuration the library does not support */
} vb_status;

/* Boundary conditions, lib/MeshInterface/src/MeshInterface.jl:74-83. */
enum { VB_BC_OUTFLOW = 0, VB_BC_PERIODIC = 1, VB_BC_REFLECTING = 2 };

/* Precision modes.  VB_FP64: every operation in float64 in the reference's
 * order, no fused multiply-add (bit-identical to the CPU restatement).
 * VB_MIXED: float64 state, pressure recovery, flux-difference accumulation and
 * reductions; float32 reconstruction and HLLC. */
enum { VB_FP64 = 0, VB_MIXED = 1 };

typedef struct vb_ctx vb_ctx;
typedef struct vb_grid vb_grid;

/* Uniform-mesh problem: mirrors Problem (src/problem.jl:20-50) on a RefMesh
 * UniformMesh (lib/RefMesh/src/RefMesh.jl:89-100).  Unused axes are ignored. */
typedef struct {
    int32_t ndim;        /* 1..3 */
    int32_t bc_lo[3];    /* VB_BC_* per axis, lo side */
    int32_t bc_hi[3];    /* VB_BC_* per axis, hi side */
    int32_t flags;       /* reserved, must be 0 */
    int64_t dims[3];     /* interior cells per axis */
    double lo[3];        /* domain lower bounds */
    double hi[3];        /* domain upper bounds */
    double gamma;        /* adiabatic index, IdealHydro(γ) src/equationset.jl:31-33 */
    double cfl;          /* Courant number, Problem.cfl */
    double aexp;         /* expansion factor in dt/(aexp*V), src/driver.jl:297-307; 1.0 without cosmology */
} vb_problem_desc;

int vb_abi_version(void);

/* Thread-local message of the last failed call; returns its full length. */
int vb_last_error(char *buf, size_t len);

/* Context: one CUDA device, one stream, cached scratch buffers. */
int vb_ctx_create(int device, vb_ctx **out);
int vb_ctx_destroy(vb_ctx *ctx);
int vb_ctx_synchronize(vb_ctx *ctx);
/* The context's cudaStream_t (as void*), e.g. to time it with CUDA events. */
int vb_ctx_stream(vb_ctx *ctx, void **stream);
/* Number of kernels this context has launched so far (graph nodes included). */
int vb_ctx_launch_count(vb_ctx *ctx, int64_t *count);
/* Device bounds checks of the check build (-DVB_CHECK: libvespa_b200_check.so,
 * `make -C vespa.jl_b200/csrc check`).  Waits for the context's stream, then
 * *line = 0 when no device bounds check failed since the last call, the
 * source line of the first failed check otherwise (the guarded access was
 * skipped), and -1 in the normal build, which has no checks.  Clears the
 * record. */
int vb_check_read(vb_ctx *ctx, int64_t *line);
/* CUDA-event timing on the context's stream (the reference's Instrumented
 * span timing, lib/MeshInterface/src/instrument.jl:30-95, moved to device
 * time): vb_ctx_mark records event `slot` (0..15); vb_ctx_elapsed_ms waits
 * for the later mark and returns the device time between two marks. */
int vb_ctx_mark(vb_ctx *ctx, int slot);
int vb_ctx_elapsed_ms(vb_ctx *ctx, int slot_a, int slot_b, float *ms);

/* Batched HLLC face fluxes from gathered left/right primitive states.
 * Replaces Vespa.compute_face_fluxes!(::KAFlux, model, F, WL, WR, axisv)
 * (ext/VespaKAFluxExt.jl:37-63; contract src/ka_flux.jl:40-53): WL, WR and F
 * are host arrays of 5*nf float64, axis holds nf 1-based axes, gamma is
 * adiabatic_index(model).  Bit-identical to HostBatchedFlux. */
int vb_hllc_faces(vb_ctx *ctx, int64_t nf, const double *WL, const double *WR,
                  const int32_t *axis, double gamma, double *F);
/* Same on device pointers, asynchronous on the context's stream. */
int vb_hllc_faces_device_async(vb_ctx *ctx, int64_t nf, const double *dWL, const double *dWR,
                               const int32_t *daxis, double gamma, double *dF);

/* No counterpart in the reference.  vb_hllc_faces without any device
 * allocation, for callers that own all of the GPU's memory (a pool allocator
 * that must not see foreign cudaMalloc/cudaFree, which synchronise the device
 * and fragment the pool, or memory reserved up front).  The host arrays are
 * staged in a fixed array compiled into the library, so at most
 * VB_NOALLOC_MAX_FACES faces per call (larger nf returns VB_EINVAL); every
 * GPU that loads the library holds that array (about 7.75 MiB) until exit.
 * Runs on the calling thread's current device and `stream` (a cudaStream_t,
 * NULL for the default stream) and returns after the results are in F.
 * The first call on a device looks up the array's device address in the
 * current context (again whenever a later call finds another context current,
 * e.g. after cudaDeviceReset); make that first call before any stream capture.
 * All calls share the array: calls whose work overlaps on the GPU race and
 * must be serialised by the caller. */
#define VB_NOALLOC_MAX_FACES 65536
int vb_hllc_faces_noalloc(int64_t nf, const double *WL, const double *WR, const int32_t *axis,
                          double gamma, double *F, void *stream);

/* Device-resident uniform grid: Simulation(UniformMesh, prob) state, u0 and
 * stage buffers (src/driver.jl:27-79).  precision is VB_FP64 or VB_MIXED. */
int vb_grid_create(vb_ctx *ctx, const vb_problem_desc *desc, int precision, vb_grid **out);
int vb_grid_destroy(vb_grid *grid);
int vb_grid_ncell(const vb_grid *grid, int64_t *ncell);
/* State I/O: 5*ncell float64 host arrays (the `sv` field views). */
int vb_grid_upload(vb_grid *grid, const double *U);
int vb_grid_download(vb_grid *grid, double *U);
/* Device pointer of the state (5*ncell float64), valid until vb_grid_destroy. */
int vb_grid_device_state(vb_grid *grid, double **dU);
/* Kernel selection and tuning knobs (no counterpart in the reference, whose
 * per-face loop has no launch shape).  VB_OPT_KERNEL: VB_KERNEL_AUTO picks the
 * tiled 3D kernel when the grid allows it (nx, ny multiples of 16, nz >= 2),
 * VB_KERNEL_CELL forces the cell-centric kernel, VB_KERNEL_TILED requires the
 * tiled one.  VB_OPT_TILE_KZ: z planes per tiled work item.
 * VB_OPT_TILE_TAPER: -1 (default) lets the autotuner choose whether the 3D
 * work queue's last z chunks taper (untuned: VB_MIXED grids taper), 0 keeps
 * uniform chunks, 1 tapers in either precision.  Results do not depend on
 * any of these knobs. */
enum { VB_OPT_KERNEL = 1, VB_OPT_TILE_KZ = 2, VB_OPT_TILE_TAPER = 3 };
enum { VB_KERNEL_AUTO = 0, VB_KERNEL_CELL = 1, VB_KERNEL_TILED = 2 };
int vb_grid_set_option(vb_grid *grid, int option, int64_t value);
int vb_grid_get_option(const vb_grid *grid, int option, int64_t *value);
/* Autotuner (no counterpart in the reference): times the tiled kernel's
 * z-chunk candidates (16 .. 128 planes) on this grid for nsteps CFL steps
 * each -- on 3D grids with VB_OPT_TILE_TAPER at -1 both as uniform and as
 * tapered work queues -- keeps the fastest, and restores the state and clock.  The choice is
 * cached for the process per (device, dims, boundaries, precision) and later
 * grids of the same kind start from it.  Allocates one state-sized scratch
 * buffer for the duration of the call.  No-op (returns the current kz) when
 * the grid uses the cell-centric kernel. */
int vb_grid_autotune(vb_grid *grid, int nsteps, int64_t *best_kz, double *best_ms_per_step);
/* Simulation clock (sim.t, sim.step). */
int vb_grid_set_time(vb_grid *grid, double t, int64_t step);
int vb_grid_get_time(vb_grid *grid, double *t, int64_t *step);

/* compute_dt(sim), src/driver.jl:169-199: cfl / max over cells and axes of
 * (|v_d| + c) / w_d; +Inf when the gas is at rest. */
int vb_compute_dt(vb_grid *grid, double *dt);
/* Slab decomposition of one grid across GPUs (no counterpart in the
 * reference, which runs on one host): a rank's grid holds its z slab plus
 * ghost planes copied from its neighbours.  vb_grid_set_zwindow marks planes
 * zw0 <= z < zw1 as the rank's own (the CFL maximum and the totals cover them
 * only), gives plane zw0 the lo-face order class zcls0 it has in the whole
 * domain (0 emitted by the plane below, 1 by itself: a wall, 2 by the
 * periodic partner above; -1 keeps the slab's own) and sets the z cell width
 * wz of the whole domain (areas and volume follow).  3D grids on the tiled
 * kernel only, without gravity or boundary-flux recording. */
int vb_grid_set_zwindow(vb_grid *grid, int64_t zw0, int64_t zw1, int zcls0, double wz);
/* One step in phases, queued on the context's stream, so the ranks can
 * all-reduce the CFL maximum (vb_grid_cfl_bits) and exchange ghost planes
 * (vb_grid_planes) between them: CFL (fold the current state's maximum if
 * stale), FINALIZE (dt from the maximum), STAGE1, STAGE2, ADVANCE (clock). */
enum { VB_PHASE_CFL = 0, VB_PHASE_FINALIZE = 1, VB_PHASE_STAGE1 = 2, VB_PHASE_STAGE2 = 3,
       VB_PHASE_ADVANCE = 4 };
int vb_grid_step_phase(vb_grid *grid, int phase);
/* Copy n whole z planes from plane z0 of the state (which = 0) or the
 * stage-1 state (which = 1) to (put = 0) or from (put = 1) the device buffer
 * dev, laid out [5 fields][n planes][ny][nx] float64. */
int vb_grid_planes(vb_grid *grid, int which, int64_t z0, int64_t n, void *dev, int put);
/* The running CFL maximum as one int64 device word at dev (put = 0 reads it
 * out, put = 1 writes it back): non-negative doubles compare like their bit
 * patterns, so an all-reduce max of the words is the max of the values. */
int vb_grid_cfl_bits(vb_grid *grid, void *dev, int put);
/* No counterpart in the reference: a self-test of the failure path.  Runs one
 * block that waits, bounded by limit_ns (1 us .. 10 s), on an mbarrier that
 * nothing completes, then takes the tiled stage kernels' abandon path, which
 * raises the grid's timeout flag; the call returns VB_ETIMEOUT exactly as a
 * stage whose TMA load never arrived would, clears the flag and leaves the
 * state and clock untouched. */
int vb_grid_selftest_wait(vb_grid *grid, int64_t limit_ns);
/* step!(sim, dt), src/driver.jl:333-359: one SSP-RK2 step, advances t. */
int vb_step(vb_grid *grid, double dt);
/* evolve!(sim), src/driver.jl:483-508: steps with dt = min(compute_dt,
 * tfinal - t) until t >= tfinal*(1-1e-12) or max_steps steps (max_steps < 0:
 * no limit).  dt is computed on the device; the loop runs as CUDA graphs. */
int vb_evolve(vb_grid *grid, double tfinal, int64_t max_steps, double *t, int64_t *nsteps);
/* nsteps CFL-limited steps without a final time, queued on the stream. */
int vb_run_steps_async(vb_grid *grid, int64_t nsteps);
/* conserved_totals(sim), src/diagnostics.jl:16-31: sum of U*V per field. */
int vb_conserved_totals(vb_grid *grid, double out[5]);
/* Profiling aid: runs nsteps CFL-limited steps with an event pair around
 * every launch and returns the mean device time of each kernel of the step
 * (dt finalisation, stage 1, stage 2) in milliseconds. */
int vb_grid_profile_step(vb_grid *grid, int nsteps, double *ms_finalize, double *ms_stage1,
                         double *ms_stage2);

/* Batch of independent uniform 3D problems stepped together (no counterpart
 * in the reference, which steps one Simulation at a time).  Every box keeps
 * its own state, clock and CFL dt (the per-box step is evolve!'s, src/driver.jl:
 * 483-508); one persistent kernel launch per RK2 stage covers the column
 * tiles of all boxes through one work queue (largest boxes first), and
 * vb_batch_run_steps replays the steps as a CUDA graph.  Each box must take
 * the tiled kernel: nx and ny multiples of 16, nz >= 2. */
typedef struct vb_batch vb_batch;
int vb_batch_create(vb_ctx *ctx, int nbox, const vb_problem_desc *descs, int precision,
                    vb_batch **out);
int vb_batch_destroy(vb_batch *batch);
/* Cells of box `box`, or of all boxes when box = -1. */
int vb_batch_ncell(const vb_batch *batch, int box, int64_t *ncell);
int vb_batch_upload(vb_batch *batch, int box, const double *U);
int vb_batch_download(vb_batch *batch, int box, double *U);
/* nsteps CFL-limited SSP-RK2 steps of every box; returns when done. */
int vb_batch_run_steps(vb_batch *batch, int64_t nsteps);
/* The same, queued on the context's stream without waiting. */
int vb_batch_run_steps_async(vb_batch *batch, int64_t nsteps);
/* Pick the depth of the batch's work items (16 x 16 x kz column tiles): the
 * default chunks (*best_cap = 0) or a cap of 16..128 planes on every box's
 * chunk, each timed over nsteps steps of the whole batch (CUDA-graph
 * replays, after a warm-up step).  States and clocks are restored; needs
 * device memory for a copy of every box's state.  Results do not depend on
 * the layout (same bits). */
int vb_batch_autotune(vb_batch *batch, int nsteps, int64_t *best_cap, double *best_ms);
int vb_batch_get_time(vb_batch *batch, int box, double *t, int64_t *step);
int vb_batch_conserved_totals(vb_batch *batch, int box, double out[5]);

/* Boundary-flux register (BoundaryFluxRegister, src/reflux.jl:113-146).
 * vb_bflux_enable(grid, VB_BFLUX_OUTER): while enabled, every domain-boundary
 * face accumulates (0.5*dt*F)*area per RK2 stage (_bflux_capture!,
 * src/reflux.jl:125-132) -- recorded by whichever stage kernel runs, the
 * tiled ones included.  VB_BFLUX_INTERIOR also records every interior face
 * (record_interior, _bflux_capture_interior!, src/reflux.jl:138-146; the
 * cell-centric kernel then runs).  VB_BFLUX_OFF stops recording and keeps the
 * values.  Changing between OUTER and INTERIOR reallocates a zeroed register.
 * Layout (vb_bflux_read): the outer planes per axis d (1..ndim) and side (lo,
 * hi), five components each, the flux axis collapsed and the other axes
 * column-major with the lowest axis fastest; then, with INTERIOR, per axis the
 * five components of every cell's hi face keyed by that (lo) cell, ncell
 * values each, zero where the hi side is a domain boundary. */
enum { VB_BFLUX_OFF = 0, VB_BFLUX_OUTER = 1, VB_BFLUX_INTERIOR = 2 };
int vb_bflux_enable(vb_grid *grid, int enable);
int vb_bflux_size(const vb_grid *grid, int64_t *n);
int vb_bflux_read(vb_grid *grid, double *out, int64_t n);
int vb_bflux_clear(vb_grid *grid);
/* bflux_plane(Val(R), dim, start, stop, g0, flux_off, comp, Vcell, lookup)
 * (src/reflux.jl:171-191) on the device: rasterises one face plane of the
 * register into out (n = prod(stop - start + 1) doubles, column-major, axis 0
 * fastest), each value the recorded flux component comp (1-based; comp <= 0
 * gives zeros) divided by vcell.  dim is the 0-based flux axis; start, stop
 * and g0 hold R = ndim global indices; along dim the active index is flux_off,
 * across it g - g0 + 1.  source replaces the reference's lookup closure:
 * VB_BFLUX_PLANE_LO / _HI read the outer register of that side (cells other
 * than the boundary cell read 0), VB_BFLUX_PLANE_INTERIOR the interior
 * register.  Cells outside the grid read 0. */
enum { VB_BFLUX_PLANE_LO = 0, VB_BFLUX_PLANE_HI = 1, VB_BFLUX_PLANE_INTERIOR = 2 };
int vb_bflux_plane(vb_grid *grid, int dim, int source, const int64_t *start, const int64_t *stop,
                   const int64_t *g0, int64_t flux_off, int comp, double vcell, double *out,
                   int64_t n);

/* Self-gravity on a uniform grid (src/gravity.jl): enable_gravity!,
 * solve_poisson!, apply_laplacian!, and the source g = -grad phi that
 * step!/evolve! add after each flux accumulation (+rho g on momentum, +rho v.g
 * on energy), with the free-fall limiter sqrt(4 pi G rho)/0.5 in compute_dt.
 *
 * The potential phi carries its own boundary codes: VB_BC_PERIODIC wraps,
 * any other code is a homogeneous Neumann wall.  The solver is matrix-free
 * conjugate gradients on A = -lap * V (the reference's operator, rows summed
 * in its order), warm-started from the stored phi, stopping when
 * ||r|| / ||b|| <= tol or after maxiter iterations; project_mean removes the
 * constant null mode of a fully periodic box (the reference's default for
 * periodic bcs).  Inner products are deterministic tree sums, so a solve
 * agrees with the reference's serial sums to the tolerance.
 *
 * While gravity is enabled: vb_evolve and vb_run_steps_async solve once per
 * step before the stages (evolve!, src/driver.jl:498) and synchronise with
 * the host for it; vb_step uses the field of the last solve (or set_phi), as
 * step! does; the stages of a 3D grid take the tiled kernels with the source
 * added (1D and 2D grids the cell-centric kernel).  The adjoint refuses a
 * grid with gravity (VB_ENOTSUP). */
enum {
    VB_GRAV_PRECOND_NONE = 0, /* plain CG (the reference's default) */
    VB_GRAV_PRECOND_MG = 1    /* CG preconditioned by one base-grid multigrid cycle
                                 (precond = :mg, ext/mg_pcg.jl); 3D cubic grids with
                                 periodic phi only, VB_ENOTSUP otherwise */
};

typedef struct {
    double G;          /* gravitational constant, code units */
    double tol;        /* relative residual target */
    int64_t maxiter;   /* CG iteration cap */
    int32_t bc_lo[3];  /* phi's boundary codes per axis */
    int32_t bc_hi[3];
    int32_t project_mean;
    int32_t precond;   /* VB_GRAV_PRECOND_* */
    int32_t flags;     /* must be 0 */
} vb_gravity_desc;

/* Enable (or reconfigure: phi is kept) gravity; phi starts at 0. */
int vb_gravity_enable(vb_grid *grid, const vb_gravity_desc *desc);
int vb_gravity_disable(vb_grid *grid);
/* solve_poisson!: iteration count and final relative residual. */
int vb_gravity_solve(vb_grid *grid, int64_t *iters, double *relres);
/* phi (ncell values, the state's cell order), read and written; writing it
 * recomputes g for the next vb_step. */
int vb_gravity_phi(vb_grid *grid, double *phi);
int vb_gravity_set_phi(vb_grid *grid, const double *phi);
/* g = -grad phi (ndim * ncell values, axis-major), as the stages use it. */
int vb_gravity_accel(vb_grid *grid, double *g);
/* Ax = A x with A = -lap * V: apply_laplacian!'s operator (src/gravity.jl:96-133)
 * in the row form of _lap_csr_cpu! (325-334), the one the solver iterates. */
int vb_gravity_laplacian(vb_grid *grid, const double *x, double *Ax);

/* lib/PPMKernels' unsplit MUSCL step, muscl_step_3d! (lib/PPMKernels/src/
 * muscl_grid.jl:314-380; Enzo HydroMethod=3): PLM with the minmod-theta
 * limiter on (rho, eint, v), HLL fluxes, SSP-RK2, float64, on five conserved
 * arrays D, S1, S2, S3, Tau (Tau = rho * specific total energy) of dims[3]
 * cells, x fastest, including ng >= 2 ghost zones per side (each dim >=
 * 2 ng + 1).  The active region per axis is ng .. dims - ng - 1 (0-based).
 * Ghost zones: VB_MUSCL_BC_NONE leaves them as they are, as the reference does
 * without a bc! callback; VB_MUSCL_BC_PERIODIC refills them from the opposite
 * side of the active region before each stage (needs each dim >= 3 ng).
 * Results are bit-identical to the reference's operation order. */
typedef struct vb_muscl vb_muscl;
enum { VB_MUSCL_BC_NONE = 0, VB_MUSCL_BC_PERIODIC = 1 };
typedef struct {
    double dt;
    double gamma;
    double theta;      /* limiter parameter (the reference's default 1.5) */
    double dx;
    double small_rho;  /* density and eint floor (default 1e-10) */
    int32_t bc;        /* VB_MUSCL_BC_* */
    int32_t flags;     /* must be 0 */
} vb_muscl_params;
/* Scratch for a grid of dims (and an owned state of 5 x N doubles, field-major).
 * ng >= 2; each dim >= 2 ng + 1; dims[1] <= 524280 and dims[2] <= 65535 (launch
 * grid); VB_EINVAL otherwise. */
int vb_muscl_create(vb_ctx *ctx, const int64_t dims[3], int32_t ng, vb_muscl **out);
int vb_muscl_destroy(vb_muscl *m);
int vb_muscl_upload(vb_muscl *m, const double *U);
int vb_muscl_download(vb_muscl *m, double *U);
/* device address of the owned state */
int vb_muscl_state(vb_muscl *m, double **dU);
/* one step of the owned state (synchronous) */
int vb_muscl_step(vb_muscl *m, const vb_muscl_params *p);
/* nsteps steps of the owned state, queued on the context's stream */
int vb_muscl_run_async(vb_muscl *m, const vb_muscl_params *p, int64_t nsteps);
/* one step of caller-owned device arrays of the handle's dims: the
 * signature of muscl_step_3d!(D, S1, S2, S3, Tau, dims, ng; ...) */
int vb_muscl_step_fields(vb_muscl *m, double *D, double *S1, double *S2, double *S3, double *Tau,
                         const vb_muscl_params *p);

/* Adjoint of the float64 SSP-RK2 step on a periodic grid (no counterpart in
 * the reference, which has no adjoint; it differentiates the map that
 * step!/evolve! apply, src/driver.jl:285-359,483-508).  Reverse mode, written
 * by hand: HLLC, minmod and the pressure floor keep the branches the forward
 * evaluation took, and each step's dt is held at its forward value.
 *
 * vb_adjoint_forward runs up to max_steps CFL-limited steps of the grid
 * (like vb_evolve), keeping a copy of the state every checkpoint_every steps
 * and every step's dt.  vb_adjoint_backward maps dJ/dU at the end of that run
 * (host, the state layout) to dJ/dU at its start, recomputing each segment
 * from its checkpoint.  Device memory: (ceil(max_steps/checkpoint_every) +
 * 2*checkpoint_every + 2 + 2*ndim) states.  checkpoint_every = 1 keeps a
 * tape instead: every step's state and stage-1 state (2*max_steps + 4 +
 * 2*ndim states), and the reverse sweep recomputes nothing.  The grid must
 * be VB_FP64 and periodic on every side (VB_ENOTSUP otherwise). */
typedef struct vb_adjoint vb_adjoint;
int vb_adjoint_create(vb_grid *grid, int64_t max_steps, int64_t checkpoint_every,
                      vb_adjoint **out);
int vb_adjoint_destroy(vb_adjoint *adj);
int vb_adjoint_forward(vb_adjoint *adj, double tfinal, int64_t max_steps, double *t,
                       int64_t *nsteps);
int vb_adjoint_steps(const vb_adjoint *adj, int64_t *nsteps);
/* dt of each recorded step; n must equal the recorded step count. */
int vb_adjoint_dts(const vb_adjoint *adj, double *dts, int64_t n);
int vb_adjoint_backward(vb_adjoint *adj, const double *lam_final, double *lam_init);
/* One step from the grid's current state with the given dt (the grid is not
 * advanced): lam_in = (dU^{n+1}/dU^n)^T lam_out. */
int vb_adjoint_step(vb_adjoint *adj, double dt, const double *lam_out, double *lam_in);
/* Device milliseconds of the last forward run, and of the last backward
 * sweep's recompute and adjoint stages. */
int vb_adjoint_timing(const vb_adjoint *adj, double ms[3]);

/* Composite AMR mesh (lib/HGBackend/src/HGBackend.jl semantics): the base
 * grid of `base` is a forest of root cells refined into a 2:1 face-balanced
 * cell tree whose leaves are the cells; float64 only.  Leaves are ordered
 * by root (column-major), then depth first with children x fastest; the state
 * is five float64 fields of nleaf values in that order.  Faces follow the
 * reference's emission rules (conforming faces from the hi side, coarse<->fine
 * sub-faces from the fine side with the fine area), PLM uses the
 * representative face neighbour (the first finer leaf when the neighbours are
 * finer), regrid is refine-only on the density-gradient indicator with
 * piecewise-constant prolongation (src/driver.jl:400-462), and the drivers
 * are evolve! with a RefinementPolicy, single rate or subcycled with flux
 * registers (src/driver.jl:483-605, src/reflux.jl:51-103). */
typedef struct vb_amr vb_amr;
int vb_amr_create(vb_ctx *ctx, const vb_problem_desc *base, vb_amr **out);
int vb_amr_destroy(vb_amr *amr);
int vb_amr_nleaf(const vb_amr *amr, int64_t *nleaf);
int vb_amr_nface(const vb_amr *amr, int64_t *nface);
/* level (0 = base) and integer coordinates at that level (3 per leaf) */
int vb_amr_leaves(const vb_amr *amr, int32_t *level, int64_t *coords);
int vb_amr_max_level(const vb_amr *amr, int32_t *level);
int vb_amr_upload(vb_amr *amr, const double *U);
int vb_amr_download(vb_amr *amr, double *U);
int vb_amr_set_time(vb_amr *amr, double t, int64_t step);
int vb_amr_get_time(const vb_amr *amr, double *t, int64_t *step);
/* refine! of the given leaves (indices in the current order), with balance */
int vb_amr_refine(vb_amr *amr, const int64_t *leaves, int64_t n);
/* density_gradient_indicator of every leaf */
int vb_amr_indicator(vb_amr *amr, double *out);
/* regrid!: refine leaves below max_level whose indicator exceeds refine_above */
int vb_amr_regrid(vb_amr *amr, double refine_above, int max_level, int64_t *ntagged);
/* compute_dt over one level (level < 0: every leaf); +Inf for an empty level */
int vb_amr_compute_dt(vb_amr *amr, int level, double *dt);
/* step!(sim, dt): one single-rate SSP-RK2 step, advances the clock */
int vb_amr_step(vb_amr *amr, double dt);
/* step!(sim, dt; level): only that level's leaves, clock unchanged */
int vb_amr_step_level(vb_amr *amr, double dt, int level);
/* evolve! with RefinementPolicy(refine_above, max_level, every); every <= 0
 * disables regrid; subcycle != 0 selects evolve_level! with flux registers. */
int vb_amr_evolve(vb_amr *amr, double tfinal, int64_t max_steps, double refine_above,
                  int max_level, int every, int subcycle, double *t, int64_t *nsteps);
/* device milliseconds spent in regrids during the last vb_amr_evolve */
int vb_amr_regrid_ms(const vb_amr *amr, double *ms);
int vb_amr_conserved_totals(vb_amr *amr, double out[5]);

#ifdef __cplusplus
}
#endif
#endif /* VESPA_B200_H */
