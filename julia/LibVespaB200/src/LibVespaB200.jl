"""
    LibVespaB200

Julia bindings of `libvespa_b200.so`, the B200 (sm_100a) implementation of
Vespa.jl's finite-volume hydro step (C ABI: `include/vespa_b200.h`).

Three layers:
  1. raw bindings, one `ccall` per C entry point, same names and argument
     order as the header (every one returns the `Cint` status);
  2. `check`/`VespaB200Error`, turning a non-zero status into an exception
     that carries `vb_last_error`'s message;
  3. the backend objects a Vespa user constructs: `B200Flux` (the drop-in for
     `KAFlux` at `compute_face_fluxes!`) and `B200Mesh` (a device-resident
     uniform mesh).  Their Vespa methods live in the package extension
     `VespaB200FluxExt` (ext/VespaB200FluxExt.jl of Vespa.jl), loaded when
     both Vespa and this package are.

The library is found through the environment variable `VESPA_B200_LIB`, else
the path this package sits at in the repository
(`vespa.jl_b200/libvespa_b200.so`); the choice is fixed at precompile time.
"""
module LibVespaB200

export B200Flux, B200Mesh, VespaB200Error, check, upload!, download!, evolve_steps

# Generic functions whose methods for Vespa's Simulation{<:B200Mesh} come from
# the VespaB200FluxExt extension (this package does not depend on Vespa).
"`upload!(sim)`: host mirror -> device state (after host code wrote the state)."
function upload! end
"`download!(sim)`: device state -> host mirror."
function download! end
"""
`evolve_steps(sim, U0, nsteps) -> U`: `nsteps` CFL steps of the device grid
from the conserved state `U0` (ncell x 5, field-major); the function that the
ChainRulesCore extension differentiates with the device adjoint.
"""
function evolve_steps end

const libvespa_b200 = get(ENV, "VESPA_B200_LIB",
                          normpath(joinpath(@__DIR__, "..", "..", "..", "vespa.jl_b200",
                                            "libvespa_b200.so")))

# ---------------------------------------------------------------- constants
# vb_status
const VB_OK = 0
const VB_EINVAL = 1
const VB_ECUDA = 2
const VB_ENOMEM = 3
const VB_ENONFINITE = 4
const VB_ETIMEOUT = 5
const VB_ENOTSUP = 6
const STATUS_NAMES = Dict(0 => "VB_OK", 1 => "VB_EINVAL", 2 => "VB_ECUDA", 3 => "VB_ENOMEM",
                          4 => "VB_ENONFINITE", 5 => "VB_ETIMEOUT", 6 => "VB_ENOTSUP")
# boundary codes (MeshInterface Outflow / Periodic / Reflecting)
const VB_BC_OUTFLOW = Int32(0)
const VB_BC_PERIODIC = Int32(1)
const VB_BC_REFLECTING = Int32(2)
# precision modes
const VB_FP64 = Cint(0)
const VB_MIXED = Cint(1)
# grid options
const VB_OPT_KERNEL = Cint(1)
const VB_OPT_TILE_KZ = Cint(2)
const VB_OPT_TILE_TAPER = Cint(3)
const VB_KERNEL_AUTO = 0
const VB_KERNEL_CELL = 1
const VB_KERNEL_TILED = 2
# gravity preconditioners
const VB_GRAV_PRECOND_NONE = Int32(0)
const VB_GRAV_PRECOND_MG = Int32(1)
# MUSCL ghost fill
const VB_MUSCL_BC_NONE = Int32(0)
const VB_MUSCL_BC_PERIODIC = Int32(1)
const VB_NOALLOC_MAX_FACES = 65536
# step phases (vb_grid_step_phase)
const VB_PHASE_CFL = Cint(0)
const VB_PHASE_FINALIZE = Cint(1)
const VB_PHASE_STAGE1 = Cint(2)
const VB_PHASE_STAGE2 = Cint(3)
const VB_PHASE_ADVANCE = Cint(4)
# boundary-flux register modes and bflux_plane sources
const VB_BFLUX_OFF = Cint(0)
const VB_BFLUX_OUTER = Cint(1)
const VB_BFLUX_INTERIOR = Cint(2)
const VB_BFLUX_PLANE_LO = Cint(0)
const VB_BFLUX_PLANE_HI = Cint(1)
const VB_BFLUX_PLANE_INTERIOR = Cint(2)

# ------------------------------------------------------------------ structs
# Field for field the C structs of the header (same order, same widths).

"vb_problem_desc: a Problem on a uniform mesh (unused axes ignored)."
struct VbProblemDesc
    ndim::Int32
    bc_lo::NTuple{3,Int32}
    bc_hi::NTuple{3,Int32}
    flags::Int32
    dims::NTuple{3,Int64}
    lo::NTuple{3,Float64}
    hi::NTuple{3,Float64}
    gamma::Float64
    cfl::Float64
    aexp::Float64
end

"vb_gravity_desc: enable_gravity!'s options."
struct VbGravityDesc
    G::Float64
    tol::Float64
    maxiter::Int64
    bc_lo::NTuple{3,Int32}
    bc_hi::NTuple{3,Int32}
    project_mean::Int32
    precond::Int32
    flags::Int32
end

"vb_muscl_params: muscl_step_3d!'s keyword arguments."
struct VbMusclParams
    dt::Float64
    gamma::Float64
    theta::Float64
    dx::Float64
    small_rho::Float64
    bc::Int32
    flags::Int32
end

# ------------------------------------------------------------- raw bindings
vb_abi_version() =
    ccall((:vb_abi_version, libvespa_b200), Cint, ())
vb_last_error(buf, len) =
    ccall((:vb_last_error, libvespa_b200), Cint, (Ptr{UInt8}, Csize_t), buf, len)
vb_ctx_create(device, out) =
    ccall((:vb_ctx_create, libvespa_b200), Cint, (Cint, Ref{Ptr{Cvoid}}), device, out)
vb_ctx_destroy(ctx) =
    ccall((:vb_ctx_destroy, libvespa_b200), Cint, (Ptr{Cvoid},), ctx)
vb_ctx_synchronize(ctx) =
    ccall((:vb_ctx_synchronize, libvespa_b200), Cint, (Ptr{Cvoid},), ctx)
vb_ctx_stream(ctx, stream) =
    ccall((:vb_ctx_stream, libvespa_b200), Cint, (Ptr{Cvoid}, Ref{Ptr{Cvoid}}), ctx, stream)
vb_ctx_launch_count(ctx, count) =
    ccall((:vb_ctx_launch_count, libvespa_b200), Cint, (Ptr{Cvoid}, Ptr{Int64}), ctx, count)
vb_check_read(ctx, line) =
    ccall((:vb_check_read, libvespa_b200), Cint, (Ptr{Cvoid}, Ptr{Int64}), ctx, line)
vb_ctx_mark(ctx, slot) =
    ccall((:vb_ctx_mark, libvespa_b200), Cint, (Ptr{Cvoid}, Cint), ctx, slot)
vb_ctx_elapsed_ms(ctx, slot_a, slot_b, ms) =
    ccall((:vb_ctx_elapsed_ms, libvespa_b200), Cint, (Ptr{Cvoid}, Cint, Cint, Ptr{Float32}), ctx, slot_a, slot_b, ms)
vb_hllc_faces(ctx, nf, WL, WR, axis, gamma, F) =
    ccall((:vb_hllc_faces, libvespa_b200), Cint, (Ptr{Cvoid}, Int64, Ptr{Float64}, Ptr{Float64}, Ptr{Int32}, Float64, Ptr{Float64}), ctx, nf, WL, WR, axis, gamma, F)
vb_hllc_faces_device_async(ctx, nf, dWL, dWR, daxis, gamma, dF) =
    ccall((:vb_hllc_faces_device_async, libvespa_b200), Cint, (Ptr{Cvoid}, Int64, Ptr{Float64}, Ptr{Float64}, Ptr{Int32}, Float64, Ptr{Float64}), ctx, nf, dWL, dWR, daxis, gamma, dF)
vb_hllc_faces_noalloc(nf, WL, WR, axis, gamma, F, stream) =
    ccall((:vb_hllc_faces_noalloc, libvespa_b200), Cint, (Int64, Ptr{Float64}, Ptr{Float64}, Ptr{Int32}, Float64, Ptr{Float64}, Ptr{Cvoid}), nf, WL, WR, axis, gamma, F, stream)
vb_grid_create(ctx, desc, precision, out) =
    ccall((:vb_grid_create, libvespa_b200), Cint, (Ptr{Cvoid}, Ref{VbProblemDesc}, Cint, Ref{Ptr{Cvoid}}), ctx, desc, precision, out)
vb_grid_destroy(grid) =
    ccall((:vb_grid_destroy, libvespa_b200), Cint, (Ptr{Cvoid},), grid)
vb_grid_ncell(grid, ncell) =
    ccall((:vb_grid_ncell, libvespa_b200), Cint, (Ptr{Cvoid}, Ptr{Int64}), grid, ncell)
vb_grid_upload(grid, U) =
    ccall((:vb_grid_upload, libvespa_b200), Cint, (Ptr{Cvoid}, Ptr{Float64}), grid, U)
vb_grid_download(grid, U) =
    ccall((:vb_grid_download, libvespa_b200), Cint, (Ptr{Cvoid}, Ptr{Float64}), grid, U)
vb_grid_device_state(grid, dU) =
    ccall((:vb_grid_device_state, libvespa_b200), Cint, (Ptr{Cvoid}, Ref{Ptr{Float64}}), grid, dU)
vb_grid_set_option(grid, option, value) =
    ccall((:vb_grid_set_option, libvespa_b200), Cint, (Ptr{Cvoid}, Cint, Int64), grid, option, value)
vb_grid_get_option(grid, option, value) =
    ccall((:vb_grid_get_option, libvespa_b200), Cint, (Ptr{Cvoid}, Cint, Ptr{Int64}), grid, option, value)
vb_grid_autotune(grid, nsteps, best_kz, best_ms_per_step) =
    ccall((:vb_grid_autotune, libvespa_b200), Cint, (Ptr{Cvoid}, Cint, Ptr{Int64}, Ptr{Float64}), grid, nsteps, best_kz, best_ms_per_step)
vb_grid_set_time(grid, t, step) =
    ccall((:vb_grid_set_time, libvespa_b200), Cint, (Ptr{Cvoid}, Float64, Int64), grid, t, step)
vb_grid_get_time(grid, t, step) =
    ccall((:vb_grid_get_time, libvespa_b200), Cint, (Ptr{Cvoid}, Ptr{Float64}, Ptr{Int64}), grid, t, step)
vb_compute_dt(grid, dt) =
    ccall((:vb_compute_dt, libvespa_b200), Cint, (Ptr{Cvoid}, Ptr{Float64}), grid, dt)
vb_grid_selftest_wait(grid, limit_ns) =
    ccall((:vb_grid_selftest_wait, libvespa_b200), Cint, (Ptr{Cvoid}, Int64), grid, limit_ns)
vb_grid_set_zwindow(grid, zw0, zw1, zcls0, wz) =
    ccall((:vb_grid_set_zwindow, libvespa_b200), Cint, (Ptr{Cvoid}, Int64, Int64, Cint, Float64), grid, zw0, zw1, zcls0, wz)
vb_grid_step_phase(grid, phase) =
    ccall((:vb_grid_step_phase, libvespa_b200), Cint, (Ptr{Cvoid}, Cint), grid, phase)
vb_grid_planes(grid, which, z0, n, dev, put) =
    ccall((:vb_grid_planes, libvespa_b200), Cint, (Ptr{Cvoid}, Cint, Int64, Int64, Ptr{Cvoid}, Cint), grid, which, z0, n, dev, put)
vb_grid_cfl_bits(grid, dev, put) =
    ccall((:vb_grid_cfl_bits, libvespa_b200), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, Cint), grid, dev, put)
vb_step(grid, dt) =
    ccall((:vb_step, libvespa_b200), Cint, (Ptr{Cvoid}, Float64), grid, dt)
vb_evolve(grid, tfinal, max_steps, t, nsteps) =
    ccall((:vb_evolve, libvespa_b200), Cint, (Ptr{Cvoid}, Float64, Int64, Ptr{Float64}, Ptr{Int64}), grid, tfinal, max_steps, t, nsteps)
vb_run_steps_async(grid, nsteps) =
    ccall((:vb_run_steps_async, libvespa_b200), Cint, (Ptr{Cvoid}, Int64), grid, nsteps)
vb_conserved_totals(grid, out) =
    ccall((:vb_conserved_totals, libvespa_b200), Cint, (Ptr{Cvoid}, Ptr{Float64}), grid, out)
vb_grid_profile_step(grid, nsteps, ms_finalize, ms_stage1, ms_stage2) =
    ccall((:vb_grid_profile_step, libvespa_b200), Cint, (Ptr{Cvoid}, Cint, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}), grid, nsteps, ms_finalize, ms_stage1, ms_stage2)
vb_batch_create(ctx, nbox, descs, precision, out) =
    ccall((:vb_batch_create, libvespa_b200), Cint, (Ptr{Cvoid}, Cint, Ptr{VbProblemDesc}, Cint, Ref{Ptr{Cvoid}}), ctx, nbox, descs, precision, out)
vb_batch_destroy(batch) =
    ccall((:vb_batch_destroy, libvespa_b200), Cint, (Ptr{Cvoid},), batch)
vb_batch_ncell(batch, box, ncell) =
    ccall((:vb_batch_ncell, libvespa_b200), Cint, (Ptr{Cvoid}, Cint, Ptr{Int64}), batch, box, ncell)
vb_batch_upload(batch, box, U) =
    ccall((:vb_batch_upload, libvespa_b200), Cint, (Ptr{Cvoid}, Cint, Ptr{Float64}), batch, box, U)
vb_batch_download(batch, box, U) =
    ccall((:vb_batch_download, libvespa_b200), Cint, (Ptr{Cvoid}, Cint, Ptr{Float64}), batch, box, U)
vb_batch_run_steps(batch, nsteps) =
    ccall((:vb_batch_run_steps, libvespa_b200), Cint, (Ptr{Cvoid}, Int64), batch, nsteps)
vb_batch_run_steps_async(batch, nsteps) =
    ccall((:vb_batch_run_steps_async, libvespa_b200), Cint, (Ptr{Cvoid}, Int64), batch, nsteps)
vb_batch_autotune(batch, nsteps, best_cap, best_ms) =
    ccall((:vb_batch_autotune, libvespa_b200), Cint, (Ptr{Cvoid}, Cint, Ptr{Int64}, Ptr{Float64}), batch, nsteps, best_cap, best_ms)
vb_batch_get_time(batch, box, t, step) =
    ccall((:vb_batch_get_time, libvespa_b200), Cint, (Ptr{Cvoid}, Cint, Ptr{Float64}, Ptr{Int64}), batch, box, t, step)
vb_batch_conserved_totals(batch, box, out) =
    ccall((:vb_batch_conserved_totals, libvespa_b200), Cint, (Ptr{Cvoid}, Cint, Ptr{Float64}), batch, box, out)
vb_bflux_enable(grid, enable) =
    ccall((:vb_bflux_enable, libvespa_b200), Cint, (Ptr{Cvoid}, Cint), grid, enable)
vb_bflux_size(grid, n) =
    ccall((:vb_bflux_size, libvespa_b200), Cint, (Ptr{Cvoid}, Ptr{Int64}), grid, n)
vb_bflux_read(grid, out, n) =
    ccall((:vb_bflux_read, libvespa_b200), Cint, (Ptr{Cvoid}, Ptr{Float64}, Int64), grid, out, n)
vb_bflux_plane(grid, dim, source, start, stop, g0, flux_off, comp, vcell, out, n) =
    ccall((:vb_bflux_plane, libvespa_b200), Cint, (Ptr{Cvoid}, Cint, Cint, Ptr{Int64}, Ptr{Int64}, Ptr{Int64}, Int64, Cint, Float64, Ptr{Float64}, Int64), grid, dim, source, start, stop, g0, flux_off, comp, vcell, out, n)
vb_bflux_clear(grid) =
    ccall((:vb_bflux_clear, libvespa_b200), Cint, (Ptr{Cvoid},), grid)
vb_gravity_enable(grid, desc) =
    ccall((:vb_gravity_enable, libvespa_b200), Cint, (Ptr{Cvoid}, Ref{VbGravityDesc}), grid, desc)
vb_gravity_disable(grid) =
    ccall((:vb_gravity_disable, libvespa_b200), Cint, (Ptr{Cvoid},), grid)
vb_gravity_solve(grid, iters, relres) =
    ccall((:vb_gravity_solve, libvespa_b200), Cint, (Ptr{Cvoid}, Ptr{Int64}, Ptr{Float64}), grid, iters, relres)
vb_gravity_phi(grid, phi) =
    ccall((:vb_gravity_phi, libvespa_b200), Cint, (Ptr{Cvoid}, Ptr{Float64}), grid, phi)
vb_gravity_set_phi(grid, phi) =
    ccall((:vb_gravity_set_phi, libvespa_b200), Cint, (Ptr{Cvoid}, Ptr{Float64}), grid, phi)
vb_gravity_accel(grid, g) =
    ccall((:vb_gravity_accel, libvespa_b200), Cint, (Ptr{Cvoid}, Ptr{Float64}), grid, g)
vb_gravity_laplacian(grid, x, Ax) =
    ccall((:vb_gravity_laplacian, libvespa_b200), Cint, (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}), grid, x, Ax)
vb_muscl_create(ctx, dims, ng, out) =
    ccall((:vb_muscl_create, libvespa_b200), Cint, (Ptr{Cvoid}, Ptr{Int64}, Int32, Ref{Ptr{Cvoid}}), ctx, dims, ng, out)
vb_muscl_destroy(m) =
    ccall((:vb_muscl_destroy, libvespa_b200), Cint, (Ptr{Cvoid},), m)
vb_muscl_upload(m, U) =
    ccall((:vb_muscl_upload, libvespa_b200), Cint, (Ptr{Cvoid}, Ptr{Float64}), m, U)
vb_muscl_download(m, U) =
    ccall((:vb_muscl_download, libvespa_b200), Cint, (Ptr{Cvoid}, Ptr{Float64}), m, U)
vb_muscl_state(m, dU) =
    ccall((:vb_muscl_state, libvespa_b200), Cint, (Ptr{Cvoid}, Ref{Ptr{Float64}}), m, dU)
vb_muscl_step(m, p) =
    ccall((:vb_muscl_step, libvespa_b200), Cint, (Ptr{Cvoid}, Ref{VbMusclParams}), m, p)
vb_muscl_run_async(m, p, nsteps) =
    ccall((:vb_muscl_run_async, libvespa_b200), Cint, (Ptr{Cvoid}, Ref{VbMusclParams}, Int64), m, p, nsteps)
vb_muscl_step_fields(m, D, S1, S2, S3, Tau, p) =
    ccall((:vb_muscl_step_fields, libvespa_b200), Cint, (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ref{VbMusclParams}), m, D, S1, S2, S3, Tau, p)
vb_adjoint_create(grid, max_steps, checkpoint_every, out) =
    ccall((:vb_adjoint_create, libvespa_b200), Cint, (Ptr{Cvoid}, Int64, Int64, Ref{Ptr{Cvoid}}), grid, max_steps, checkpoint_every, out)
vb_adjoint_destroy(adj) =
    ccall((:vb_adjoint_destroy, libvespa_b200), Cint, (Ptr{Cvoid},), adj)
vb_adjoint_forward(adj, tfinal, max_steps, t, nsteps) =
    ccall((:vb_adjoint_forward, libvespa_b200), Cint, (Ptr{Cvoid}, Float64, Int64, Ptr{Float64}, Ptr{Int64}), adj, tfinal, max_steps, t, nsteps)
vb_adjoint_steps(adj, nsteps) =
    ccall((:vb_adjoint_steps, libvespa_b200), Cint, (Ptr{Cvoid}, Ptr{Int64}), adj, nsteps)
vb_adjoint_dts(adj, dts, n) =
    ccall((:vb_adjoint_dts, libvespa_b200), Cint, (Ptr{Cvoid}, Ptr{Float64}, Int64), adj, dts, n)
vb_adjoint_backward(adj, lam_final, lam_init) =
    ccall((:vb_adjoint_backward, libvespa_b200), Cint, (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}), adj, lam_final, lam_init)
vb_adjoint_step(adj, dt, lam_out, lam_in) =
    ccall((:vb_adjoint_step, libvespa_b200), Cint, (Ptr{Cvoid}, Float64, Ptr{Float64}, Ptr{Float64}), adj, dt, lam_out, lam_in)
vb_adjoint_timing(adj, ms) =
    ccall((:vb_adjoint_timing, libvespa_b200), Cint, (Ptr{Cvoid}, Ptr{Float64}), adj, ms)
vb_amr_create(ctx, base, out) =
    ccall((:vb_amr_create, libvespa_b200), Cint, (Ptr{Cvoid}, Ref{VbProblemDesc}, Ref{Ptr{Cvoid}}), ctx, base, out)
vb_amr_destroy(amr) =
    ccall((:vb_amr_destroy, libvespa_b200), Cint, (Ptr{Cvoid},), amr)
vb_amr_nleaf(amr, nleaf) =
    ccall((:vb_amr_nleaf, libvespa_b200), Cint, (Ptr{Cvoid}, Ptr{Int64}), amr, nleaf)
vb_amr_nface(amr, nface) =
    ccall((:vb_amr_nface, libvespa_b200), Cint, (Ptr{Cvoid}, Ptr{Int64}), amr, nface)
vb_amr_leaves(amr, level, coords) =
    ccall((:vb_amr_leaves, libvespa_b200), Cint, (Ptr{Cvoid}, Ptr{Int32}, Ptr{Int64}), amr, level, coords)
vb_amr_max_level(amr, level) =
    ccall((:vb_amr_max_level, libvespa_b200), Cint, (Ptr{Cvoid}, Ptr{Int32}), amr, level)
vb_amr_upload(amr, U) =
    ccall((:vb_amr_upload, libvespa_b200), Cint, (Ptr{Cvoid}, Ptr{Float64}), amr, U)
vb_amr_download(amr, U) =
    ccall((:vb_amr_download, libvespa_b200), Cint, (Ptr{Cvoid}, Ptr{Float64}), amr, U)
vb_amr_set_time(amr, t, step) =
    ccall((:vb_amr_set_time, libvespa_b200), Cint, (Ptr{Cvoid}, Float64, Int64), amr, t, step)
vb_amr_get_time(amr, t, step) =
    ccall((:vb_amr_get_time, libvespa_b200), Cint, (Ptr{Cvoid}, Ptr{Float64}, Ptr{Int64}), amr, t, step)
vb_amr_refine(amr, leaves, n) =
    ccall((:vb_amr_refine, libvespa_b200), Cint, (Ptr{Cvoid}, Ptr{Int64}, Int64), amr, leaves, n)
vb_amr_indicator(amr, out) =
    ccall((:vb_amr_indicator, libvespa_b200), Cint, (Ptr{Cvoid}, Ptr{Float64}), amr, out)
vb_amr_regrid(amr, refine_above, max_level, ntagged) =
    ccall((:vb_amr_regrid, libvespa_b200), Cint, (Ptr{Cvoid}, Float64, Cint, Ptr{Int64}), amr, refine_above, max_level, ntagged)
vb_amr_compute_dt(amr, level, dt) =
    ccall((:vb_amr_compute_dt, libvespa_b200), Cint, (Ptr{Cvoid}, Cint, Ptr{Float64}), amr, level, dt)
vb_amr_step(amr, dt) =
    ccall((:vb_amr_step, libvespa_b200), Cint, (Ptr{Cvoid}, Float64), amr, dt)
vb_amr_step_level(amr, dt, level) =
    ccall((:vb_amr_step_level, libvespa_b200), Cint, (Ptr{Cvoid}, Float64, Cint), amr, dt, level)
vb_amr_evolve(amr, tfinal, max_steps, refine_above, max_level, every, subcycle, t, nsteps) =
    ccall((:vb_amr_evolve, libvespa_b200), Cint, (Ptr{Cvoid}, Float64, Int64, Float64, Cint, Cint, Cint, Ptr{Float64}, Ptr{Int64}), amr, tfinal, max_steps, refine_above, max_level, every, subcycle, t, nsteps)
vb_amr_regrid_ms(amr, ms) =
    ccall((:vb_amr_regrid_ms, libvespa_b200), Cint, (Ptr{Cvoid}, Ptr{Float64}), amr, ms)
vb_amr_conserved_totals(amr, out) =
    ccall((:vb_amr_conserved_totals, libvespa_b200), Cint, (Ptr{Cvoid}, Ptr{Float64}), amr, out)

# ------------------------------------------------------------------- errors
struct VespaB200Error <: Exception
    status::Int
    message::String
end
Base.showerror(io::IO, e::VespaB200Error) =
    print(io, get(STATUS_NAMES, e.status, string(e.status)), ": ", e.message)

"The calling thread's last error message."
function last_error()
    buf = Vector{UInt8}(undef, 1024)
    vb_last_error(buf, length(buf))
    return unsafe_string(pointer(buf))
end

"Throw `VespaB200Error` for a non-zero status; return nothing otherwise."
check(st::Integer) = st == VB_OK ? nothing : throw(VespaB200Error(Int(st), last_error()))

# ----------------------------------------------------------------- contexts
"One CUDA device and stream (`vb_ctx`); destroyed by its finalizer."
mutable struct Context
    handle::Ptr{Cvoid}
    device::Int
    function Context(device::Integer = 0)
        r = Ref{Ptr{Cvoid}}(C_NULL)
        check(vb_ctx_create(Cint(device), r))
        c = new(r[], Int(device))
        finalizer(x -> (x.handle == C_NULL || vb_ctx_destroy(x.handle); x.handle = C_NULL), c)
        return c
    end
end

const _default_ctx = Dict{Int,Context}()
const _ctx_lock = ReentrantLock()
"The process-wide context of `device`, created on first use."
default_context(device::Integer = 0) =
    lock(_ctx_lock) do
        get!(() -> Context(device), _default_ctx, Int(device))
    end

# ------------------------------------------------------- the flux drop-in
"""
    B200Flux(device = 0)

Flux backend for `sim.flux`: the drop-in replacement of `KAFlux(CUDABackend())`
at `Vespa.compute_face_fluxes!` (src/ka_flux.jl:40-53).  Its method is defined
by the `VespaB200FluxExt` extension and calls `vb_hllc_faces`.
"""
struct B200Flux
    ctx::Context
end
B200Flux(device::Integer = 0) = B200Flux(default_context(device))

# Float64 pointer to face data of any dense layout (a Vector{NTuple{5,Float64}}
# or a 5 x nf Matrix{Float64}); the caller keeps the array alive (GC.@preserve)
_f64ptr(x::DenseArray) = Ptr{Float64}(pointer(x))

"""
    hllc_faces!(ctx, F, WL, WR, axis, gamma)

`vb_hllc_faces` on face data holding 5 Float64 per face (a
`Vector{NTuple{5,Float64}}` or a 5 x nf matrix), 1-based `Int32` axes.
"""
function hllc_faces!(ctx::Context, F::DenseArray, WL::DenseArray, WR::DenseArray,
                     axis::Vector{Int32}, gamma::Real)
    nf = length(axis)
    (sizeof(F) == sizeof(WL) == sizeof(WR) == 40nf) ||
        throw(DimensionMismatch("face data must hold 5 Float64 per face"))
    nf == 0 && return F
    GC.@preserve F WL WR begin
        check(vb_hllc_faces(ctx.handle, Int64(nf), _f64ptr(WL), _f64ptr(WR), axis,
                            Float64(gamma), _f64ptr(F)))
    end
    return F
end

"""
    hllc_faces_noalloc!(F, WL, WR, axis, gamma; stream = C_NULL)

`vb_hllc_faces_noalloc`: the same fluxes without any device allocation (for a
process whose GPU memory belongs to another allocator), at most
`VB_NOALLOC_MAX_FACES` faces per call, on the current device and `stream`.
"""
function hllc_faces_noalloc!(F::DenseArray, WL::DenseArray, WR::DenseArray,
                             axis::Vector{Int32}, gamma::Real; stream::Ptr{Cvoid} = C_NULL)
    nf = length(axis)
    (sizeof(F) == sizeof(WL) == sizeof(WR) == 40nf) ||
        throw(DimensionMismatch("face data must hold 5 Float64 per face"))
    GC.@preserve F WL WR begin
        check(vb_hllc_faces_noalloc(Int64(nf), _f64ptr(WL), _f64ptr(WR), axis,
                                    Float64(gamma), _f64ptr(F), stream))
    end
    return F
end

# ------------------------------------------------------ the device mesh
"""
    B200Mesh(dims, domain; precision = :fp64, device = 0, T = Float64)

A uniform mesh whose conserved state lives in GPU memory.  It forwards the
mesh interface (rank, cells, geometry, host field storage) to a RefMesh
`UniformMesh` with the same `dims` and `domain`, which holds the host mirror
of the state; the `VespaB200FluxExt` extension specialises `step!`,
`compute_dt`, `evolve!` and `conserved_totals` on `Simulation{<:B200Mesh}` to
run on the device (`vb_grid_*`).  `precision` is `:fp64` (bit-identical to
the float64 reference arithmetic) or `:mixed` (float32 reconstruction and
HLLC, float64 state and sums).

The device grid is created at the first device call from the simulation's
problem and filled from the host mirror.  After host code writes the state,
call `upload!(sim)`; after device steps, `download!(sim)` refreshes the host
mirror (`evolve!` does this once at its end).
"""
mutable struct B200Mesh{N,M}
    inner::M                 # RefMesh.UniformMesh{N}: geometry and host mirror
    precision::Cint
    ctx::Context
    grid::Ptr{Cvoid}         # vb_grid, C_NULL until the first device call
    device_newer::Bool       # the device state is ahead of the host mirror
end
function B200Mesh(inner; precision::Symbol = :fp64, device::Integer = 0)
    precision in (:fp64, :mixed) || throw(ArgumentError("precision must be :fp64 or :mixed"))
    N = length(inner.dims)
    m = B200Mesh{N,typeof(inner)}(inner, precision === :mixed ? VB_MIXED : VB_FP64,
                                  default_context(device), C_NULL, false)
    finalizer(x -> (x.grid == C_NULL || vb_grid_destroy(x.grid); x.grid = C_NULL), m)
    return m
end

"""
    problem_desc(dims, lo, hi, bc_lo, bc_hi, gamma, cfl; aexp = 1.0)

A `VbProblemDesc` from per-axis tuples (boundary codes `VB_BC_*`); axes beyond
`length(dims)` are filled as unused.
"""
function problem_desc(dims, lo, hi, bc_lo, bc_hi, gamma, cfl; aexp = 1.0)
    N = length(dims)
    pad(x, v, T) = ntuple(d -> d <= N ? T(x[d]) : T(v), 3)
    return VbProblemDesc(Int32(N), pad(bc_lo, 1, Int32), pad(bc_hi, 1, Int32), Int32(0),
                         pad(dims, 1, Int64), pad(lo, 0.0, Float64), pad(hi, 1.0, Float64),
                         Float64(gamma), Float64(cfl), Float64(aexp))
end

"""
    ensure_grid!(mesh, desc, U)

Create `mesh`'s device grid from `desc` and upload the host state `U` (5 x
ncell Float64, x fastest) unless it exists already.
"""
function ensure_grid!(m::B200Mesh, desc::VbProblemDesc, U)
    m.grid == C_NULL || return m.grid
    r = Ref{Ptr{Cvoid}}(C_NULL)
    check(vb_grid_create(m.ctx.handle, Ref(desc), m.precision, r))
    m.grid = r[]
    check(vb_grid_upload(m.grid, U))
    m.device_newer = false
    return m.grid
end

end # module
