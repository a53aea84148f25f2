# VespaB200FluxExt -- the libvespa_b200 backend of Vespa.jl, in place of
# VespaKAFluxExt (ext/VespaKAFluxExt.jl) as the device path.
#
# Loaded when Vespa and LibVespaB200 are both loaded (Project.toml:
# [weakdeps] LibVespaB200, [extensions] VespaB200FluxExt = "LibVespaB200").
# Two levels:
#   1. compute_face_fluxes!(::B200Flux, ...) -- the batched-face boundary of
#      src/ka_flux.jl:40-53, bit-identical to HostBatchedFlux;
#   2. Simulation{<:B200Mesh} -- the state stays in GPU memory and step!,
#      compute_dt, evolve! and conserved_totals (src/driver.jl:169-199,
#      333-359, 483-508; src/diagnostics.jl:16-31) run on the device.  The
#      mesh interface is forwarded to the RefMesh UniformMesh inside the
#      B200Mesh, which holds the host mirror of the state, so Simulation
#      construction, initial conditions and host diagnostics are unchanged.
#
# Not run in this repository (no Julia in its build image): the test suite
# checks every ccall signature against include/vespa_b200.h mechanically.
module VespaB200FluxExt

using Vespa
using MeshInterface
using LibVespaB200
const L = LibVespaB200
const MI = MeshInterface

# ----------------------------------------------------------- 1. face batches
# Same contract as the KAFlux method (ext/VespaKAFluxExt.jl:37-63): F, WL, WR
# are Vector{NTuple{5,Float64}}, axisv the 1-based face axes.
function Vespa.compute_face_fluxes!(b::L.B200Flux, model, F, WL, WR, axisv)
    nf = length(F)
    nf == 0 && return F
    eltype(eltype(F)) === Float64 ||
        throw(ArgumentError("B200Flux computes Float64 face batches"))
    L.hllc_faces!(b.ctx, F, WL, WR, convert(Vector{Int32}, axisv), Vespa.adiabatic_index(model))
    return F
end

# ------------------------------------------------ 2. the mesh interface
for f in (:rank, :domain, :n_cells, :max_level, :field_eltype, :coord_eltype)
    @eval MI.$f(m::L.B200Mesh) = MI.$f(m.inner)
end
for f in (:level_of, :cell_center, :cell_width, :cell_volume, :face_area, :neighbor,
          :face_neighbor_handles, :field_view, :restrict!, :prolong!)
    @eval MI.$f(m::L.B200Mesh, args...; kw...) = MI.$f(m.inner, args...; kw...)
end
MI.for_each_cell(f, m::L.B200Mesh; kw...) = MI.for_each_cell(f, m.inner; kw...)
MI.for_each_face(f, m::L.B200Mesh; kw...) = MI.for_each_face(f, m.inner; kw...)
MI.allocate_fields(m::L.B200Mesh, spec::MI.FieldSpec; kw...) =
    MI.allocate_fields(m.inner, spec; kw...)

const B200Sim = Vespa.Simulation{<:L.B200Mesh}

# boundary code of one side (lib/MeshInterface/src/MeshInterface.jl:74-83)
_bc_code(::MI.Outflow) = L.VB_BC_OUTFLOW
_bc_code(::MI.Periodic) = L.VB_BC_PERIODIC
_bc_code(::MI.Reflecting) = L.VB_BC_REFLECTING
_bc_code(bc) = throw(ArgumentError("$(typeof(bc)) has no device form (ParentGhost needs a host callback)"))

function _desc(sim::B200Sim)
    sim.cosmo === nothing || throw(ArgumentError("B200Mesh: cosmological expansion is not supported"))
    m = sim.backend.inner
    N = length(m.dims)
    lo = ntuple(d -> _bc_code(MI.bc_on(sim.bcs, d, :lo)), N)
    hi = ntuple(d -> _bc_code(MI.bc_on(sim.bcs, d, :hi)), N)
    return L.problem_desc(m.dims, m.lo, m.hi, lo, hi, Float64(sim.γ), Float64(sim.problem.cfl))
end

# the host mirror as one 5 x ncell field-major array (x fastest within a field)
function _host_state(sim::B200Sim)
    n = MI.n_cells(sim.backend)
    U = Matrix{Float64}(undef, n, 5)
    for k in 1:5
        copyto!(view(U, :, k), vec(sim.sv[k]))
    end
    return U
end

function _grid(sim::B200Sim)
    m = sim.backend
    m.grid == C_NULL && L.ensure_grid!(m, _desc(sim), _host_state(sim))
    return m.grid
end

function L.upload!(sim::B200Sim)
    m = sim.backend
    U = _host_state(sim)
    m.grid == C_NULL ? L.ensure_grid!(m, _desc(sim), U) : L.check(L.vb_grid_upload(m.grid, U))
    L.check(L.vb_grid_set_time(m.grid, Float64(sim.t), Int64(sim.step)))
    m.device_newer = false
    return sim
end

function L.download!(sim::B200Sim)
    m = sim.backend
    (m.grid == C_NULL || !m.device_newer) && return sim
    n = MI.n_cells(m)
    U = Matrix{Float64}(undef, n, 5)
    L.check(L.vb_grid_download(m.grid, U))
    for k in 1:5
        copyto!(vec(sim.sv[k]), view(U, :, k))
    end
    m.device_newer = false
    return sim
end

function Vespa.compute_dt(sim::B200Sim; level = nothing)
    level === nothing || throw(ArgumentError("B200Mesh is single-level"))
    sim.grav === nothing || throw(ArgumentError("B200Mesh: enable gravity through vb_gravity_enable"))
    dt = Ref(0.0)
    L.check(L.vb_compute_dt(_grid(sim), dt))
    return dt[]
end

function Vespa.step!(sim::B200Sim, dt::Real; level = nothing, bflux = nothing)
    level === nothing || throw(ArgumentError("B200Mesh is single-level"))
    bflux === nothing ||
        throw(ArgumentError("B200Mesh records boundary fluxes through vb_bflux_enable/vb_bflux_read"))
    L.check(L.vb_step(_grid(sim), Float64(dt)))
    sim.t += dt          # the device clock advances the same way
    sim.step += 1
    sim.backend.device_newer = true
    return sim
end

# evolve! (src/driver.jl:483-508): without a policy, callback or subcycling the
# whole loop runs on the device (dt never leaves it); otherwise the reference's
# loop drives the device step!/compute_dt and refreshes the host mirror before
# every callback.
function Vespa.evolve!(sim::B200Sim; verbose::Bool = false, policy = nothing,
                       callback = nothing, callback_every::Int = 1, subcycle::Bool = false)
    (policy === nothing && !subcycle) ||
        throw(ArgumentError("B200Mesh is single-level: use the vb_amr_* mesh for AMR"))
    tfinal = sim.problem.tfinal
    g = _grid(sim)
    if callback === nothing
        L.check(L.vb_grid_set_time(g, Float64(sim.t), Int64(sim.step)))
        t = Ref(0.0)
        n = Ref{Int64}(0)
        L.check(L.vb_evolve(g, Float64(tfinal), Int64(-1), t, n))
        sim.t = t[]
        sim.step += n[]
        sim.backend.device_newer = true
        L.download!(sim)
        verbose && println("evolve!: $(n[]) device steps, t = $(sim.t)")
        return sim
    end
    L.download!(sim)
    callback(sim, :init)
    while sim.t < tfinal * (1 - 1e-12)
        dt = min(Vespa.compute_dt(sim), tfinal - sim.t)
        Vespa.step!(sim, dt)
        if callback_every > 0 && sim.step % callback_every == 0
            L.download!(sim)
            callback(sim, :step)
        end
    end
    L.download!(sim)
    return sim
end

function Vespa.conserved_totals(sim::B200Sim)
    tot = zeros(5)
    L.check(L.vb_conserved_totals(_grid(sim), tot))
    return (mass = tot[1], momentum_x = tot[2], momentum_y = tot[3], momentum_z = tot[4],
            energy = tot[5])
end

# evolve_steps: the primal that VespaB200ChainRulesExt differentiates
function L.evolve_steps(sim::B200Sim, U0::AbstractMatrix{Float64}, nsteps::Integer)
    g = _grid(sim)
    L.check(L.vb_grid_upload(g, U0))
    t = Ref(0.0)
    n = Ref{Int64}(0)
    L.check(L.vb_evolve(g, Inf, Int64(nsteps), t, n))
    U = similar(U0)
    L.check(L.vb_grid_download(g, U))
    return U
end

end # module
