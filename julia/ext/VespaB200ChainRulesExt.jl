# VespaB200ChainRulesExt -- reverse-mode rule for LibVespaB200.evolve_steps
# through the device adjoint (vb_adjoint_*), so that Zygote or any
# ChainRulesCore-aware AD differentiates an objective of a device run.
#
# The differentiated map is the float64 evolve! of a periodic grid with each
# step's dt held at its forward value; minmod, the pressure floor and the HLLC
# wave pattern keep the branch the forward took.  The forward stores a
# checkpoint every `checkpoint_every` steps and the pullback recomputes each
# segment before its adjoint stages.
#
# Loaded when Vespa, LibVespaB200 and ChainRulesCore are loaded ([extensions]
# VespaB200ChainRulesExt = ["LibVespaB200", "ChainRulesCore"]).  Not run in
# this repository (no Julia in its build image).
module VespaB200ChainRulesExt

using Vespa
using LibVespaB200
using ChainRulesCore
const L = LibVespaB200

const CHECKPOINT_EVERY = 20

function ChainRulesCore.rrule(::typeof(L.evolve_steps), sim::Vespa.Simulation{<:L.B200Mesh},
                              U0::AbstractMatrix{Float64}, nsteps::Integer)
    g = sim.backend.grid == C_NULL ? (L.upload!(sim); sim.backend.grid) : sim.backend.grid
    L.check(L.vb_grid_upload(g, U0))
    adj = Ref{Ptr{Cvoid}}(C_NULL)
    L.check(L.vb_adjoint_create(g, Int64(nsteps), Int64(CHECKPOINT_EVERY), adj))
    t = Ref(0.0)
    n = Ref{Int64}(0)
    st = L.vb_adjoint_forward(adj[], Inf, Int64(nsteps), t, n)
    if st != L.VB_OK
        L.vb_adjoint_destroy(adj[])
        L.check(st)
    end
    UT = similar(U0)
    L.check(L.vb_grid_download(g, UT))
    handle = adj[]
    function evolve_steps_pullback(dUT)
        lam = Matrix{Float64}(collect(unthunk(dUT)))
        dU0 = similar(lam)
        st = L.vb_adjoint_backward(handle, lam, dU0)
        L.vb_adjoint_destroy(handle)
        L.check(st)
        return NoTangent(), NoTangent(), dU0, NoTangent()
    end
    return UT, evolve_steps_pullback
end

end # module
