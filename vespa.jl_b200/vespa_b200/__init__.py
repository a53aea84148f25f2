"""vespa_b200 -- host-side mirror of Vespa.jl's hydro-step API over libvespa_b200.

The compute path is the CUDA library (sm_100a) behind the C ABI in
include/vespa_b200.h; this package only marshals arguments and mirrors the
reference's public names (Simulation, step!, evolve!, compute_dt,
conserved_totals, compute_face_fluxes!, enable_gravity!, solve_poisson!).
"""
from ._lib import Context, VespaB200Error, default_context, load
from . import amr
from .amr import AmrMesh, AmrSimulation, RefinementPolicy
from .adjoint import Adjoint, EvolveFunction, evolve_with_adjoint, rho2_integral, rho2_seed
from .flux import AbstractFluxBackend, B200Flux, compute_face_fluxes
from .gravity import GravityField, apply_laplacian, disable_gravity, enable_gravity, solve_poisson
from .muscl import MusclGrid, muscl_step_3d
from .problem import (BC, IdealHydro, Outflow, Periodic, Problem, Reflecting, cons2prim,
                      initial_primitive, initial_state, kelvin_helmholtz_problem, prim2cons,
                      riemann_box_problem, sedov_problem, smooth_random_problem,
                      sod_problem_defaults, uniform01)
from .simulation import (B200Mesh, Batch, Simulation, Totals, cell_samples, compute_dt,
                         conserved_totals, dump_fields, evolve, primitive_at, primitive_state,
                         run_steps_async, step)

__all__ = [
    "Context", "VespaB200Error", "default_context", "load",
    "amr", "AmrMesh", "AmrSimulation", "RefinementPolicy",
    "Adjoint", "EvolveFunction", "evolve_with_adjoint", "rho2_integral", "rho2_seed",
    "AbstractFluxBackend", "B200Flux", "compute_face_fluxes",
    "GravityField", "apply_laplacian", "disable_gravity", "enable_gravity", "solve_poisson",
    "MusclGrid", "muscl_step_3d",
    "BC", "IdealHydro", "Outflow", "Periodic", "Problem", "Reflecting", "cons2prim",
    "initial_primitive", "initial_state", "kelvin_helmholtz_problem", "prim2cons",
    "riemann_box_problem", "sedov_problem", "smooth_random_problem", "sod_problem_defaults",
    "uniform01",
    "B200Mesh", "Batch", "Simulation", "Totals", "cell_samples", "compute_dt", "conserved_totals",
    "dump_fields", "evolve", "primitive_at", "primitive_state", "run_steps_async", "step",
]
