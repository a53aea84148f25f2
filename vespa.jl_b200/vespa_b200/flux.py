"""The batched flux backend: the drop-in for ``KAFlux``.

``compute_face_fluxes(backend, model, F, WL, WR, axisv)`` has the contract of
``Vespa.compute_face_fluxes!`` (src/ka_flux.jl:40-53): fill ``F[f]`` with the
HLLC flux across face ``f`` from the gathered primitive states ``WL[f]``,
``WR[f]`` and the 1-based face-normal axis ``axisv[f]``, mutate ``F`` and
return it.  ``B200Flux`` runs it on the GPU through ``vb_hllc_faces``
(replacing ext/VespaKAFluxExt.jl:37-63); results are bit-identical to the
reference's host loop (``HostBatchedFlux``).
"""
from __future__ import annotations

import numpy as np

from . import _lib


class AbstractFluxBackend:
    """Swappable flux backend (src/ka_flux.jl:28)."""


class B200Flux(AbstractFluxBackend):
    """GPU flux backend on a libvespa_b200 context."""

    def __init__(self, ctx: _lib.Context | None = None):
        self.ctx = ctx or _lib.default_context()


def _gamma_of(model) -> float:
    if hasattr(model, "adiabatic_index"):
        return float(model.adiabatic_index())
    return float(model)


def compute_face_fluxes(backend: AbstractFluxBackend, model, F: np.ndarray, WL: np.ndarray,
                        WR: np.ndarray, axisv) -> np.ndarray:
    """compute_face_fluxes!(backend, model, F, WL, WR, axisv).

    ``F``, ``WL``, ``WR`` are ``(nf, 5)`` float64 arrays (a Vector{NTuple{5}}
    in memory); ``axisv`` holds nf 1-based axes.  Returns ``F``."""
    if not isinstance(backend, B200Flux):
        raise TypeError(f"no compute_face_fluxes method for {type(backend).__name__}")
    nf = len(F)
    if nf == 0:
        return F
    for name, a in (("F", F), ("WL", WL), ("WR", WR)):
        if a.shape != (nf, 5) or a.dtype != np.float64 or not a.flags.c_contiguous:
            raise ValueError(f"{name} must be a C-contiguous ({nf}, 5) float64 array")
    ax = np.ascontiguousarray(axisv, dtype=np.int32)
    if ax.shape != (nf,):
        raise ValueError("axisv must have one entry per face")
    _lib.call("vb_hllc_faces", backend.ctx.handle, nf, _lib.dptr(WL), _lib.dptr(WR),
              _lib.i32ptr(ax), _gamma_of(model), _lib.dptr(F))
    return F
