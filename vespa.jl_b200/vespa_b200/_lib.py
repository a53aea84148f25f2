"""ctypes binding of libvespa_b200.so (the C ABI declared in include/vespa_b200.h).

There is no CPU fallback: loading fails loudly when the shared library is
missing, and every entry point raises ``VespaB200Error`` on a non-zero status.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(PKG_DIR), "libvespa_b200.so")

VB_OK, VB_EINVAL, VB_ECUDA, VB_ENOMEM, VB_ENONFINITE, VB_ETIMEOUT, VB_ENOTSUP = range(7)
STATUS_NAMES = {0: "VB_OK", 1: "VB_EINVAL", 2: "VB_ECUDA", 3: "VB_ENOMEM", 4: "VB_ENONFINITE",
                5: "VB_ETIMEOUT", 6: "VB_ENOTSUP"}
BC_OUTFLOW, BC_PERIODIC, BC_REFLECTING = 0, 1, 2
FP64, MIXED = 0, 1
OPT_KERNEL, OPT_TILE_KZ, OPT_TILE_TAPER = 1, 2, 3
KERNELS = {"auto": 0, "cell": 1, "tiled": 2}
BFLUX_OFF, BFLUX_OUTER, BFLUX_INTERIOR = 0, 1, 2
PHASE_CFL, PHASE_FINALIZE, PHASE_STAGE1, PHASE_STAGE2, PHASE_ADVANCE = 0, 1, 2, 3, 4
BFLUX_PLANE_LO, BFLUX_PLANE_HI, BFLUX_PLANE_INTERIOR = 0, 1, 2


class VespaB200Error(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class ProblemDesc(C.Structure):
    """vb_problem_desc"""
    _fields_ = [
        ("ndim", C.c_int32),
        ("bc_lo", C.c_int32 * 3),
        ("bc_hi", C.c_int32 * 3),
        ("flags", C.c_int32),
        ("dims", C.c_int64 * 3),
        ("lo", C.c_double * 3),
        ("hi", C.c_double * 3),
        ("gamma", C.c_double),
        ("cfl", C.c_double),
        ("aexp", C.c_double),
    ]


class GravityDesc(C.Structure):
    """vb_gravity_desc"""
    _fields_ = [
        ("G", C.c_double),
        ("tol", C.c_double),
        ("maxiter", C.c_int64),
        ("bc_lo", C.c_int32 * 3),
        ("bc_hi", C.c_int32 * 3),
        ("project_mean", C.c_int32),
        ("precond", C.c_int32),
        ("flags", C.c_int32),
    ]


class MusclParams(C.Structure):
    """vb_muscl_params"""
    _fields_ = [
        ("dt", C.c_double),
        ("gamma", C.c_double),
        ("theta", C.c_double),
        ("dx", C.c_double),
        ("small_rho", C.c_double),
        ("bc", C.c_int32),
        ("flags", C.c_int32),
    ]


# name -> (argtypes); every entry point returns int
_VP = C.c_void_p
_DP = C.POINTER(C.c_double)
_I32P = C.POINTER(C.c_int32)
_I64P = C.POINTER(C.c_int64)
SIGNATURES = {
    "vb_abi_version": [],
    "vb_last_error": [C.c_char_p, C.c_size_t],
    "vb_ctx_create": [C.c_int, C.POINTER(_VP)],
    "vb_ctx_destroy": [_VP],
    "vb_ctx_synchronize": [_VP],
    "vb_ctx_stream": [_VP, C.POINTER(_VP)],
    "vb_ctx_launch_count": [_VP, _I64P],
    "vb_check_read": [_VP, _I64P],
    "vb_ctx_mark": [_VP, C.c_int],
    "vb_ctx_elapsed_ms": [_VP, C.c_int, C.c_int, C.POINTER(C.c_float)],
    "vb_hllc_faces": [_VP, C.c_int64, _DP, _DP, _I32P, C.c_double, _DP],
    "vb_hllc_faces_device_async": [_VP, C.c_int64, _VP, _VP, _VP, C.c_double, _VP],
    "vb_hllc_faces_noalloc": [C.c_int64, _DP, _DP, _I32P, C.c_double, _DP, _VP],
    "vb_grid_create": [_VP, C.POINTER(ProblemDesc), C.c_int, C.POINTER(_VP)],
    "vb_grid_destroy": [_VP],
    "vb_grid_ncell": [_VP, _I64P],
    "vb_grid_upload": [_VP, _DP],
    "vb_grid_download": [_VP, _DP],
    "vb_grid_device_state": [_VP, C.POINTER(_VP)],
    "vb_grid_set_option": [_VP, C.c_int, C.c_int64],
    "vb_grid_get_option": [_VP, C.c_int, _I64P],
    "vb_grid_autotune": [_VP, C.c_int, _I64P, _DP],
    "vb_grid_set_time": [_VP, C.c_double, C.c_int64],
    "vb_grid_get_time": [_VP, _DP, _I64P],
    "vb_compute_dt": [_VP, _DP],
    "vb_step": [_VP, C.c_double],
    "vb_grid_selftest_wait": [_VP, C.c_int64],
    "vb_grid_set_zwindow": [_VP, C.c_int64, C.c_int64, C.c_int, C.c_double],
    "vb_grid_step_phase": [_VP, C.c_int],
    "vb_grid_planes": [_VP, C.c_int, C.c_int64, C.c_int64, _VP, C.c_int],
    "vb_grid_cfl_bits": [_VP, _VP, C.c_int],
    "vb_evolve": [_VP, C.c_double, C.c_int64, _DP, _I64P],
    "vb_run_steps_async": [_VP, C.c_int64],
    "vb_conserved_totals": [_VP, _DP],
    "vb_grid_profile_step": [_VP, C.c_int, _DP, _DP, _DP],
    "vb_batch_create": [_VP, C.c_int, C.POINTER(ProblemDesc), C.c_int, C.POINTER(_VP)],
    "vb_batch_destroy": [_VP],
    "vb_batch_ncell": [_VP, C.c_int, _I64P],
    "vb_batch_upload": [_VP, C.c_int, _DP],
    "vb_batch_download": [_VP, C.c_int, _DP],
    "vb_batch_run_steps": [_VP, C.c_int64],
    "vb_batch_run_steps_async": [_VP, C.c_int64],
    "vb_batch_autotune": [_VP, C.c_int, _I64P, _DP],
    "vb_batch_get_time": [_VP, C.c_int, _DP, _I64P],
    "vb_batch_conserved_totals": [_VP, C.c_int, _DP],
    "vb_bflux_enable": [_VP, C.c_int],
    "vb_bflux_size": [_VP, _I64P],
    "vb_bflux_read": [_VP, _DP, C.c_int64],
    "vb_bflux_clear": [_VP],
    "vb_bflux_plane": [_VP, C.c_int, C.c_int, _I64P, _I64P, _I64P, C.c_int64, C.c_int, C.c_double,
                       _DP, C.c_int64],
    "vb_gravity_enable": [_VP, C.POINTER(GravityDesc)],
    "vb_gravity_disable": [_VP],
    "vb_gravity_solve": [_VP, _I64P, _DP],
    "vb_gravity_phi": [_VP, _DP],
    "vb_gravity_set_phi": [_VP, _DP],
    "vb_gravity_accel": [_VP, _DP],
    "vb_gravity_laplacian": [_VP, _DP, _DP],
    "vb_muscl_create": [_VP, _I64P, C.c_int32, C.POINTER(_VP)],
    "vb_muscl_destroy": [_VP],
    "vb_muscl_upload": [_VP, _DP],
    "vb_muscl_download": [_VP, _DP],
    "vb_muscl_state": [_VP, C.POINTER(_VP)],
    "vb_muscl_step": [_VP, C.POINTER(MusclParams)],
    "vb_muscl_run_async": [_VP, C.POINTER(MusclParams), C.c_int64],
    "vb_muscl_step_fields": [_VP, _VP, _VP, _VP, _VP, _VP, C.POINTER(MusclParams)],
    "vb_adjoint_create": [_VP, C.c_int64, C.c_int64, C.POINTER(_VP)],
    "vb_adjoint_destroy": [_VP],
    "vb_adjoint_forward": [_VP, C.c_double, C.c_int64, _DP, _I64P],
    "vb_adjoint_steps": [_VP, _I64P],
    "vb_adjoint_dts": [_VP, _DP, C.c_int64],
    "vb_adjoint_backward": [_VP, _DP, _DP],
    "vb_adjoint_step": [_VP, C.c_double, _DP, _DP],
    "vb_adjoint_timing": [_VP, _DP],
    "vb_amr_create": [_VP, C.POINTER(ProblemDesc), C.POINTER(_VP)],
    "vb_amr_destroy": [_VP],
    "vb_amr_nleaf": [_VP, _I64P],
    "vb_amr_nface": [_VP, _I64P],
    "vb_amr_leaves": [_VP, _I32P, _I64P],
    "vb_amr_max_level": [_VP, _I32P],
    "vb_amr_upload": [_VP, _DP],
    "vb_amr_download": [_VP, _DP],
    "vb_amr_set_time": [_VP, C.c_double, C.c_int64],
    "vb_amr_get_time": [_VP, _DP, _I64P],
    "vb_amr_refine": [_VP, _I64P, C.c_int64],
    "vb_amr_indicator": [_VP, _DP],
    "vb_amr_regrid": [_VP, C.c_double, C.c_int, _I64P],
    "vb_amr_compute_dt": [_VP, C.c_int, _DP],
    "vb_amr_step": [_VP, C.c_double],
    "vb_amr_step_level": [_VP, C.c_double, C.c_int],
    "vb_amr_evolve": [_VP, C.c_double, C.c_int64, C.c_double, C.c_int, C.c_int, C.c_int, _DP,
                      _I64P],
    "vb_amr_regrid_ms": [_VP, _DP],
    "vb_amr_conserved_totals": [_VP, _DP],
}

_lib = None


def load(path: str | None = None):
    """Load the shared library once; raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    p = path or os.environ.get("VESPA_B200_LIB", LIB_PATH)
    if not os.path.exists(p):
        raise ImportError(
            f"libvespa_b200.so not found at {p}; build it with `make -C vespa.jl_b200/csrc` "
            "(there is no CPU fallback)")
    L = C.CDLL(p)
    for name, args in SIGNATURES.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = C.c_int
    _lib = L
    return L


def last_error() -> str:
    buf = C.create_string_buffer(1024)
    load().vb_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(status: int) -> None:
    if status != VB_OK:
        raise VespaB200Error(status, last_error())


def call(name: str, *args) -> None:
    check(getattr(load(), name)(*args))


def dptr(a: np.ndarray):
    if a.dtype != np.float64 or not a.flags.c_contiguous:
        raise TypeError("expected a C-contiguous float64 array")
    return a.ctypes.data_as(_DP)


def i32ptr(a: np.ndarray):
    if a.dtype != np.int32 or not a.flags.c_contiguous:
        raise TypeError("expected a C-contiguous int32 array")
    return a.ctypes.data_as(_I32P)


def i64ptr(a: np.ndarray):
    if a.dtype != np.int64 or not a.flags.c_contiguous:
        raise TypeError("expected a C-contiguous int64 array")
    return a.ctypes.data_as(_I64P)


class Context:
    """A vb_ctx: one device, one stream."""

    def __init__(self, device: int = 0):
        h = _VP()
        call("vb_ctx_create", int(device), C.byref(h))
        self.handle = h
        self.device = device

    def close(self):
        if self.handle:
            load().vb_ctx_destroy(self.handle)
            self.handle = _VP()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def synchronize(self):
        call("vb_ctx_synchronize", self.handle)

    @property
    def stream(self) -> int:
        s = _VP()
        call("vb_ctx_stream", self.handle, C.byref(s))
        return s.value or 0

    def mark(self, slot: int) -> None:
        call("vb_ctx_mark", self.handle, int(slot))

    def elapsed_ms(self, a: int, b: int) -> float:
        ms = C.c_float()
        call("vb_ctx_elapsed_ms", self.handle, int(a), int(b), C.byref(ms))
        return ms.value

    @property
    def launch_count(self) -> int:
        n = C.c_int64()
        call("vb_ctx_launch_count", self.handle, C.byref(n))
        return n.value

    def check_read(self) -> int:
        """Device bounds-check record (vb_check_read): 0 = no check failed
        since the last read, else the source line of the first failed check;
        -1 in the normal build (no checks).  Waits for the stream; clears."""
        n = C.c_int64()
        call("vb_check_read", self.handle, C.byref(n))
        return n.value


_default_ctx: Context | None = None


def default_context() -> Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(int(os.environ.get("VESPA_B200_DEVICE", "0")))
    return _default_ctx
