"""ctypes binding of libvlasolve_b200.so (the C-ABI of include/vlasolve_b200.h).

The library is the only compute path: there is no CPU fallback.  Importing
this module raises if the shared object is missing or does not load.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libvlasolve_b200.so")

VLS_OK, VLS_EINVAL, VLS_ECUDA, VLS_ENAN, VLS_EIO, VLS_ENOMEM, VLS_ESTATE = range(7)
STATUS_NAMES = {0: "VLS_OK", 1: "VLS_EINVAL", 2: "VLS_ECUDA", 3: "VLS_ENAN",
                4: "VLS_EIO", 5: "VLS_ENOMEM", 6: "VLS_ESTATE"}

SCALES = {"linear": 0, "logarithmic": 1, "quadratic": 2}
KERNELS = {"delayed": 0, "reflective": 1}
PROFILES = {"UDF": 0, "PLDF": 1, "Plummer": 2, "Hernquist": 3}
PRECISIONS = {"fp64": 0, "fp32": 1, "fp32all": 2}

# every symbol include/vlasolve_b200.h declares
EXPORTED = [
    "vls_version", "vls_device_ok", "vls_create", "vls_create_layout", "vls_get_layout",
    "vls_destroy", "vls_last_error",
    "vls_dims", "vls_coords", "vls_init_profile", "vls_set_f", "vls_get_f",
    "vls_get_footpoints", "vls_set_footpoints", "vls_get_chains",
    "vls_set_chain_values", "vls_step", "vls_sync", "vls_kernel_launches",
    "vls_moments", "vls_last_mass", "vls_last_mass_async", "vls_stats", "vls_get_time", "vls_set_time",
    "vls_write_ndfield", "vls_read_ndfield", "vls_stream", "vls_set_profiling",
    "vls_profile_read", "vls_radial_mass_noalloc", "vls_noalloc_last_error",
    "vls_adjoint_forward", "vls_adjoint_backward", "vls_adjoint_set_inner",
    "vls_adjoint_inner_used", "vls_adjoint_init_dot", "vls_device_bytes", "vls_write_restart",
    "vls_restart_info", "vls_read_restart",
    "vls_spline2d_create", "vls_spline2d_destroy", "vls_spline2d_dims", "vls_spline2d_scale",
    "vls_spline2d_assign", "vls_spline2d_build", "vls_spline2d_coefficients",
    "vls_spline2d_pos2coord", "vls_spline2d_evaluate_c", "vls_spline2d_evaluate_nxpy",
    "vls_spline2d_evaluate", "vls_spline2d_last_error", "vls_interp_create_init",
    "vls_interp_create", "vls_interp_evaluate", "vls_interp_destroy", "vls_interp_last_error",
]
KERNEL_KINDS = ["ucol_kick", "ucol", "prer", "tails", "drift", "scan", "moment",
                "stats", "convert", "adj_drift", "adj_tails", "adj_prer", "adj_ucol",
                "adj_shift", "adj_moment"]


class VlsError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


class GridDesc(ctypes.Structure):
    _fields_ = [("Pmin", ctypes.c_double), ("Pmax", ctypes.c_double),
                ("Pres", ctypes.c_int32), ("Pscale", ctypes.c_int32),
                ("Umin", ctypes.c_double * 2), ("Umax", ctypes.c_double * 2),
                ("Ures", ctypes.c_int32 * 2), ("Uscale", ctypes.c_int32 * 2)]


class SolverDesc(ctypes.Structure):
    _fields_ = [("G", ctypes.c_double), ("T0", ctypes.c_double),
                ("Tmax", ctypes.c_double), ("dt", ctypes.c_double),
                ("noLinking", ctypes.c_int32), ("kernelType", ctypes.c_int32),
                ("kernelBufferSize", ctypes.c_int32), ("precision", ctypes.c_int32),
                ("device", ctypes.c_int32)]


# vls_layout_desc: kernel layouts of a handle (zeroes = the defaults)
PREFILTERS = {"auto": 0, "register": 1, "segment": 2}
DRIFTS = {"auto": 0, "window": 1, "strip2": 2, "strip1": 3}


class LayoutDesc(ctypes.Structure):
    _fields_ = [("prefilter", ctypes.c_int32), ("drift", ctypes.c_int32),
                ("slices_per_batch", ctypes.c_int32), ("streams", ctypes.c_int32),
                ("drift_wait_spins", ctypes.c_int32), ("u_chunk_rows", ctypes.c_int32),
                ("r_chunk_rows", ctypes.c_int32)]


class Spline2dDesc(ctypes.Structure):
    _fields_ = [("start", ctypes.c_double * 2), ("stop", ctypes.c_double * 2),
                ("N", ctypes.c_int32 * 2), ("scaleType", ctypes.c_int32 * 2),
                ("vlType", ctypes.c_int32 * 2), ("bCond", (ctypes.c_int32 * 2) * 2),
                ("precision", ctypes.c_int32), ("device", ctypes.c_int32)]


class InterpInit(ctypes.Structure):
    _fields_ = [("xstart", ctypes.c_double), ("xend", ctypes.c_double),
                ("ystart", ctypes.c_double), ("yend", ctypes.c_double),
                ("nx", ctypes.c_int32), ("ny", ctypes.c_int32),
                ("xbc", ctypes.c_int32 * 2), ("ybc", ctypes.c_int32 * 2),
                ("xbcv", ctypes.c_double * 2), ("ybcv", ctypes.c_double * 2),
                ("xscaleType", ctypes.c_int32), ("yscaleType", ctypes.c_int32),
                ("rescaleNeeded", ctypes.c_int32), ("useLog", ctypes.c_int32)]


# localSpline::boundaryTypeV and einspline's bc_code (interpolSpline)
BC = {"periodic": 0, "flat": 1, "natural": 2, "supra_natural": 3, "not_a_knot": 4, "local": 5}
EBC = {"periodic": 0, "deriv1": 1, "deriv2": 2, "flat": 3, "natural": 4, "antiperiodic": 5}


class InitDesc(ctypes.Structure):
    _fields_ = [("type", ctypes.c_int32), ("M", ctypes.c_double),
                ("R0", ctypes.c_double), ("alpha", ctypes.c_double),
                ("smoothingRadius", ctypes.c_double), ("gap", ctypes.c_double * 2),
                ("eta", ctypes.c_double), ("n", ctypes.c_double),
                ("Ra", ctypes.c_double), ("R0_given", ctypes.c_int32)]


class StatsOut(ctypes.Structure):
    _fields_ = [("time", ctypes.c_double), ("step", ctypes.c_int64),
                ("Mass", ctypes.c_double), ("E", ctypes.c_double),
                ("Ek", ctypes.c_double), ("Ep", ctypes.c_double),
                ("S", ctypes.c_double), ("L1", ctypes.c_double),
                ("L2", ctypes.c_double)]


_lib = None


def load(path: str = LIB_PATH):
    """Load the shared library and declare every signature."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(
            f"{path} is missing: build it with `python -m vlasolve_b200.build` "
            "(the CUDA path is the only implementation)")
    L = ctypes.CDLL(path)
    P = ctypes.POINTER
    H = ctypes.c_void_p
    i32, i64, d, u8 = ctypes.c_int32, ctypes.c_int64, ctypes.c_double, ctypes.c_uint8
    sig = {
        "vls_version": [P(i32), P(i32)],
        "vls_device_ok": [i32],
        "vls_create": [P(GridDesc), P(SolverDesc), P(H)],
        "vls_create_layout": [P(GridDesc), P(SolverDesc), P(LayoutDesc), P(H)],
        "vls_get_layout": [H, P(LayoutDesc)],
        "vls_destroy": [H],
        "vls_dims": [H, P(i64), P(i64), P(i64)],
        "vls_coords": [H, P(d), P(d), P(d), P(d)],
        "vls_init_profile": [H, P(InitDesc), P(d)],
        "vls_set_f": [H, P(d), ctypes.c_size_t],
        "vls_get_f": [H, P(d), ctypes.c_size_t],
        "vls_get_footpoints": [H, P(i32), P(d), P(i32), P(d), P(u8), P(d)],
        "vls_set_footpoints": [H, P(i32), P(d), P(i32), P(d), P(u8), P(d)],
        "vls_get_chains": [H, P(i64), P(i64), P(i64), P(i64), P(i32), P(d), P(d), P(d)],
        "vls_set_chain_values": [H, P(d), i64],
        "vls_step": [H, i32],
        "vls_sync": [H],
        "vls_kernel_launches": [H, P(i64)],
        "vls_moments": [H, P(d), P(d), P(d)],
        "vls_last_mass": [H, P(d)],
        "vls_last_mass_async": [H, P(d)],
        "vls_stats": [H, P(StatsOut)],
        "vls_get_time": [H, P(d), P(i64)],
        "vls_set_time": [H, d, i64],
        "vls_write_ndfield": [H, ctypes.c_char_p],
        "vls_read_ndfield": [H, ctypes.c_char_p],
        "vls_stream": [H, P(ctypes.c_void_p)],
        "vls_set_profiling": [H, i32],
        "vls_profile_read": [H, P(d), P(i64), i32],
        "vls_write_restart": [H, ctypes.c_char_p, i64, i64, i64],
        "vls_restart_info": [ctypes.c_char_p, P(GridDesc), P(SolverDesc), P(i64), P(d),
                             P(i64)],
        "vls_read_restart": [H, ctypes.c_char_p],
        "vls_adjoint_forward": [H, i32, i32],
        "vls_adjoint_backward": [H, P(d), i64, P(d), ctypes.c_size_t, P(d), i64],
        "vls_adjoint_set_inner": [H, i32],
        "vls_adjoint_inner_used": [H, P(i32)],
        "vls_adjoint_init_dot": [H, P(InitDesc), P(InitDesc), P(d), P(d)],
        "vls_device_bytes": [H, P(ctypes.c_size_t)],
        "vls_spline2d_create": [P(Spline2dDesc), i64, P(H)],
        "vls_spline2d_destroy": [H],
        "vls_spline2d_dims": [H, P(i32), P(i32), P(i64)],
        "vls_spline2d_scale": [H, P(d), P(d)],
        "vls_spline2d_assign": [H, P(d), i64],
        "vls_spline2d_build": [H],
        "vls_spline2d_coefficients": [H, i64, P(d)],
        "vls_spline2d_pos2coord": [H, i32, i64, P(d), P(i32), P(d)],
        "vls_spline2d_evaluate_c": [H, i64, P(i64), P(i32), P(d), P(i32), P(d), P(d)],
        "vls_spline2d_evaluate_nxpy": [H, i64, P(i64), P(i32), P(d), P(d)],
        "vls_spline2d_evaluate": [H, i64, P(i64), P(d), P(d), P(d)],
        "vls_interp_create_init": [d, d, i32, d, d, i32, i32, i32, i32, i32, i32, i32, i32, i32,
                                   d, d, d, d, P(InterpInit)],
        "vls_interp_create": [P(InterpInit), P(d), i32, P(H)],
        "vls_interp_evaluate": [H, i64, P(d), P(d), P(d), P(d), P(d)],
        "vls_interp_destroy": [H],
        "vls_radial_mass_noalloc": [ctypes.c_void_p, i32, i64, i64, i64, P(d), P(d), P(d),
                                    P(d), ctypes.c_void_p, ctypes.c_void_p,
                                    ctypes.c_void_p, ctypes.c_void_p, i32],
    }
    for name, args in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = ctypes.c_int
    L.vls_last_error.argtypes = [H]
    L.vls_last_error.restype = ctypes.c_char_p
    for name in ("vls_spline2d_last_error", "vls_interp_last_error"):
        getattr(L, name).argtypes = [H]
        getattr(L, name).restype = ctypes.c_char_p
    L.vls_noalloc_last_error.argtypes = []
    L.vls_noalloc_last_error.restype = ctypes.c_char_p
    _lib = L
    return L


def check(code: int, handle=None):
    if code != VLS_OK:
        msg = _lib.vls_last_error(handle).decode(errors="replace")
        raise VlsError(code, msg)
