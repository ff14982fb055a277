"""ctypes binding of the in-tree CUDA library libh3dmg.so (C ABI: include/h3d_mg.h).

There is no fallback: if the library is missing or fails to load, every
entry point raises.  Build it with ``python -m hydro3d_b200.build``.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libh3dmg.so")

H3D_OK = 0
H3D_ERR_BAD_CONFIG = -1
H3D_ERR_CUDA = -2
H3D_ERR_NOT_CONVERGED = -3
H3D_ERR_DIVERGED = -4
H3D_ERR_TIMEOUT = -5
H3D_ERR_NO_DEVICE = -6
H3D_ERR_ARG = -7
H3D_ERR_OOM = -8
H3D_ERR_INTERNAL = -9

PREC_FP64 = 0
PREC_MIXED = 1
FIELD_P = 0
FIELD_B = 1
FIELD_U, FIELD_V, FIELD_W = 2, 3, 4
FIELD_USTAR, FIELD_VSTAR, FIELD_WSTAR = 5, 6, 7
FIELD_PP = 8


class BlockDesc(C.Structure):
    """h3d_block_desc."""

    _fields_ = [
        ("n", C.c_int32 * 3),
        ("ttc", C.c_int32 * 3),
        ("pl", C.c_int32),
        ("ngrid", C.c_int32),
        ("h", C.c_double * 3),
        ("nb_face", C.c_int32 * 6),
        ("nb_corner", C.c_int32 * 8),
        ("nb_edge", C.c_int32 * 12),
        ("nb_periodic", C.c_int32 * 6),
        ("bc", C.c_int32 * 6),
        ("rdiv", C.c_int32),
        ("origin", C.c_int32 * 3),
    ]


class MGDesc(C.Structure):
    """h3d_mg_desc."""

    _fields_ = [
        ("nblocks", C.c_int32),
        ("ngrd_gl", C.c_int32),
        ("mg_itrsch", C.c_int32),
        ("irestr", C.c_int32),
        ("iproln", C.c_int32),
        ("maxcy", C.c_int32),
        ("precision", C.c_int32),
        ("var_coef", C.c_int32),
        ("device", C.c_int32),
        ("coarse_sweeps", C.c_int32),
        ("inner_cycles", C.c_int32),
        ("use_graph", C.c_int32),
        ("coarse_op", C.c_int32),
        ("coarse_direct", C.c_int32),
        ("rb_order", C.c_int32),
        ("omega", C.c_float),
        ("blocks", C.POINTER(BlockDesc)),
    ]


class SolveOpts(C.Structure):
    _fields_ = [
        ("tol", C.c_double),
        ("maxcy", C.c_int32),
        ("stop_rule", C.c_int32),
        ("remove_mean", C.c_int32),
        ("record_history", C.c_int32),
    ]


class SolveInfo(C.Structure):
    _fields_ = [
        ("cycles", C.c_int32),
        ("outer", C.c_int32),
        ("relres", C.c_double),
        ("rmax", C.c_double),
        ("bnorm", C.c_double),
        ("device_ms", C.c_double),
        ("smoother_ms", C.c_double),
        ("smoother_launches", C.c_int64),
        ("kernel_launches", C.c_int64),
        ("smoother_bytes", C.c_double),
        ("relres_block_max", C.c_double),
    ]


# Every exported entry point, as declared in include/h3d_mg.h.
EXPORTS = [
    "h3d_mg_create", "h3d_mg_destroy", "h3d_mg_set_density", "h3d_mg_coeff", "h3d_mg_mgkcyc",
    "h3d_mg_newsolv", "h3d_mg_upload", "h3d_mg_download", "h3d_mg_zero_field", "h3d_mg_solve_resident", "h3d_mg_residual",
    "h3d_mg_history", "h3d_mg_put_level", "h3d_mg_get_level", "h3d_mg_mgrelax", "h3d_mg_mgrestr",
    "h3d_mg_mgcorr", "h3d_mg_mgbound", "h3d_mg_exchangepp", "h3d_mg_vcycle", "h3d_mg_sync",
    "h3d_mg_set_profiling", "h3d_mg_smoother_bytes", "h3d_mg_set_smoother", "h3d_mg_get_smoother",
    "h3d_mg_set_restriction", "h3d_mg_get_restriction", "h3d_topology", "h3d_halo_table", "h3d_halo_expr",
    "h3d_mg_strerror", "h3d_mg_last_error", "h3d_residual_noalloc",
    "h3d_mg_calvel", "h3d_mg_calmas", "h3d_mg_pbound", "h3d_mg_project_resident", "h3d_mg_project",
    "h3d_mg_set_wait_limit", "h3d_mg_wait_probe", "h3d_mg_sipsol", "h3d_mg_pressure_1sweep",
]

_lib = None


class H3DError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{msg} (code {code})")
        self.code = code


def lib():
    """Load libh3dmg.so (raises if it is not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is not built; run `python -m hydro3d_b200.build`")
    L = C.CDLL(LIB_PATH)
    vp, i32, i64, dbl = C.c_void_p, C.c_int32, C.c_int64, C.c_double
    pd = C.POINTER(C.c_double)
    ppd = C.POINTER(pd)
    pu32 = C.POINTER(C.c_uint32)
    sig = {
        "h3d_mg_create": (i32, [C.POINTER(vp), C.POINTER(MGDesc)]),
        "h3d_mg_destroy": (i32, [vp]),
        "h3d_mg_set_density": (i32, [vp, i32, pd]),
        "h3d_mg_coeff": (i32, [vp]),
        "h3d_mg_mgkcyc": (i32, [vp, ppd, ppd]),
        "h3d_mg_newsolv": (i32, [vp, ppd, ppd, C.POINTER(SolveOpts), C.POINTER(SolveInfo)]),
        "h3d_mg_upload": (i32, [vp, i32, i32, pd]),
        "h3d_mg_download": (i32, [vp, i32, i32, pd]),
        "h3d_mg_zero_field": (i32, [vp, i32]),
        "h3d_mg_solve_resident": (i32, [vp, C.POINTER(SolveOpts), C.POINTER(SolveInfo)]),
        "h3d_mg_residual": (i32, [vp, pd, pd, pd]),
        "h3d_mg_history": (i32, [vp, pd, i32, C.POINTER(i32)]),
        "h3d_mg_put_level": (i32, [vp, i32, i32, i32, pd]),
        "h3d_mg_get_level": (i32, [vp, i32, i32, i32, pd]),
        "h3d_mg_mgrelax": (i32, [vp, i32, i32]),
        "h3d_mg_mgrestr": (i32, [vp, i32]),
        "h3d_mg_mgcorr": (i32, [vp, i32]),
        "h3d_mg_mgbound": (i32, [vp, i32]),
        "h3d_mg_exchangepp": (i32, [vp, i32]),
        "h3d_mg_vcycle": (i32, [vp]),
        "h3d_mg_sync": (i32, [vp]),
        "h3d_mg_set_profiling": (i32, [vp, i32]),
        "h3d_mg_smoother_bytes": (i32, [vp, pd]),
        "h3d_mg_set_smoother": (i32, [vp, i32, i32, i32]),
        "h3d_mg_get_smoother": (i32, [vp, i32, C.POINTER(i32), C.POINTER(i32), C.POINTER(i32)]),
        "h3d_mg_set_restriction": (i32, [vp, i32, i32, i32]),
        "h3d_mg_get_restriction": (i32, [vp, i32, C.POINTER(i32), C.POINTER(i32), C.POINTER(i32)]),
        "h3d_topology": (i32, [i32, C.POINTER(C.c_int32), C.POINTER(C.c_int32), pd, i32, C.POINTER(BlockDesc)]),
        "h3d_halo_table": (i32, [i32, C.POINTER(BlockDesc), i32, i32, pu32, pu32, i64, C.POINTER(i64)]),
        "h3d_halo_expr": (i32, [i32, C.POINTER(BlockDesc), i32, i32, pu32, i64, C.POINTER(i64), pu32, pu32, i64,
                                C.POINTER(i64)]),
        "h3d_residual_noalloc": (i32, [C.c_void_p, C.c_void_p, i32, i32, i32, pd, i32, pd, C.c_void_p]),
        "h3d_mg_set_wait_limit": (i32, [vp, i64]),
        "h3d_mg_wait_probe": (i32, [vp]),
        "h3d_mg_sipsol": (i32, [vp, i32, C.POINTER(i32), pd]),
        "h3d_mg_pressure_1sweep": (i32, [vp, dbl, dbl, dbl, i32, i32, C.POINTER(SolveInfo)]),
        "h3d_mg_calvel": (i32, [vp, dbl, dbl]),
        "h3d_mg_calmas": (i32, [vp, dbl, pd, pd]),
        "h3d_mg_pbound": (i32, [vp]),
        "h3d_mg_project_resident": (i32, [vp, dbl, dbl, C.POINTER(SolveOpts), C.POINTER(SolveInfo)]),
        "h3d_mg_project": (i32, [vp, ppd, ppd, ppd, ppd, ppd, ppd, ppd, dbl, dbl, C.POINTER(SolveOpts),
                                 C.POINTER(SolveInfo)]),
        "h3d_mg_strerror": (C.c_char_p, [C.c_int]),
        "h3d_mg_last_error": (C.c_char_p, [vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def check(rc, handle=None, what=""):
    if rc == H3D_OK:
        return rc
    L = lib()
    detail = L.h3d_mg_last_error(handle).decode() if handle is not None or rc != H3D_OK else ""
    raise H3DError(rc, f"{what}: {L.h3d_mg_strerror(rc).decode()}: {detail}")
