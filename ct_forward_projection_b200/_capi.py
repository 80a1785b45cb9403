"""ctypes binding of the C ABI in include/ctfp.h (libctfp.so, built in-tree).

The library is loaded from the package directory only; importing this module
on a machine where it has not been built raises immediately, so no caller can
silently run without the CUDA path.
"""
from __future__ import annotations

import ctypes as C
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libctfp.so")

CTFP_OK, CTFP_INVALID_ARG, CTFP_OOM, CTFP_CUDA_ERROR, CTFP_TIMEOUT, CTFP_UNSUPPORTED, CTFP_NOT_READY = range(7)
STATUS_NAMES = {0: "OK", 1: "INVALID_ARG", 2: "OOM", 3: "CUDA_ERROR", 4: "TIMEOUT", 5: "UNSUPPORTED",
                6: "NOT_READY"}

INTERP_TRILINEAR, INTERP_TEXEMU, INTERP_TEXTURE = 0, 1, 2
GRID_NONE, GRID_COLUMN, GRID_PIXEL = 0, 1, 2
SAMPLER_GLOBAL, SAMPLER_LAYERED, SAMPLER_BRICK, SAMPLER_AXIS = 1, 2, 3, 4
MAX_MATERIALS = 4


class CtfpError(RuntimeError):
    def __init__(self, status: int, where: str, msg: str):
        super().__init__(f"{where}: {STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


class Geometry(C.Structure):
    """ctfp_geometry — CTScanParas fields the projector reads (DataType.h:33-55)."""
    _fields_ = [("pNumX", C.c_int64), ("pNumY", C.c_int64), ("pNumZ", C.c_int64),
                ("pLengthX", C.c_float), ("pLengthY", C.c_float), ("pLengthZ", C.c_float),
                ("projNum", C.c_int64), ("dNumU", C.c_int64), ("dNumV", C.c_int64),
                ("dSize", C.c_float), ("sod", C.c_float), ("sdd", C.c_float),
                ("rotatedDirection", C.c_int32), ("reserved", C.c_int32)]


class SystemInfo(C.Structure):
    """ctfp_system_info — CTScanSystemInfo as computeParas fills it (DataType.h:78-111)."""
    _fields_ = [(n, C.c_float) for n in ("thetaStep", "dHalfLU", "dHalfLV", "FOVR", "FOVH", "pHalfX", "pHalfY",
                                          "pHalfZ", "pSizeX", "pSizeY", "pSizeZ", "dx", "dy", "dz")] + \
               [("intNum", C.c_int64)]


class LaunchShape(C.Structure):
    """ctfp_launch_shape — the autotuner's choice."""
    _fields_ = [("tile_u", C.c_int32), ("tile_v", C.c_int32), ("views_per_cta", C.c_int32),
                ("min_ctas_per_sm", C.c_int32), ("ms", C.c_float), ("from_cache", C.c_int32)]


class GridParams(C.Structure):
    """ctfp_grid_params — GridInfo geometry (DataType.h:57-75)."""
    _fields_ = [("gridStripsWidth", C.c_int32), ("interspaceWidth", C.c_int32), ("h", C.c_float),
                ("FD", C.c_float)]


_P = C.c_void_p
_FP = C.POINTER(C.c_float)

# name -> (restype, argtypes)
_SIGNATURES = {
    "ctfp_compute_paras": (C.c_int, [C.POINTER(Geometry), C.POINTER(SystemInfo)]),
    "ctfp_view_angle": (C.c_int, [C.POINTER(Geometry), C.c_int64, _FP]),
    "ctfp_plan_create": (C.c_int, [C.POINTER(Geometry), C.c_int32, C.c_int32, C.c_int32, C.POINTER(_P)]),
    "ctfp_plan_destroy": (C.c_int, [_P]),
    "ctfp_plan_get_system_info": (C.c_int, [_P, C.POINTER(SystemInfo)]),
    "ctfp_plan_set_interp": (C.c_int, [_P, C.c_int32]),
    "ctfp_plan_set_sampler": (C.c_int, [_P, C.c_int32]),
    "ctfp_plan_set_skip_empty": (C.c_int, [_P, C.c_int32]),
    "ctfp_plan_check_status": (C.c_int, [_P, C.POINTER(C.c_uint32)]),
    "ctfp_plan_set_focal_spot": (C.c_int, [_P, _P, _P]),
    "ctfp_focal_spot_offsets": (C.c_int, [C.c_int64, C.c_float, _P, _P]),
    "ctfp_plan_set_launch_shape": (C.c_int, [_P, C.c_int32, C.c_int32, C.c_int32, C.c_int32]),
    "ctfp_set_spectral_tables": (C.c_int, [_P, C.c_int32, _P, _P, _P, C.c_int32, _P, C.c_float]),
    "ctfp_line_integrals": (C.c_int, [_P, _P, _P, _P]),
    "ctfp_forward": (C.c_int, [_P, _P, _P, _P, _P, _P, _P]),
    "ctfp_spectral_from_L": (C.c_int, [_P, _P, _P, _P, _P]),
    "ctfp_forward_views": (C.c_int, [_P, _P, C.c_int64, C.c_int64, _P, _P, _P, _P, _P]),
    "ctfp_backward_views": (C.c_int, [_P, _P, _P, _P, C.c_int64, C.c_int64, _P, _P]),
    "ctfp_finalize_counts": (C.c_int, [C.c_int64, C.c_int64, _P, _P, _P, _P, _P, _P, _P]),
    "ctfp_backward": (C.c_int, [_P, _P, _P, _P, _P, _P]),
    "ctfp_line_integrals_adjoint": (C.c_int, [_P, _P, _P, _P]),
    "ctfp_sample_volume": (C.c_int, [_P, C.c_int64, C.c_int64, C.c_int64, C.c_int32, _P, C.c_int64, _P, _P]),
    "ctfp_count_support_samples": (C.c_int, [_P, C.POINTER(C.c_int64)]),
    "ctfp_axis_gather_count": (C.c_int, [_P, C.POINTER(C.c_double)]),
    "ctfp_forward_host": (C.c_int, [_P, _P, _P, _P, _P, _P]),
    "ctfp_build_grid_table": (C.c_int, [C.POINTER(Geometry), C.POINTER(GridParams), C.c_int32, _P, _P, C.c_int32,
                                        _P, _P]),
    "ctfp_scintillator_thickness": (C.c_int, [C.c_int64, C.c_float, C.c_float, _P]),
    "ctfp_build_det_response": (C.c_int, [C.c_int32, C.c_int64, _P, _P, C.c_float, _P, _P]),
    "ctfp_labels_to_density": (C.c_int, [_P, C.c_int64, C.c_int32, _P, _P, _P]),
    "ctfp_forward_noalloc": (C.c_int, [C.POINTER(Geometry), C.c_int32, C.c_int32, C.c_int32, _P, _P, _P, C.c_int32,
                                       _P, C.c_float, _P, _P, _P, _P, _P]),
    "ctfp_sampler_peak": (C.c_int, [C.c_int32, C.c_int32, C.POINTER(C.c_double)]),
    "ctfp_plan_autotune": (C.c_int, [_P, _P, _P, _P, C.c_int32, C.POINTER(LaunchShape), _P]),
    "ctfp_batch_create": (C.c_int, [C.c_int32, _P, C.POINTER(_P)]),
    "ctfp_batch_destroy": (C.c_int, [_P]),
    "ctfp_batch_forward": (C.c_int, [_P, _P, _P, _P, _P, _P]),
    "ctfp_batch_forward_adjoint": (C.c_int, [_P, _P, _P, _P, _P, _P, _P]),
    "ctfp_batch_info": (C.c_int, [_P, C.POINTER(C.c_int64), C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "ctfp_batch_set_shape": (C.c_int, [_P, C.c_int32, C.c_int32]),
    "ctfp_batch_autotune": (C.c_int, [_P, _P, _P, _P, _P]),
    "ctfp_batch_get_shapes": (C.c_int, [_P, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                        C.POINTER(C.c_int32)]),
    "ctfp_batch_set_views": (C.c_int, [_P, C.c_int32, C.c_int32]),
    "ctfp_check_division": (C.c_int, [C.c_int32, C.c_float, C.c_int64, C.c_uint64, C.POINTER(C.c_int64)]),
    "ctfp_batch_get_views": (C.c_int, [_P, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "ctfp_last_error_string": (C.c_char_p, []),
    "ctfp_version": (C.c_char_p, []),
}


def exported_symbols_from_header(header: str | None = None) -> list[str]:
    """Function names declared in include/ctfp.h."""
    import re
    header = header or os.path.join(os.path.dirname(PKG), "include", "ctfp.h")
    text = open(header).read()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[\w ]+?\**\s*\b(ctfp_\w+)\s*\(", text, re.M)))


_lib = None


def lib() -> C.CDLL:
    """Loads libctfp.so (raises OSError if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(f"{LIB_PATH} not built; run python -m ct_forward_projection_b200.build")
        h = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGNATURES.items():
            if hasattr(h, name):
                f = getattr(h, name)
                f.restype = res
                f.argtypes = args
        _lib = h
    return _lib


def check(status: int, where: str) -> None:
    if status != CTFP_OK:
        raise CtfpError(status, where, lib().ctfp_last_error_string().decode())


def call(name: str, *args) -> None:
    check(getattr(lib(), name)(*args), name)


def ptr_array(ptrs) -> C.Array:
    """Host array of device pointers (const float* const*)."""
    arr = (C.c_void_p * max(1, len(ptrs)))()
    for i, p in enumerate(ptrs):
        arr[i] = p
    return arr
