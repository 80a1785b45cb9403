"""Python binding of the FP64 CPU oracle (oracle/ctfp_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline leg of bench.py as the checker.  The product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libctfp_oracle.so")

TRILINEAR, TEXEMU = 0, 1


class OGeom(C.Structure):
    _fields_ = [("pNumX", C.c_int64), ("pNumY", C.c_int64), ("pNumZ", C.c_int64),
                ("pLengthX", C.c_float), ("pLengthY", C.c_float), ("pLengthZ", C.c_float),
                ("projNum", C.c_int64), ("dNumU", C.c_int64), ("dNumV", C.c_int64),
                ("dSize", C.c_float), ("sod", C.c_float), ("sdd", C.c_float),
                ("rotatedDirection", C.c_int32), ("reserved", C.c_int32)]


class OInfo(C.Structure):
    _fields_ = [(n, C.c_float) for n in ("thetaStep", "dHalfLU", "dHalfLV", "FOVR", "FOVH", "pHalfX", "pHalfY",
                                          "pHalfZ", "pSizeX", "pSizeY", "pSizeZ", "dx", "dy", "dz")] + \
               [("intNum", C.c_int64)]


_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        src = os.path.join(HERE, "ctfp_oracle.c")
        if not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(src):
            build()
        _lib = C.CDLL(LIB)
        _lib.orc_view_angle.restype = C.c_float
        _lib.orc_num_threads.restype = C.c_int
        _lib.orc_grid_column.restype = C.c_int
        _lib.orc_grid_pixel.restype = C.c_int
    return _lib


def geom(d: dict) -> OGeom:
    g = OGeom()
    for k in ("pNumX", "pNumY", "pNumZ", "projNum", "dNumU", "dNumV"):
        setattr(g, k, int(d[k]))
    for k in ("pLengthX", "pLengthY", "pLengthZ", "dSize", "sod", "sdd"):
        setattr(g, k, float(d[k]))
    g.rotatedDirection = int(d.get("rotatedDirection", 1))
    return g


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _f32(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float32)


def compute_paras(d: dict) -> dict:
    info = OInfo()
    lib().orc_compute_paras(C.byref(geom(d)), C.byref(info))
    return {k: getattr(info, k) for k, _ in OInfo._fields_}


def view_angle(d: dict, p: int) -> float:
    g = geom(d)
    info = OInfo()
    lib().orc_compute_paras(C.byref(g), C.byref(info))
    return float(lib().orc_view_angle(C.byref(g), C.byref(info), C.c_int64(p)))


def _vol_array(vols):
    vols = [_f32(v) for v in vols]
    arr = (C.c_void_p * len(vols))(*[v.ctypes.data for v in vols])
    return arr, vols


def _rays(d, ray_ids):
    if ray_ids is None:
        return int(d["projNum"] * d["dNumV"] * d["dNumU"]), None
    r = np.ascontiguousarray(ray_ids, dtype=np.int64)
    return len(r), r


def line_integrals(d: dict, vols, mode: int = TRILINEAR, ray_ids=None, focal_spot=None) -> np.ndarray:
    """focal_spot: (offset_u, offset_v) per view in mm, or None."""
    n, r = _rays(d, ray_ids)
    arr, keep = _vol_array(vols)
    L = np.empty((n, len(keep)), np.float64)
    if focal_spot is None:
        lib().orc_line_integrals(C.byref(geom(d)), len(keep), arr, mode, C.c_int64(n), _p(r), _p(L))
    else:
        fu, fv = _f32(focal_spot[0]), _f32(focal_spot[1])
        lib().orc_line_integrals_focal_spot(C.byref(geom(d)), len(keep), arr, mode, C.c_int64(n), _p(r), _p(fu),
                                            _p(fv), _p(L))
    return L


def shift_views(d: dict, L, M: int, focal_spot, mode: int = TRILINEAR) -> np.ndarray:
    """Focal-spot re-alignment of all views' line integrals L [P*V*U][M]."""
    P, V, U = int(d["projNum"]), int(d["dNumV"]), int(d["dNumU"])
    L = np.ascontiguousarray(L, dtype=np.float64).reshape(P * V * U, M)
    out = np.empty_like(L)
    fu, fv = _f32(focal_spot[0]), _f32(focal_spot[1])
    lib().orc_shift_views(mode, C.c_int64(P), C.c_int64(V), C.c_int64(U), M, C.c_float(float(d["dSize"])), _p(fu),
                          _p(fv), _p(L), _p(out))
    return out


def focal_spot_offsets(n: int, size: float):
    u = np.empty(n, np.float32)
    v = np.empty(n, np.float32)
    lib().orc_focal_spot_offsets(C.c_int64(n), C.c_float(size), _p(u), _p(v))
    return u, v


def forward_focal_spot(d: dict, vols, mu, W, focal_spot, mode: int = TRILINEAR) -> dict:
    """The focal-spot forward: shifted march, re-alignment, spectral epilogue."""
    M = len(vols)
    L = shift_views(d, line_integrals(d, vols, mode, focal_spot=focal_spot), M, focal_spot, mode)
    I, A = spectral(d, mu, W, L)
    return {"I": I, "IAbsorb": A, "L": L}


def energy_weights(d: dict, spectrum, grid=None, grid_layout: int = 0, det=None, I0Val: float = 1.0) -> np.ndarray:
    S = _f32(spectrum)
    G = _f32(grid)
    D = _f32(det)
    E = len(S)
    W = np.empty((E, int(d["dNumV"]), int(d["dNumU"])), np.float64)
    lib().orc_energy_weights(C.byref(geom(d)), E, _p(S), _p(G), grid_layout if G is not None else 0, _p(D),
                             C.c_double(I0Val), _p(W))
    return W


def spectral(d: dict, mu, W, L, ray_ids=None):
    mu = _f32(mu)
    E, M = mu.shape
    n, r = _rays(d, ray_ids)
    L = np.ascontiguousarray(L, dtype=np.float64).reshape(n, M)
    W = np.ascontiguousarray(W, dtype=np.float64)
    I = np.empty(n, np.float64)
    A = np.empty(n, np.float64)
    lib().orc_spectral(C.byref(geom(d)), M, E, _p(mu), _p(W), C.c_int64(n), _p(r), _p(L), _p(I), _p(A))
    return I, A


def forward(d: dict, vols, mu, W, mode: int = TRILINEAR, ray_ids=None) -> dict:
    L = line_integrals(d, vols, mode, ray_ids)
    I, A = spectral(d, mu, W, L, ray_ids)
    return {"I": I, "IAbsorb": A, "L": L, "I0": W.sum(axis=0)}


def backward(d: dict, mu, W, L, gI=None, gIAbs=None, mode: int = TRILINEAR, ray_ids=None):
    mu = _f32(mu)
    E, M = mu.shape
    n, r = _rays(d, ray_ids)
    L = np.ascontiguousarray(L, dtype=np.float64).reshape(n, M)
    W = np.ascontiguousarray(W, dtype=np.float64)
    gI = None if gI is None else np.ascontiguousarray(gI, dtype=np.float64).reshape(n)
    gA = None if gIAbs is None else np.ascontiguousarray(gIAbs, dtype=np.float64).reshape(n)
    shape = (int(d["pNumZ"]), int(d["pNumY"]), int(d["pNumX"]))
    grads = [np.zeros(shape, np.float64) for _ in range(M)]
    arr = (C.c_void_p * M)(*[g.ctypes.data for g in grads])
    lib().orc_backward(C.byref(geom(d)), M, mode, E, _p(mu), _p(W), C.c_int64(n), _p(r), _p(L), _p(gI), _p(gA), arr)
    return grads


def line_integrals_adjoint(d: dict, gL, M: int, mode: int = TRILINEAR, ray_ids=None):
    n, r = _rays(d, ray_ids)
    gL = np.ascontiguousarray(gL, dtype=np.float64).reshape(n, M)
    shape = (int(d["pNumZ"]), int(d["pNumY"]), int(d["pNumX"]))
    grads = [np.zeros(shape, np.float64) for _ in range(M)]
    arr = (C.c_void_p * M)(*[g.ctypes.data for g in grads])
    lib().orc_line_integrals_adjoint(C.byref(geom(d)), M, mode, C.c_int64(n), _p(r), _p(gL), arr)
    return grads


def finalize(I, I0):
    I = _f32(I)
    I0 = _f32(I0)
    n_pix = I0.size
    n_views = I.size // n_pix
    Ip = np.empty(I.shape, np.uint32)
    proj = np.empty(I.shape, np.float32)
    lib().orc_finalize(C.c_int64(n_pix), C.c_int64(n_views), _p(I), _p(I0), _p(Ip), _p(proj))
    return Ip, proj


def scint_thickness(n_pix: int, thickness: float, err: float) -> np.ndarray:
    out = np.empty(n_pix, np.float32)
    lib().orc_scint_thickness(C.c_int64(n_pix), C.c_float(thickness), C.c_float(err), _p(out))
    return out


def det_response(mu_scint, thick, factor: float) -> np.ndarray:
    mu = _f32(mu_scint)
    t = _f32(thick)
    D = np.empty((len(mu), t.size), np.float32)
    lib().orc_det_response(len(mu), C.c_int64(t.size), _p(mu), _p(t), C.c_float(factor), _p(D))
    return D


def grid_column(dNumU: int, dSize_mm: float, strip_um: int, inter_um: int, h_mm: float, FD_mm: float,
                mu_strip_mm: float, mu_inter_mm: float) -> np.ndarray:
    out = np.empty(dNumU, np.float32)
    rc = lib().orc_grid_column(C.c_int64(dNumU), C.c_float(dSize_mm), strip_um, inter_um, C.c_float(h_mm),
                               C.c_float(FD_mm), C.c_float(mu_strip_mm), C.c_float(mu_inter_mm), _p(out))
    if rc != 0:
        raise ValueError("grid parameters out of range")
    return out


def grid_pixel(dNumU: int, dNumV: int, dSize_mm: float, strip_um: int, inter_um: int, h_mm: float, FD_mm: float,
               mu_strip_mm, mu_inter_mm, rows=None) -> np.ndarray:
    """Per-pixel, per-energy grid transmission [E][len(rows)][dNumU] in FP64
    for the detector rows listed (all rows when None)."""
    ms, mi = _f32(np.atleast_1d(mu_strip_mm)), _f32(np.atleast_1d(mu_inter_mm))
    rows = np.arange(dNumV, dtype=np.int64) if rows is None else np.ascontiguousarray(rows, dtype=np.int64)
    out = np.empty((len(ms), len(rows), dNumU), np.float64)
    rc = lib().orc_grid_pixel(C.c_int64(dNumU), C.c_int64(dNumV), C.c_float(dSize_mm), strip_um, inter_um,
                              C.c_float(h_mm), C.c_float(FD_mm), len(ms), _p(ms), _p(mi), C.c_int64(len(rows)),
                              _p(rows), _p(out))
    if rc != 0:
        raise ValueError("grid parameters out of range")
    return out


def num_threads() -> int:
    return int(lib().orc_num_threads())
