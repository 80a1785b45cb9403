"""Python host mirror of the projector over the C ABI (include/ctfp.h).

`Projector` is one plan: the geometry of CTScanParas (DataType.h:33-55), the
number of materials, the sampler, and the spectral tables.  Device memory is
torch tensors on the plan's CUDA device; every compute call goes through
libctfp.so, and there is no other compute path.
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence

import numpy as np

from . import _capi as capi
from ._capi import Geometry, GridParams, SystemInfo, call, lib, ptr_array

INTERP = {"trilinear": capi.INTERP_TRILINEAR, "texemu": capi.INTERP_TEXEMU, "texture": capi.INTERP_TEXTURE}


def make_geometry(d: dict) -> Geometry:
    g = Geometry()
    for k in ("pNumX", "pNumY", "pNumZ", "projNum", "dNumU", "dNumV"):
        setattr(g, k, int(d[k]))
    for k in ("pLengthX", "pLengthY", "pLengthZ", "dSize", "sod", "sdd"):
        setattr(g, k, float(d[k]))
    g.rotatedDirection = int(d.get("rotatedDirection", 1))
    g.reserved = 0
    return g


def compute_paras(geom: dict) -> dict:
    """CBCTForwardProj::computeParas (CBCTForwardProj.cpp:23-62) via the library."""
    info = SystemInfo()
    call("ctfp_compute_paras", C.byref(make_geometry(geom)), C.byref(info))
    return {k: getattr(info, k) for k, _ in SystemInfo._fields_}


def _np_ptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.float32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.c_void_p)


def _dptr(t) -> int | None:
    if t is None:
        return None
    import torch
    assert isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float32 and t.is_contiguous(), \
        "device tensors must be contiguous float32 CUDA tensors"
    return t.data_ptr()


def _dp(t, numel: int, name: str, device: int) -> int | None:
    """Device pointer of an argument after the checks the C ABI cannot make
    (it sees only the pointer): a contiguous float32 tensor on the plan's
    device with exactly the number of elements the call reads or writes."""
    if t is None:
        return None
    import torch
    if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float32 and t.is_contiguous()):
        raise TypeError(f"{name}: a contiguous float32 CUDA tensor is required")
    if t.device.index != device:
        raise ValueError(f"{name} is on {t.device}; the plan is on cuda:{device}")
    if t.numel() != numel:
        raise ValueError(f"{name} holds {t.numel()} elements; the call needs {numel}")
    return t.data_ptr()


def _hp(a, numel: int, name: str):
    """Host pointer of an argument (numpy array or CPU tensor, float32,
    contiguous) holding exactly numel elements."""
    if a is None:
        return None
    n = a.size if isinstance(a, np.ndarray) else a.numel()
    if n != numel:
        raise ValueError(f"{name} holds {n} elements; the call needs {numel}")
    return _host_ptr(a)


def _stream(stream) -> int | None:
    import torch
    if stream is None:
        return torch.cuda.current_stream().cuda_stream
    return stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream)


class Projector:
    """One projection plan (replaces the reference's initDevice* + forward*GPU)."""

    def __init__(self, geometry: dict, n_materials: int, interp: str = "trilinear", device: int = 0):
        self.geometry = dict(geometry)
        self.M = int(n_materials)
        self.interp = interp
        self.device = int(device)
        self._g = make_geometry(self.geometry)
        h = C.c_void_p()
        call("ctfp_plan_create", C.byref(self._g), self.M, INTERP[interp], self.device, C.byref(h))
        self._h = h
        info = SystemInfo()
        call("ctfp_plan_get_system_info", self._h, C.byref(info))
        self.info = {k: getattr(info, k) for k, _ in SystemInfo._fields_}
        self.E = 0

    # -- lifetime -----------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().ctfp_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    @property
    def shape_proj(self) -> tuple[int, int, int]:
        g = self.geometry
        return (int(g["projNum"]), int(g["dNumV"]), int(g["dNumU"]))

    @property
    def shape_vol(self) -> tuple[int, int, int]:
        g = self.geometry
        return (int(g["pNumZ"]), int(g["pNumY"]), int(g["pNumX"]))

    def set_interp(self, interp: str) -> None:
        call("ctfp_plan_set_interp", self._h, INTERP[interp])
        self.interp = interp

    def set_sampler(self, sampler: str) -> None:
        """'global' (linear volumes through L1), 'layered' (texture gathers
        from z-layered copies), 'axis' (gathers from copies layered along the
        view's major in-plane axis, reused across samples) or 'brick'
        (per-bundle voxel boxes in shared memory)."""
        call("ctfp_plan_set_sampler", self._h, {"global": capi.SAMPLER_GLOBAL, "layered": capi.SAMPLER_LAYERED,
                                                 "brick": capi.SAMPLER_BRICK, "axis": capi.SAMPLER_AXIS}[sampler])

    def set_focal_spot(self, offset_u=None, offset_v=None) -> None:
        """Per-view focal-spot offsets in mm (ctfp_plan_set_focal_spot); None clears."""
        if offset_u is None:
            call("ctfp_plan_set_focal_spot", self._h, None, None)
            return
        u = np.ascontiguousarray(offset_u, dtype=np.float32)
        v = np.ascontiguousarray(offset_v, dtype=np.float32)
        assert u.shape == v.shape == (self.shape_proj[0],), "one offset pair per view"
        call("ctfp_plan_set_focal_spot", self._h, _np_ptr(u), _np_ptr(v))

    def set_skip_empty(self, enable: bool = True) -> None:
        """Empty-space skipping for the layered sampler (ctfp_plan_set_skip_empty)."""
        call("ctfp_plan_set_skip_empty", self._h, 1 if enable else 0)

    def check_status(self, raise_on_timeout: bool = False) -> int:
        """ctfp_plan_check_status: waits for the device, returns and clears
        the plan's status bits (1: a TMA-staged brick wait ran out; outputs
        stay correct).  raise_on_timeout raises CtfpError(CTFP_TIMEOUT) then.
        Bit 2 (the wait at a CTA's exit ran out too: outputs not trusted)
        always raises CtfpError(CTFP_CUDA_ERROR)."""
        flags = C.c_uint32()
        st = lib().ctfp_plan_check_status(self._h, C.byref(flags))
        if st == capi.CTFP_TIMEOUT and not raise_on_timeout:
            return int(flags.value)
        capi.check(st, "ctfp_plan_check_status")
        return int(flags.value)

    def set_launch_shape(self, tile_u: int, tile_v: int, views_per_cta: int = 1, min_ctas_per_sm: int = 2) -> None:
        call("ctfp_plan_set_launch_shape", self._h, tile_u, tile_v, views_per_cta, min_ctas_per_sm)

    def autotune(self, volumes: Sequence, n_sample_views: int = 64, stream=None) -> dict:
        """ctfp_plan_autotune: times launch shapes on a sample of views and
        sets the fastest; returns it with its time and whether it was cached."""
        import torch
        P, V, U = self.shape_proj
        dev = f"cuda:{self.device}"
        I = torch.empty((P, V, U), device=dev)
        A = torch.empty((P, V, U), device=dev)
        r = capi.LaunchShape()
        call("ctfp_plan_autotune", self._h, self._vol_ptrs(volumes), _dptr(I), _dptr(A), int(n_sample_views),
             C.byref(r), _stream(stream))
        return {k: getattr(r, k) for k, _ in capi.LaunchShape._fields_}

    # -- tables -------------------------------------------------------------
    def set_spectral_tables(self, spectrum, mu, grid=None, grid_layout: int | None = None, det_response=None,
                            I0Val: float = 60000.0) -> None:
        """spectrum [E]; mu [E][M] (1/mm per g/cm^3); grid [E][U] or [E][V][U];
        det_response [E][V][U]; host numpy arrays."""
        S = np.ascontiguousarray(spectrum, dtype=np.float32)
        mu = np.ascontiguousarray(mu, dtype=np.float32).reshape(len(S), self.M)
        G = None if grid is None else np.ascontiguousarray(grid, dtype=np.float32)
        if G is not None and grid_layout is None:
            grid_layout = capi.GRID_COLUMN if G.ndim == 2 else capi.GRID_PIXEL
        D = None if det_response is None else np.ascontiguousarray(det_response, dtype=np.float32)
        call("ctfp_set_spectral_tables", self._h, len(S), _np_ptr(S), _np_ptr(mu), _np_ptr(G),
             int(grid_layout or 0), _np_ptr(D), float(I0Val))
        self.E = len(S)

    def set_tables_from_workload(self, w, device_tables: bool = True) -> None:
        """Builds grid/scintillator tables for a physics.Workload on the device
        and installs the spectral tables."""
        import torch
        E = len(w.energies)
        U, V = int(self.geometry["dNumU"]), int(self.geometry["dNumV"])
        G = D = None
        layout = 0
        if w.grid is not None:
            ms, mi = w.grid_mu()
            layout = w.grid_layout
            G = build_grid_table(self.geometry, w.grid, ms, mi, layout, device=self.device).cpu().numpy()
        if w.scint_mm is not None:
            t = scintillator_thickness(U * V, w.scint_mm, w.scint_err_mm)
            D = build_det_response(w.scint_mu(), torch.from_numpy(t).to(f"cuda:{self.device}"), 1.0).cpu().numpy()
            D = D.reshape(E, V, U)
        self.set_spectral_tables(w.spectrum(), w.mu_table(), G, layout if G is not None else 0, D, w.I0Val)

    # -- compute ------------------------------------------------------------
    @property
    def n_voxels(self) -> int:
        z, y, x = self.shape_vol
        return z * y * x

    def _vol_ptrs(self, volumes: Sequence, name: str = "volume"):
        if len(volumes) != self.M:
            raise ValueError(f"expected {self.M} {name}s, got {len(volumes)}")
        for v in volumes:
            if tuple(v.shape) != self.shape_vol:
                raise ValueError(f"{name} shape {tuple(v.shape)} != {self.shape_vol}")
        return ptr_array([_dp(v, self.n_voxels, name, self.device) for v in volumes])

    def forward(self, volumes: Sequence, want_L: bool = False, out=None, stream=None, views=None) -> dict:
        """Fused march + spectral epilogue. Returns dict(I, IAbsorb, I0[, L]).
        views=(view0, n): only those views, in compact [n][V][U] outputs
        (ctfp_forward_views)."""
        import torch
        dev = f"cuda:{self.device}"
        P, V, U = self.shape_proj
        n = P if views is None else int(views[1])
        if out is None:
            out = {"I": torch.empty((n, V, U), device=dev), "IAbsorb": torch.empty((n, V, U), device=dev),
                   "I0": torch.empty((V, U), device=dev)}
            if want_L:
                out["L"] = torch.empty((n, V, U, self.M), device=dev)
        d = self.device
        ptrs = (_dp(out.get("I"), n * V * U, "I", d), _dp(out.get("IAbsorb"), n * V * U, "IAbsorb", d),
                _dp(out.get("I0"), V * U, "I0", d), _dp(out.get("L"), n * V * U * self.M, "L", d))
        if views is None:
            call("ctfp_forward", self._h, self._vol_ptrs(volumes), *ptrs, _stream(stream))
        else:
            call("ctfp_forward_views", self._h, self._vol_ptrs(volumes), int(views[0]), n, *ptrs, _stream(stream))
        return out

    def forward_host(self, host_volumes: Sequence[np.ndarray], out: dict | None = None) -> dict:
        """ctfp_forward_host: host volumes in, host I/IAbsorb/I0 out."""
        P, V, U = self.shape_proj
        if out is None:
            out = {"I": np.empty((P, V, U), np.float32), "IAbsorb": np.empty((P, V, U), np.float32),
                   "I0": np.empty((V, U), np.float32)}
        if len(host_volumes) != self.M:
            raise ValueError(f"expected {self.M} volumes, got {len(host_volumes)}")
        ptrs = ptr_array([_hp(v, self.n_voxels, "volume") for v in host_volumes])
        call("ctfp_forward_host", self._h, ptrs, _hp(out["I"], P * V * U, "I"),
             _hp(out["IAbsorb"], P * V * U, "IAbsorb"), _hp(out.get("I0"), V * U, "I0"), _stream(None))
        return out

    def line_integrals(self, volumes: Sequence, out=None, stream=None):
        import torch
        P, V, U = self.shape_proj
        if out is None:
            out = torch.empty((P, V, U, self.M), device=f"cuda:{self.device}")
        call("ctfp_line_integrals", self._h, self._vol_ptrs(volumes), _dp(out, P * V * U * self.M, "L", self.device),
             _stream(stream))
        return out

    def spectral_from_L(self, L, stream=None) -> dict:
        import torch
        P, V, U = self.shape_proj
        dev = f"cuda:{self.device}"
        out = {"I": torch.empty((P, V, U), device=dev), "IAbsorb": torch.empty((P, V, U), device=dev)}
        call("ctfp_spectral_from_L", self._h, _dp(L, P * V * U * self.M, "L", self.device), _dptr(out["I"]),
             _dptr(out["IAbsorb"]), _stream(stream))
        return out

    def backward(self, L, gI=None, gIAbsorb=None, grads=None, stream=None, views=None) -> list:
        """Adds dLoss/drho_m into grads (created as zeros if None).
        views=(view0, n): L, gI, gIAbsorb are the compact buffers of those
        views (ctfp_backward_views)."""
        import torch
        if grads is None:
            grads = [torch.zeros(self.shape_vol, device=f"cuda:{self.device}") for _ in range(self.M)]
        P, V, U = self.shape_proj
        n = P if views is None else int(views[1])
        d = self.device
        gp = self._vol_ptrs(grads, "gradient")
        args = (_dp(L, n * V * U * self.M, "L", d), _dp(gI, n * V * U, "gI", d),
                _dp(gIAbsorb, n * V * U, "gIAbsorb", d))
        if views is None:
            call("ctfp_backward", self._h, *args, gp, _stream(stream))
        else:
            call("ctfp_backward_views", self._h, *args, int(views[0]), n, gp, _stream(stream))
        return grads

    def line_integrals_adjoint(self, gL, grads=None, stream=None) -> list:
        import torch
        if grads is None:
            grads = [torch.zeros(self.shape_vol, device=f"cuda:{self.device}") for _ in range(self.M)]
        P, V, U = self.shape_proj
        call("ctfp_line_integrals_adjoint", self._h, _dp(gL, P * V * U * self.M, "gL", self.device),
             self._vol_ptrs(grads, "gradient"), _stream(stream))
        return grads

    def axis_gather_count(self) -> float:
        """ctfp_axis_gather_count: texture quad-gathers per voxel-sample of the
        axis sampler's march (0.5 = both gathers of every sample in full warps)."""
        r = C.c_double()
        call("ctfp_axis_gather_count", self._h, C.byref(r))
        return float(r.value)

    def count_support_samples(self) -> int:
        n = C.c_int64()
        call("ctfp_count_support_samples", self._h, C.byref(n))
        return int(n.value)


class Batch:
    """ctfp_batch: several plans in one persistent launch replayed as a CUDA
    graph.  Keeps references to its projectors; close it before them."""

    def __init__(self, projectors: Sequence[Projector]):
        self.projectors = list(projectors)
        plans = ptr_array([p.handle.value for p in self.projectors])
        h = C.c_void_p()
        call("ctfp_batch_create", len(self.projectors), plans, C.byref(h))
        self._h = h
        self._keep = []

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().ctfp_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_shape(self, tile_u: int, tile_v: int) -> None:
        """ctfp_batch_set_shape: tile_u x tile_v (= 64) rays per work unit."""
        call("ctfp_batch_set_shape", self._h, tile_u, tile_v)

    def set_views(self, fwd_views: int, adj_views: int) -> None:
        """ctfp_batch_set_views: views per work unit of the forward and of the
        fused forward + adjoint (1 to 8)."""
        call("ctfp_batch_set_views", self._h, fwd_views, adj_views)

    def autotune(self, volumes: Sequence[Sequence], targets: Sequence, stream=None) -> dict:
        """ctfp_batch_autotune: times the forward and the fused kernels with
        candidate ray tiles and views per unit and keeps the fastest of each;
        returns the fused kernel's tile (tile_u, tile_v), views per unit and
        ms, and the forward's tile (fwd_tile_u, fwd_tile_v) and views."""
        self._keep = []
        vt = self._vol_table(volumes)
        T = self._item_ptrs(targets, 1, "target")
        r = capi.LaunchShape()
        call("ctfp_batch_autotune", self._h, vt, T, C.byref(r), _stream(stream))
        sh = self.shapes()
        return {"tile_u": r.tile_u, "tile_v": r.tile_v, "views": r.views_per_cta, "ms": r.ms,
                "fwd_tile_u": sh["fwd"][0], "fwd_tile_v": sh["fwd"][1], "fwd_views": sh["views"][0]}

    def shapes(self) -> dict:
        """ctfp_batch_get_shapes and ctfp_batch_get_views: the work-unit ray
        tiles of the two kinds of call, and their views per unit
        ("views": (forward, fused))."""
        a, b, c, d = C.c_int32(), C.c_int32(), C.c_int32(), C.c_int32()
        call("ctfp_batch_get_shapes", self._h, C.byref(a), C.byref(b), C.byref(c), C.byref(d))
        f, j = C.c_int32(), C.c_int32()
        call("ctfp_batch_get_views", self._h, C.byref(f), C.byref(j))
        return {"fwd": (int(a.value), int(b.value)), "fwd_adjoint": (int(c.value), int(d.value)),
                "views": (int(f.value), int(j.value))}

    def info(self) -> dict:
        u, g0, g1 = C.c_int64(), C.c_int32(), C.c_int32()
        call("ctfp_batch_info", self._h, C.byref(u), C.byref(g0), C.byref(g1))
        return {"units": int(u.value), "grid_forward": int(g0.value), "grid_adjoint": int(g1.value)}

    def _vol_table(self, volumes, name: str = "volume"):
        if len(volumes) != len(self.projectors):
            raise ValueError(f"expected {len(self.projectors)} items, got {len(volumes)}")
        per = [p._vol_ptrs(v, name) for p, v in zip(self.projectors, volumes)]
        self._keep = self._keep + per
        return ptr_array([C.cast(a, C.c_void_p).value for a in per])

    def _item_ptrs(self, tensors, per_ray: int, name: str):
        """One pointer per item: tensors[k] holds rays(k) * per_ray floats."""
        if len(tensors) != len(self.projectors):
            raise ValueError(f"expected {len(self.projectors)} {name} entries, got {len(tensors)}")
        out = []
        for p, t in zip(self.projectors, tensors):
            P, V, U = p.shape_proj
            out.append(_dp(t, P * V * U * (p.M if per_ray < 0 else per_ray), name, p.device))
        return ptr_array(out)

    def _out(self, want_L: bool = False) -> list:
        import torch
        outs = []
        for p in self.projectors:
            dev = f"cuda:{p.device}"
            P, V, U = p.shape_proj
            o = {"I": torch.empty((P, V, U), device=dev), "IAbsorb": torch.empty((P, V, U), device=dev)}
            if want_L:
                o["L"] = torch.empty((P, V, U, p.M), device=dev)
            outs.append(o)
        return outs

    def forward(self, volumes: Sequence[Sequence], want_L: bool = False, out: list | None = None, stream=None) -> list:
        """volumes[k] = the M density maps of item k; returns [dict(I, IAbsorb[, L])]."""
        out = out if out is not None else self._out(want_L)
        self._keep = []
        vt = self._vol_table(volumes)
        I = self._item_ptrs([o["I"] for o in out], 1, "I")
        A = self._item_ptrs([o.get("IAbsorb") for o in out], 1, "IAbsorb")
        L = self._item_ptrs([o.get("L") for o in out], -1, "L") if any("L" in o for o in out) else None
        call("ctfp_batch_forward", self._h, vt, I, A, L, _stream(stream))
        return out

    def forward_adjoint(self, volumes: Sequence[Sequence], targets: Sequence, grads: list | None = None,
                        I_out: list | None = None, loss=None, stream=None) -> dict:
        """Fused forward + sum (log I - log T)^2 + adjoint; grads accumulate."""
        import torch
        if grads is None:
            grads = [[torch.zeros(p.shape_vol, device=f"cuda:{p.device}") for _ in range(p.M)]
                     for p in self.projectors]
        if loss is None:
            loss = torch.zeros(len(self.projectors), device=f"cuda:{self.projectors[0].device}")
        self._keep = []
        vt = self._vol_table(volumes)
        G = self._vol_table(grads, "gradient")
        T = self._item_ptrs(targets, 1, "target")
        I = self._item_ptrs(I_out, 1, "I") if I_out is not None else None
        lp = _dp(loss, len(self.projectors), "loss", self.projectors[0].device) if loss is not None else None
        call("ctfp_batch_forward_adjoint", self._h, vt, T, I, G, lp, _stream(stream))
        return {"grads": grads, "loss": loss, "I": I_out}


def _host_ptr(a):
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return _np_ptr(a)
    import torch
    assert isinstance(a, torch.Tensor) and not a.is_cuda and a.dtype == torch.float32 and a.is_contiguous()
    return a.data_ptr()


def finalize_counts(I, IAbsorb, I0, stream=None) -> dict:
    """Ipoly = floor(I) (uint32 as int32 tensor bits), IAbsPoly, proj = log(I0/Ipoly)."""
    import torch
    P, V, U = I.shape
    Ip = torch.empty((P, V, U), dtype=torch.int32, device=I.device)
    Ap = torch.empty((P, V, U), dtype=torch.int32, device=I.device)
    proj = torch.empty((P, V, U), dtype=torch.float32, device=I.device)
    call("ctfp_finalize_counts", V * U, P, _dptr(I), _dptr(IAbsorb), _dptr(I0), Ip.data_ptr(), Ap.data_ptr(),
         _dptr(proj), _stream(stream))
    return {"Ipoly": Ip, "IAbsPoly": Ap, "proj": proj}


def sample_volume(volume, points, interp: str, stream=None):
    """Samples volume [nz][ny][nx] at points [n][3] (x, y, z voxel coordinates)."""
    import torch
    nz, ny, nx = volume.shape
    out = torch.empty(points.shape[0], device=volume.device)
    call("ctfp_sample_volume", _dptr(volume), nx, ny, nz, INTERP[interp], _dptr(points.contiguous()),
         points.shape[0], _dptr(out), _stream(stream))
    return out


def focal_spot_offsets(n_views: int, focal_spot_size: float) -> tuple[np.ndarray, np.ndarray]:
    """The reference's per-view focal-spot offsets (ctfp_focal_spot_offsets), mm."""
    u = np.empty(int(n_views), np.float32)
    v = np.empty(int(n_views), np.float32)
    call("ctfp_focal_spot_offsets", int(n_views), float(focal_spot_size), _np_ptr(u), _np_ptr(v))
    return u, v


def sampler_peak(device: int = 0, kind: str = "layered") -> float:
    """ctfp_sampler_peak: voxel-samples/s the texture path delivers at most
    ('layered': two tld4 gathers per sample; 'tex3d': one filtered fetch)."""
    r = C.c_double()
    call("ctfp_sampler_peak", int(device), capi.SAMPLER_LAYERED if kind == "layered" else 0, C.byref(r))
    return float(r.value)


def build_grid_table(geometry: dict, grid, mu_strip, mu_inter, layout: int, device: int = 0):
    import torch
    g = make_geometry(geometry)
    gp = GridParams(int(grid.strip_um), int(grid.inter_um), float(grid.h_mm), float(grid.FD_mm))
    ms = np.ascontiguousarray(mu_strip, dtype=np.float32)
    mi = np.ascontiguousarray(mu_inter, dtype=np.float32)
    E = len(ms)
    shape = (E, int(geometry["dNumU"])) if layout == capi.GRID_COLUMN else \
        (E, int(geometry["dNumV"]), int(geometry["dNumU"]))
    out = torch.empty(shape, device=f"cuda:{device}")
    call("ctfp_build_grid_table", C.byref(g), C.byref(gp), E, _np_ptr(ms), _np_ptr(mi), layout, _dptr(out),
         _stream(None))
    return out


def scintillator_thickness(n_pix: int, thickness: float, thickness_err: float) -> np.ndarray:
    out = np.empty(n_pix, np.float32)
    call("ctfp_scintillator_thickness", n_pix, float(thickness), float(thickness_err), _np_ptr(out))
    return out


def build_det_response(mu_scint, thickness_dev, factor: float):
    import torch
    mu = np.ascontiguousarray(mu_scint, dtype=np.float32)
    n = thickness_dev.numel()
    out = torch.empty((len(mu), n), device=thickness_dev.device)
    call("ctfp_build_det_response", len(mu), n, _np_ptr(mu), _dptr(thickness_dev), float(factor), _dptr(out),
         _stream(None))
    return out


def labels_to_density(labels_dev, density: Sequence[float]):
    import torch
    M = len(density)
    d = np.ascontiguousarray(density, dtype=np.float32)
    outs = [torch.empty(labels_dev.shape, device=labels_dev.device) for _ in range(M)]
    call("ctfp_labels_to_density", labels_dev.data_ptr(), labels_dev.numel(), M, _np_ptr(d),
         ptr_array([o.data_ptr() for o in outs]), _stream(None))
    return outs
