"""ctfp_forward_noalloc, the forward for callers that cannot allocate device
memory (a host framework that owns every byte through its own pool, a
real-time loop that may not allocate after start-up, a process on a fixed
memory budget).  It is checked through the C ABI against the plan-based
ctfp_forward, on two calls in a row; the scratch it keeps in a fixed device
array holds the previous call's tables when the second call starts.

This file is collected last so that a run stopping at its first failure has
already run every other test."""
import ctypes as C

import numpy as np
import pytest
import torch

from ct_forward_projection_b200 import Projector
from ct_forward_projection_b200 import _capi as capi
from ct_forward_projection_b200.projector import make_geometry
from tests.conftest import random_volumes, small_geometry, spectral_setup

pytestmark = pytest.mark.gpu

RTOL = 1e-5  # the tolerance of the forward parity tests


def _prepare(d, vols, S, mu, G, D):
    """Device inputs and outputs of one call, allocated by the test beforehand."""
    P, V, U = d["projNum"], d["dNumV"], d["dNumU"]
    return dict(d=d, vols=vols, S=np.ascontiguousarray(S, np.float32), mu=np.ascontiguousarray(mu, np.float32),
                G=None if G is None else torch.from_numpy(G).cuda(), D=None if D is None else torch.from_numpy(D).cuda(),
                I=torch.empty((P, V, U), device="cuda"), A=torch.empty((P, V, U), device="cuda"),
                I0=torch.empty((V, U), device="cuda"), ptrs=capi.ptr_array([v.data_ptr() for v in vols]),
                g=make_geometry(d))


def _noalloc(c, layout, I0Val, interp):
    capi.call("ctfp_forward_noalloc", C.byref(c["g"]), len(c["vols"]), interp, len(c["S"]),
              c["S"].ctypes.data_as(C.c_void_p), c["mu"].ctypes.data_as(C.c_void_p),
              None if c["G"] is None else c["G"].data_ptr(), layout,
              None if c["D"] is None else c["D"].data_ptr(), C.c_float(I0Val), c["ptrs"], c["I"].data_ptr(),
              c["A"].data_ptr(), c["I0"].data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return c["I"].clone(), c["A"].clone(), c["I0"].clone()


def _rel(a, b):
    a = a.double().cpu().numpy()
    b = b.double().cpu().numpy()
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-30)))


def _free_bytes():
    torch.cuda.synchronize()
    return torch.cuda.mem_get_info()[0]


@pytest.mark.parametrize("interp", [0, 1])
def test_noalloc_matches_plan_forward_twice(interp):
    cases = []
    for k, (geo, M, E, layout) in enumerate([(dict(n=20, views=7, U=24, V=14), 2, 13, 2),
                                             (dict(n=(18, 14, 11), views=5, U=17, V=9, rot=-1), 3, 21, 1)]):
        d = small_geometry(**geo)
        vols = [torch.from_numpy(v).cuda() for v in random_volumes(d, M, 900 + k)]
        S, mu, G, D = spectral_setup(d, M, E, 40 + k)
        if layout == 1:
            G = np.ascontiguousarray(G[:, 0, :])
        with Projector(d, M, "trilinear" if interp == 0 else "texemu") as pr:
            pr.set_spectral_tables(S, mu, G, layout, D, 60000.0)
            ref = pr.forward(vols)
            torch.cuda.synchronize()
        cases.append((_prepare(d, vols, S, mu, G, D), layout, ref))
    _noalloc(cases[0][0], cases[0][1], 60000.0, interp)  # first call on this device: looks up the scratch address
    # two calls in a row of different problems, then the first again: each call
    # must rewrite the scratch the previous one left behind
    results = []
    free0 = _free_bytes()
    for c, layout, ref in cases + cases[:1]:
        capi.call("ctfp_forward_noalloc", C.byref(c["g"]), len(c["vols"]), interp, len(c["S"]),
                  c["S"].ctypes.data_as(C.c_void_p), c["mu"].ctypes.data_as(C.c_void_p),
                  None if c["G"] is None else c["G"].data_ptr(), layout,
                  None if c["D"] is None else c["D"].data_ptr(), C.c_float(60000.0), c["ptrs"], c["I"].data_ptr(),
                  c["A"].data_ptr(), c["I0"].data_ptr(), torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        # copies straight to host memory: no device allocation inside the measured window
        results.append((c["I"].cpu().double(), c["A"].cpu().double(), c["I0"].cpu().double(), ref))
    # the calls took no device memory (every buffer above was allocated by the test beforehand)
    assert _free_bytes() == free0
    for I, A, I0, ref in results:
        assert _rel(I, ref["I"]) < RTOL
        assert _rel(A, ref["IAbsorb"]) < RTOL
        assert _rel(I0, ref["I0"]) < RTOL


def test_noalloc_rejects_sizes_beyond_its_scratch():
    d = small_geometry(views=8193)
    v = torch.zeros((d["pNumZ"], d["pNumY"], d["pNumX"]), device="cuda")
    S = np.ones(3, np.float32) / 3
    mu = np.full((3, 1), 0.02, np.float32)
    out = torch.empty(1, device="cuda")
    st = capi.lib().ctfp_forward_noalloc(C.byref(make_geometry(d)), 1, 0, 3, S.ctypes.data_as(C.c_void_p),
                                         mu.ctypes.data_as(C.c_void_p), None, 0, None, C.c_float(1.0),
                                         capi.ptr_array([v.data_ptr()]), out.data_ptr(), out.data_ptr(), None,
                                         None)
    assert st == capi.CTFP_INVALID_ARG
    assert "CTFP_NOALLOC_MAX_VIEWS" in capi.lib().ctfp_last_error_string().decode()
    d = small_geometry(views=4)
    S = np.ones(300, np.float32)
    mu = np.zeros((300, 1), np.float32)
    st = capi.lib().ctfp_forward_noalloc(C.byref(make_geometry(d)), 1, 0, 300, S.ctypes.data_as(C.c_void_p),
                                         mu.ctypes.data_as(C.c_void_p), None, 0, None, C.c_float(1.0),
                                         capi.ptr_array([v.data_ptr()]), out.data_ptr(), out.data_ptr(), None,
                                         None)
    assert st == capi.CTFP_INVALID_ARG
    st = capi.lib().ctfp_forward_noalloc(C.byref(make_geometry(d)), 1, 2, 3, S.ctypes.data_as(C.c_void_p),
                                         mu.ctypes.data_as(C.c_void_p), None, 0, None, C.c_float(1.0),
                                         capi.ptr_array([v.data_ptr()]), out.data_ptr(), out.data_ptr(), None,
                                         None)
    assert st == capi.CTFP_UNSUPPORTED


@pytest.mark.parametrize("interp", [0, 1])
def test_noalloc_without_grid_response_or_flat_field(interp):
    """The optional inputs: no grid table (layout 0), no detector response
    (D NULL) and no flat-field output (I0 NULL, its kernel skipped), with one
    material and with four, against the plan forward on the same inputs."""
    for k, (geo, M, layout, with_D) in enumerate([(dict(n=16, views=5, U=19, V=11), 1, 0, False),
                                                  (dict(n=(14, 18, 12), views=6, U=15, V=13), 4, 2, False),
                                                  (dict(n=12, views=3, U=9, V=21, rot=-1), 4, 0, True)]):
        d = small_geometry(**geo)
        vols = [torch.from_numpy(v).cuda() for v in random_volumes(d, M, 950 + k)]
        S, mu, G, D = spectral_setup(d, M, 9, 60 + k, grid=layout != 0, det=with_D)
        with Projector(d, M, "trilinear" if interp == 0 else "texemu") as pr:
            pr.set_spectral_tables(S, mu, G, layout, D, 1000.0)
            ref = pr.forward(vols)
            torch.cuda.synchronize()
        c = _prepare(d, vols, S, mu, G, D)
        for _ in range(2):
            capi.call("ctfp_forward_noalloc", C.byref(c["g"]), M, interp, len(c["S"]),
                      c["S"].ctypes.data_as(C.c_void_p), c["mu"].ctypes.data_as(C.c_void_p),
                      None if c["G"] is None else c["G"].data_ptr(), layout,
                      None if c["D"] is None else c["D"].data_ptr(), C.c_float(1000.0), c["ptrs"],
                      c["I"].data_ptr(), c["A"].data_ptr(), None, torch.cuda.current_stream().cuda_stream)
            torch.cuda.synchronize()
            assert _rel(c["I"], ref["I"]) < RTOL
            assert _rel(c["A"], ref["IAbsorb"]) < RTOL


def test_noalloc_refuses_a_capturing_stream():
    """Each call copies its host tables from pageable memory, which a graph
    capture cannot record: on a capturing stream the call returns
    CTFP_UNSUPPORTED before it issues anything, and the capture stays valid."""
    d = small_geometry(n=12, views=3, U=9, V=7)
    vols = [torch.from_numpy(v).cuda() for v in random_volumes(d, 1, 990)]
    S, mu, G, D = spectral_setup(d, 1, 5, 70, grid=False, det=False)
    c = _prepare(d, vols, S, mu, G, D)
    x = torch.zeros(4, device="cuda")
    s = torch.cuda.Stream()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=s):
        st = capi.lib().ctfp_forward_noalloc(C.byref(c["g"]), 1, 0, len(c["S"]), c["S"].ctypes.data_as(C.c_void_p),
                                             c["mu"].ctypes.data_as(C.c_void_p), None, 0, None, C.c_float(1.0),
                                             c["ptrs"], c["I"].data_ptr(), c["A"].data_ptr(), None,
                                             C.c_void_p(s.cuda_stream))
        x.add_(1.0)
    assert st == capi.CTFP_UNSUPPORTED
    assert "capturing" in capi.lib().ctfp_last_error_string().decode()
    graph.replay()
    torch.cuda.synchronize()
    assert float(x[0]) == 1.0
    # outside the capture the same call runs
    _noalloc(c, 0, 1.0, 0)
