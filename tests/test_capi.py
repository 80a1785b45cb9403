"""The C-ABI library without a GPU: it loads, exports every declared symbol,
computes the reference's FP32 geometry exactly, and rejects bad input."""
import ctypes as C
import glob
import os
import re
import subprocess

import numpy as np
import pytest

from ct_forward_projection_b200 import _capi as capi
from ct_forward_projection_b200.projector import compute_paras, make_geometry
from oracle import oracle as O
from tests.conftest import ROOT, small_geometry


def _declared(header):
    text = open(header).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ctfp_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = capi.lib()
    headers = glob.glob(os.path.join(ROOT, "include", "*.h"))
    assert headers
    missing = []
    for h in headers:
        for name in _declared(h):
            if not hasattr(lib, name):
                missing.append((os.path.basename(h), name))
    assert not missing, missing


def test_version_string():
    assert capi.lib().ctfp_version().decode().startswith("ctfp")


@pytest.mark.parametrize("views,U,V,dsize,n,length", [(60, 256, 256, 1.0, 128, 128.0), (360, 512, 384, 0.8, 256, 128.0),
                                                     (720, 1024, 768, 0.4, 512, 204.8), (7, 21, 9, 0.37, 17, 9.3)])
def test_compute_paras_bit_exact_vs_oracle(views, U, V, dsize, n, length):
    d = dict(pNumX=n, pNumY=n, pNumZ=n, pLengthX=length, pLengthY=length, pLengthZ=length, projNum=views,
             dNumU=U, dNumV=V, dSize=dsize, sod=1000.0, sdd=1500.0, rotatedDirection=1)
    assert compute_paras(d) == O.compute_paras(d)


def test_view_angles_bit_exact_vs_oracle():
    for rot in (1, -1):
        d = small_geometry(views=13, rot=rot)
        g = make_geometry(d)
        for p in range(13):
            a = C.c_float()
            capi.call("ctfp_view_angle", C.byref(g), p, C.byref(a))
            assert a.value == O.view_angle(d, p)


@pytest.mark.parametrize("field,value", [("pNumX", 0), ("projNum", 0), ("dSize", 0.0), ("sdd", 100.0),
                                         ("rotatedDirection", 2), ("reserved", 1)])
def test_bad_geometry_rejected(field, value):
    d = small_geometry()
    g = make_geometry(d)
    setattr(g, field, value)
    info = capi.SystemInfo()
    st = capi.lib().ctfp_compute_paras(C.byref(g), C.byref(info))
    assert st == capi.CTFP_INVALID_ARG
    assert capi.lib().ctfp_last_error_string().decode()


def test_null_arguments_rejected():
    lib = capi.lib()
    assert lib.ctfp_compute_paras(None, None) == capi.CTFP_INVALID_ARG
    assert lib.ctfp_forward(None, None, None, None, None, None, None) == capi.CTFP_INVALID_ARG
    assert lib.ctfp_backward(None, None, None, None, None, None) == capi.CTFP_INVALID_ARG
    assert lib.ctfp_plan_destroy(None) == capi.CTFP_OK


def test_scintillator_thickness_matches_oracle():
    out = np.empty(1000, np.float32)
    capi.call("ctfp_scintillator_thickness", 1000, C.c_float(0.4), C.c_float(0.05),
              out.ctypes.data_as(C.c_void_p))
    np.testing.assert_array_equal(out, O.scint_thickness(1000, 0.4, 0.05))


def test_no_gpu_plan_create_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    g = make_geometry(small_geometry())
    h = C.c_void_p()
    st = capi.lib().ctfp_plan_create(C.byref(g), 1, 0, 0, C.byref(h))
    assert st in (capi.CTFP_CUDA_ERROR, capi.CTFP_OOM)
    assert not h.value


C_SRC = os.path.join(os.path.dirname(os.path.abspath(__file__)), "c_abi", "forward_host.c")


def _build_c_example(tmp_path):
    exe = str(tmp_path / "forward_host")
    pkg = os.path.dirname(capi.LIB_PATH)
    inc = os.path.join(os.path.dirname(pkg), "include")
    r = subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-I", inc, C_SRC, "-o", exe, "-L", pkg,
                        "-lctfp", f"-Wl,-rpath,{pkg}", "-lm"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_c_caller_compiles_against_the_header(tmp_path):
    # the boundary is plain C: a C99 program builds against include/ctfp.h and links libctfp.so
    assert os.access(_build_c_example(tmp_path), os.X_OK)


@pytest.mark.gpu
def test_c_caller_matches_python_mirror(tmp_path):
    import numpy as np
    exe = _build_c_example(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    got = np.array([[float(x) for x in line.split()] for line in r.stdout.strip().splitlines()], np.float32)
    from ct_forward_projection_b200 import Projector
    d = dict(pNumX=16, pNumY=14, pNumZ=12, pLengthX=16.0, pLengthY=14.0, pLengthZ=12.0, projNum=4, dNumU=20, dNumV=15,
             dSize=1.6, sod=300.0, sdd=450.0, rotatedDirection=1)
    rho = (0.5 + (np.arange(16 * 14 * 12) % 7) * 0.25).astype(np.float32).reshape(12, 14, 16)
    with Projector(d, 1, "trilinear") as pr:
        pr.set_spectral_tables(np.array([0.2, 0.5, 0.3], np.float32), np.array([[0.040], [0.025], [0.018]], np.float32),
                               None, 0, None, 1000.0)
        out = pr.forward_host([rho])
    np.testing.assert_array_equal(got[:, 0], out["I"].ravel())
    np.testing.assert_array_equal(got[:, 1], out["IAbsorb"].ravel())
