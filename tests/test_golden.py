"""Parity with the reference's own projector.

tests/golden/reference_cases.npz holds the outputs of the reference's CUDA
pipeline (built from its sources by oracle/build_ref.sh, run on a B200 by
tests/golden/make_golden.py) for one small seeded case per dispatch branch of
ForwardProjection::run, with the inputs.  The reference samples through
tex3D, so the comparisons use the texture-unit emulation (oracle and CUDA) and
the hardware texture (CUDA); the bound is 1e-3 relative per pixel on the
counts, as the reference's FP32 coordinates move samples across the texture
unit's 1/256 steps.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O

FIX = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_cases.npz")
CASES = ["grid_response_multi", "grid_response_sinmat", "nogrid_response_multi", "nogrid_response_sinmat",
         "grid_noresponse_sinmat", "nogrid_noresponse_sinmat", "test_i0"]
RTOL_COUNTS = 1e-3
ATOL_PROJ = 1e-3


@pytest.fixture(scope="module")
def fx():
    if not os.path.exists(FIX):
        pytest.fail(f"missing golden fixtures {FIX}")
    return np.load(FIX)


def inputs(z, name):
    gv = z["geometry"]
    keys = ("pNumX", "pNumY", "pNumZ", "pLengthX", "pLengthY", "pLengthZ", "projNum", "dNumU", "dNumV", "dSize",
            "sod", "sdd", "rotatedDirection")
    g = {k: (int(v) if k in ("pNumX", "pNumY", "pNumZ", "projNum", "dNumU", "dNumV", "rotatedDirection")
             else float(v)) for k, v in zip(keys, gv)}
    p = name + "/"
    flags = dict(zip(("IsTestI0", "IsDetResponse", "IsGrid", "IsSingleMaterial"), z[p + "flags"].tolist()))
    lab = z[p + "labels"]
    dens = z[p + "densities"]
    ma = z[p + "mass_atten"]  # [M][E] cm^2/g
    S = z[p + "spectrum"]
    E = S.size
    f32 = np.float32
    if flags["IsSingleMaterial"]:
        vols = [(lab.astype(f32) * dens[0]).astype(f32)]  # PhantomObject::computeDesity (PhantomObject.cpp:65-71)
    else:
        vols = [np.where(lab == m + 1, dens[m], f32(0)).astype(f32) for m in range(len(dens))]
    mu = (ma.T.astype(f32) / f32(10)).astype(f32)  # (mu/rho)/10 (PhantomObject.cpp:56, 62)
    sd, st, se, sf = z["scint_params"]
    FD, h, strip, inter, sdens, idens = z["grid_params"]
    U, V = g["dNumU"], g["dNumV"]
    G = None
    if flags["IsGrid"] and not flags["IsTestI0"]:
        ms = (z[p + "grid_strip_ma"] * f32(sdens)) / f32(10)
        mi = (z[p + "grid_inter_ma"] * f32(idens)) / f32(10)
        G = np.stack([O.grid_column(U, g["dSize"], int(strip), int(inter), float(h), float(FD), float(ms[e]),
                                    float(mi[e])) for e in range(E)])
    D = None
    if flags["IsDetResponse"]:
        thick = O.scint_thickness(U * V, float(st), float(se))
        mus = (z[p + "scint_ma"] * f32(sd)) / f32(10)
        D = O.det_response(mus, thick, float(sf)).reshape(E, V, U)
    return g, flags, vols, S, mu, G, D, float(z["I0Val"][0])


def check_counts(name, I, IAbs, I0, z):
    p = name + "/"
    ref_I0 = z[p + "out_BgImgPro"].astype(np.float64)
    assert np.max(np.abs(I0 - ref_I0) / ref_I0) < 1e-5
    if name == "test_i0":
        return
    for key, mine in (("PhoImgPro", I), ("PhoImgAbsorb", IAbs)):
        ref = z[p + "out_" + key].astype(np.float64)
        got = np.floor(mine)
        # floor() turns any difference at an integer boundary into one count
        err = np.maximum(np.abs(got - ref) - 1.0, 0.0) / np.maximum(ref, 1.0)
        assert np.max(err) < RTOL_COUNTS, (key, float(np.max(err)))
    ref_proj = z[p + "out_Projection"].astype(np.float64)
    Ip = np.floor(I)
    mine_proj = np.log(I0[None] / Ip)
    fin = np.isfinite(ref_proj) & np.isfinite(mine_proj)
    # a one-count flip moves proj by up to 1/count; compare where counts are
    # large enough for the 1e-3 bound to be meaningful
    big = fin & (Ip > 1000)
    assert np.max(np.abs(mine_proj[big] - ref_proj[big])) < ATOL_PROJ


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_reference_binary(fx, name):
    g, flags, vols, S, mu, G, D, I0Val = inputs(fx, name)
    W = O.energy_weights(g, S, G, 1 if G is not None else 0, D, I0Val)
    if name == "test_i0":
        check_counts(name, None, None, W.sum(axis=0), fx)
        return
    out = O.forward(g, vols, mu, W, O.TEXEMU)
    P, V, U = g["projNum"], g["dNumV"], g["dNumU"]
    check_counts(name, out["I"].reshape(P, V, U), out["IAbsorb"].reshape(P, V, U), W.sum(axis=0), fx)


@pytest.mark.parametrize("name", ["grid_response_sinmat", "nogrid_response_sinmat"])
def test_detector_response_sample_matches_reference(fx, name):
    # ADetResponse.txt: detResponse at flat index (U + V) / 2 per energy
    # (CBCTForwardProj.cpp:255-296), written with 6 significant digits
    g, flags, vols, S, mu, G, D, I0Val = inputs(fx, name)
    ref = fx[name + "/out_ADetResponse"]
    k = (g["dNumU"] + g["dNumV"]) // 2
    mine = D.reshape(D.shape[0], -1)[:, k]
    np.testing.assert_allclose(mine, ref, rtol=1e-5, atol=1e-6)


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["texture", "texemu"])
@pytest.mark.parametrize("name", CASES)
def test_cuda_path_matches_reference_binary(fx, cuda_ok, name, mode):
    import torch

    from ct_forward_projection_b200 import Projector, finalize_counts
    g, flags, vols, S, mu, G, D, I0Val = inputs(fx, name)
    with Projector(g, len(vols), mode) as pr:
        pr.set_spectral_tables(S, mu, G, 1 if G is not None else 0, D, I0Val)
        out = pr.forward([torch.from_numpy(v).cuda() for v in vols])
        fin = finalize_counts(out["I"], out["IAbsorb"], out["I0"])
        torch.cuda.synchronize()
    I0 = out["I0"].double().cpu().numpy()
    if name == "test_i0":
        check_counts(name, None, None, I0, fx)
        return
    check_counts(name, out["I"].double().cpu().numpy(), out["IAbsorb"].double().cpu().numpy(), I0, fx)
    # the device finalize (floor, log) agrees with the reference's host code
    ref = fx[name + "/out_PhoImgPro"].astype(np.float64)
    ip = fin["Ipoly"].cpu().numpy().view(np.uint32).astype(np.float64)
    assert np.max(np.maximum(np.abs(ip - ref) - 1.0, 0.0) / np.maximum(ref, 1.0)) < RTOL_COUNTS
