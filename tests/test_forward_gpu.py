"""Parity of the CUDA forward path (through the C ABI) with the FP64 oracle.

Tolerances (relative, per pixel, against the FP64 oracle on the same inputs):
  software trilinear (CTFP_INTERP_TRILINEAR)     1e-5
  texture emulation  (CTFP_INTERP_TEXEMU)        1e-4   (8-bit weights flip on
                     FP32-vs-FP64 coordinate differences at quantisation edges)
  hardware texture   (CTFP_INTERP_TEXTURE)       1e-4 against the emulation
"""
import numpy as np
import pytest
import torch

from ct_forward_projection_b200 import Projector, finalize_counts, sample_volume
from oracle import oracle as O
from tests.conftest import random_volumes, small_geometry, spectral_setup

pytestmark = pytest.mark.gpu

RTOL_TRI = 1e-5
RTOL_TEX = 1e-4


def rel_err(x, ref):
    x = np.asarray(x, np.float64).reshape(-1)
    ref = np.asarray(ref, np.float64).reshape(-1)
    den = np.maximum(np.abs(ref), 1e-30)
    return float(np.max(np.abs(x - ref) / den)) if ref.size else 0.0


def rel_err_scaled(x, ref, floor_frac=1e-6):
    """Relative error with a floor of floor_frac * max|ref| (for L, where rays
    that graze the volume have tiny path integrals)."""
    x = np.asarray(x, np.float64).reshape(-1)
    ref = np.asarray(ref, np.float64).reshape(-1)
    den = np.maximum(np.abs(ref), floor_frac * max(np.max(np.abs(ref)), 1e-30))
    return float(np.max(np.abs(x - ref) / den)) if ref.size else 0.0


def to_dev(vols):
    return [torch.from_numpy(v).cuda() for v in vols]


GEOMS = [
    dict(n=24, views=6, U=20, V=12),
    dict(n=(20, 16, 12), views=5, U=17, V=11),
    dict(n=16, views=4, U=33, V=9, rot=-1),
    dict(n=(9, 23, 14), views=3, U=8, V=40),
]


@pytest.mark.parametrize("sampler", ["layered", "global", "brick", "axis"])
@pytest.mark.parametrize("gi", range(len(GEOMS)))
@pytest.mark.parametrize("M", [1, 2, 3, 4])
def test_line_integrals_trilinear_vs_oracle(cuda_ok, gi, M, sampler):
    d = small_geometry(**GEOMS[gi])
    vols = random_volumes(d, M, 100 + gi * 7 + M)
    with Projector(d, M, "trilinear") as pr:
        pr.set_sampler(sampler)
        L = pr.line_integrals(to_dev(vols)).cpu().numpy().reshape(-1, M)
    Lref = O.line_integrals(d, vols, O.TRILINEAR)
    assert rel_err_scaled(L, Lref) < RTOL_TRI


@pytest.mark.parametrize("sampler", ["layered", "global", "brick", "axis"])
@pytest.mark.parametrize("gi", range(len(GEOMS)))
@pytest.mark.parametrize("M", [1, 2, 4])
def test_forward_trilinear_vs_oracle(cuda_ok, gi, M, sampler):
    d = small_geometry(**GEOMS[gi])
    vols = random_volumes(d, M, 200 + gi + M)
    S, mu, G, D = spectral_setup(d, M, 17, 5 + gi)
    W = O.energy_weights(d, S, G, 2, D, 60000.0)
    ref = O.forward(d, vols, mu, W, O.TRILINEAR)
    with Projector(d, M, "trilinear") as pr:
        pr.set_sampler(sampler)
        pr.set_spectral_tables(S, mu, G, 2, D, 60000.0)
        out = pr.forward(to_dev(vols), want_L=True)
        torch.cuda.synchronize()
    assert rel_err(out["I"].cpu(), ref["I"]) < RTOL_TRI
    assert rel_err(out["IAbsorb"].cpu(), ref["IAbsorb"]) < RTOL_TRI
    assert rel_err(out["I0"].cpu(), W.sum(axis=0)) < 1e-6
    assert rel_err_scaled(out["L"].cpu().numpy().reshape(-1, M), ref["L"]) < RTOL_TRI


# voxels of different size on each axis (1.0 x 0.75 x 2.5 mm): the reference
# divides each texture coordinate by its own axis's voxel size
# (CBCTPolyProjGPU.cu:1915-1920) while the ray step is half the x voxel
ANISO = dict(pNumX=20, pNumY=16, pNumZ=10, pLengthX=20.0, pLengthY=12.0, pLengthZ=25.0, projNum=5, dNumU=24,
             dNumV=16, dSize=2.0, sod=300.0, sdd=450.0, rotatedDirection=1)


@pytest.mark.parametrize("mode,sampler", [("trilinear", "layered"), ("trilinear", "global"), ("trilinear", "brick"),
                                          ("trilinear", "axis"), ("texemu", "layered"), ("texemu", "axis"),
                                          ("texture", None)])
def test_anisotropic_voxels_vs_oracle(cuda_ok, mode, sampler):
    d = dict(ANISO)
    M = 2
    vols = random_volumes(d, M, 404)
    S, mu, G, D = spectral_setup(d, M, 9, 41)
    W = O.energy_weights(d, S, G, 2, D, 60000.0)
    ref = O.forward(d, vols, mu, W, O.TRILINEAR if mode == "trilinear" else O.TEXEMU)
    with Projector(d, M, mode) as pr:
        if sampler:
            pr.set_sampler(sampler)
        pr.set_spectral_tables(S, mu, G, 2, D, 60000.0)
        out = pr.forward(to_dev(vols), want_L=True)
        torch.cuda.synchronize()
    tol = RTOL_TRI if mode == "trilinear" else RTOL_TEX
    assert rel_err(out["I"].cpu(), ref["I"]) < tol
    assert rel_err(out["IAbsorb"].cpu(), ref["IAbsorb"]) < tol
    assert rel_err_scaled(out["L"].cpu().numpy().reshape(-1, M), ref["L"]) < (RTOL_TRI if mode == "trilinear" else 1e-3)


@pytest.mark.parametrize("layout", [0, 1, 2])
def test_forward_grid_layouts_and_no_response(cuda_ok, layout):
    d = small_geometry(n=16, views=4, U=24, V=10)
    M = 2
    vols = random_volumes(d, M, 77)
    rng = np.random.RandomState(3)
    E = 9
    S = rng.uniform(0.1, 1, E).astype(np.float32)
    mu = rng.uniform(0.01, 0.05, (E, M)).astype(np.float32)
    G = None if layout == 0 else (rng.uniform(0.5, 1, (E, 24)) if layout == 1 else
                                  rng.uniform(0.5, 1, (E, 10, 24))).astype(np.float32)
    W = O.energy_weights(d, S, G, layout, None, 1234.0)
    ref = O.forward(d, vols, mu, W)
    with Projector(d, M, "trilinear") as pr:
        pr.set_spectral_tables(S, mu, G, layout, None, 1234.0)
        out = pr.forward(to_dev(vols))
        torch.cuda.synchronize()
    assert rel_err(out["I"].cpu(), ref["I"]) < RTOL_TRI
    assert rel_err(out["IAbsorb"].cpu(), ref["IAbsorb"]) < RTOL_TRI


@pytest.mark.parametrize("sampler", ["layered", "global", "brick", "axis"])
@pytest.mark.parametrize("M", [1, 2, 3])
def test_forward_texemu_vs_oracle(cuda_ok, M, sampler):
    d = small_geometry(n=20, views=5, U=24, V=14)
    vols = random_volumes(d, M, 300 + M)
    S, mu, G, D = spectral_setup(d, M, 11, 9)
    W = O.energy_weights(d, S, G, 2, D, 60000.0)
    ref = O.forward(d, vols, mu, W, O.TEXEMU)
    with Projector(d, M, "texemu") as pr:
        pr.set_sampler(sampler)
        pr.set_spectral_tables(S, mu, G, 2, D, 60000.0)
        out = pr.forward(to_dev(vols), want_L=True)
        torch.cuda.synchronize()
    assert rel_err(out["I"].cpu(), ref["I"]) < RTOL_TEX
    assert rel_err(out["IAbsorb"].cpu(), ref["IAbsorb"]) < RTOL_TEX


@pytest.mark.parametrize("M", [1, 2, 4])
def test_hardware_texture_vs_emulation(cuda_ok, M):
    d = small_geometry(n=20, views=5, U=24, V=14)
    vols = to_dev(random_volumes(d, M, 400 + M))
    S, mu, G, D = spectral_setup(d, M, 11, 19)
    outs = {}
    for mode in ("texemu", "texture"):
        with Projector(d, M, mode) as pr:
            pr.set_spectral_tables(S, mu, G, 2, D, 60000.0)
            outs[mode] = pr.forward(vols, want_L=True)
            torch.cuda.synchronize()
    assert rel_err(outs["texture"]["I"].cpu(), outs["texemu"]["I"].cpu()) < RTOL_TEX
    assert rel_err_scaled(outs["texture"]["L"].cpu(), outs["texemu"]["L"].cpu()) < RTOL_TEX


def test_texture_weight_rounding_pinned(cuda_ok):
    # the hardware sampler at random points against the 8-bit emulation, per
    # sample; pins the weight quantisation rule the emulation uses
    rng = np.random.RandomState(0)
    vol = torch.from_numpy(rng.uniform(-1, 1, (6, 7, 8)).astype(np.float32)).cuda()
    pts = rng.uniform(-1.5, 8.5, (20000, 3)).astype(np.float32)
    pts[:5000] = np.round(pts[:5000] * 512) / 512  # exact quantisation edges
    pts_d = torch.from_numpy(pts).cuda()
    hw = sample_volume(vol, pts_d, "texture").cpu().numpy()
    em = sample_volume(vol, pts_d, "texemu").cpu().numpy()
    tri = sample_volume(vol, pts_d, "trilinear").cpu().numpy()
    # same 8 corner weights; only the FP32 summation order of the unit differs
    assert np.max(np.abs(hw - em)) < 1e-6
    assert np.max(np.abs(hw - tri)) < 2e-2


def test_zero_volume_is_flat_field(cuda_ok):
    d = small_geometry()
    S, mu, G, D = spectral_setup(d, 2, 5, 1)
    with Projector(d, 2, "trilinear") as pr:
        pr.set_spectral_tables(S, mu, G, 2, D, 1000.0)
        z = [torch.zeros(pr.shape_vol, device="cuda") for _ in range(2)]
        out = pr.forward(z)
        torch.cuda.synchronize()
    I0 = out["I0"].cpu().numpy()
    assert np.array_equal(out["I"].cpu().numpy(), np.broadcast_to(I0, out["I"].shape))
    assert float(out["IAbsorb"].abs().max()) == 0.0


def test_spectral_from_L_matches_fused(cuda_ok):
    d = small_geometry()
    vols = to_dev(random_volumes(d, 3, 5))
    S, mu, G, D = spectral_setup(d, 3, 13, 2)
    with Projector(d, 3, "trilinear") as pr:
        pr.set_spectral_tables(S, mu, G, 2, D, 60000.0)
        f = pr.forward(vols, want_L=True)
        s = pr.spectral_from_L(f["L"])
        torch.cuda.synchronize()
    assert torch.equal(f["I"], s["I"]) and torch.equal(f["IAbsorb"], s["IAbsorb"])


@pytest.mark.parametrize("views,pinned,focal", [(6, False, False), (13, True, False), (17, True, True),
                                                 (3, False, True)])
def test_forward_host_matches_device(cuda_ok, views, pinned, focal):
    # ctfp_forward_host marches in view chunks whose results travel back on a
    # second stream; pageable or page-locked host buffers, with and without a
    # focal spot, give the device path's results exactly
    d = small_geometry(views=views)
    vols = random_volumes(d, 2, 8)
    S, mu, G, D = spectral_setup(d, 2, 7, 3)
    with Projector(d, 2, "trilinear") as pr:
        pr.set_spectral_tables(S, mu, G, 2, D, 60000.0)
        if focal:
            from ct_forward_projection_b200.projector import focal_spot_offsets
            pr.set_focal_spot(*focal_spot_offsets(views, 0.8))
        dev = pr.forward(to_dev(vols))
        torch.cuda.synchronize()
        out = None
        if pinned:
            P, V, U = pr.shape_proj
            out = {"I": torch.empty((P, V, U)).pin_memory(), "IAbsorb": torch.empty((P, V, U)).pin_memory(),
                   "I0": torch.empty((V, U)).pin_memory()}
            hv = [torch.from_numpy(v).pin_memory() for v in vols]
        else:
            hv = vols
        host = pr.forward_host(hv, out=out)
        host = {k: np.asarray(v) for k, v in host.items()}
    assert np.array_equal(host["I"], dev["I"].cpu().numpy())
    assert np.array_equal(host["IAbsorb"], dev["IAbsorb"].cpu().numpy())
    assert np.array_equal(host["I0"], dev["I0"].cpu().numpy())


def test_finalize_counts_vs_oracle(cuda_ok):
    rng = np.random.RandomState(1)
    I = (rng.uniform(0, 5e4, (3, 4, 5)).astype(np.float32))
    I[0, 0, :2] = [0.3, 0.0]
    I0 = rng.uniform(5e4, 6e4, (4, 5)).astype(np.float32)
    A = rng.uniform(0, 5e4, (3, 4, 5)).astype(np.float32)
    out = finalize_counts(torch.from_numpy(I).cuda(), torch.from_numpy(A).cuda(), torch.from_numpy(I0).cuda())
    Ip, proj = O.finalize(I, I0)
    assert np.array_equal(out["Ipoly"].cpu().numpy().view(np.uint32), Ip)
    assert np.array_equal(out["IAbsPoly"].cpu().numpy().view(np.uint32), np.floor(A).astype(np.uint32))
    p = out["proj"].cpu().numpy()
    fin = np.isfinite(proj)
    assert np.array_equal(np.isinf(p), ~fin)
    assert np.max(np.abs(p[fin] - proj[fin])) < 2e-6


@pytest.mark.parametrize("U,V,P", [(1, 1, 1), (1, 7, 2), (33, 1, 3)])
def test_degenerate_detectors(cuda_ok, U, V, P):
    d = small_geometry(n=10, views=P, U=U, V=V, pitch=1.5)
    vols = random_volumes(d, 1, 4)
    with Projector(d, 1, "trilinear") as pr:
        L = pr.line_integrals(to_dev(vols)).cpu().numpy().reshape(-1, 1)
    assert rel_err_scaled(L, O.line_integrals(d, vols)) < RTOL_TRI


def test_more_views_than_one_launch_holds(cuda_ok):
    # 70000 views at one view per CTA exceed the 65535 CTAs of grid.z: the
    # forward and the adjoint launch in view chunks and still equal the oracle
    d = small_geometry(n=4, views=70000, U=2, V=2, length=4.0)
    M = 1
    vols = random_volumes(d, M, 90)
    S, mu, G, D = spectral_setup(d, M, 3, 91)
    W = O.energy_weights(d, S, G, 2, D, 60000.0)
    ref = O.forward(d, vols, mu, W, O.TRILINEAR)
    rng = np.random.RandomState(4)
    gL = rng.normal(size=(d["projNum"] * 4, M)).astype(np.float32)
    gref = O.line_integrals_adjoint(d, gL, M, O.TRILINEAR)
    with Projector(d, M, "trilinear") as pr:
        pr.set_launch_shape(32, 1, 1, 2)
        pr.set_spectral_tables(S, mu, G, 2, D, 60000.0)
        out = pr.forward(to_dev(vols), want_L=True)
        g = pr.line_integrals_adjoint(torch.from_numpy(gL.reshape(d["projNum"], 2, 2, M)).cuda())
        torch.cuda.synchronize()
    assert rel_err(out["I"].cpu(), ref["I"]) < RTOL_TRI
    assert rel_err_scaled(out["L"].cpu().numpy().reshape(-1, M), ref["L"]) < RTOL_TRI
    a = g[0].double().cpu().numpy()
    assert np.max(np.abs(a - gref[0])) / np.max(np.abs(gref[0])) < 1e-5


def test_host_mirror_rejects_wrong_buffers(cuda_ok):
    # the C ABI sees only pointers; the Python mirror checks every buffer's
    # element count, dtype and device before a call, so a wrong buffer is an
    # exception on the host and never an out-of-bounds access on the GPU
    from ct_forward_projection_b200 import Batch
    d = small_geometry(n=8, views=3, U=10, V=6)
    M = 2
    vols = to_dev(random_volumes(d, M, 11))
    S, mu, G, D = spectral_setup(d, M, 4, 12)
    with Projector(d, M, "trilinear") as pr:
        pr.set_spectral_tables(S, mu, G, 2, D, 1000.0)
        good = pr.forward(vols, want_L=True)
        bad_I = {**good, "I": torch.empty(3 * 6 * 10 - 1, device="cuda")}
        with pytest.raises(ValueError):
            pr.forward(vols, out=bad_I)
        with pytest.raises(ValueError):
            pr.forward(vols[:1])
        with pytest.raises(TypeError):
            pr.forward([v.double() for v in vols])
        with pytest.raises(ValueError):
            pr.forward(vols, out={**good, "L": torch.empty(3, 6, 10, 1, device="cuda")})
        with pytest.raises(ValueError):
            pr.backward(good["L"], gI=torch.ones(3, 6, 9, device="cuda"))
        with pytest.raises(ValueError):
            pr.backward(good["L"], gI=torch.ones_like(good["I"]), grads=[torch.zeros(8, 8, 7, device="cuda")] * M)
        with pytest.raises(ValueError):
            pr.forward_host([v.cpu().numpy() for v in vols], out={"I": np.empty(5, np.float32),
                                                                   "IAbsorb": np.empty((3, 6, 10), np.float32)})
        b = Batch([pr])
        with pytest.raises(ValueError):
            b.forward_adjoint([vols], [torch.ones(3, 6, 11, device="cuda")])
        out = b.forward_adjoint([vols], [good["I"] * 0.9])
        torch.cuda.synchronize()
        assert torch.isfinite(out["loss"]).all()
        b.close()


def test_rays_missing_volume_are_zero(cuda_ok):
    # a detector offset so far that every ray passes beside the volume
    d = small_geometry(n=8, views=2, U=6, V=6, length=8.0, pitch=60.0)
    vols = [np.ones((8, 8, 8), np.float32)]
    with Projector(d, 1, "trilinear") as pr:
        L = pr.line_integrals(to_dev(vols)).cpu().numpy().reshape(-1)
    ref = O.line_integrals(d, vols).reshape(-1)
    assert np.array_equal(L == 0, ref == 0)
    assert rel_err_scaled(L, ref) < RTOL_TRI


@pytest.mark.parametrize("mode", ["trilinear", "texemu"])
@pytest.mark.parametrize("pitch", [None, 9.0])
@pytest.mark.parametrize("n,staging", [((40, 36, 30), "tma"), ((40, 36, 30), "loads"), ((41, 36, 30), "tma")])
def test_brick_sampler_equals_layered(cuda_ok, mode, pitch, n, staging, monkeypatch):
    # same corner values, weights and summation order: identical results,
    # whether the bundle's boxes fit (default pitch) or not (rays many voxels
    # apart: every segment reads the caller's volume instead), and whether the
    # boxes are staged by TMA tensor loads (pNumX a multiple of 4) or by plain
    # loads (CTFP_BRICK_STAGING=loads, or pNumX = 41)
    monkeypatch.setenv("CTFP_BRICK_STAGING", staging)
    d = small_geometry(n=n, views=5, U=37, V=35, pitch=pitch)
    vols = random_volumes(d, 3, 12)
    S, mu, G, D = spectral_setup(d, 3, 6, 2)
    with Projector(d, 3, mode) as pr:
        pr.set_spectral_tables(S, mu, G, 2, D, 1000.0)
        pr.set_sampler("layered")
        a = pr.forward(to_dev(vols), want_L=True)
        pr.set_sampler("brick")
        b = pr.forward(to_dev(vols), want_L=True)
        torch.cuda.synchronize()
        assert pr.check_status() == 0
    assert torch.equal(a["L"], b["L"]) and torch.equal(a["I"], b["I"]) and torch.equal(a["IAbsorb"], b["IAbsorb"])


def test_brick_tma_wait_that_runs_out(cuda_ok, monkeypatch):
    # with CTFP_WAIT_LIMIT=0 every CTA gives up its first TMA wait at once:
    # it reads the volume instead (identical outputs), waits for the load
    # still in flight before exiting, and the plan's status reports
    # CTFP_TIMEOUT once, then reads clear
    from ct_forward_projection_b200._capi import CTFP_TIMEOUT, CtfpError
    d = small_geometry(n=(40, 36, 30), views=4, U=37, V=35)
    vols = random_volumes(d, 2, 13)
    S, mu, G, D = spectral_setup(d, 2, 5, 3)
    with Projector(d, 2, "trilinear") as pr:
        pr.set_spectral_tables(S, mu, G, 2, D, 1000.0)
        pr.set_sampler("layered")
        a = pr.forward(to_dev(vols), want_L=True)
        pr.set_sampler("brick")
        monkeypatch.setenv("CTFP_WAIT_LIMIT", "0")
        b = pr.forward(to_dev(vols), want_L=True)
        torch.cuda.synchronize()
        with pytest.raises(CtfpError) as e:
            pr.check_status(raise_on_timeout=True)
        assert e.value.status == CTFP_TIMEOUT
        assert pr.check_status() == 0
        monkeypatch.delenv("CTFP_WAIT_LIMIT")
        c = pr.forward(to_dev(vols), want_L=True)
        torch.cuda.synchronize()
        assert pr.check_status() == 0
    for o in (b, c):
        assert torch.equal(a["L"], o["L"]) and torch.equal(a["I"], o["I"])


def _sparse_volumes(d, M, seed):
    # random densities with large all-zero regions (as air around a body)
    vols = random_volumes(d, M, seed)
    z, y, x = vols[0].shape
    for v in vols:
        v[:, :, : x // 3] = 0.0
        v[: z // 2, y // 2:, :] = 0.0
    return vols


@pytest.mark.parametrize("mode", ["trilinear", "texemu", "texture"])
@pytest.mark.parametrize("M", [1, 2, 3])
def test_skip_empty_matches_full_march(cuda_ok, mode, M):
    d = small_geometry(n=(40, 36, 30), views=6, U=37, V=29)
    vols = _sparse_volumes(d, M, 40 + M)
    S, mu, G, D = spectral_setup(d, M, 7, 3)
    with Projector(d, M, mode) as pr:
        pr.set_spectral_tables(S, mu, G, 2, D, 1000.0)
        full = pr.forward(to_dev(vols), want_L=True)
        pr.set_skip_empty(True)
        skip = pr.forward(to_dev(vols), want_L=True)
        skip2 = pr.forward(to_dev(vols), want_L=True)  # occupancy rebuilt per call
        torch.cuda.synchronize()
    for k in ("I", "IAbsorb"):
        assert rel_err(skip[k].cpu().numpy(), full[k].cpu().numpy()) < 1e-6
    assert rel_err_scaled(skip["L"].cpu().numpy(), full["L"].cpu().numpy()) < 1e-6
    assert torch.equal(skip["I"], skip2["I"])
    if mode == "trilinear":
        W = O.energy_weights(d, S, G, 2, D, 1000.0)
        ref = O.forward(d, vols, mu, W, O.TRILINEAR)
        assert rel_err(skip["I"].cpu().numpy(), ref["I"]) < RTOL_TRI


@pytest.mark.parametrize("mode", ["trilinear", "texture"])
@pytest.mark.parametrize("pos", [(0, 0, 0), (6, 7, 8), (7, 15, 23), (8, 16, 24), (15, 9, 31), (31, 31, 31)])
def test_skip_empty_isolated_voxels_at_brick_edges(cuda_ok, pos, mode):
    # one non-zero voxel on either side of the 8-voxel brick boundaries and at
    # the volume's faces: a brick missed by the dilation would drop every ray
    # through that voxel's footprint
    d = small_geometry(n=32, views=5, U=41, V=41, pitch=0.9)
    vol = np.zeros((32, 32, 32), np.float32)
    vol[pos[2], pos[1], pos[0]] = 1.5
    with Projector(d, 1, mode) as pr:
        full = pr.line_integrals(to_dev([vol])).cpu().numpy()
        pr.set_skip_empty(True)
        skip = pr.line_integrals(to_dev([vol])).cpu().numpy()
    assert np.count_nonzero(full) > 0
    np.testing.assert_array_equal(skip != 0, full != 0)
    assert rel_err_scaled(skip, full) < 1e-6


@pytest.mark.parametrize("mode", ["trilinear", "texemu"])
@pytest.mark.parametrize("M", [1, 2])
def test_focal_spot_forward_vs_oracle(cuda_ok, mode, M):
    from ct_forward_projection_b200.projector import focal_spot_offsets
    d = small_geometry(n=(20, 18, 14), views=6, U=23, V=15)
    vols = random_volumes(d, M, 70 + M)
    S, mu, G, D = spectral_setup(d, M, 6, 5)
    fs = focal_spot_offsets(d["projNum"], 1.2)  # up to ~1.3 detector pitches
    W = O.energy_weights(d, S, G, 2, D, 1000.0)
    omode = O.TRILINEAR if mode == "trilinear" else O.TEXEMU
    ref = O.forward_focal_spot(d, vols, mu, W, fs, omode)
    with Projector(d, M, mode) as pr:
        pr.set_spectral_tables(S, mu, G, 2, D, 1000.0)
        pr.set_focal_spot(*fs)
        f = pr.forward(to_dev(vols), want_L=True)
        L_only = pr.line_integrals(to_dev(vols))
        torch.cuda.synchronize()
    tol = RTOL_TRI if mode == "trilinear" else RTOL_TEX
    assert rel_err(f["I"].cpu().numpy(), ref["I"]) < tol
    assert rel_err(f["IAbsorb"].cpu().numpy(), ref["IAbsorb"]) < tol * 10
    assert rel_err_scaled(f["L"].cpu().numpy().reshape(-1, M), ref["L"]) < tol
    assert torch.equal(L_only, f["L"])


@pytest.mark.parametrize("mode", ["trilinear", "texemu", "texture"])
def test_focal_spot_zero_offsets_equal_plain_forward(cuda_ok, mode):
    d = small_geometry(n=16, views=4, U=19, V=13)
    vols = random_volumes(d, 2, 9)
    S, mu, G, D = spectral_setup(d, 2, 5, 1)
    with Projector(d, 2, mode) as pr:
        pr.set_spectral_tables(S, mu, G, 2, D, 1000.0)
        a = pr.forward(to_dev(vols), want_L=True)
        z = np.zeros(d["projNum"], np.float32)
        pr.set_focal_spot(z, z)
        b = pr.forward(to_dev(vols), want_L=True)
        c = pr.forward(to_dev(vols), views=(1, 2))
        with pytest.raises(Exception):
            pr.backward(b["L"], gI=torch.ones_like(b["I"]))
        pr.set_focal_spot(None)
        torch.cuda.synchronize()
    assert torch.equal(a["L"], b["L"])
    assert rel_err(b["I"].cpu().numpy(), a["I"].cpu().numpy()) < 1e-6
    assert rel_err(c["I"].cpu().numpy(), a["I"][1:3].cpu().numpy()) < 1e-6


def test_deep_volume_default_sampler_and_layered_refused(cuda_ok):
    # layered textures hold at most 2048 layers: a volume 2050 slices deep is
    # marched by the default axis sampler (layers along x and y), and asking
    # for the z-layered one is refused
    from ct_forward_projection_b200._capi import CtfpError, CTFP_UNSUPPORTED
    d = small_geometry(n=(6, 5, 2050), views=2, U=7, V=9, length=6.0, pitch=2.0)
    vols = random_volumes(d, 1, 3)
    with Projector(d, 1, "trilinear") as pr:
        L = pr.line_integrals(to_dev(vols)).cpu().numpy().reshape(-1, 1)
        with pytest.raises(CtfpError) as e:
            pr.set_sampler("layered")
        assert e.value.status == CTFP_UNSUPPORTED
    assert rel_err_scaled(L, O.line_integrals(d, vols)) < RTOL_TRI


def test_wide_volume_falls_back_to_layered_sampler(cuda_ok):
    # the axis sampler's copies hold at most 2046 voxel layers along x and y:
    # a volume 2050 voxels wide is marched by the z-layered sampler
    d = small_geometry(n=(2050, 4, 3), views=3, U=9, V=5, length=20.0, pitch=2.0)
    vols = random_volumes(d, 1, 4)
    with Projector(d, 1, "trilinear") as pr:
        L = pr.line_integrals(to_dev(vols)).cpu().numpy().reshape(-1, 1)
    assert rel_err_scaled(L, O.line_integrals(d, vols)) < RTOL_TRI


# geometries for the axis sampler: views all round the rotation (both copies,
# rays marching up and down each axis), anisotropic voxels, the reversed
# rotation, detector sizes that leave partial tiles and partial lane quads
AXIS_GEOMS = [
    dict(n=(26, 22, 18), views=37, U=21, V=14),
    dict(n=16, views=24, U=33, V=9, rot=-1),
    dict(n=(9, 23, 14), views=19, U=8, V=41),
]


@pytest.mark.parametrize("mode", ["trilinear", "texemu"])
@pytest.mark.parametrize("gi", range(len(AXIS_GEOMS)))
@pytest.mark.parametrize("M", [1, 2, 3, 4])
def test_axis_sampler_equals_layered(cuda_ok, mode, gi, M):
    """The axis sampler reads the same voxel values with the same weights as
    the layered sampler, interpolating the layer axis last: outputs agree to
    FP32 rounding (and each matches the oracle in the parity tests)."""
    d = small_geometry(**AXIS_GEOMS[gi])
    vols = random_volumes(d, M, 500 + 10 * gi + M)
    S, mu, G, D = spectral_setup(d, M, 7, 3 + gi)
    with Projector(d, M, mode) as pr:
        pr.set_spectral_tables(S, mu, G, 2, D, 1000.0)
        pr.set_sampler("layered")
        a = pr.forward(to_dev(vols), want_L=True)
        pr.set_sampler("axis")
        b = pr.forward(to_dev(vols), want_L=True)
        torch.cuda.synchronize()
    assert torch.equal(a["I0"], b["I0"])
    for k in ("I", "IAbsorb"):
        assert rel_err(b[k].cpu().numpy(), a[k].cpu().numpy()) < 1e-6, k
    assert rel_err_scaled(b["L"].cpu().numpy(), a["L"].cpu().numpy()) < 1e-6


@pytest.mark.parametrize("mode", ["trilinear", "texemu"])
@pytest.mark.parametrize("shape", [(16, 16, 1, 3), (32, 8, 2, 4), (8, 32, 4, 2), (16, 4, 1, 3), (64, 2, 1, 3)])
def test_axis_sampler_launch_shapes(cuda_ok, mode, shape):
    """Every launch shape gives the same outputs (tiles whose height is not a
    multiple of 4 run as 16 x 16): bitwise, since each ray is marched alone."""
    d = small_geometry(n=(20, 24, 16), views=9, U=37, V=23)
    vols = random_volumes(d, 2, 77)
    S, mu, G, D = spectral_setup(d, 2, 5, 8)
    with Projector(d, 2, mode) as pr:
        pr.set_spectral_tables(S, mu, G, 2, D, 1000.0)
        pr.set_sampler("axis")
        a = pr.forward(to_dev(vols), want_L=True)
        pr.set_launch_shape(*shape)
        b = pr.forward(to_dev(vols), want_L=True)
        torch.cuda.synchronize()
    assert torch.equal(a["L"], b["L"]) and torch.equal(a["I"], b["I"])


@pytest.mark.parametrize("mode", ["trilinear", "texemu"])
def test_axis_sampler_skip_empty(cuda_ok, mode):
    d = small_geometry(n=(40, 36, 30), views=11, U=37, V=29)
    vols = _sparse_volumes(d, 2, 91)
    S, mu, G, D = spectral_setup(d, 2, 7, 3)
    with Projector(d, 2, mode) as pr:
        pr.set_spectral_tables(S, mu, G, 2, D, 1000.0)
        pr.set_sampler("axis")
        full = pr.forward(to_dev(vols), want_L=True)
        pr.set_skip_empty(True)
        skip = pr.forward(to_dev(vols), want_L=True)
        torch.cuda.synchronize()
    for k in ("I", "IAbsorb"):
        assert rel_err(skip[k].cpu().numpy(), full[k].cpu().numpy()) < 1e-6
    assert rel_err_scaled(skip["L"].cpu().numpy(), full["L"].cpu().numpy()) < 1e-6


def test_axis_sampler_limits(cuda_ok):
    # the copies are layered along x and y: at most 2048 layers each
    from ct_forward_projection_b200._capi import CtfpError, CTFP_UNSUPPORTED
    d = small_geometry(n=(2050, 4, 3), views=2, U=7, V=5, length=20.0, pitch=2.0)
    with Projector(d, 1, "trilinear") as pr:
        with pytest.raises(CtfpError) as e:
            pr.set_sampler("axis")
        assert e.value.status == CTFP_UNSUPPORTED


@pytest.mark.parametrize("gi", range(len(AXIS_GEOMS)))
@pytest.mark.parametrize("mode", ["trilinear", "texemu"])
def test_axis_gather_count_bounds(cuda_ok, gi, mode):
    """The axis march's texture work per voxel-sample is positive and at most
    both slots of every sample with one live lane per quad (2.0); it does not
    depend on the volumes and is the same on every call."""
    d = small_geometry(**AXIS_GEOMS[gi])
    with Projector(d, 2, mode) as pr:
        pr.set_sampler("axis")
        g = pr.axis_gather_count()
        assert pr.axis_gather_count() == g
    assert 0.0 < g <= 2.0


def test_axis_gather_count_reuse_on_a_fine_march(cuda_ok):
    # a 64^3 volume sampled at half a voxel by a 128-column detector: most
    # samples keep or advance their footprint, so fewer than 60 % of the
    # two-gather work is fetched
    d = small_geometry(n=64, views=12, U=128, V=32, length=64.0)
    with Projector(d, 1, "trilinear") as pr:
        pr.set_sampler("axis")
        g = pr.axis_gather_count()
    assert g < 0.3


def test_reciprocal_division_is_the_ieee_division(cuda_ok):
    """The texture emulation's coordinates divide by the voxel size through the
    plan's FP32 reciprocal and two exact-remainder correction steps; every
    quotient must equal the IEEE division bit for bit (the reference divides),
    for the voxel sizes of the benchmark workloads, divisors whose mantissa
    sits at either end of its binade, and seeded random divisors."""
    import ctypes as C

    from ct_forward_projection_b200 import _capi as capi
    fixed = [0.5, 0.4, 0.8, 1.0, 0.75, 2.5, 0.3, 1.0 / 3.0, 0.7, 0.1, 0.390625, 1.2, 0.123456,
             float(np.nextafter(np.float32(1.0), np.float32(0))), float(np.nextafter(np.float32(1.0), np.float32(2))),
             float(np.nextafter(np.float32(2.0), np.float32(0))), 1.5, 3.0, 7.0, 0.0625]
    rng = np.random.RandomState(17)
    rand = [float(np.float32(x)) for x in np.exp(rng.uniform(np.log(0.02), np.log(8.0), 200))]
    for k, y in enumerate(fixed + rand):
        bad = C.c_int64(-1)
        capi.call("ctfp_check_division", 0, C.c_float(y), 4_000_000 if k < len(fixed) else 500_000, 1000 + k,
                  C.byref(bad))
        assert bad.value == 0, (y, bad.value)
