"""The batched form (ctfp_batch_*; no reference counterpart): persistent
kernels over a work queue of (item, view, 8 x 8 ray tile) units, replayed as
a CUDA graph; items in every interpolation mode, the hardware texture included.  Every item's outputs must equal the plain per-plan calls on the same
inputs; the fused forward + loss + adjoint must equal ctfp_forward followed by
ctfp_backward with dLoss/dI formed on the host."""
import numpy as np
import pytest
import torch

from ct_forward_projection_b200 import Batch, Projector
from ct_forward_projection_b200._capi import CtfpError, CTFP_NOT_READY, CTFP_UNSUPPORTED
from oracle import oracle as O
from tests.conftest import random_volumes, small_geometry, spectral_setup

pytestmark = pytest.mark.gpu

# items of uneven size, material count, spectrum length and sampler
ITEMS = [
    dict(n=(20, 16, 12), views=5, U=24, V=12, M=2, E=7, mode="trilinear", seed=1),
    dict(n=(12, 12, 12), views=3, U=13, V=9, M=1, E=4, mode="texemu", seed=2),
    dict(n=(26, 18, 9), views=7, U=33, V=17, M=3, E=11, mode="trilinear", seed=3),
    dict(n=(9, 11, 14), views=2, U=8, V=8, M=4, E=5, mode="texemu", seed=4),
    dict(n=(16, 14, 12), views=4, U=19, V=13, M=2, E=6, mode="texture", seed=5),
]


def make_items(specs):
    out = []
    for sp in specs:
        d = small_geometry(n=sp["n"], views=sp["views"], U=sp["U"], V=sp["V"])
        vols = random_volumes(d, sp["M"], sp["seed"])
        S, mu, G, D = spectral_setup(d, sp["M"], sp["E"], sp["seed"] + 10)
        pr = Projector(d, sp["M"], sp["mode"])
        pr.set_spectral_tables(S, mu, G, 2, D, 1000.0)
        out.append((pr, [torch.from_numpy(v).cuda() for v in vols], (d, S, mu, G, D, vols)))
    return out


def rel(a, b):
    a = a.double().cpu().numpy()
    b = b.double().cpu().numpy()
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-30))


def test_batch_forward_equals_plain_calls(cuda_ok):
    items = make_items(ITEMS)
    b = Batch([it[0] for it in items])
    info = b.info()
    # forward units: one view of an 8 x 16 ray tile (the fused kernel's 8 x 8, twice as high)
    assert b.shapes() == {"fwd": (8, 16), "fwd_adjoint": (8, 8), "views": (1, 1)}
    assert info["units"] == sum(((sp["U"] + 7) // 8) * ((sp["V"] + 15) // 16) * sp["views"] for sp in ITEMS)
    assert info["grid_forward"] % 148 == 0 and info["grid_adjoint"] % 148 == 0
    outs = b.forward([it[1] for it in items], want_L=True)
    torch.cuda.synchronize()
    for (pr, vols, _), o in zip(items, outs):
        ref = pr.forward(vols, want_L=True)
        torch.cuda.synchronize()
        assert rel(o["I"], ref["I"]) < 2e-6
        assert rel(o["IAbsorb"], ref["IAbsorb"]) < 2e-6
        assert rel(o["L"], ref["L"]) < 1e-6
    b.close()


def test_batch_forward_vs_oracle(cuda_ok):
    items = make_items(ITEMS[:2])
    b = Batch([it[0] for it in items])
    outs = b.forward([it[1] for it in items])
    torch.cuda.synchronize()
    for (pr, _, (d, S, mu, G, D, vols)), o in zip(items, outs):
        mode = O.TRILINEAR if pr.interp == "trilinear" else O.TEXEMU
        ref = O.forward(d, vols, mu, O.energy_weights(d, S, G, 2, D, 1000.0), mode)
        tol = 1e-5 if mode == O.TRILINEAR else 1e-4
        assert np.max(np.abs(o["I"].double().cpu().numpy().ravel() - ref["I"]) / np.maximum(ref["I"], 1e-3)) < tol
    b.close()


def test_graph_replay_reads_current_contents(cuda_ok):
    # a replayed graph reads the buffers' contents at replay time; a new
    # pointer re-records it
    items = make_items(ITEMS[:3])
    b = Batch([it[0] for it in items])
    vols = [it[1] for it in items]
    o1 = b.forward(vols)
    I1 = [o["I"].clone() for o in o1]
    o2 = b.forward(vols, out=o1)
    torch.cuda.synchronize()
    for a, c in zip(I1, o2):
        assert torch.equal(a, c["I"])
    for v in vols[1]:
        v.mul_(0.5)
    o3 = b.forward(vols, out=o1)
    torch.cuda.synchronize()
    ref = items[1][0].forward(vols[1])
    torch.cuda.synchronize()
    assert rel(o3[1]["I"], ref["I"]) < 2e-6
    assert not torch.equal(o3[1]["I"], I1[1])
    vols2 = [[v.clone() for v in vk] for vk in vols]
    o4 = b.forward(vols2)
    torch.cuda.synchronize()
    for a, c in zip(o3, o4):
        assert torch.equal(a["I"], c["I"])
    b.close()


@pytest.mark.parametrize("specs", [ITEMS, ITEMS[1:2]])
def test_batch_forward_adjoint_equals_plain(cuda_ok, specs):
    items = make_items(specs)
    rng = np.random.RandomState(5)
    targets, ref_grads, ref_loss = [], [], []
    for pr, vols, _ in items:
        f = pr.forward(vols, want_L=True)
        torch.cuda.synchronize()
        I = f["I"].double()
        T = (I * torch.from_numpy(np.exp(rng.normal(scale=0.05, size=tuple(I.shape)))).cuda()).float()
        targets.append(T)
        r = torch.log(I) - torch.log(T.double())
        ref_loss.append(float(torch.sum(r * r)))
        gI = (2.0 * r / I).float()
        ref_grads.append(pr.backward(f["L"], gI=gI))
    torch.cuda.synchronize()
    b = Batch([it[0] for it in items])
    res = b.forward_adjoint([it[1] for it in items], targets)
    torch.cuda.synchronize()
    for k, (pr, _, _) in enumerate(items):
        assert abs(float(res["loss"][k]) - ref_loss[k]) / ref_loss[k] < 1e-4
        for m in range(pr.M):
            assert rel(res["grads"][k][m], ref_grads[k][m]) < 1e-4
    # second call: graph replay, gradients accumulate
    res2 = b.forward_adjoint([it[1] for it in items], targets, grads=res["grads"])
    torch.cuda.synchronize()
    for k, (pr, _, _) in enumerate(items):
        for m in range(pr.M):
            assert rel(res2["grads"][k][m], 2 * ref_grads[k][m]) < 1e-4
    b.close()


def test_batch_rejects_focal_spot_other_samplers_and_missing_tables(cuda_ok):
    d = small_geometry(n=8, views=2, U=8, V=8)
    S, mu, G, D = spectral_setup(d, 1, 3, 1)
    with Projector(d, 1, "texture") as pr:
        pr.set_spectral_tables(S, mu, G, 2, D, 1000.0)
        pr.set_focal_spot(np.full(2, 0.1, np.float32), np.zeros(2, np.float32))
        with pytest.raises(CtfpError) as e:
            Batch([pr])
        assert e.value.status == CTFP_UNSUPPORTED
    for sampler in ("global", "brick"):
        with Projector(d, 1, "trilinear") as pr:
            pr.set_spectral_tables(S, mu, G, 2, D, 1000.0)
            pr.set_sampler(sampler)
            with pytest.raises(CtfpError) as e:
                Batch([pr])
            assert e.value.status == CTFP_UNSUPPORTED
    with Projector(d, 1, "trilinear") as pr:
        with pytest.raises(CtfpError) as e:
            Batch([pr])
        assert e.value.status == CTFP_NOT_READY


@pytest.mark.parametrize("shape", [(16, 4), (4, 16), (32, 2), (64, 1)])
def test_batch_unit_shapes_equal_plain_calls(cuda_ok, shape):
    # any ray tile covers every ray of every view exactly once
    items = make_items(ITEMS)
    b = Batch([it[0] for it in items])
    b.set_shape(*shape)
    tu, tv = shape
    tvf = 2 * tv  # the forward's tile: twice as high
    assert b.shapes() == {"fwd": (tu, tvf), "fwd_adjoint": (tu, tv), "views": (1, 1)}
    assert b.info()["units"] == sum(((sp["U"] + tu - 1) // tu) * ((sp["V"] + tvf - 1) // tvf) * sp["views"]
                                    for sp in ITEMS)
    with pytest.raises(CtfpError):
        b.set_shape(8, 4)
    outs = b.forward([it[1] for it in items], want_L=True)
    torch.cuda.synchronize()
    for (pr, vols, _), o in zip(items, outs):
        ref = pr.forward(vols, want_L=True)
        torch.cuda.synchronize()
        assert rel(o["I"], ref["I"]) < 2e-6 and rel(o["L"], ref["L"]) < 1e-6
    b.close()


@pytest.mark.parametrize("views", [(1, 2), (4, 4), (3, 1)])
def test_batch_views_per_unit(cuda_ok, views):
    # a unit marches its rays for several consecutive views: every ray of every
    # view still runs exactly once, forward and fused
    items = make_items(ITEMS)
    b = Batch([it[0] for it in items])
    with pytest.raises(CtfpError):
        b.set_views(0, 1)
    with pytest.raises(CtfpError):
        b.set_views(1, 9)
    b.set_views(*views)
    fv, av = views
    assert b.shapes()["views"] == views
    assert b.info()["units"] == sum(((sp["U"] + 7) // 8) * ((sp["V"] + 15) // 16) * ((sp["views"] + fv - 1) // fv)
                                    for sp in ITEMS)
    outs = b.forward([it[1] for it in items], want_L=True)
    targets, ref_grads = [], []
    for (pr, vols, _), o in zip(items, outs):
        ref = pr.forward(vols, want_L=True)
        torch.cuda.synchronize()
        assert rel(o["I"], ref["I"]) < 2e-6 and rel(o["L"], ref["L"]) < 1e-6
        T = (ref["I"] * 0.98).contiguous()
        targets.append(T)
        r = torch.log(ref["I"].double()) - torch.log(T.double())
        ref_grads.append(pr.backward(ref["L"], gI=(2.0 * r / ref["I"].double()).float()))
    grads = [[torch.zeros_like(v) for v in it[1]] for it in items]
    res = b.forward_adjoint([it[1] for it in items], targets, grads=grads)
    torch.cuda.synchronize()
    for k, (pr, _, _) in enumerate(items):
        for m in range(pr.M):
            assert rel(res["grads"][k][m], ref_grads[k][m]) < 1e-4
    b.close()


def test_batch_autotune_keeps_results(cuda_ok):
    # the tuner changes only the unit shape: the fused step afterwards equals
    # the plain calls, and nothing the caller owns was written while tuning
    items = make_items(ITEMS)
    targets, ref_grads = [], []
    for pr, vols, _ in items:
        f = pr.forward(vols, want_L=True)
        T = (f["I"] * 1.03).contiguous()
        targets.append(T)
        r = torch.log(f["I"].double()) - torch.log(T.double())
        ref_grads.append(pr.backward(f["L"], gI=(2.0 * r / f["I"].double()).float()))
    torch.cuda.synchronize()
    b = Batch([it[0] for it in items])
    grads = [[torch.zeros_like(v) for v in it[1]] for it in items]
    shape = b.autotune([it[1] for it in items], targets)
    assert shape["tile_u"] * shape["tile_v"] == 64 and shape["ms"] > 0
    sh = b.shapes()  # the forward's and the fused kernel's tiles and views, tuned apart
    assert sh["fwd_adjoint"] == (shape["tile_u"], shape["tile_v"])
    assert sh["fwd"][0] * sh["fwd"][1] == 128 and sh["fwd"] == (shape["fwd_tile_u"], shape["fwd_tile_v"])
    assert sh["views"] == (shape["fwd_views"], shape["views"]) and set(sh["views"]) <= {1, 2, 4}
    assert all(float(g.abs().max()) == 0.0 for gk in grads for g in gk)
    res = b.forward_adjoint([it[1] for it in items], targets, grads=grads)
    torch.cuda.synchronize()
    for k, (pr, _, _) in enumerate(items):
        for m in range(pr.M):
            assert rel(res["grads"][k][m], ref_grads[k][m]) < 1e-4
    b.close()


def test_batch_mixed_samplers_equal_plain_calls(cuda_ok):
    # items on the axis sampler (the default) and on the z-layered one run in
    # groups of their own, each equal to its plain calls
    items = make_items(ITEMS[:4])
    items[0][0].set_sampler("layered")
    items[2][0].set_sampler("layered")
    b = Batch([it[0] for it in items])
    outs = b.forward([it[1] for it in items], want_L=True)
    torch.cuda.synchronize()
    for (pr, vols, _), o in zip(items, outs):
        ref = pr.forward(vols, want_L=True)
        torch.cuda.synchronize()
        assert rel(o["I"], ref["I"]) < 2e-6 and rel(o["L"], ref["L"]) < 1e-6
    b.close()
