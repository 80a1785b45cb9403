"""The hand-written adjoint (no reference counterpart): dot-product test,
FP64 oracle adjoint, central finite differences of an FP64 loss."""
import numpy as np
import pytest
import torch

from ct_forward_projection_b200 import Projector
from oracle import oracle as O
from tests.conftest import random_volumes, small_geometry, spectral_setup

pytestmark = pytest.mark.gpu


def to_dev(vols):
    return [torch.from_numpy(v).cuda() for v in vols]


@pytest.mark.parametrize("mode", ["trilinear", "texemu"])
@pytest.mark.parametrize("M", [1, 2, 3])
def test_line_integral_adjoint_dot_product(cuda_ok, mode, M):
    # <A x, y> = <x, A^T y>, both sides accumulated in FP64
    d = small_geometry(n=(18, 14, 11), views=5, U=21, V=13)
    x = random_volumes(d, M, 50 + M)
    rng = np.random.RandomState(M)
    with Projector(d, M, mode) as pr:
        Ax = pr.line_integrals(to_dev(x)).double().cpu().numpy()
        y = rng.normal(size=Ax.shape).astype(np.float32)
        g = pr.line_integrals_adjoint(torch.from_numpy(y).cuda())
        torch.cuda.synchronize()
    lhs = float(np.sum(Ax * y.astype(np.float64)))
    rhs = float(sum(np.sum(g[m].double().cpu().numpy() * x[m].astype(np.float64)) for m in range(M)))
    assert abs(lhs - rhs) / max(abs(lhs), 1e-30) < 1e-5


@pytest.mark.parametrize("mode", ["trilinear", "texemu"])
def test_adjoint_anisotropic_voxels_vs_oracle(cuda_ok, mode):
    # voxels of 1.0 x 0.75 x 2.5 mm: the adjoint against the oracle's
    from tests.test_forward_gpu import ANISO
    d = dict(ANISO)
    M = 2
    rng = np.random.RandomState(5)
    gL = rng.normal(size=(d["projNum"] * d["dNumV"] * d["dNumU"], M)).astype(np.float32)
    with Projector(d, M, mode) as pr:
        g = pr.line_integrals_adjoint(torch.from_numpy(gL.reshape(d["projNum"], d["dNumV"], d["dNumU"], M)).cuda())
        torch.cuda.synchronize()
    ref = O.line_integrals_adjoint(d, gL, M, O.TRILINEAR if mode == "trilinear" else O.TEXEMU)
    for m in range(M):
        a = g[m].double().cpu().numpy()
        assert np.max(np.abs(a - ref[m])) / np.max(np.abs(ref[m])) < (1e-5 if mode == "trilinear" else 1e-3)


@pytest.mark.parametrize("mode", ["trilinear", "texemu"])
def test_line_integral_adjoint_vs_oracle(cuda_ok, mode):
    d = small_geometry(n=12, views=4, U=14, V=9)
    M = 2
    rng = np.random.RandomState(2)
    gL = rng.normal(size=(d["projNum"] * d["dNumV"] * d["dNumU"], M)).astype(np.float32)
    with Projector(d, M, mode) as pr:
        g = pr.line_integrals_adjoint(torch.from_numpy(gL.reshape(d["projNum"], d["dNumV"], d["dNumU"], M)).cuda())
        torch.cuda.synchronize()
    ref = O.line_integrals_adjoint(d, gL, M, O.TRILINEAR if mode == "trilinear" else O.TEXEMU)
    for m in range(M):
        a = g[m].double().cpu().numpy()
        scale = np.max(np.abs(ref[m]))
        assert np.max(np.abs(a - ref[m])) / scale < (1e-5 if mode == "trilinear" else 1e-3)


def test_backward_vs_oracle(cuda_ok):
    d = small_geometry(n=14, views=4, U=16, V=10)
    M = 2
    vols = random_volumes(d, M, 31)
    S, mu, G, D = spectral_setup(d, M, 9, 4)
    W = O.energy_weights(d, S, G, 2, D, 1000.0)
    rng = np.random.RandomState(7)
    n = d["projNum"] * d["dNumV"] * d["dNumU"]
    gI = rng.normal(size=n).astype(np.float32)
    gA = rng.normal(size=n).astype(np.float32)
    with Projector(d, M, "trilinear") as pr:
        pr.set_spectral_tables(S, mu, G, 2, D, 1000.0)
        f = pr.forward(to_dev(vols), want_L=True)
        shp = f["I"].shape
        g = pr.backward(f["L"], torch.from_numpy(gI).cuda().view(shp), torch.from_numpy(gA).cuda().view(shp))
        torch.cuda.synchronize()
        L = f["L"].double().cpu().numpy().reshape(n, M)
    ref = O.backward(d, mu, W, L, gI, gA, O.TRILINEAR)
    for m in range(M):
        a = g[m].double().cpu().numpy()
        assert np.max(np.abs(a - ref[m])) / np.max(np.abs(ref[m])) < 1e-4


def test_backward_central_differences(cuda_ok):
    # loss = sum (log I - log I_t)^2; gradient from the GPU adjoint against FP64
    # central differences of the oracle loss on 64 seeded voxels
    d = small_geometry(n=10, views=3, U=12, V=8)
    M = 2
    vols = random_volumes(d, M, 61)
    S, mu, G, D = spectral_setup(d, M, 7, 6)
    W = O.energy_weights(d, S, G, 2, D, 1000.0)
    rng = np.random.RandomState(9)
    target = O.forward(d, [v * np.float32(0.97) for v in vols], mu, W)["I"]
    logt = np.log(target)

    def loss(vs):
        I = O.forward(d, vs, mu, W)["I"]
        return float(np.sum((np.log(I) - logt) ** 2))

    with Projector(d, M, "trilinear") as pr:
        pr.set_spectral_tables(S, mu, G, 2, D, 1000.0)
        f = pr.forward(to_dev(vols), want_L=True)
        I = f["I"].double()
        gI = (2.0 * (torch.log(I) - torch.from_numpy(logt).cuda().view(I.shape)) / I).float()
        g = pr.backward(f["L"], gI)
        torch.cuda.synchronize()
    g = [x.double().cpu().numpy() for x in g]
    shape = vols[0].shape
    worst = 0.0
    for k in range(64):
        m = k % M
        idx = tuple(rng.randint(0, s) for s in shape)
        h = 1e-3
        vp = [v.astype(np.float64).copy() for v in vols]
        vm = [v.astype(np.float64).copy() for v in vols]
        vp[m][idx] += h
        vm[m][idx] -= h
        fd = (loss([v.astype(np.float32) for v in vp]) - loss([v.astype(np.float32) for v in vm])) / (2 * h)
        # the perturbation itself is rounded to float32; use the realised step
        hp = np.float32(vols[m][idx] + np.float32(h)) - vols[m][idx]
        hm = vols[m][idx] - np.float32(vols[m][idx] - np.float32(h))
        fd = fd * 2 * h / (float(hp) + float(hm))
        scale = max(abs(fd), 1e-3 * np.max(np.abs(g[m])))
        worst = max(worst, abs(g[m][idx] - fd) / scale)
    assert worst < 2e-2


def test_autograd_binding(cuda_ok):
    # project() through torch.autograd equals ctfp_backward with the same
    # dLoss/dI, dLoss/dIAbsorb, and its directional derivative matches FP64
    # central differences of the oracle loss
    from ct_forward_projection_b200.autograd import project
    d = small_geometry(n=(11, 10, 9), views=3, U=12, V=9)
    M = 2
    vols = random_volumes(d, M, 71)
    S, mu, G, D = spectral_setup(d, M, 6, 8)
    W = O.energy_weights(d, S, G, 2, D, 1000.0)
    target = O.forward(d, [v * np.float32(0.95) for v in vols], mu, W)["I"]
    logt = torch.from_numpy(np.log(target)).cuda().float()
    with Projector(d, M, "trilinear") as pr:
        pr.set_spectral_tables(S, mu, G, 2, D, 1000.0)
        xs = [torch.from_numpy(v).cuda().requires_grad_(True) for v in vols]
        I, A, I0 = project(pr, *xs)
        loss = torch.sum((torch.log(I) - logt.view(I.shape)) ** 2) + 1e-4 * torch.sum(A)
        loss.backward()
        f = pr.forward(to_dev(vols), want_L=True)
        gI = 2.0 * (torch.log(f["I"]) - logt.view(I.shape)) / f["I"]
        ref = pr.backward(f["L"], gI=gI, gIAbsorb=torch.full_like(f["I"], 1e-4))
        torch.cuda.synchronize()
        assert not I0.requires_grad
    for m in range(M):
        assert torch.max(torch.abs(xs[m].grad - ref[m])) / torch.max(torch.abs(ref[m])) < 1e-5
    rng = np.random.RandomState(3)
    dirs = [rng.normal(size=v.shape) for v in vols]

    def f64_loss(t):
        vs = [(v.astype(np.float64) + t * dv).astype(np.float32) for v, dv in zip(vols, dirs)]
        r = O.forward(d, vs, mu, W)
        return float(np.sum((np.log(r["I"]) - np.log(target)) ** 2) + 1e-4 * np.sum(r["IAbsorb"]))

    h = 1e-3
    fd = (f64_loss(h) - f64_loss(-h)) / (2 * h)
    an = sum(float(np.sum(xs[m].grad.double().cpu().numpy() * dirs[m])) for m in range(M))
    assert abs(an - fd) / abs(fd) < 1e-2


def test_fused_log_loss_binding(cuda_ok):
    # LogIntensityLoss (the fused forward + loss + adjoint kernel) gives the
    # loss and gradients of sum (log I - log T)^2 computed through project(),
    # scales its gradient by the incoming one, and replays its graph on a
    # second call, in the exact and the hardware-texture modes
    from ct_forward_projection_b200._capi import CtfpError
    from ct_forward_projection_b200.autograd import LogIntensityLoss, project
    d = small_geometry(n=(13, 12, 10), views=4, U=14, V=10)
    M = 2
    vols = random_volumes(d, M, 72)
    S, mu, G, D = spectral_setup(d, M, 7, 9)
    W = O.energy_weights(d, S, G, 2, D, 1000.0)
    target = O.forward(d, [v * np.float32(0.95) for v in vols], mu, W)["I"]
    with Projector(d, M, "trilinear") as pr:
        pr.set_spectral_tables(S, mu, G, 2, D, 1000.0)
        T = torch.from_numpy(target.astype(np.float32)).cuda().view(pr.shape_proj)
        xs = [torch.from_numpy(v).cuda().requires_grad_(True) for v in vols]
        I, _, _ = project(pr, *xs)
        ref = torch.sum((torch.log(I) - torch.log(T)) ** 2)
        ref.backward()
        with LogIntensityLoss(pr) as lf:
            for _ in range(2):
                ys = [torch.from_numpy(v).cuda().requires_grad_(True) for v in vols]
                loss = lf(T, *ys)
                (2.0 * loss).backward()
                torch.cuda.synchronize()
                assert abs(float(loss.detach()) - float(ref.detach())) <= 1e-5 * abs(float(ref.detach()))
                for m in range(M):
                    err = torch.max(torch.abs(ys[m].grad - 2.0 * xs[m].grad)) / torch.max(torch.abs(2.0 * xs[m].grad))
                    assert float(err) < 1e-5
    # the reference's own sampler: the same loss and gradients as project()
    with Projector(d, M, "texture") as pt:
        pt.set_spectral_tables(S, mu, G, 2, D, 1000.0)
        xs = [torch.from_numpy(v).cuda().requires_grad_(True) for v in vols]
        I, _, _ = project(pt, *xs)
        ref = torch.sum((torch.log(I) - torch.log(T)) ** 2)
        ref.backward()
        with LogIntensityLoss(pt) as lf:
            ys = [torch.from_numpy(v).cuda().requires_grad_(True) for v in vols]
            loss = lf(T, *ys)
            loss.backward()
            torch.cuda.synchronize()
        assert abs(float(loss.detach()) - float(ref.detach())) <= 1e-5 * abs(float(ref.detach()))
        for m in range(M):
            assert float(torch.max(torch.abs(ys[m].grad - xs[m].grad)) / torch.max(torch.abs(xs[m].grad))) < 1e-5
        # a plan with a focal spot has no adjoint
        pt.set_focal_spot(np.full(d["projNum"], 0.1, np.float32), np.zeros(d["projNum"], np.float32))
        with pytest.raises(CtfpError):
            LogIntensityLoss(pt)


def test_view_ranges_compose_the_full_projection(cuda_ok):
    # ctfp_forward_views / ctfp_backward_views on three contiguous ranges (what
    # three GPUs of a view-sharded projection run) give the full forward
    # exactly and the full adjoint once the partial gradients are summed
    from ct_forward_projection_b200.shard import view_range
    d = small_geometry(n=(16, 14, 12), views=7, U=15, V=9)
    M = 2
    vols = to_dev(random_volumes(d, M, 8))
    S, mu, G, D = spectral_setup(d, M, 5, 2)
    with Projector(d, M, "trilinear") as pr:
        pr.set_spectral_tables(S, mu, G, 2, D, 1000.0)
        full = pr.forward(vols, want_L=True)
        gI = torch.randn(full["I"].shape, device="cuda", generator=torch.Generator("cuda").manual_seed(1)) * 1e-3
        ref = pr.backward(full["L"], gI=gI)
        acc = [torch.zeros_like(v) for v in vols]
        for r in range(3):
            v0, n = view_range(d["projNum"], r, 3)
            part = pr.forward(vols, want_L=True, views=(v0, n))
            assert torch.equal(part["I"], full["I"][v0:v0 + n])
            assert torch.equal(part["L"], full["L"][v0:v0 + n])
            g = pr.backward(part["L"], gI=gI[v0:v0 + n].contiguous(), views=(v0, n))
            for a, b in zip(acc, g):
                a += b
        torch.cuda.synchronize()
    for a, b in zip(acc, ref):
        assert torch.max(torch.abs(a - b)) / torch.max(torch.abs(b)) < 1e-5
