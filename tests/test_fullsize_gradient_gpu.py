"""The adjoint at full size: the three-material 256^3 workload (180 views,
384 x 384 detector, 101 energies, grid and scintillator tables), loss
sum (log I - log T)^2 with T the projection of the phantom scaled by 0.97.
The GPU gradient (ctfp_backward from the forward's L checkpoint) is compared
with central differences of the loss, taken by two full forwards per voxel on
64 seeded voxels.  The loss difference is summed per ray in FP64, so the rays
a perturbation does not reach (bit-identical in both forwards) cancel
exactly and the difference carries no rounding from the other 2.65e7 terms."""
import numpy as np
import pytest
import torch

from ct_forward_projection_b200 import Projector, physics

pytestmark = pytest.mark.gpu

N_VOXELS = 64
H = 0.01  # g/cm^3: keeps the iodine term's third-order error near 1e-4


@pytest.fixture(scope="module")
def problem(cuda_ok):
    w = physics.workload("diff_3mat_256")
    vols = physics.phantom(w, "cuda:0")
    pr = Projector(w.geometry, len(vols), "trilinear")
    pr.set_tables_from_workload(w)
    logT = torch.log(pr.forward([v * 0.97 for v in vols])["I"].double())
    yield w, vols, pr, logT
    pr.close()


def residual(pr, vols, logT):
    return torch.log(pr.forward(vols)["I"].double()) - logT


def test_gradient_matches_central_differences(problem):
    w, vols, pr, logT = problem
    f = pr.forward(vols, want_L=True)
    r = torch.log(f["I"].double()) - logT
    gI = (2.0 * r / f["I"].double()).float()
    grads = pr.backward(f["L"], gI)
    torch.cuda.synchronize()
    del f, gI
    gmax = [float(g.abs().max()) for g in grads]
    assert all(m > 0 for m in gmax)

    nz, ny, nx = vols[0].shape
    rng = np.random.RandomState(2024)
    worst = 0.0
    for k in range(N_VOXELS):
        m = k % len(vols)
        # voxels of the central part of the volume, which every view's rays cross
        z = rng.randint(int(0.3 * nz), int(0.7 * nz))
        y = rng.randint(int(0.3 * ny), int(0.7 * ny))
        x = rng.randint(int(0.3 * nx), int(0.7 * nx))
        v0 = np.float32(vols[m][z, y, x].item())
        vp, vm = np.float32(v0 + np.float32(H)), np.float32(v0 - np.float32(H))
        vols[m][z, y, x] = float(vp)
        rp = residual(pr, vols, logT)
        vols[m][z, y, x] = float(vm)
        rm = residual(pr, vols, logT)
        vols[m][z, y, x] = float(v0)
        fd = float(torch.sum(rp * rp - rm * rm)) / (float(vp) - float(vm))
        g = float(grads[m][z, y, x])
        scale = max(abs(fd), 1e-2 * gmax[m])
        worst = max(worst, abs(g - fd) / scale)
    assert worst < 2e-3, worst
