"""Device table builders against the oracle restatements of the reference's
host builders (Grid.cpp, CBCTForwardProj.cpp, PhantomObject.cpp)."""
import numpy as np
import pytest
import torch

from ct_forward_projection_b200 import (build_det_response, build_grid_table, labels_to_density,
                                        scintillator_thickness)
from ct_forward_projection_b200.physics import GridSpec
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("U,dsize,strip,inter", [(64, 0.2, 50, 200), (63, 0.2, 50, 200), (64, 0.2, 49, 201),
                                                 (63, 0.201, 30, 201), (600, 0.2, 210, 220), (512, 0.8, 50, 200)])
def test_grid_column_vs_oracle(cuda_ok, U, dsize, strip, inter):
    E = 5
    ms = np.linspace(2.0, 20.0, E).astype(np.float32)
    mi = np.linspace(0.001, 0.05, E).astype(np.float32)
    geom = dict(pNumX=8, pNumY=8, pNumZ=8, pLengthX=8., pLengthY=8., pLengthZ=8., projNum=1, dNumU=U, dNumV=5,
                dSize=dsize, sod=1000., sdd=1500.)
    g = build_grid_table(geom, GridSpec(strip, inter, 1.5, 1400.0), ms, mi, 1).cpu().numpy()
    for e in range(E):
        ref = O.grid_column(U, dsize, strip, inter, 1.5, 1400.0, float(ms[e]), float(mi[e]))
        assert np.max(np.abs(g[e] - ref) / np.maximum(ref, 1e-30)) < 2e-6


def _pixel_case_rows(V):
    rng = np.random.RandomState(V)
    rows = {0, 1, V // 2 - 1, V // 2, V - 2, V - 1} | set(rng.randint(0, V, 4).tolist())
    return np.array(sorted(r for r in rows if 0 <= r < V), np.int64)


# (U, V, dSize mm, strip um, interspace um, h mm, FD mm): the four parity cases of the
# reference's fill loops (units N = U * dSize even/odd x interspace even/odd), even and odd
# row counts (V = 384, the headline detector, has no row at y = 0), the headline's 0.8 mm
# pitch with its 50/200 um grid, the large configuration's 27/140 um grid, a strip wider
# than a pixel
PIXEL_CASES = [(64, 5, 0.2, 50, 200, 2.0, 1500.0),     # N even, interspace even
               (64, 384, 0.2, 49, 201, 2.0, 1500.0),   # N even, interspace odd
               (63, 7, 0.201, 50, 200, 1.5, 1400.0),   # N odd, interspace even
               (63, 384, 0.201, 30, 201, 1.5, 1400.0),  # N odd, interspace odd
               (40, 384, 0.8, 50, 200, 2.0, 1500.0),
               (33, 6, 0.8, 27, 140, 1.68, 1500.0),
               (21, 9, 0.2, 210, 220, 2.0, 1000.0)]


@pytest.mark.parametrize("U,V,dsize,strip,inter,h,FD", PIXEL_CASES)
def test_grid_pixel_vs_oracle(cuda_ok, U, V, dsize, strip, inter, h, FD):
    """CTFP_GRID_PIXEL against the oracle's FP64 unit-by-unit incidence-angle
    model (orc_grid_pixel) on off-centre rows.  Tolerance: 2e-6 relative plus
    1.2e-7 per unit of optical depth -ln(T), the FP32 rounding of the
    exponent's argument that the device (like the reference) evaluates in FP32,
    and 1e-35 absolute: a unit behind 160 optical depths of lead transmits
    below FP32's range and reads 0 on the device."""
    E = 4
    ms = np.array([80.0, 20.0, 6.0, 2.5], np.float32)   # lead, 1/mm, low to high energy
    mi = np.array([0.05, 0.01, 0.003, 0.001], np.float32)
    geom = dict(pNumX=8, pNumY=8, pNumZ=8, pLengthX=8., pLengthY=8., pLengthZ=8., projNum=1, dNumU=U, dNumV=V,
                dSize=dsize, sod=1000., sdd=1500.)
    g = build_grid_table(geom, GridSpec(strip, inter, h, FD), ms, mi, 2).cpu().numpy().astype(np.float64)
    rows = _pixel_case_rows(V)
    ref = O.grid_pixel(U, V, dsize, strip, inter, h, FD, ms, mi, rows)
    got = g[:, rows, :]
    tol = 2e-6 * ref + 1.2e-7 * ref * np.maximum(-np.log(np.maximum(ref, 1e-300)), 0.0) + 1e-35
    bad = np.abs(got - ref) > tol
    assert not bad.any(), (f"{bad.sum()} pixels off; worst rel "
                           f"{np.max(np.abs(got - ref) / np.maximum(ref, 1e-300)):.3e}")
    # rows further from the centre see longer slant paths: transmission falls with |y|
    if V % 2 == 0:
        np.testing.assert_allclose(g[:, V // 2 - 1, :], g[:, V // 2, :], rtol=1e-6, atol=0)
    assert np.all(g[:, 0, :] <= g[:, V // 2, :] * (1 + 1e-6))


def test_grid_pixel_layout_central_row_equals_column(cuda_ok):
    E, U, V = 3, 40, 7
    ms = np.array([5.0, 10.0, 15.0], np.float32)
    mi = np.array([0.01, 0.02, 0.03], np.float32)
    geom = dict(pNumX=8, pNumY=8, pNumZ=8, pLengthX=8., pLengthY=8., pLengthZ=8., projNum=1, dNumU=U, dNumV=V,
                dSize=0.2, sod=1000., sdd=1500.)
    spec = GridSpec(50, 200, 2.0, 1500.0)
    col = build_grid_table(geom, spec, ms, mi, 1).cpu().numpy()
    pix = build_grid_table(geom, spec, ms, mi, 2).cpu().numpy()
    assert np.array_equal(pix[:, V // 2, :], col)
    # off-centre rows see a longer slant path: less transmission
    assert np.all(pix[:, 0, :] <= col + 1e-7)


def test_det_response_vs_oracle(cuda_ok):
    t = scintillator_thickness(600 * 4, 0.4, 0.05)
    mu = np.linspace(0.5, 8.0, 11).astype(np.float32)
    D = build_det_response(mu, torch.from_numpy(t).cuda(), 0.8).cpu().numpy()
    ref = O.det_response(mu, t, 0.8)
    # CUDA expf vs the host expf differ by an ulp; 1 - exp(-x) amplifies that
    assert np.max(np.abs(D - ref) / ref) < 1e-6


def test_labels_to_density(cuda_ok):
    rng = np.random.RandomState(0)
    lab = rng.randint(0, 4, (7, 9, 11)).astype(np.uint8)
    dens = [1.0, 2.699, 0.5]
    outs = labels_to_density(torch.from_numpy(lab).cuda(), dens)
    for m in range(3):
        ref = np.where(lab == m + 1, np.float32(dens[m]), np.float32(0))
        assert np.array_equal(outs[m].cpu().numpy(), ref)
