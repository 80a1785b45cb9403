"""The oracle against known answers (CPU).

The reference ships no tests or golden data; these pins come from physics and
arithmetic that the reference's algorithm must satisfy, plus the committed
fixtures of the reference's own CUDA pipeline (test_golden.py)."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.conftest import small_geometry, random_volumes


def test_compute_paras_known_values():
    # 128 mm phantom at 1 mm, 256 x 1 mm detector, SOD 1000 / SDD 1500:
    # FOVR = 1000 * 128 / sqrt(128^2 + 1500^2), K = round(2 FOVR / 0.5)
    d = dict(pNumX=128, pNumY=128, pNumZ=128, pLengthX=128., pLengthY=128., pLengthZ=128., projNum=60,
             dNumU=256, dNumV=256, dSize=1.0, sod=1000., sdd=1500., rotatedDirection=1)
    s = O.compute_paras(d)
    assert abs(s["FOVR"] - 1000 * 128 / np.hypot(128, 1500)) < 1e-4
    assert s["dx"] == 0.5 and s["intNum"] == 340 and s["thetaStep"] == np.float32(6.0)


def test_view_angle_fp32():
    d = small_geometry(views=7)
    a = O.view_angle(d, 3)
    step = np.float32(360) / np.float32(7)
    expect = np.float32(np.float32(np.float32(3) * step) / np.float32(180)) * np.float32(np.arccos(np.float32(-1)))
    assert a == pytest.approx(float(expect), rel=0, abs=1e-7)
    d["rotatedDirection"] = -1
    assert O.view_angle(d, 3) == pytest.approx(-float(expect), abs=1e-7)


def test_zero_volume_gives_flat_field():
    d = small_geometry()
    vols = [np.zeros((d["pNumZ"], d["pNumY"], d["pNumX"]), np.float32)]
    S = np.array([0.3, 0.7], np.float32)
    W = O.energy_weights(d, S, I0Val=1000.0)
    out = O.forward(d, vols, np.array([[0.02], [0.01]], np.float32), W)
    assert np.all(out["L"] == 0)
    I0 = W.sum(axis=0).reshape(-1)
    np.testing.assert_allclose(out["I"].reshape(d["projNum"], -1), np.broadcast_to(I0, (d["projNum"], I0.size)),
                               rtol=1e-15)
    assert np.all(out["IAbsorb"] == 0)


def test_uniform_volume_central_ray_chord():
    # uniform density 1: with an odd detector the central pixel lies on the
    # axis, so its ray runs through the middle of the volume along x (view 0)
    # or y (view 1); the trilinear support is (-1, n) voxels, whose integral
    # is n voxels: L = n * pSize up to the sampling quadrature.
    n = 32
    d = dict(pNumX=n, pNumY=n, pNumZ=n, pLengthX=32., pLengthY=32., pLengthZ=32., projNum=4, dNumU=101,
             dNumV=101, dSize=1.0, sod=200., sdd=400., rotatedDirection=1)
    assert O.compute_paras(d)["FOVR"] > 23.0
    vols = [np.ones((n, n, n), np.float32)]
    ids = np.array([p * 101 * 101 + 50 * 101 + 50 for p in range(4)])
    L = O.line_integrals(d, vols, ray_ids=ids)[:, 0]
    np.testing.assert_allclose(L, 32.0, atol=0.3)


def test_linearity_in_density():
    d = small_geometry()
    a, b = random_volumes(d, 2, 5)
    La = O.line_integrals(d, [a])
    Lb = O.line_integrals(d, [b])
    Lab = O.line_integrals(d, [2.0 * a + 3.0 * b])
    # the combined volume is rounded to float32 once per voxel
    np.testing.assert_allclose(Lab, 2 * La + 3 * Lb, rtol=5e-7, atol=1e-9)


def test_single_vs_multi_material_equivalence():
    # the reference's multi-material path integrates mu_E = sum_m mu_em rho_m;
    # the single-material path integrates rho then multiplies; both equal
    # sum_m mu_em L_m because interpolation is linear
    d = small_geometry()
    vols = random_volumes(d, 2, 9)
    mu = np.array([[0.02, 0.05], [0.01, 0.03]], np.float32)
    S = np.array([0.4, 0.6], np.float32)
    W = O.energy_weights(d, S, I0Val=500.0)
    multi = O.forward(d, vols, mu, W)
    for e in range(2):
        mix = (mu[e, 0].astype(np.float64) * vols[0] + mu[e, 1].astype(np.float64) * vols[1])
        Lmix = O.line_integrals(d, [mix.astype(np.float32)])[:, 0]
        Lsum = multi["L"] @ mu[e].astype(np.float64)
        np.testing.assert_allclose(Lmix, Lsum, rtol=2e-6, atol=1e-9)


def test_texemu_close_to_trilinear():
    d = small_geometry()
    vols = random_volumes(d, 1, 3)
    a = O.line_integrals(d, vols, O.TRILINEAR)
    b = O.line_integrals(d, vols, O.TEXEMU)
    # the texture unit holds each fraction and each corner-weight product with
    # 8 fractional bits, so a sample can move by a few 1/256 of its corner
    # spread; on white-noise volumes that stays well under 1 %
    assert np.max(np.abs(a - b) / np.maximum(np.abs(a), 1)) < 1e-2


def test_adjoint_dot_product():
    d = small_geometry(n=12, views=3, U=8, V=6)
    M = 2
    vols = random_volumes(d, M, 11)
    rng = np.random.RandomState(4)
    gL = rng.normal(size=(d["projNum"] * d["dNumU"] * d["dNumV"], M))
    L = O.line_integrals(d, vols)
    g = O.line_integrals_adjoint(d, gL, M)
    lhs = float(np.sum(L * gL))
    rhs = float(sum(np.sum(g[m] * vols[m].astype(np.float64)) for m in range(M)))
    assert lhs == pytest.approx(rhs, rel=1e-10)


def test_msvc_rand_known_sequence():
    # MSVC rand() after srand(1) returns 41, 18467, 6334, 26500; the thickness
    # jitter uses the same generator seeded with 100 (CBCTForwardProj.cpp:101)
    st = 1
    seq = []
    for _ in range(4):
        st = (st * 214013 + 2531011) & 0xFFFFFFFF
        seq.append((st >> 16) & 0x7FFF)
    assert seq == [41, 18467, 6334, 26500]
    t = O.scint_thickness(5, 0.4, 0.05)
    st = 100
    exp = []
    for _ in range(5):
        st = (st * 214013 + 2531011) & 0xFFFFFFFF
        r = (st >> 16) & 0x7FFF
        exp.append(np.float32(0.4) + (np.float32(-0.05) + np.float32(r % 1001) / np.float32(10000.0)))
    np.testing.assert_array_equal(t, np.array(exp, np.float32))


def test_grid_column_no_attenuation_is_one():
    g = O.grid_column(64, 0.2, 50, 200, 2.0, 1500.0, 0.0, 0.0)
    np.testing.assert_allclose(g, 1.0, rtol=0, atol=1e-7)


@pytest.mark.parametrize("U,dsize,inter", [(64, 0.2, 200), (63, 0.2, 200), (64, 0.2, 201), (63, 0.201, 201)])
def test_grid_column_parity_cases_mean_open_fraction(U, dsize, inter):
    # opaque strips and a transparent interspace: each column's value is the
    # open fraction of its micron units; over the whole detector it tends to
    # inter / period (the four even/odd cases of Grid.cpp:90-270)
    g = O.grid_column(U, dsize, 50, inter, 2.0, 1500.0, 1e6, 0.0)
    frac = g.mean()
    assert abs(frac - inter / (50 + inter)) < 0.02
    assert np.all((g >= 0) & (g <= 1))
    # symmetric about the centre up to the one-unit mirror offset
    assert np.max(np.abs(g - g[::-1])) < 0.02


@pytest.mark.parametrize("U,dsize,strip,inter", [(64, 0.2, 50, 200), (64, 0.2, 49, 201), (63, 0.201, 50, 200),
                                                 (63, 0.201, 30, 201), (40, 0.8, 50, 200)])
def test_grid_pixel_central_row_is_the_column_model(U, dsize, strip, inter):
    """The FP64 incidence-angle grid at y = 0 (the central row of an odd
    detector) is the reference's column model (FP32 as the reference computes
    it); rows off the centre transmit less, symmetrically about it."""
    ms = np.array([30.0, 6.0, 2.0], np.float32)
    mi = np.array([0.05, 0.01, 0.002], np.float32)
    V = 9
    g = O.grid_pixel(U, V, dsize, strip, inter, 2.0, 1500.0, ms, mi)
    for e in range(3):
        col = O.grid_column(U, dsize, strip, inter, 2.0, 1500.0, float(ms[e]), float(mi[e]))
        assert np.max(np.abs(g[e, V // 2] - col) / col) < 3e-6
    assert np.all(g[:, 0] < g[:, 1]) and np.all(g[:, 1] < g[:, V // 2])
    np.testing.assert_allclose(g[:, 0], g[:, V - 1], rtol=1e-14)


def test_finalize_floor_and_log():
    I = np.array([[[10.7, 0.4]]], np.float32)
    I0 = np.array([[20.0, 5.0]], np.float32)
    Ip, proj = O.finalize(I, I0)
    assert Ip.tolist() == [[[10, 0]]]
    assert proj[0, 0, 0] == pytest.approx(np.log(2.0), rel=1e-6)
    assert np.isinf(proj[0, 0, 1])


def _msvc_offsets(n, size):
    # restatement of CBCTForwardProj::computeFoSpOffset in numpy float32
    state = 10
    r = np.float32(size / 2.0)
    sz = int(np.float32(size) * np.float32(10000))
    bound = np.float32(np.arccos(np.float32(-1.0))) * r * r

    def rnd():
        nonlocal state
        state = (state * 214013 + 2531011) & 0xFFFFFFFF
        return (state >> 16) & 0x7FFF

    us, vs = [], []
    for _ in range(n):
        while True:
            du = -r + np.float32(rnd() % sz) / np.float32(10000.0)
            dv = -r + np.float32(rnd() % sz) / np.float32(10000.0)
            if not (du * du + dv * dv > bound):
                break
        us.append(du)
        vs.append(dv)
    return np.array(us, np.float32), np.array(vs, np.float32)


@pytest.mark.parametrize("size", [0.4, 1.0, 0.0123])
def test_focal_spot_offsets_restatements_agree(size):
    # the oracle's C restatement, the library's and a numpy restatement of the
    # reference's srand(10) / MSVC rand() draw
    from ct_forward_projection_b200.projector import focal_spot_offsets
    u, v = O.focal_spot_offsets(300, size)
    lu, lv = focal_spot_offsets(300, size)
    nu, nv = _msvc_offsets(300, size)
    np.testing.assert_array_equal(u, lu)
    np.testing.assert_array_equal(v, lv)
    np.testing.assert_array_equal(u, nu)
    np.testing.assert_array_equal(v, nv)
    r = size / 2
    assert np.all(u >= -r - 1e-6) and np.all(u < r + 1e-6)
    assert np.all(u * u + v * v <= np.pi * r * r + 1e-6)


def test_shift_views_integer_offsets_move_the_image():
    # an offset of exactly k detector pitches moves the image by k pixels,
    # zero-filled at the edge, in both weight modes
    d = dict(pNumX=4, pNumY=4, pNumZ=4, pLengthX=4.0, pLengthY=4.0, pLengthZ=4.0, projNum=2, dNumU=6, dNumV=5,
             dSize=0.5, sod=100.0, sdd=200.0, rotatedDirection=1)
    rng = np.random.RandomState(0)
    L = rng.uniform(0, 1, (2, 5, 6, 2))
    fu = np.array([1.0, -0.5], np.float32)  # +2 and -1 pixels
    fv = np.array([0.0, 0.5], np.float32)   # 0 and +1 pixel
    for mode in (O.TRILINEAR, O.TEXEMU):
        out = O.shift_views(d, L.reshape(-1, 2), 2, (fu, fv), mode).reshape(2, 5, 6, 2)
        ref0 = np.zeros_like(L[0])
        ref0[:, :4] = L[0][:, 2:]
        ref1 = np.zeros_like(L[1])
        ref1[:4, 1:] = L[1][1:, :5]
        np.testing.assert_array_equal(out[0], ref0)
        np.testing.assert_array_equal(out[1], ref1)
