"""Full-size parity with the reference's own projector: the reference binary
(oracle/_ref/ctfp_ref, built from the reference sources by oracle/build_ref.sh)
and the drop-in CLI run the same case directory -- the 256^3 two-material grid
workload (label phantom, 120 one-keV energies, focused grid, scintillator
response) on 6 of its views -- and every output file is compared, in both the
reference's own sampler (hardware texture) and its exact emulation."""
import os
import subprocess

import numpy as np
import pytest

from ct_forward_projection_b200 import physics
from oracle import ref_runner
from tests.test_dropin import CLI
from tests.test_golden import RTOL_COUNTS

pytestmark = pytest.mark.gpu

VIEWS = 6


@pytest.fixture(scope="module")
def ref_case():
    if not os.path.exists(ref_runner.REF_BIN):
        pytest.skip("reference binary not built (oracle/build_ref.sh)")
    w = physics.workload("poly_grid_256")
    g = dict(w.geometry)
    g["projNum"] = VIEWS
    case = ref_runner.reference_case_from_workload(w, g)
    # the reference's grid projector never copies InterspaceDensity from its
    # configuration (CBCTPolyForwardProjGrid.cpp:53-63, the one GridInfo field
    # left out), so its interspace attenuation uses an uninitialised density;
    # an air interspace (density 0) is the configuration where that bug and
    # the intended behaviour agree
    case["grid"]["inter_density"] = 0.0
    outs, _, _ = ref_runner.run(case, timeout=900)
    return case, outs


@pytest.mark.parametrize("interp", ["texture", "texemu"])
def test_fullsize_cli_matches_reference_binary(cuda_ok, tmp_path, ref_case, interp):
    case, ref = ref_case
    ref_runner.write_case(str(tmp_path), case)
    env = dict(os.environ, CTFP_INTERP=interp)
    r = subprocess.run([CLI, str(tmp_path)], capture_output=True, text=True, timeout=900, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    ours = ref_runner.read_outputs(str(tmp_path), case)
    r0 = ref["BgImgPro"].astype(np.float64)
    assert np.max(np.abs(ours["BgImgPro"] - r0) / r0) < 1e-5
    for key in ("PhoImgPro", "PhoImgAbsorb"):
        a, b = ours[key].astype(np.float64), ref[key].astype(np.float64)
        assert a.shape == b.shape
        err = np.maximum(np.abs(a - b) - 1.0, 0.0) / np.maximum(b, 1.0)
        assert np.max(err) < RTOL_COUNTS, (key, float(np.max(err)))
    proj, rproj = ours["Projection"].astype(np.float64), ref["Projection"].astype(np.float64)
    big = np.isfinite(proj) & np.isfinite(rproj) & (ours["PhoImgPro"] > 1000)
    assert big.sum() > 0.5 * proj.size
    assert np.max(np.abs(proj[big] - rproj[big])) < 1e-3
