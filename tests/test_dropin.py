"""The drop-in C++ classes and CLI (ct_forward_projection_b200/compat):
ForwardProjection::run reads the reference's ScanSetting.ini / OutPutFolder.ini
and writes the reference's output files.  CPU tests cover the configuration
contract; GPU tests run the CLI on the golden cases' inputs (in the reference's
file formats) and compare its files with the reference binary's outputs."""
import os
import subprocess

import numpy as np
import pytest

from oracle import ref_runner
from tests.test_golden import CASES, FIX, RTOL_COUNTS

CLI = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "ct_forward_projection_b200",
                   "ctfp_forward_projection")


def run_cli(run_dir, env_extra=None, timeout=300):
    env = dict(os.environ)
    env.update(env_extra or {})
    return subprocess.run([CLI, run_dir], capture_output=True, text=True, timeout=timeout, env=env)


def case_from_fixture(z, name):
    p = name + "/"
    gv = z["geometry"]
    keys = ("pNumX", "pNumY", "pNumZ", "pLengthX", "pLengthY", "pLengthZ", "projNum", "dNumU", "dNumV", "dSize",
            "sod", "sdd", "rotatedDirection")
    g = {k: (int(v) if k in ("pNumX", "pNumY", "pNumZ", "projNum", "dNumU", "dNumV", "rotatedDirection")
             else float(v)) for k, v in zip(keys, gv)}
    sd, st, se, sf = [float(x) for x in z["scint_params"]]
    FD, h, strip, inter, sdens, idens = [float(x) for x in z["grid_params"]]
    return {
        "flags": dict(zip(("IsTestI0", "IsDetResponse", "IsGrid", "IsSingleMaterial"), z[p + "flags"].tolist())),
        "geometry": g, "I0Val": float(z["I0Val"][0]), "spectrum": z[p + "spectrum"], "labels": z[p + "labels"],
        "densities": [float(d) for d in z[p + "densities"]], "mass_atten": list(z[p + "mass_atten"]),
        "scint": {"density": sd, "thickness": st, "err": se, "factor": sf, "mass_atten": z[p + "scint_ma"]},
        "grid": {"FD": FD, "h": h, "strip": int(strip), "inter": int(inter), "strip_density": sdens,
                 "inter_density": idens, "strip_ma": z[p + "grid_strip_ma"], "inter_ma": z[p + "grid_inter_ma"]},
    }


@pytest.fixture(scope="module")
def fx():
    return np.load(FIX)


def test_cli_built():
    assert os.access(CLI, os.X_OK), "build the drop-in CLI: python -m ct_forward_projection_b200.build"


def test_missing_config_is_an_error(tmp_path):
    r = run_cli(str(tmp_path))
    assert r.returncode == 1 and "ScanPara" in r.stderr


def test_multimaterial_without_response_is_rejected(tmp_path, fx):
    # the reference silently does nothing for IsDetResponse=0, IsSingleMaterial=0
    case = case_from_fixture(fx, "grid_response_multi")
    case["flags"]["IsDetResponse"] = 0
    ref_runner.write_case(str(tmp_path), case)
    r = run_cli(str(tmp_path))
    assert r.returncode == 1 and "no projector" in r.stderr


def test_missing_input_file_is_an_error(tmp_path, fx):
    case = case_from_fixture(fx, "nogrid_response_sinmat")
    ref_runner.write_case(str(tmp_path), case)
    os.unlink(os.path.join(str(tmp_path), "InputData", "spectrum.dat"))
    r = run_cli(str(tmp_path))
    assert r.returncode == 1 and "spectrum" in r.stderr


def test_ini_comments_and_whitespace(tmp_path, fx):
    # values end at ';' and are trimmed (ScanSetting.ini:2,9 carry ';' and tabs);
    # a key missing from its section is reported
    case = case_from_fixture(fx, "nogrid_response_sinmat")
    ref_runner.write_case(str(tmp_path), case)
    ini = os.path.join(str(tmp_path), "Config", "ScanSetting.ini")
    text = open(ini).read().replace("DNumV=", "DNumW=")
    open(ini, "w").write(text)
    r = run_cli(str(tmp_path))
    assert r.returncode == 1 and "Detector" in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("interp", ["texture", "texemu"])
@pytest.mark.parametrize("name", CASES)
def test_cli_files_match_reference_binary(fx, cuda_ok, tmp_path, name, interp):
    case = case_from_fixture(fx, name)
    ref_runner.write_case(str(tmp_path), case)
    r = run_cli(str(tmp_path), {"CTFP_INTERP": interp})
    assert r.returncode == 0, r.stderr[-2000:]
    outs = ref_runner.read_outputs(str(tmp_path), case)
    p = name + "/"
    ref_I0 = fx[p + "out_BgImgPro"].astype(np.float64)
    assert np.max(np.abs(outs["BgImgPro"] - ref_I0) / ref_I0) < 1e-5
    if name == "test_i0":
        return
    for key in ("PhoImgPro", "PhoImgAbsorb"):
        ref = fx[p + "out_" + key].astype(np.float64)
        got = outs[key].astype(np.float64)
        err = np.maximum(np.abs(got - ref) - 1.0, 0.0) / np.maximum(ref, 1.0)
        assert np.max(err) < RTOL_COUNTS, (key, float(np.max(err)))
    proj, rproj = outs["Projection"].astype(np.float64), fx[p + "out_Projection"].astype(np.float64)
    big = np.isfinite(proj) & np.isfinite(rproj) & (outs["PhoImgPro"] > 1000)
    assert np.max(np.abs(proj[big] - rproj[big])) < 1e-3
    if (p + "out_ADetResponse") in fx.files:
        np.testing.assert_allclose(outs["ADetResponse"], fx[p + "out_ADetResponse"], rtol=1e-5, atol=1e-6)


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_cli_skip_empty_matches_reference_binary(fx, cuda_ok, tmp_path, name):
    # CTFP_SKIP_EMPTY=1 (empty-space skipping in the hardware-texture march)
    # writes the same files within the same bounds
    case = case_from_fixture(fx, name)
    ref_runner.write_case(str(tmp_path), case)
    r = run_cli(str(tmp_path), {"CTFP_INTERP": "texture", "CTFP_SKIP_EMPTY": "1"})
    assert r.returncode == 0, r.stderr[-2000:]
    outs = ref_runner.read_outputs(str(tmp_path), case)
    p = name + "/"
    if name == "test_i0":
        return
    for key in ("PhoImgPro", "PhoImgAbsorb"):
        ref = fx[p + "out_" + key].astype(np.float64)
        got = outs[key].astype(np.float64)
        err = np.maximum(np.abs(got - ref) - 1.0, 0.0) / np.maximum(ref, 1.0)
        assert np.max(err) < RTOL_COUNTS, (key, float(np.max(err)))
