"""Host logic of bench.py that needs no GPU: the clock sampler keeps only the
nvidia-smi samples taken inside the timed region and reads the throttle
reasons from them (a stand-in nvidia-smi on PATH prints the samples)."""
import os
import stat
import sys
import time

import bench
import numpy as np

FAKE = """#!{python}
import datetime, sys, time
reason = "{reason}"
while True:
    now = datetime.datetime.now()
    ts = now.strftime("%Y/%m/%d %H:%M:%S.") + "%03d" % (now.microsecond // 1000)
    print(ts + ", 0, {mhz}, 1965, 700.0, 0x0, Not Active, Not Active, Not Active, " + reason, flush=True)
    time.sleep(0.05)
"""


def fake_smi(tmp_path, monkeypatch, mhz, reason):
    p = tmp_path / "nvidia-smi"
    p.write_text(FAKE.format(python=sys.executable, mhz=mhz, reason=reason))
    p.chmod(p.stat().st_mode | stat.S_IEXEC)
    monkeypatch.setenv("PATH", str(tmp_path) + os.pathsep + os.environ["PATH"])


def test_clock_samples_inside_the_timed_region(tmp_path, monkeypatch):
    fake_smi(tmp_path, monkeypatch, 1965, "Active")
    c = bench.ClockSampler(0)
    c.start()
    time.sleep(0.3)  # samples before the timed region are left out
    c.begin()
    time.sleep(0.5)
    c.end()
    time.sleep(0.3)
    r = c.stop()
    assert r["window"] == "timed region"
    assert 4 <= r["samples"] <= 14
    assert r["sm_mhz"] == 1965.0 and r["sm_max_mhz"] == 1965.0
    assert r["reasons"] == ["sw_power_cap"]


def test_clock_sampler_without_a_window_keeps_every_sample(tmp_path, monkeypatch):
    fake_smi(tmp_path, monkeypatch, 1500, "Not Active")
    c = bench.ClockSampler(0)
    c.start()
    time.sleep(0.3)
    r = c.stop()
    assert r["window"].startswith("whole run")
    assert r["samples"] >= 1 and r["sm_mhz"] == 1500.0 and r["reasons"] == []


def test_reference_arm_other_ranks_exit_at_once():
    # under torchrun only rank 0 runs the reference arm; the others leave with
    # status 0 and print nothing, before any process group or GPU work
    import subprocess
    env = dict(os.environ, RANK="1", LOCAL_RANK="1", WORLD_SIZE="2", MASTER_ADDR="127.0.0.1", MASTER_PORT="29591")
    r = subprocess.run([sys.executable, os.path.join(os.path.dirname(bench.__file__), "bench.py"), "--impl",
                        "reference", "--gpus", "2"], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == ""


def test_reference_arm_finds_its_runner_in_a_fresh_process():
    # the reference arm imports oracle/ref_runner before anything else has
    # imported the oracle package
    import subprocess
    code = "import bench; r = bench._ref_runner(); assert r.REF_BIN.endswith('ctfp_ref')"
    r = subprocess.run([sys.executable, "-c", code], cwd=os.path.dirname(bench.__file__), capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]


def test_cpu_baseline_accuracy_figures():
    # the bench's accuracy block on a small problem whose "GPU" outputs are the
    # oracle's own, rounded to float32: per-ray errors at FP32 rounding, the
    # projection error likewise, and the sample sized from the time budget
    import types

    import numpy as np
    import torch

    from oracle import oracle as O
    from tests.conftest import random_volumes, small_geometry, spectral_setup
    d = small_geometry(n=(16, 16, 16), views=4, U=20, V=10)
    vols = random_volumes(d, 2, 3)
    S, mu, G, D = spectral_setup(d, 2, 6, 11)
    W = O.energy_weights(d, S, G, 2, D, 1000.0)
    n = 4 * 20 * 10
    w = types.SimpleNamespace(geometry=d, n_rays=n, _vols=[torch.from_numpy(v) for v in vols], _W=W,
                              mu_table=lambda: mu)
    ref = O.forward(d, vols, mu, W, O.TRILINEAR, np.arange(n))
    gpu = {"I": ref["I"].astype(np.float32), "IAbsorb": ref["IAbsorb"].astype(np.float32),
           "I0": ref["I0"].astype(np.float32)}
    cpu, acc = bench.cpu_baseline(w, gpu, 0.2)
    assert cpu["kind"] == "port" and cpu["value"] > 0 and cpu["cores"] >= 1
    for k in ("I", "IAbsorb", "I0"):
        assert acc[k]["max"] < 1e-7 and acc[k]["p99"] <= acc[k]["max"]
    assert acc["proj_abs"]["max"] < 1e-3
    assert acc["rays"] == n


def test_reference_arm_extrapolates_the_full_view_step(monkeypatch):
    # the reference arm's runs alternate between two view counts; a line
    # T(n) = F + n t through their wall times predicts the full-view step.
    # A stand-in for the reference binary takes F = 5 s + 0.25 s per view.
    import types

    from ct_forward_projection_b200 import physics
    from oracle import ref_runner
    calls = []

    def fake_run(case, timeout=600.0, keep_dir=None):
        n = case["geometry"]["projNum"]
        calls.append(n)
        return {}, 5.0 + 0.25 * n, ""

    monkeypatch.setattr(ref_runner, "run", fake_run)
    monkeypatch.setattr(ref_runner, "reference_case_from_workload",
                        lambda w, g: {"geometry": g, "spectrum": np.zeros(120)})
    w = physics.workload("poly_grid_256")
    args = types.SimpleNamespace(steps=4, warmup=2)
    line = ref_runner.bench_line(args, w)
    assert calls == [1, 1, 8, 24, 8, 24]
    split = line["reference_split"]
    assert abs(split["fixed_s"] - 5.0) < 1e-9 and abs(split["per_view_s"] - 0.25) < 1e-9
    assert abs(line["value"] - 360 * 512 * 384 / (5.0 + 0.25 * 360)) < 1e-3
    assert abs(line["ms_per_step"] - 1e3 * (5.0 + 0.25 * 16)) < 1e-6  # mean of the 8- and 24-view runs
    assert line["config"]["views"] == 360 and line["steps"] == 4 and line["warmup"] == 2
    assert line["e2e"]["value"] == line["value"] and line["cpu_baseline"]["kind"] == "reference"
