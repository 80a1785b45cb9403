"""The launch-shape autotuner (ctfp_plan_autotune; no reference counterpart):
it picks a valid shape, leaves results unchanged, caches per process and in
the CTFP_TUNE_CACHE file."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest
import torch

from ct_forward_projection_b200 import Projector
from tests.conftest import random_volumes, small_geometry, spectral_setup

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def setup(pr, d, M, seed):
    S, mu, G, D = spectral_setup(d, M, 9, seed)
    pr.set_spectral_tables(S, mu, G, 2, D, 1000.0)
    return [torch.from_numpy(v).cuda() for v in random_volumes(d, M, seed)]


@pytest.mark.parametrize("mode", ["trilinear", "texemu", "texture"])
def test_autotune_picks_valid_shape_and_keeps_results(cuda_ok, mode):
    d = small_geometry(n=(40, 36, 30), views=24, U=70, V=44)
    with Projector(d, 2, mode) as pr:
        vols = setup(pr, d, 2, 4)
        before = pr.forward(vols)["I"].clone()
        r = pr.autotune(vols, n_sample_views=8)
        t = r["tile_u"] * r["tile_v"]
        assert t % 32 == 0 and 32 <= t <= 256 and 2 <= r["min_ctas_per_sm"] <= 4 and r["views_per_cta"] in (1, 2, 4)
        assert r["ms"] > 0 and r["from_cache"] == 0
        after = pr.forward(vols)["I"]
        torch.cuda.synchronize()
        err = torch.max(torch.abs(after - before) / before).item()
        assert err < 1e-6
        r2 = pr.autotune(vols, n_sample_views=8)
        assert r2["from_cache"] == 1
        assert {k: r2[k] for k in ("tile_u", "tile_v", "views_per_cta", "min_ctas_per_sm")} == \
            {k: r[k] for k in ("tile_u", "tile_v", "views_per_cta", "min_ctas_per_sm")}


CHILD = r'''
import json, sys
sys.path.insert(0, {root!r})
import torch
from ct_forward_projection_b200 import Projector
from tests.conftest import small_geometry
from tests.test_autotune_gpu import setup
d = small_geometry(n=20, views=8, U=32, V=16)
with Projector(d, 1, "trilinear") as pr:
    vols = setup(pr, d, 1, 2)
    print(json.dumps(pr.autotune(vols, n_sample_views=4)))
'''


def test_autotune_file_cache(cuda_ok, tmp_path):
    cache = str(tmp_path / "tune.txt")
    env = dict(os.environ, CTFP_TUNE_CACHE=cache)
    code = CHILD.format(root=ROOT)
    outs = []
    for _ in range(2):
        r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env, cwd=ROOT,
                           timeout=300)
        assert r.returncode == 0, r.stderr[-2000:]
        outs.append(json.loads(r.stdout.strip().splitlines()[-1]))
    assert outs[0]["from_cache"] == 0 and outs[1]["from_cache"] == 1
    assert outs[0]["tile_u"] == outs[1]["tile_u"] and outs[0]["tile_v"] == outs[1]["tile_v"]
    lines = open(cache).read().strip().splitlines()
    assert len(lines) == 1 and len(lines[0].split()) == 6
