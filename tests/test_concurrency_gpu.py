"""Threading contract of the C ABI: one plan per thread, plans on different
streams run concurrently, and the library keeps no process-global state that
one plan's calls could disturb.  The last-error message is per thread.  (The
reference is single-threaded and keeps its textures in file-scope globals,
Source/CUDAFun/CBCTPolyProjGPU.cu:8-10.)

Four threads, each with its own plan (geometry, material count, sampler) and
its own CUDA stream, run forward + backward repeatedly at the same time;
every iteration must equal the same plan run alone: I, IAbsorb and the L
checkpoint bit for bit (the forward has no reductions across threads), the
gradients to float rounding (their order of atomic additions varies).  A
fifth thread creates invalid plans meanwhile and must see its own error
message every time."""
import threading

import pytest
import torch

from ct_forward_projection_b200 import Projector
from ct_forward_projection_b200._capi import CtfpError, CTFP_INVALID_ARG
from tests.conftest import random_volumes, small_geometry, spectral_setup

pytestmark = pytest.mark.gpu

PLANS = [
    dict(n=(22, 20, 16), views=7, U=26, V=14, M=2, E=9, mode="trilinear", sampler="layered", seed=31),
    dict(n=(16, 16, 16), views=5, U=17, V=11, M=1, E=6, mode="texemu", sampler="brick", seed=32),
    dict(n=(20, 18, 12), views=6, U=21, V=13, M=3, E=7, mode="trilinear", sampler="brick", seed=33),
    dict(n=(18, 18, 18), views=4, U=19, V=15, M=2, E=8, mode="texture", sampler=None, seed=34),
]
ITERS = 6


def make(sp):
    d = small_geometry(n=sp["n"], views=sp["views"], U=sp["U"], V=sp["V"])
    vols = [torch.from_numpy(v).cuda() for v in random_volumes(d, sp["M"], sp["seed"])]
    S, mu, G, D = spectral_setup(d, sp["M"], sp["E"], sp["seed"] + 100)
    pr = Projector(d, sp["M"], sp["mode"])
    if sp["sampler"]:
        pr.set_sampler(sp["sampler"])
    pr.set_spectral_tables(S, mu, G, 2, D, 1000.0)
    return pr, vols


def run_once(pr, vols, stream):
    with torch.cuda.stream(stream):
        out = pr.forward(vols, want_L=True, stream=stream)
        gI = torch.rsqrt(out["I"] + 1.0)
        grads = pr.backward(out["L"], gI=gI, stream=stream)
    stream.synchronize()
    return {k: out[k].clone() for k in ("I", "IAbsorb", "L")}, [g.clone() for g in grads]


def test_plans_on_threads_and_streams(cuda_ok):
    plans = [make(sp) for sp in PLANS]
    torch.cuda.synchronize()
    alone = [run_once(pr, vols, torch.cuda.Stream()) for pr, vols in plans]

    results = [[] for _ in plans]
    errors = []
    bad_msgs = []
    start = threading.Barrier(len(plans) + 1)

    def worker(k):
        try:
            torch.cuda.set_device(0)
            st = torch.cuda.Stream()
            pr, vols = plans[k]
            start.wait()
            for _ in range(ITERS):
                results[k].append(run_once(pr, vols, st))
        except Exception as e:  # reported below
            errors.append((k, repr(e)))

    def bad_plans():
        try:
            torch.cuda.set_device(0)
            d = small_geometry()
            d["sdd"] = d["sod"] * 0.5
            start.wait()
            for _ in range(40):
                try:
                    Projector(d, 1, "trilinear")
                    bad_msgs.append("created")
                except CtfpError as e:
                    if e.status != CTFP_INVALID_ARG or "need 0 < sod < sdd" not in str(e):
                        bad_msgs.append(str(e))
        except Exception as e:
            errors.append(("bad", repr(e)))

    threads = [threading.Thread(target=worker, args=(k,)) for k in range(len(plans))]
    threads.append(threading.Thread(target=bad_plans))
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=300)
    assert not any(t.is_alive() for t in threads)
    assert not errors, errors
    assert not bad_msgs, bad_msgs

    for k, (ref_out, ref_g) in enumerate(alone):
        assert len(results[k]) == ITERS
        for out, g in results[k]:
            for key in ("I", "IAbsorb", "L"):
                assert torch.equal(out[key], ref_out[key]), (k, key)
            for a, b in zip(g, ref_g):
                scale = float(b.abs().max())
                assert float((a - b).abs().max()) <= 1e-5 * scale, k
    for pr, _ in plans:
        pr.close()
