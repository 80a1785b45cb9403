#!/usr/bin/env python3
"""Benchmark: polyenergetic cone-beam forward projection on B200.

Workload (default): two-material polyenergetic projection with a focused
anti-scatter grid and scintillator response -- 256^3 soft-tissue + bone density
maps at 0.5 mm, 360 views, 512 x 384 detector at 0.8 mm, 120 kVp in 1-keV bins
20-120 keV (101 bins), SOD 1000 / SDD 1500 mm, grid 10:1 at 40 lines/cm with
per-pixel per-energy transmission.  A step is one full forward projection
(all 70.8 M rays).  Synthetic seeded phantom.

  value  rays/s with inputs resident in HBM (CUDA events, L2 flushed between steps)
  e2e    rays/s through ctfp_forward_host: host volumes in, host I/IAbsorb out
  roofline  the march kernel against its binding ceiling, the texture path's
            measured peak, with 32 B (8 FP32 corners) per voxel-sample of
            algorithmic traffic; the compulsory HBM bytes beside it
  cpu_baseline  the FP64 oracle on the host cores over a seeded ray subset

Multi-GPU (torchrun): by default every rank projects its own seeded object
(independent objects, weak scaling, no data-path collective); with --shard views
the ranks split one object's views (strong scaling; the adjoint sums the ranks'
partial gradients with an all-reduce).  Time is the max over ranks.
--impl reference runs the reference's own implementation of the path (see
reference_arm below).
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

HBM_FALLBACK_GBS = 6650.0
# DRAM bytes (read + write) per full forward launch, from one ncu capture
# (dram__bytes_read.sum + dram__bytes_write.sum) of k_forward on the 36-view
# case of the same problem (poly_grid_256_v36, default launch shape): 5.95 GB +
# 0.09 GB, scaled by 10 for 360 views (traffic grows with the views marched).
# DRAM bytes (read + write) of one forward launch over the 360-view workload:
# ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch on the 36-view
# case (every tenth view), x10.  An upper estimate: in the full run adjacent
# views are 1 degree apart and share more L2 lines than the 36-view case's.
TRAFFIC_PER_LAUNCH = {("poly_grid_256", "trilinear", "layered"): 60.37e9,
                      ("poly_grid_256", "trilinear", "axis"): 73.20e9}
BYTES_PER_VOXEL_SAMPLE = 32  # 8 FP32 corners, the reuse-free trilinear footprint


def measured_peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle sampling.  Started before the timed region
    (and waited on until its first sample lands), it keeps only the samples
    whose timestamps fall between begin() and end()."""

    FIELDS = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.path = os.path.join("/tmp", f"ctfp_clocks_{os.getpid()}.csv")
        self.t0 = self.t1 = None

    def start(self):
        if not shutil.which("nvidia-smi"):
            return
        self.f = open(self.path, "w")
        self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits", "-lms", "50"], stdout=self.f,
                                     stderr=subprocess.DEVNULL)
        deadline = time.time() + 3.0
        while time.time() < deadline and os.path.getsize(self.path) == 0:
            time.sleep(0.02)

    def begin(self):
        self.t0 = time.time()

    def end(self):
        self.t1 = time.time()

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        import datetime
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 10:
                continue
            try:
                ts = datetime.datetime.strptime(parts[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                rows.append((ts, float(parts[2]), float(parts[3]), parts[6:10]))
            except ValueError:
                continue
        os.unlink(self.path)
        inside = [r for r in rows if self.t0 is not None and self.t0 - 0.05 <= r[0] <= self.t1 + 0.05]
        window = "timed region"
        if not inside:
            inside, window = rows, "whole run (no sample inside the timed region)"
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = {n for r in inside for n, v in zip(names, r[3]) if v.lower() == "active"}
        sm = [r[1] for r in inside]
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(r[2] for r in inside) if inside else None,
                "reasons": sorted(reasons), "samples": len(sm), "window": window}


def dist_setup(n_gpus):
    import torch
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    else:
        if torch.cuda.is_available():
            torch.cuda.set_device(0)
    return ws, rank, local


def barrier_sync(ws):
    import torch
    torch.cuda.synchronize()
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()


def max_over_ranks(x: float, ws: int) -> float:
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def step_times(fn, n: int, ws: int, stream) -> tuple:
    """n back-to-back calls of fn on stream, an event recorded after each: the
    mean ms per call over the whole run and the per-call spread (min, median,
    max), each the max over ranks."""
    import torch
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(n + 1)]
    barrier_sync(ws)
    ev[0].record(stream)
    for k in range(n):
        fn()
        ev[k + 1].record(stream)
    barrier_sync(ws)
    per = sorted(ev[k].elapsed_time(ev[k + 1]) for k in range(n))
    mean = max_over_ranks(ev[0].elapsed_time(ev[n]) / n, ws)
    spread = {"min": max_over_ranks(per[0], ws), "median": max_over_ranks(per[n // 2], ws),
              "max": max_over_ranks(per[-1], ws), "steps": n}
    return mean, spread


def _err_stats(x: np.ndarray) -> dict:
    return {"max": float(np.max(x)), "p99": float(np.percentile(x, 99))}


def _ray_ids(rng, g, rows, n):
    """n distinct seeded ray ids (view, row, column) whose detector row is one
    of rows (every row when rows is None), sorted."""
    P, V, U = int(g["projNum"]), int(g["dNumV"]), int(g["dNumU"])
    rows = np.arange(V) if rows is None else np.asarray(rows)
    n_sel = P * len(rows) * U
    k = np.sort(rng.choice(n_sel, min(n, n_sel), replace=False))
    p, rem = np.divmod(k, len(rows) * U)
    r, u = np.divmod(rem, U)
    return np.sort((p * V + rows[r]) * U + u).astype(np.int64)


def cpu_baseline(w, gpu: dict, budget_s: float):
    """FP64 oracle over a seeded subset of rays on all host cores; also the
    error of the GPU result on those rays: per-ray relative error of I,
    IAbsorb and I0 (max and 99th percentile) and the absolute error of the
    compat projection log(I0 / floor(I)) (CBCTForwardProj.cpp:376-387).
    The rays lie on the detector rows whose oracle energy weights were built
    (w._rows, oracle_weights)."""
    from oracle import oracle as O
    g = w.geometry
    rows = getattr(w, "_rows", None)
    rng = np.random.RandomState(7)
    vols = [v.cpu().numpy() for v in w._vols]
    W = w._W
    mu = w.mu_table()
    # warm the thread pool, calibrate on a subset, then size the sample to the budget
    n0 = min(8192, w.n_rays)
    O.forward(g, vols, mu, W, O.TRILINEAR, _ray_ids(rng, g, rows, 512))
    ids = _ray_ids(rng, g, rows, n0)
    t0 = time.perf_counter()
    O.forward(g, vols, mu, W, O.TRILINEAR, ids)
    dt = time.perf_counter() - t0
    n = int(max(len(ids), len(ids) * budget_s / max(dt, 1e-6)))
    ids = _ray_ids(rng, g, rows, n)
    n = len(ids)
    t0 = time.perf_counter()
    ref = O.forward(g, vols, mu, W, O.TRILINEAR, ids)
    dt = time.perf_counter() - t0
    def rel(a, b):
        return np.abs(a - b) / np.maximum(np.abs(b), 1e-30)

    pix = ids % (g["dNumU"] * g["dNumV"])
    got = {k: gpu[k].reshape(-1)[pix if k == "I0" else ids].astype(np.float64) for k in ("I", "IAbsorb", "I0")}
    ref_I0 = ref["I0"].reshape(-1)[pix]
    acc = {k: _err_stats(rel(got[k], r)) for k, r in (("I", ref["I"]), ("IAbsorb", ref["IAbsorb"]), ("I0", ref_I0))}
    with np.errstate(divide="ignore"):
        proj_got = np.log(got["I0"] / np.floor(got["I"]))
        proj_ref = np.log(ref_I0 / np.floor(ref["I"]))
    acc["proj_abs"] = _err_stats(np.abs(proj_got - proj_ref))
    acc["proj_abs"]["note"] = "includes the floor to integer counts: I one count apart near an integer gives ~1/I"
    acc["rays"] = n
    acc["tables"] = getattr(w, "_tables", "as given")
    if rows is not None:
        acc["detector_rows"] = [int(r) for r in rows]
    where = "all detector rows" if rows is None else f"{len(rows)} seeded detector rows"
    cpu = {"value": n / dt, "unit": "rays/s", "cores": O.num_threads(), "kind": "port",
           "cpu_model": _cpu_model(),
           "sample": f"{n} seeded random rays (seed 7) on {where} of the full workload, FP64 oracle, {dt:.1f} s"}
    return cpu, acc


def _cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def _ref_runner():
    """oracle/ref_runner (the package module, whatever was imported before)."""
    from oracle import ref_runner
    return ref_runner


def reference_arm(args, w, ws, rank):
    """The reference's own implementation of the path.  Its projector is CUDA
    (Source/CUDAFun/CBCTPolyProjGPU.cu); oracle/build_ref.sh builds it from the
    reference sources into oracle/_ref/ctfp_ref.  When that binary is absent the
    oracle port on the host cores stands in."""
    if rank != 0:
        return None
    ref_bin = os.path.join(ROOT, "oracle", "_ref", "ctfp_ref")
    if os.path.exists(ref_bin):
        return _ref_runner().bench_line(args, w)
    from oracle import oracle as O
    g = w.geometry
    rng = np.random.RandomState(7)
    mu = w.mu_table()
    vals = []
    vols = [v.cpu().numpy() for v in w._vols]
    n = 4096
    for s in range(args.warmup + args.steps):
        ids = _ray_ids(rng, g, getattr(w, "_rows", None), n)
        t0 = time.perf_counter()
        O.forward(g, vols, mu, w._W, O.TRILINEAR, ids)
        dt = time.perf_counter() - t0
        if s >= args.warmup:
            vals.append(n / dt)
    v = statistics.mean(vals)
    return {"impl": "reference", "metric": "rays/s (forward projection)", "value": v, "unit": "rays/s",
            "n_gpus": 0, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "config": {"workload": w.name}, "dtype": "f64",
            "cpu_baseline": {"value": v, "unit": "rays/s", "cores": O.num_threads(), "kind": "port",
                             "sample": f"{n} seeded random rays per step"},
            "e2e": {"value": v, "unit": "rays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="poly_grid_256")
    ap.add_argument("--interp", default="trilinear", choices=["trilinear", "texemu", "texture"])
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--shard", default="objects", choices=["objects", "views"],
                    help="N > 1: each rank projects its own object (weak scaling) or a slab of one "
                         "object's views (strong scaling; the adjoint sums gradients with all-reduce)")
    ap.add_argument("--sampler", default="axis", choices=["axis", "layered", "global", "brick"],
                    help="where the software interp modes read corners")
    ap.add_argument("--batch-items", type=int, default=48,
                    help="problems in the uneven batch leg (0 skips it)")
    ap.add_argument("--no-batch-autotune", action="store_true",
                    help="batch leg with the default work units (no ctfp_batch_autotune)")
    ap.add_argument("--batch-passes", type=int, default=3,
                    help="timed passes per arm of the batch leg (after one warm-up pass; arms interleaved)")
    ap.add_argument("--launch-shape", default=None,
                    help="tile_u,tile_v,views_per_cta,min_ctas_per_sm for the march (instead of the autotuner)")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the other benchmark configurations (the `configs` block)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    import torch

    from ct_forward_projection_b200 import physics
    from ct_forward_projection_b200.projector import Projector

    if args.impl == "reference":
        # rank 0 alone runs the reference's implementation; under torchrun the
        # other ranks exit at once, and no process group is formed, so nothing
        # waits on a rank that has left
        ws = int(os.environ.get("WORLD_SIZE", "1"))
        rank = int(os.environ.get("RANK", "0"))
        local = int(os.environ.get("LOCAL_RANK", "0"))
        if rank != 0:
            return
        torch.cuda.set_device(local)
        w = physics.workload(args.workload)
        w._vols = physics.phantom(w, "cpu")
        if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "ctfp_ref")):
            # the oracle port stands in, with its own tables
            w._rows = oracle_rows(w)
            w._W, w._tables = oracle_weights(w, w._rows)
        line = reference_arm(args, w, ws, rank)
        if line is not None:
            print(json.dumps(line), flush=True)
        return

    ws, rank, local = dist_setup(args.gpus)
    w = physics.workload(args.workload)
    sharded = args.shard == "views" and ws > 1
    if not sharded:
        w.seed += rank  # each rank projects its own object
    dev = f"cuda:{local}"

    vols = physics.phantom(w, dev)
    M = len(vols)
    pr = Projector(w.geometry, M, args.interp, local)
    if args.interp != "texture":
        pr.set_sampler(args.sampler)
    pr.set_tables_from_workload(w)
    P, V, U = pr.shape_proj
    rays = P * U * V
    vr = None  # this rank's (first view, count) when one object's views are sharded
    if sharded:
        from ct_forward_projection_b200.shard import view_range
        vr = view_range(P, rank, ws)
        args.batch_items = 0
    n_local = vr[1] if sharded else P
    out = {"I": torch.empty((n_local, V, U), device=dev), "IAbsorb": torch.empty((n_local, V, U), device=dev)}
    stream = torch.cuda.current_stream()
    shape = {"tile_u": 16, "tile_v": 8, "views_per_cta": 2, "min_ctas_per_sm": 4, "source": "default"}
    if args.launch_shape:
        tu, tv, vpc, mc = (int(x) for x in args.launch_shape.split(","))
        pr.set_launch_shape(tu, tv, vpc, mc)
        shape = {"tile_u": tu, "tile_v": tv, "views_per_cta": vpc, "min_ctas_per_sm": mc, "source": "--launch-shape"}
    elif not args.no_autotune:
        # candidates timed on every view of the step (four launches of a
        # quarter of the views each): shorter samples end in a partial wave of
        # CTAs that weighs more for CTAs of more views, and picked 1 view per
        # CTA where 2 run the full step 2.7 % faster
        r = pr.autotune(vols, n_sample_views=n_local)
        shape = {k: r[k] for k in ("tile_u", "tile_v", "views_per_cta", "min_ctas_per_sm")}
        shape["source"] = "cache" if r["from_cache"] else "autotuned"
        shape["sample_views"] = n_local
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # 256 MB > 126 MB L2

    # ---------------- device-resident forward (value) -----------------------
    for _ in range(args.warmup):
        pr.forward(vols, out=out, views=vr)
    barrier_sync(ws)
    clocks = ClockSampler(local)
    clocks.start()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    barrier_sync(ws)
    clocks.begin()
    for s in range(args.steps):
        flush.fill_(float(s))
        ev[s][0].record(stream)
        pr.forward(vols, out=out, views=vr)
        ev[s][1].record(stream)
    barrier_sync(ws)
    clocks.end()
    clk = clocks.stop()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    ms = max_over_ranks(statistics.mean(step_ms), ws)
    total_rays = rays if sharded else ws * rays
    value = total_rays / (ms / 1e3)

    # ---------------- optional empty-space skipping (not the headline) -------
    skip = None
    if args.interp == "texture" or args.sampler in ("layered", "axis"):
        ref_I = out["I"].clone()
        pr.set_skip_empty(True)
        o2 = {"I": torch.empty_like(out["I"]), "IAbsorb": torch.empty_like(out["IAbsorb"])}
        for _ in range(2):
            pr.forward(vols, out=o2, views=vr)
        barrier_sync(ws)
        sk = []
        for s_ in range(args.steps):
            flush.fill_(float(s_))
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            pr.forward(vols, out=o2, views=vr)
            e1.record(stream)
            sk.append((e0, e1))
        barrier_sync(ws)
        pr.set_skip_empty(False)
        sk_ms = max_over_ranks(statistics.mean([a.elapsed_time(b) for a, b in sk]), ws)
        diff = float(torch.max(torch.abs(o2["I"] - ref_I) / ref_I.abs().clamp_min(1e-30)))
        skip = {"ms_per_step": sk_ms, "value": total_rays / (sk_ms / 1e3), "unit": "rays/s", "speedup": ms / sk_ms,
                "max_rel_diff_vs_full_march": diff,
                "note": "ctfp_plan_set_skip_empty: footprints in all-zero 8^3 bricks are not fetched; "
                        "occupancy rebuilt inside every timed step"}
        del o2, ref_I

    # roofline of the dominant kernel (the march): its algorithmic bytes are
    # the 8 FP32 corners of every voxel-sample (32 B, reuse-free), which the
    # texture path returns to registers; the binding ceiling is that path's
    # rate for the march's own gathers, measured in this run (texture_roof).
    # DRAM sees far fewer bytes (the texture cache serves neighbouring rays'
    # shared corners): the compulsory HBM bytes (volumes once, outputs once)
    # are reported beside it against the measured copy bandwidth.
    support = pr.count_support_samples()
    vs_launch = support * M * n_local // P  # sharded: this rank's share of the views, pro rata
    nominal_vs = M * rays * int(pr.info["intNum"])
    hbm_peak, peak_kind = measured_peak_hbm()
    vs_rate = vs_launch / (ms / 1e3)
    achieved = vs_rate * BYTES_PER_VOXEL_SAMPLE / 1e9
    tex_peak, tex_src = texture_roof(pr, args.interp, args.sampler, local, {})
    traffic = TRAFFIC_PER_LAUNCH.get((w.name, args.interp, args.sampler if args.interp != "texture" else "tex3d"))
    nvox = int(np.prod(pr.shape_vol))
    compulsory = M * nvox * 4 + n_local * U * V * 8
    roofline = {"bound": "texture" if tex_peak else "hbm",
                "achieved": achieved, "unit": "GB/s",
                "peak": (tex_peak * BYTES_PER_VOXEL_SAMPLE / 1e9) if tex_peak else hbm_peak,
                "frac": (vs_rate / tex_peak) if tex_peak else achieved / hbm_peak,
                "peak_source": (tex_src + " x 32 B") if tex_peak else f"{peak_kind} HBM copy bandwidth",
                "traffic": traffic,
                "traffic_source": None if traffic is None else
                    "not measured in this run: ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch on "
                    "the 36-view case of this workload (every tenth view), x10 for 360 views (the committed ncu "
                    "summary of this kernel); an upper estimate, adjacent views sharing more L2 lines in the full run",
                "voxel_samples_per_launch": vs_launch, "voxel_samples_per_s": vs_rate,
                "nominal_voxel_samples_per_launch": nominal_vs,
                "hbm": {"compulsory_bytes_per_launch": compulsory,
                        "achieved_GBs": compulsory / (ms / 1e3) / 1e9, "peak_GBs": hbm_peak,
                        "frac": compulsory / (ms / 1e3) / 1e9 / hbm_peak, "peak_source": peak_kind,
                        "note": "volumes read once + I and IAbsorb written once, against the HBM copy peak"},
                "note": "achieved = 32 B (the 8 FP32 corners a trilinear sample reads, reuse-free) x support "
                        "voxel-samples / kernel time; peak = the texture path's measured rate for the same "
                        "gathers x 32 B"}

    # ---------------- end to end through ctfp_forward_host (e2e) ------------
    e2e = None
    if not args.no_e2e and not sharded:
        host_vols = [v.cpu().pin_memory() for v in vols]
        host_out = {"I": torch.empty((P, V, U)).pin_memory(), "IAbsorb": torch.empty((P, V, U)).pin_memory(),
                    "I0": torch.empty((V, U)).pin_memory()}
        for _ in range(2):
            pr.forward_host(host_vols, out=host_out)
        barrier_sync(ws)
        t_e2e = []
        for s in range(args.steps):
            t0 = time.perf_counter()
            pr.forward_host(host_vols, out=host_out)
            t_e2e.append(time.perf_counter() - t0)
        barrier_sync(ws)
        e2e_s = max_over_ranks(statistics.mean(t_e2e), ws)
        h2d = sum(v.numel() * 4 for v in host_vols)
        d2h = 2 * rays * 4 + U * V * 4
        e2e = {"value": ws * rays / e2e_s, "unit": "rays/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
               "s_per_step": e2e_s}

    # ---------------- forward + adjoint (extra) -----------------------------
    # loss = sum (log I - log T)^2 against the projection T of the same phantom
    # with every density scaled by 0.97 (made once, untimed); a step is the
    # forward with checkpoint, dLoss/dI in torch, the adjoint and the fold
    fa = None
    if not args.no_adjoint:
        L = torch.empty((n_local, V, U, M), device=dev)
        T = pr.forward([v * 0.97 for v in vols], views=vr)["I"]
        logT = torch.log(T)
        grads = [torch.zeros_like(v) for v in vols]
        loss = torch.zeros((), device=dev)
        sp = None
        if sharded:
            from ct_forward_projection_b200.shard import ViewShardedProjector
            sp = ViewShardedProjector(pr)

        def fa_step():
            pr.forward(vols, out={**out, "L": L}, views=vr)
            r = torch.log(out["I"]) - logT
            loss.copy_(torch.sum(r * r))
            if sp is None:
                pr.backward(L, 2.0 * r / out["I"], None, grads)
            else:
                sp.backward(L, gI=2.0 * r / out["I"], grads=grads)  # partial adjoint + all-reduce

        for _ in range(2):
            fa_step()
        n_fa = max(1, min(args.steps, 10))
        fa_ms, fa_spread = step_times(fa_step, n_fa, ws, stream)
        fa = {"value": total_rays / (fa_ms / 1e3), "unit": "rays/s", "ms_per_step": fa_ms, "step_ms": fa_spread,
              "loss": "sum (log I - log T)^2, T = projection of the phantom x 0.97", "last_loss": float(loss)}
        fa["fused"] = None if sharded else fused_fwd_adjoint(pr, vols, T, fa_step, grads, loss, n_fa, total_rays,
                                                             fa_ms, ws, stream)
        del L, logT, T

    # ---------------- uneven batch: batched vs loop of plain calls ----------
    batch = None
    if args.batch_items > 0:
        batch = batch_leg(args, ws, rank, local, stream)

    # ---------------- the other configurations (rank 0, N = 1) -------------
    configs = None
    if rank == 0 and ws == 1 and not args.no_configs and not sharded:
        configs = config_legs(args, local, stream, flush)

    # ---------------- CPU baseline (rank 0, N = 1) --------------------------
    cpu = None
    err = acc = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        w._vols = vols
        w._rows = oracle_rows(w)
        w._W, w._tables = oracle_weights(w, w._rows)
        gpu = {k: out[k].cpu().numpy() for k in ("I", "IAbsorb")}
        gpu["I0"] = pr.forward(vols, views=(0, 1))["I0"].cpu().numpy()  # view-independent; not in the timed step
        cpu, acc = cpu_baseline(w, gpu, args.cpu_budget)
        err = acc["I"]["max"]

    if rank == 0:
        line = {
            "metric": "rays/s (polyenergetic cone-beam forward projection)",
            "value": value, "unit": "rays/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms, "higher_is_better": True, "scaling": "strong" if sharded else "weak",
            "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded phantom per rank)",
            "config": {"workload": w.name, "interp": args.interp,
                       "sampler": args.sampler if args.interp != "texture" else "tex3d",
                       "volume": list(pr.shape_vol[::-1]), "materials": M,
                       "views": P, "detector": [U, V], "energies": pr.E, "samples_per_ray": int(pr.info["intNum"]),
                       "rays_per_step": rays, "l2": "flushed (256 MB write) between timed steps",
                       "parallelism": (f"one object, views sharded x{ws} (adjoint: all-reduce of gradients)"
                                       if sharded else f"independent objects x{ws}")},
            "e2e": e2e,
            "roofline": roofline,
            "cpu_baseline": cpu,
            "max_rel_err_vs_fp64_oracle": err,
            "accuracy_vs_fp64_oracle": acc,
            "fwd_adjoint": fa,
            "fwd_skip_empty": skip,
            "batch": batch,
            "configs": configs,
            "launch_shape": shape,
            "gpu_launches": args.steps,
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    pr.close()
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


# The other benchmark configurations, each timed like the headline (CUDA
# events on the launching stream, L2 flushed between steps) and checked
# against the FP64 oracle on seeded rays: (workload, interp, timed steps,
# forward + adjoint too).  poly_grid_256 in the two modes that reproduce the
# reference's texture sampler; the single-material 128^3 case; the
# differentiable three-material case; the large four-material case.
CONFIG_LEGS = [("sinmat_nogrid_128", "trilinear", 5, False),
               ("poly_grid_256", "texemu", 3, False),
               ("poly_grid_256", "texture", 3, False),
               ("diff_3mat_256", "trilinear", 3, True),
               ("large_4mat_512", "trilinear", 2, True)]


def texture_roof(pr, interp, sampler, local, cache):
    """The march's binding ceiling in voxel-samples/s, measured in this run,
    and how it was measured.  Layered sampler: ctfp_sampler_peak (two 4-texel
    gathers per voxel-sample from an L1-resident texture, full warps, full
    occupancy).  Axis sampler: the same lane-gather rate divided by the
    gathers its march issues per voxel-sample on this geometry, counted by
    active lane quads (ctfp_axis_gather_count; 0.5 = the layered sampler's
    two full-warp gathers).  Hardware texture: one filtered tex3D fetch per
    voxel-sample (ctfp_sampler_peak tex3d).  cache holds the probe results."""
    from ct_forward_projection_b200.projector import sampler_peak
    kind = "tex3d" if interp == "texture" else ("layered" if sampler in ("layered", "axis") else None)
    if kind is None:
        return None, None
    if kind not in cache:
        cache[kind] = sampler_peak(local, kind)
    peak = cache[kind]
    if interp != "texture" and sampler == "axis":
        g = pr.axis_gather_count()
        return peak * 0.5 / g, (f"measured in this run: ctfp_sampler_peak (layered, {peak:.3e}/s at 0.5 quad-gathers "
                                f"per voxel-sample) x 0.5 / {g:.4f} quad-gathers per voxel-sample of this march "
                                f"(ctfp_axis_gather_count)")
    return peak, f"measured in this run: ctfp_sampler_peak ({kind})"


def _accuracy(w, pr, vols, out, interp, n_rays=100000):
    """Per-ray relative error of I and IAbsorb against the FP64 oracle on
    seeded rays of the oracle's detector rows (max, p99): trilinear against the
    exact oracle; the texture-unit modes against its texture emulation."""
    from oracle import oracle as O
    g = w.geometry
    rows = oracle_rows(w)
    W, tables = oracle_weights(w, rows)
    rng = np.random.RandomState(17)
    ids = _ray_ids(rng, g, rows, n_rays)
    mode = O.TRILINEAR if interp == "trilinear" else O.TEXEMU
    ref = O.forward(g, [v.cpu().numpy() for v in vols], w.mu_table(), W, mode, ids)
    import torch
    idx = torch.from_numpy(ids).to(out["I"].device)
    acc = {}
    for k, r in (("I", ref["I"]), ("IAbsorb", ref["IAbsorb"])):
        got = out[k].reshape(-1)[idx].double().cpu().numpy()
        acc[k] = _err_stats(np.abs(got - r) / np.maximum(np.abs(r), 1e-30))
    acc["rays"] = int(len(ids))
    acc["against"] = "FP64 oracle, " + ("exact trilinear" if mode == O.TRILINEAR else "texture-unit emulation")
    acc["tables"] = tables
    return acc


def config_legs(args, local, stream, flush):
    import torch

    from ct_forward_projection_b200 import physics
    from ct_forward_projection_b200.projector import Projector
    dev = f"cuda:{local}"
    res = {}
    peaks = {}
    for name, interp, steps, adjoint in CONFIG_LEGS:
        key = f"{name}/{interp}"
        try:
            w = physics.workload(name)
            vols = physics.phantom(w, dev)
            M = len(vols)
            pr = Projector(w.geometry, M, interp, local)
            if interp != "texture":
                pr.set_sampler(args.sampler)
            pr.set_tables_from_workload(w)
            P, V, U = pr.shape_proj
            rays = P * U * V
            out = {"I": torch.empty((P, V, U), device=dev), "IAbsorb": torch.empty((P, V, U), device=dev)}
            pr.forward(vols, out=out)
            ev = []
            for s_ in range(steps):
                flush.fill_(float(s_))
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                pr.forward(vols, out=out)
                e1.record(stream)
                ev.append((e0, e1))
            torch.cuda.synchronize()
            ms = statistics.mean(a.elapsed_time(b) for a, b in ev)
            vs = pr.count_support_samples() * M
            r = {"ms_per_forward": ms, "rays_per_s": rays / (ms / 1e3), "voxel_samples_per_s": vs / (ms / 1e3),
                 "rays": rays, "voxel_samples": vs, "steps": steps,
                 "volume": list(pr.shape_vol[::-1]), "materials": M, "views": P, "detector": [U, V], "energies": pr.E,
                 "sampler": "tex3d" if interp == "texture" else args.sampler}
            tpeak, tsrc = texture_roof(pr, interp, args.sampler, local, peaks)
            if tpeak:
                r["texture_frac"] = r["voxel_samples_per_s"] / tpeak
                r["texture_peak_voxel_samples_per_s"] = tpeak
                r["texture_peak_source"] = tsrc
            if adjoint:
                L = torch.empty((P, V, U, M), device=dev)
                T = pr.forward([v * 0.97 for v in vols])["I"]
                logT = torch.log(T)
                del T
                grads = [torch.zeros_like(v) for v in vols]

                def fa_step():
                    pr.forward(vols, out={**out, "L": L})
                    rr = torch.log(out["I"]) - logT
                    pr.backward(L, 2.0 * rr / out["I"], None, grads)

                fa_step()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                for _ in range(steps):
                    fa_step()
                e1.record(stream)
                torch.cuda.synchronize()
                fa_ms = e0.elapsed_time(e1) / steps
                r["fwd_adjoint"] = {"ms_per_step": fa_ms, "rays_per_s": rays / (fa_ms / 1e3),
                                    "step": "forward with checkpoint, dLoss/dI of sum (log I - log T)^2 in torch, "
                                            "adjoint and fold; T = projection of the phantom x 0.97"}
                del L, logT, grads
            if not args.no_cpu:
                r["accuracy_vs_fp64_oracle"] = _accuracy(w, pr, vols, out, interp)
            pr.close()
            del vols, out
            torch.cuda.empty_cache()
            res[key] = r
        except Exception as e:  # a failed leg is reported, the bench line still prints
            res[key] = {"error": f"{type(e).__name__}: {e}"}
            torch.cuda.empty_cache()
    return res


def fused_fwd_adjoint(pr, vols, T, fa_step, grads, loss, n_fa, total_rays, fa_ms, ws, stream):
    """The same forward + loss + adjoint step as one persistent kernel
    (ctfp_batch_forward_adjoint on a one-item batch: no L checkpoint, no
    separate dLoss/dI and backward launches), timed like the unfused step; then
    one step of each into zeroed gradients to compare them."""
    import torch

    from ct_forward_projection_b200._capi import CtfpError
    from ct_forward_projection_b200.projector import Batch
    try:
        b1 = Batch([pr])
    except CtfpError as e:
        return {"unsupported": str(e)}
    g_f = [torch.zeros_like(v) for v in vols]
    loss_f = torch.zeros(1, device=vols[0].device)
    I_f = torch.empty_like(T)

    def step():
        loss_f.zero_()
        b1.forward_adjoint([vols], [T], grads=[g_f], I_out=[I_f], loss=loss_f)

    for _ in range(2):
        step()
    ms, spread = step_times(step, n_fa, ws, stream)
    for x in g_f + grads:
        x.zero_()
    step()
    fa_step()
    torch.cuda.synchronize()
    gdiff = max(float(torch.max(torch.abs(a - c)) / torch.max(torch.abs(c)).clamp_min(1e-30))
                for a, c in zip(g_f, grads))
    ldiff = abs(float(loss_f[0]) - float(loss)) / max(abs(float(loss)), 1e-30)
    b1.close()
    return {"value": total_rays / (ms / 1e3), "unit": "rays/s", "ms_per_step": ms, "step_ms": spread,
            "speedup_vs_unfused": fa_ms / ms,
            "max_rel_diff_grad_vs_unfused": gdiff, "rel_diff_loss_vs_unfused": ldiff,
            "note": "ctfp_batch_forward_adjoint on a one-item batch: forward, loss and adjoint in one "
                    "persistent kernel replayed as a CUDA graph, then the fold"}


def batch_leg(args, ws, rank, local, stream):
    """The uneven batch (physics.batch_workloads): every problem forward, and
    forward + loss sum (log I - log T)^2 + adjoint, as one graph-replayed
    persistent launch (ctfp_batch_*) against a loop of plain calls (ctfp_forward,
    dLoss/dI in torch, ctfp_backward) over the same problems.  One untimed
    warm-up (records the graphs) and one timed pass per arm; L2 is irrelevant
    at these sizes (tens of GB per pass)."""
    import torch

    from ct_forward_projection_b200 import physics
    from ct_forward_projection_b200.projector import Batch, Projector
    dev = f"cuda:{local}"
    wl = physics.batch_workloads(args.batch_items, seed=4000 + 97 * rank)
    prs, vols, outs, Ls, targets, grads_loop, grads_b = [], [], [], [], [], [], []
    rays = 0
    for w in wl:
        pr = Projector(w.geometry, len(w.materials), "trilinear", local)
        pr.set_tables_from_workload(w)
        v = physics.phantom(w, dev)
        P, V, U = pr.shape_proj
        prs.append(pr)
        vols.append(v)
        outs.append({"I": torch.empty((P, V, U), device=dev), "IAbsorb": torch.empty((P, V, U), device=dev)})
        Ls.append(torch.empty((P, V, U, pr.M), device=dev))
        grads_loop.append([torch.zeros_like(x) for x in v])
        grads_b.append([torch.zeros_like(x) for x in v])
        rays += P * V * U
    # targets: the plain forward of each problem, perturbed multiplicatively
    gen = torch.Generator(device=dev)
    gen.manual_seed(11 + rank)
    for pr, v, o in zip(prs, vols, outs):
        pr.forward(v, out=o)
        targets.append(o["I"] * torch.exp(0.05 * torch.randn(o["I"].shape, device=dev, generator=gen)))
    b = Batch(prs)
    # the work units, tuned for each kind of call (untimed)
    if args.no_batch_autotune:
        sh = b.shapes()
        unit_shape = {"tile_u": sh["fwd_adjoint"][0], "tile_v": sh["fwd_adjoint"][1], "views": sh["views"][1],
                      "fwd_tile_u": sh["fwd"][0], "fwd_tile_v": sh["fwd"][1], "fwd_views": sh["views"][0]}
    else:
        unit_shape = b.autotune(vols, targets)
    b_outs = [{"I": torch.empty_like(o["I"]), "IAbsorb": torch.empty_like(o["I"])} for o in outs]
    b_I = [torch.empty_like(o["I"]) for o in outs]
    loss_b = torch.zeros(len(prs), device=dev)

    def loop_fwd():
        for pr, v, o in zip(prs, vols, outs):
            pr.forward(v, out=o)

    def loop_fwd_adj():
        for pr, v, o, L, T, g in zip(prs, vols, outs, Ls, targets, grads_loop):
            pr.forward(v, out={**o, "L": L})
            gI = 2.0 * (torch.log(o["I"]) - torch.log(T)) / o["I"]
            pr.backward(L, gI=gI, grads=g)

    def batched_fwd():
        b.forward(vols, out=b_outs)

    def batched_fwd_adj():
        b.forward_adjoint(vols, targets, grads=grads_b, I_out=b_I, loss=loss_b)

    def one_pass(fn):
        barrier_sync(ws)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        barrier_sync(ws)
        return max_over_ranks(e0.elapsed_time(e1), ws)

    def timed_pair(loop_fn, batch_fn):
        # one warm-up pass each (records the batch's graph), then the timed
        # passes with the arms interleaved; per arm the median pass and the
        # spread
        loop_fn()
        batch_fn()
        tl, tb = [], []
        for _ in range(max(1, args.batch_passes)):
            tl.append(one_pass(loop_fn))
            tb.append(one_pass(batch_fn))
        tl.sort()
        tb.sort()
        return tl, tb

    def arm(t_loop, t_b):
        ml, mb = t_loop[len(t_loop) // 2], t_b[len(t_b) // 2]
        return {"loop_rays_s": n_rays / (ml / 1e3), "batched_rays_s": n_rays / (mb / 1e3),
                "loop_ms": ml, "batched_ms": mb, "speedup": ml / mb,
                "loop_ms_min_max": [t_loop[0], t_loop[-1]], "batched_ms_min_max": [t_b[0], t_b[-1]],
                "speedup_min_max": [t_loop[0] / t_b[-1], t_loop[-1] / t_b[0]], "passes": len(t_loop)}

    n_rays = ws * rays
    t_loop_f, t_b_f = timed_pair(loop_fwd, batched_fwd)
    for g in grads_loop + grads_b:
        for x in g:
            x.zero_()
    t_loop_fa, t_b_fa = timed_pair(loop_fwd_adj, batched_fwd_adj)
    torch.cuda.synchronize()
    # both arms ran the same number of passes into their gradients
    gerr = max(float(torch.max(torch.abs(a - c)) / torch.max(torch.abs(c)).clamp_min(1e-30))
               for ga, gc in zip(grads_b, grads_loop) for a, c in zip(ga, gc))
    ierr = max(float(torch.max(torch.abs(a["I"] - c["I"]) / c["I"].abs().clamp_min(1e-30)))
               for a, c in zip(b_outs, outs))
    # the batched forward against the FP64 oracle on seeded rays of three problems
    oerr = None
    if rank == 0 and not args.no_cpu:
        from oracle import oracle as O
        oerr = 0.0
        rng = np.random.RandomState(3)
        for k in (0, len(wl) // 2, len(wl) - 1):
            w = wl[k]
            rows = oracle_rows(w, 4)
            W, _ = oracle_weights(w, rows)
            ids = _ray_ids(rng, w.geometry, rows, 1024)
            ref = O.forward(w.geometry, [x.cpu().numpy() for x in vols[k]], w.mu_table(), W, O.TRILINEAR, ids)
            got = b_outs[k]["I"].reshape(-1)[torch.from_numpy(ids).to(dev)].double().cpu().numpy()
            oerr = max(oerr, float(np.max(np.abs(got - ref["I"]) / np.abs(ref["I"]))))
    info = b.info()
    b.close()
    for pr in prs:
        pr.close()
    return {
        "items": len(wl), "rays_per_pass": rays, "work_units": info["units"],
        "persistent_grid": [info["grid_forward"], info["grid_adjoint"]],
        "unit_tile": {"fwd": [unit_shape["fwd_tile_u"], unit_shape["fwd_tile_v"]],
                      "fwd_adjoint": [unit_shape["tile_u"], unit_shape["tile_v"]]},
        "unit_views": {"fwd": unit_shape["fwd_views"], "fwd_adjoint": unit_shape["views"]},
        "fwd": arm(t_loop_f, t_b_f),
        "fwd_adjoint": arm(t_loop_fa, t_b_fa),
        "max_rel_diff_I_batched_vs_loop": ierr, "max_rel_diff_grad_batched_vs_loop": gerr,
        "max_rel_err_batched_I_vs_fp64_oracle": oerr,
        "note": "one warm-up pass per arm, then the timed passes with the arms interleaved; ms and speedup "
                "from the median pass; loop = ctfp_forward + torch dLoss/dI + ctfp_backward per problem",
    }


def oracle_rows(w, n_rows: int = 16, seed: int = 5):
    """The detector rows on which the oracle checks a workload with a per-pixel
    grid table: the outermost, the two central and n_rows - 4 seeded rows
    (None, meaning every row, for tables without a per-row dependence)."""
    V = int(w.geometry["dNumV"])
    if w.grid is None or w.grid_layout != 2 or V <= n_rows:
        return None
    rng = np.random.RandomState(seed)
    rows = {0, V - 1, V // 2 - 1, V // 2}
    while len(rows) < n_rows:
        rows.add(int(rng.randint(0, V)))
    return np.array(sorted(rows), np.int64)


def oracle_weights(w, rows=None):
    """Energy weights W[e][v][u] = I0Val * S_e * G_e * D_e in FP64 for the
    oracle, built from the oracle's own tables and nothing of the library:
    the grid by orc_grid_column (column layout) or orc_grid_pixel (per-pixel
    incidence-angle layout, on the rows listed; other rows hold NaN so that a
    ray there cannot pass unnoticed), the scintillator response by
    orc_scint_thickness and orc_det_response.  Returns (W, description)."""
    from oracle import oracle as O
    g = w.geometry
    U, V = int(g["dNumU"]), int(g["dNumV"])
    E = len(w.energies)
    W = np.full((E, V, U), w.I0Val, np.float64) * w.spectrum().astype(np.float64)[:, None, None]
    built = ["spectrum"]
    sel = np.arange(V) if rows is None else np.asarray(rows)
    if w.grid is not None:
        ms, mi = w.grid_mu()
        gs = w.grid
        if w.grid_layout == 2:
            G = O.grid_pixel(U, V, float(g["dSize"]), gs.strip_um, gs.inter_um, gs.h_mm, gs.FD_mm, ms, mi, sel)
            built.append(f"grid orc_grid_pixel ({len(sel)} rows)")
        else:
            col = np.stack([O.grid_column(U, float(g["dSize"]), gs.strip_um, gs.inter_um, gs.h_mm, gs.FD_mm,
                                          float(ms[e]), float(mi[e])) for e in range(E)]).astype(np.float64)
            G = np.repeat(col[:, None, :], len(sel), axis=1)
            built.append("grid orc_grid_column")
        W[:, sel, :] *= G
    if w.scint_mm is not None:
        t = O.scint_thickness(U * V, w.scint_mm, w.scint_err_mm)
        D = O.det_response(w.scint_mu(), t, 1.0).reshape(E, V, U).astype(np.float64)
        W *= D
        built.append("scintillator orc_scint_thickness + orc_det_response")
    if rows is not None:
        keep = np.zeros(V, bool)
        keep[sel] = True
        W[:, ~keep, :] = np.nan
    return W, "oracle: " + ", ".join(built)


if __name__ == "__main__":
    main()
