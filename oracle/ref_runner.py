"""Runs the reference's own projector (oracle/_ref/ctfp_ref, built from the
reference sources by oracle/build_ref.sh) on inputs written in its formats.

TEST INFRASTRUCTURE ONLY: used to make the golden fixtures under tests/golden/
and as the reference arm of bench.py.  The reference reads Config/ScanSetting.ini
and Config/OutputFolder.ini relative to its working directory
(ForwardProjection.cpp:201, 376), tables with one value per line where line e
holds energy e+1 keV, and a uint8 label volume; it writes raw little-endian
outputs (CBCTPolyForwardProjGrid.cpp:310-418, CBCTForwardProj.cpp:261-296).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_BIN = os.path.join(HERE, "_ref", "ctfp_ref")


def _write_table(path, values):
    with open(path, "w") as f:
        for v in np.asarray(values, dtype=np.float64):
            f.write(f"{v:.9g}\n")


def write_case(run_dir: str, case: dict) -> None:
    """case keys: flags (IsTestI0, IsDetResponse, IsGrid, IsSingleMaterial),
    geometry (pNumX..rotatedDirection), I0Val, spectrum [E], labels uint8
    [Z][Y][X], densities [M], mass_atten [M][E] (cm^2/g), scint (density,
    thickness, err, factor, mass_atten [E]), grid (FD, h, strip, inter,
    strip_density, inter_density, strip_ma [E], inter_ma [E])."""
    os.makedirs(os.path.join(run_dir, "Config"), exist_ok=True)
    os.makedirs(os.path.join(run_dir, "InputData"), exist_ok=True)
    g = case["geometry"]
    E = len(case["spectrum"])
    _write_table(os.path.join(run_dir, "InputData", "spectrum.dat"), case["spectrum"])
    case["labels"].astype(np.uint8).tofile(os.path.join(run_dir, "InputData", "labels.raw"))
    for m, ma in enumerate(case["mass_atten"]):
        _write_table(os.path.join(run_dir, "InputData", f"mat{m + 1}.dat"), ma)
    sc = case["scint"]
    _write_table(os.path.join(run_dir, "InputData", "scint.txt"), sc["mass_atten"])
    gr = case["grid"]
    _write_table(os.path.join(run_dir, "InputData", "grid_strip.txt"), gr["strip_ma"])
    _write_table(os.path.join(run_dir, "InputData", "grid_inter.txt"), gr["inter_ma"])
    f = case["flags"]
    lines = [
        "[ScanPara]",
        f"IsTestI0={f['IsTestI0']};", f"IsDetResponse={f['IsDetResponse']};", f"IsGrid={f['IsGrid']};",
        f"IsSingleMaterial={f['IsSingleMaterial']};",
        f"SDD={g['sdd']:.9g}\t\t;mm", f"SOD={g['sod']:.9g}\t\t;mm", f"ScanAngleNum={g['projNum']}",
        f"RotatedDirection={g.get('rotatedDirection', 1)};\t\t;comment", "",
        "[RaySource]", f"Photons={int(case['I0Val'])}", f"SpecEnergyNum={E}",
        "SpectrumPath=InputData/spectrum.dat", "",
        "[PhantomVox]", f"PNumX={g['pNumX']}", f"PNumY={g['pNumY']}", f"PNumZ={g['pNumZ']}",
        f"PLengthX={g['pLengthX']:.9g}", f"PLengthY={g['pLengthY']:.9g}", f"PLengthZ={g['pLengthZ']:.9g}", "",
        "[Detector]", f"DNumU={g['dNumU']}", f"DNumV={g['dNumV']}", f"DSize={g['dSize']:.9g}", "",
        "[Scintillator]", f"Density={sc['density']:.9g}", f"Thickness={sc['thickness']:.9g}",
        f"ThicknessErr={sc['err']:.9g}", f"PhotoelectConverFactor={sc['factor']:.9g}",
        "ScintillatorMAPath=InputData/scint.txt", "",
        "[PostGrid]", f"FD={gr['FD']:.9g}", f"Height={gr['h']:.9g}", f"GridStripsWidth={gr['strip']}",
        f"InterspcaceWidth={gr['inter']}", "GridStripMaterial=Pb", "InterspaceMaterial=Air",
        f"GridStripDensity={gr['strip_density']:.9g}", f"InterspaceDensity={gr['inter_density']:.9g}",
        "GridStripMAPath=InputData/grid_strip.txt", "InterspaceMAPath=InputData/grid_inter.txt", "",
        "[PhantomMaterial]", f"MaterialNum={len(case['densities'])}", "StructureMarkPath=InputData/labels.raw",
    ]
    for m, dens in enumerate(case["densities"]):
        lines += [f"Density{m + 1}={dens:.9g}", f"MassAttenPath{m + 1}=InputData/mat{m + 1}.dat"]
    with open(os.path.join(run_dir, "Config", "ScanSetting.ini"), "w") as fh:
        fh.write("\n".join(lines) + "\n")
    out = ["[GridNoResponse]", "OutFolder=Out/GridNoResponse", "", "[GridResponse]", "OutFolder=Out/GridResponse",
           "", "[NoGridNoResponse]", "OutFolder=Out/NoGridNoResponse", "", "[NoGridResponse]",
           "OutFolder=Out/NoGridResponse", "", "[NoGridResponseTestI0]", "OutFolder=Out/NoGridResponseTestI0"]
    text = "\n".join(out) + "\n"
    # the reference opens OutputFolder.ini while its shipped file is OutPutFolder.ini
    for name in ("OutPutFolder.ini", "OutputFolder.ini"):
        with open(os.path.join(run_dir, "Config", name), "w") as fh:
            fh.write(text)


def out_folder(flags: dict) -> str:
    if flags["IsTestI0"]:
        return "Out/NoGridResponseTestI0"
    return "Out/" + ("Grid" if flags["IsGrid"] else "NoGrid") + ("Response" if flags["IsDetResponse"] else "NoResponse")


def read_outputs(run_dir: str, case: dict) -> dict:
    g = case["geometry"]
    U, V, P = g["dNumU"], g["dNumV"], g["projNum"]
    f = case["flags"]
    tag = "Grid" if (f["IsGrid"] and not f["IsTestI0"]) else "NoGrid"
    d = os.path.join(run_dir, out_folder(f))
    res = {}

    def load(name, dtype, shape):
        p = os.path.join(d, name)
        if os.path.exists(p):
            res[name.split("_")[0]] = np.fromfile(p, dtype=dtype).reshape(shape)

    load(f"PhoImgPro_{tag}_{U}x{V}x{P}_uint32.raw", np.uint32, (P, V, U))
    load(f"PhoImgAbsorb_{tag}_{U}x{V}x{P}_uint32.raw", np.uint32, (P, V, U))
    load(f"BgImgPro_{tag}_{U}x{V}_float.raw", np.float32, (V, U))
    load(f"Projection_{tag}_{U}x{V}x{P}_float.raw", np.float32, (P, V, U))
    adr = os.path.join(d, "ADetResponse.txt")
    if os.path.exists(adr):
        res["ADetResponse"] = np.loadtxt(adr, dtype=np.float64).reshape(-1)
    return res


def run(case: dict, timeout: float = 600.0, keep_dir: str | None = None) -> tuple[dict, float, str]:
    """Runs the reference binary on one case; returns (outputs, wall seconds, stdout)."""
    if not os.path.exists(REF_BIN):
        raise FileNotFoundError(REF_BIN)
    g = case["geometry"]
    # the reference sizes its density-projection buffer K*U*V but indexes it
    # U*V*P (CBCTPolyProjGPU.cu:659): P > K would write out of bounds
    from oracle import oracle as O
    K = O.compute_paras(g)["intNum"]
    if g["projNum"] > K:
        raise ValueError(f"projNum {g['projNum']} > intNum {K}: the reference would write out of bounds")
    run_dir = keep_dir or tempfile.mkdtemp(prefix="ctfp_refrun_")
    try:
        write_case(run_dir, case)
        t0 = time.perf_counter()
        p = subprocess.run([REF_BIN], cwd=run_dir, capture_output=True, timeout=timeout, stdin=subprocess.DEVNULL)
        dt = time.perf_counter() - t0
        log = p.stdout.decode("utf-8", "replace") + p.stderr.decode("utf-8", "replace")
        outs = read_outputs(run_dir, case)
    finally:
        if keep_dir is None:
            shutil.rmtree(run_dir, ignore_errors=True)
    if p.returncode != 0:
        # The reference's destructors delete[] members its constructors never
        # set (aDetResponse, CBCTForwardProj.h:99, in the multi-material and
        # TestI0 paths), which can abort the process at exit, after the
        # outputs are written.  Accept that case only when the run printed its
        # completion message and every expected output is present.
        want = {"BgImgPro"} if case["flags"]["IsTestI0"] else {"PhoImgPro", "PhoImgAbsorb", "BgImgPro", "Projection"}
        done = ("完成" in log) and want <= set(outs)
        if not done:
            raise RuntimeError(f"reference exited {p.returncode}: {log[-2000:]}")
        log += f"\n[ref_runner] exit status {p.returncode} after the outputs were written (destructor)\n"
    return outs, dt, log


def bench_line(args, w) -> dict:
    """The reference arm of bench.py: the reference's own pipeline (one host
    thread driving the GPU, per-energy and per-view launches) on the workload's
    volume, detector, energies and grid, run as the stock binary end to end
    (process wall time, inputs from files).

    A full 360-view run takes the reference about a hundred seconds, so the
    timed steps sample it: they alternate between two view counts (8 and 24 by
    default, CTFP_REF_VIEWS="8,24"), a least-squares line T(n) = F + n * t over
    the timed steps splits each run into its fixed cost F (process and context
    start-up, per-energy host rebuild and upload of the attenuation volume,
    file I/O) and its cost per view t, and `value` is the rays/s of the
    full-view step predicted by that line, F + P * t.  `ms_per_step` is the
    wall time per timed step as run (the sample), so that steps x ms_per_step
    is the time the arm spent timing.  Warm-up runs use one view."""
    g = dict(w.geometry)
    P_full = int(g["projNum"])
    counts = [int(x) for x in os.environ.get("CTFP_REF_VIEWS", "8,24").split(",") if x.strip()]
    if len(counts) == 1:
        counts = counts * 2
    pix = int(g["dNumU"] * g["dNumV"])
    cases = {}

    def case_for(n):
        if n not in cases:
            gn = dict(g)
            gn["projNum"] = n
            cases[n] = reference_case_from_workload(w, gn)
        return cases[n]

    for _ in range(args.warmup):
        run(case_for(1), timeout=900)
    ns, ts = [], []
    for s in range(args.steps):
        n = counts[s % len(counts)]
        _, dt, _ = run(case_for(n), timeout=900)
        ns.append(n)
        ts.append(dt)
    ns_a, ts_a = np.array(ns, np.float64), np.array(ts, np.float64)
    if len(set(ns)) >= 2:
        t_view, fixed = np.polyfit(ns_a, ts_a, 1)
    else:  # one view count: no split; the per-view cost absorbs the fixed cost
        t_view, fixed = float(np.mean(ts_a / ns_a)), 0.0
    t_full = fixed + P_full * t_view
    v = P_full * pix / t_full
    E = int(case_for(counts[0])["spectrum"].size)
    return {"impl": "reference", "metric": "rays/s (polyenergetic cone-beam forward projection)", "value": v,
            "unit": "rays/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": float(np.mean(ts_a)) * 1e3, "higher_is_better": True,
            "dtype": "f32", "data": "synthetic (seeded label phantom)",
            "config": {"workload": w.name, "views": P_full, "volume": [g["pNumX"], g["pNumY"], g["pNumZ"]],
                       "detector": [g["dNumU"], g["dNumV"]], "energies": E,
                       "energies_note": "the reference's tables start at 1 keV (line e holds e + 1 keV), so the "
                                        f"{int(w.e_min)}-{int(w.kvp)} keV spectrum is {E} bins, the lowest with "
                                        "zero weight; it marches all of them",
                       "value": f"extrapolated to the {P_full}-view step: fixed + {P_full} x per-view cost, both "
                                f"fitted to the timed runs at {sorted(set(ns))} views",
                       "ms_per_step": "wall time per timed run as sampled (alternating view counts)"},
            "reference_split": {"fixed_s": float(fixed), "per_view_s": float(t_view),
                                "full_step_s_extrapolated": float(t_full),
                                "marginal_rays_per_s": pix / float(t_view) if t_view > 0 else None,
                                "runs": [{"views": int(n), "s": float(t)} for n, t in zip(ns, ts)],
                                "note": "marginal = one view's rays / per-view cost: the reference's per-view "
                                        "kernels, syncs, device-to-host copies and host sums, without its fixed "
                                        "start-up"},
            "cpu_baseline": {"value": v, "unit": "rays/s", "cores": 1, "kind": "reference",
                             "sample": f"the reference's CUDA pipeline (CBCTPolyForwardProjGrid, sm_100a build), one "
                                       f"host thread, process wall time incl. file I/O, runs at {sorted(set(ns))} "
                                       f"of {P_full} views extrapolated to {P_full}"},
            "e2e": {"value": v, "unit": "rays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def reference_case_from_workload(w, g: dict) -> dict:
    """The reference's multi-material grid mode on a label version of the
    workload's phantom; tables on the 1-keV grid from 1 keV to kVp."""
    from ct_forward_projection_b200 import physics
    E = int(w.kvp)
    energies = np.arange(1, E + 1, dtype=np.float64)
    spec = np.zeros(E)
    e_all, s_all = physics.kramers_spectrum(w.kvp, w.e_min, w.al_mm)
    spec[(e_all - 1).astype(int)] = s_all
    labels = physics.label_phantom(w)
    dens = [physics.MATERIALS[m][2] for m in w.materials]
    return {
        "flags": {"IsTestI0": 0, "IsDetResponse": 1, "IsGrid": 1, "IsSingleMaterial": 0},
        "geometry": g, "I0Val": w.I0Val, "spectrum": spec, "labels": labels, "densities": dens,
        "mass_atten": [physics.mass_attenuation(m, energies) for m in w.materials],
        "scint": {"density": physics.MATERIALS["csi"][2], "thickness": w.scint_mm or 0.6, "err": w.scint_err_mm,
                  "factor": 1.0, "mass_atten": physics.mass_attenuation("csi", energies)},
        "grid": {"FD": w.grid.FD_mm, "h": w.grid.h_mm, "strip": w.grid.strip_um, "inter": w.grid.inter_um,
                 "strip_density": physics.MATERIALS[w.grid.strip_material][2],
                 "inter_density": physics.MATERIALS[w.grid.inter_material][2],
                 "strip_ma": physics.mass_attenuation(w.grid.strip_material, energies),
                 "inter_ma": physics.mass_attenuation(w.grid.inter_material, energies)},
    }

