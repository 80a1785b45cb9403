"""Makes tests/golden/reference_cases.npz: outputs of the reference's own
projector (oracle/_ref/ctfp_ref, built from the reference sources by
oracle/build_ref.sh) on small seeded inputs, one case per dispatch branch of
ForwardProjection::run (ForwardProjection.cpp:20-84).

Run on a machine with a GPU after oracle/build_ref.sh:
    python tests/golden/make_golden.py [out.npz]
The inputs are stored next to the outputs, so the tests do not depend on this
script's generators.
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from ct_forward_projection_b200 import physics  # noqa: E402
from oracle import ref_runner  # noqa: E402

GEOM = dict(pNumX=32, pNumY=32, pNumZ=32, pLengthX=16.0, pLengthY=16.0, pLengthZ=16.0, projNum=12, dNumU=40,
            dNumV=32, dSize=0.8, sod=150.0, sdd=300.0, rotatedDirection=1)
E = 40  # energy bins e <-> (e + 1) keV, 1..40 keV

# (IsTestI0, IsDetResponse, IsGrid, IsSingleMaterial) for each reachable branch of run()
CASES = {
    "grid_response_multi": (0, 1, 1, 0),
    "grid_response_sinmat": (0, 1, 1, 1),
    "nogrid_response_multi": (0, 1, 0, 0),
    "nogrid_response_sinmat": (0, 1, 0, 1),
    "grid_noresponse_sinmat": (0, 0, 1, 1),
    "nogrid_noresponse_sinmat": (0, 0, 0, 1),
    "test_i0": (1, 1, 0, 0),
}


def labels(single: bool, seed: int) -> np.ndarray:
    rng = np.random.RandomState(seed)
    n = 32
    z, y, x = np.mgrid[0:n, 0:n, 0:n].astype(np.float64) - (n - 1) / 2
    lab = np.zeros((n, n, n), np.uint8)
    lab[(x ** 2 + y ** 2 <= (0.42 * n) ** 2) & (np.abs(z) <= 0.45 * n)] = 1
    for _ in range(4):
        c = rng.uniform(-0.22, 0.22, 3) * n
        r = rng.uniform(0.06, 0.14) * n
        m = (x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2 <= r * r
        lab[m] = 0 if single else 2
    return lab


def make_case(flags, seed):
    single = bool(flags[3])
    energies = np.arange(1, E + 1, dtype=np.float64)
    spec = np.zeros(E)
    e_s, s_s = physics.kramers_spectrum(40.0, 15.0, 1.0)
    spec[(e_s - 1).astype(int)] = s_s
    mats = ["water"] if single else ["water", "aluminium"]
    return {
        "flags": dict(zip(("IsTestI0", "IsDetResponse", "IsGrid", "IsSingleMaterial"), flags)),
        "geometry": dict(GEOM), "I0Val": 60000.0, "spectrum": spec, "labels": labels(single, seed),
        "densities": [1.0] if single else [1.0, 2.699],
        "mass_atten": [physics.mass_attenuation(m, energies) for m in mats],
        "scint": {"density": 4.51, "thickness": 0.4, "err": 0.05, "factor": 1.0,
                  "mass_atten": physics.mass_attenuation("csi", energies)},
        "grid": {"FD": 300.0, "h": 1.5, "strip": 50, "inter": 150, "strip_density": 11.35, "inter_density": 0.0,
                 "strip_ma": physics.mass_attenuation("lead", energies),
                 "inter_ma": physics.mass_attenuation("fiber", energies)},
    }


def main(out_path: str) -> None:
    store = {}
    for k, (name, flags) in enumerate(CASES.items()):
        case = make_case(flags, 40 + k)
        outs, dt, log = ref_runner.run(case, timeout=300)
        print(f"{name}: {sorted(outs)} in {dt:.2f} s", flush=True)
        p = name + "/"
        store[p + "flags"] = np.array(flags, np.int32)
        store[p + "labels"] = case["labels"]
        store[p + "spectrum"] = case["spectrum"].astype(np.float32)
        store[p + "densities"] = np.array(case["densities"], np.float32)
        store[p + "mass_atten"] = np.array(case["mass_atten"], np.float32)
        store[p + "scint_ma"] = case["scint"]["mass_atten"].astype(np.float32)
        store[p + "grid_strip_ma"] = case["grid"]["strip_ma"].astype(np.float32)
        store[p + "grid_inter_ma"] = case["grid"]["inter_ma"].astype(np.float32)
        for key, v in outs.items():
            store[p + "out_" + key] = v
    store["geometry"] = np.array([GEOM[k] for k in ("pNumX", "pNumY", "pNumZ", "pLengthX", "pLengthY", "pLengthZ",
                                                    "projNum", "dNumU", "dNumV", "dSize", "sod", "sdd",
                                                    "rotatedDirection")], np.float64)
    store["scint_params"] = np.array([4.51, 0.4, 0.05, 1.0], np.float32)
    store["grid_params"] = np.array([300.0, 1.5, 50, 150, 11.35, 0.0], np.float32)
    store["I0Val"] = np.array([60000.0], np.float32)
    np.savez_compressed(out_path, **store)
    print("wrote", out_path)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(os.path.dirname(os.path.abspath(__file__)),
                                                             "reference_cases.npz"))
