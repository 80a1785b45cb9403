"""Shared fixtures. GPU tests are marked `gpu` and need a CUDA device."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libctfp.so")


def small_geometry(n=24, views=6, U=20, V=12, pitch=None, length=24.0, sod=300.0, sdd=450.0, rot=1):
    """A small cone-beam geometry whose FOV covers most of the volume."""
    if pitch is None:
        pitch = 1.6 * length / U * sdd / sod
    nx, ny, nz = (n, n, n) if isinstance(n, int) else n
    return dict(pNumX=nx, pNumY=ny, pNumZ=nz, pLengthX=length * nx / max(nx, ny), pLengthY=length * ny / max(nx, ny),
                pLengthZ=length * nz / max(nx, ny), projNum=views, dNumU=U, dNumV=V, dSize=pitch, sod=sod, sdd=sdd,
                rotatedDirection=rot)


def random_volumes(geom, M, seed, smooth=False):
    rng = np.random.RandomState(seed)
    shape = (geom["pNumZ"], geom["pNumY"], geom["pNumX"])
    vols = []
    for m in range(M):
        v = rng.uniform(0.0, 2.0, shape).astype(np.float32)
        # a few zero voxels and an empty border slab, as label-derived maps have
        v[rng.uniform(size=shape) < 0.2] = 0.0
        vols.append(v)
    return vols


def spectral_setup(geom, M, E, seed, grid=True, det=True):
    rng = np.random.RandomState(seed)
    S = rng.uniform(0.1, 1.0, E).astype(np.float32)
    S /= S.sum()
    mu = rng.uniform(0.005, 0.06, (E, M)).astype(np.float32)
    U, V = geom["dNumU"], geom["dNumV"]
    G = rng.uniform(0.6, 0.9, (E, V, U)).astype(np.float32) if grid else None
    D = rng.uniform(0.3, 0.95, (E, V, U)).astype(np.float32) if det else None
    return S, mu, G, D


@pytest.fixture(scope="session")
def cuda_ok():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return True
