"""Synthetic physics tables and seeded phantoms for the projector's workloads.

The reference reads its spectra and attenuation tables from text files
(InputData/Spectrum, InputData/PhantomMaterial, InputData/Scintillator,
InputData/Grid; one value per line, index e <-> (e+1) keV), which stop at
80 keV for CsI and Pb.  The workloads here run to 140 keV, so the tables are
synthetic but physically shaped:

  mass attenuation  mu/rho(E) = a * E^-3 + N_A * (Z/A) * sigma_KN(E)     [cm^2/g]
  spectrum          Kramers (kVp - E) / E, filtered by exp(-mu_Al(E) rho_Al t)

with a per-material photoelectric constant a (keV^3 cm^2/g, a K-edge jump for
iodine and lead) and the Klein-Nishina total cross-section per electron.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

N_A_BARN = 0.6022140857  # Avogadro * 1e-24: electrons/g per (Z/A) times barn -> cm^2/g
R_E2_BARN = 0.0794077     # classical electron radius squared, barn (2.8179403e-13 cm)^2

# name: (photoelectric a [keV^3 cm^2/g], Z/A, density g/cm^3, K-edge keV or 0, jump ratio)
MATERIALS = {
    "water": (4800.0, 0.5551, 1.0, 0.0, 1.0),
    "soft_tissue": (4900.0, 0.5497, 1.06, 0.0, 1.0),
    "fat": (2900.0, 0.5558, 0.92, 0.0, 1.0),
    "bone": (30400.0, 0.5148, 1.92, 0.0, 1.0),
    "iodine": (95000.0, 0.4176, 4.93, 33.17, 5.8),
    "aluminium": (26500.0, 0.4818, 2.699, 0.0, 1.0),
    "lead": (1.05e6, 0.3958, 11.35, 88.0, 4.6),
    "csi": (1.10e5, 0.4160, 4.51, 33.17, 5.2),
    "fiber": (3000.0, 0.52, 0.8, 0.0, 1.0),
}


def klein_nishina_barn(E_keV) -> np.ndarray:
    """Total Klein-Nishina cross-section per electron, barn."""
    k = np.asarray(E_keV, dtype=np.float64) / 510.99895
    a = (1 + k) / k ** 2 * (2 * (1 + k) / (1 + 2 * k) - np.log1p(2 * k) / k)
    b = np.log1p(2 * k) / (2 * k) - (1 + 3 * k) / (1 + 2 * k) ** 2
    return 2 * math.pi * R_E2_BARN * (a + b)


def mass_attenuation(material: str, E_keV) -> np.ndarray:
    """mu/rho in cm^2/g at the given energies (keV)."""
    a, za, _, edge, jump = MATERIALS[material]
    E = np.asarray(E_keV, dtype=np.float64)
    photo = a * E ** -3.0
    if edge > 0:
        photo = np.where(E >= edge, photo, photo / jump)
    return photo + N_A_BARN * za * klein_nishina_barn(E)


def kramers_spectrum(kvp: float, e_min: float, al_mm: float) -> tuple[np.ndarray, np.ndarray]:
    """(energies keV, normalised spectrum) in 1-keV bins e_min..kvp."""
    E = np.arange(int(e_min), int(kvp) + 1, dtype=np.float64)
    phi = np.clip(kvp - E, 0.0, None) / E
    phi = phi * np.exp(-mass_attenuation("aluminium", E) * MATERIALS["aluminium"][2] * al_mm / 10.0)
    s = phi.sum()
    return E, (phi / s if s > 0 else phi)


@dataclass
class GridSpec:
    strip_um: int
    inter_um: int
    h_mm: float
    FD_mm: float
    strip_material: str = "lead"
    inter_material: str = "fiber"


@dataclass
class Workload:
    """One projector problem: geometry, materials and spectral setup."""
    name: str
    geometry: dict
    materials: list[str]
    kvp: float
    e_min: float
    al_mm: float = 2.0
    grid: GridSpec | None = None
    grid_layout: int = 2  # 1 column table (reference), 2 per-pixel incidence angle
    scint_mm: float | None = 0.6
    scint_err_mm: float = 0.0
    I0Val: float = 60000.0
    seed: int = 1000
    extra: dict = field(default_factory=dict)

    @property
    def energies(self) -> np.ndarray:
        return kramers_spectrum(self.kvp, self.e_min, self.al_mm)[0]

    def spectrum(self) -> np.ndarray:
        return kramers_spectrum(self.kvp, self.e_min, self.al_mm)[1].astype(np.float32)

    def mu_table(self) -> np.ndarray:
        """[E][M] attenuation per density, 1/mm per g/cm^3 ((mu/rho)/10)."""
        E = self.energies
        return np.stack([mass_attenuation(m, E) / 10.0 for m in self.materials], axis=1).astype(np.float32)

    def scint_mu(self) -> np.ndarray:
        """CsI linear attenuation, 1/mm, per energy (table * density / 10)."""
        return (mass_attenuation("csi", self.energies) * MATERIALS["csi"][2] / 10.0).astype(np.float32)

    def grid_mu(self) -> tuple[np.ndarray, np.ndarray]:
        g = self.grid
        E = self.energies
        ms = mass_attenuation(g.strip_material, E) * MATERIALS[g.strip_material][2] / 10.0
        mi = mass_attenuation(g.inter_material, E) * MATERIALS[g.inter_material][2] / 10.0
        return ms.astype(np.float32), mi.astype(np.float32)

    @property
    def n_rays(self) -> int:
        g = self.geometry
        return int(g["projNum"] * g["dNumU"] * g["dNumV"])


def _geom(n, length, views, U, V, pitch, sod=1000.0, sdd=1500.0, rot=1):
    nx, ny, nz = (n, n, n) if isinstance(n, int) else n
    lx, ly, lz = (length, length, length) if isinstance(length, (int, float)) else length
    return dict(pNumX=nx, pNumY=ny, pNumZ=nz, pLengthX=lx, pLengthY=ly, pLengthZ=lz, projNum=views, dNumU=U,
                dNumV=V, dSize=pitch, sod=sod, sdd=sdd, rotatedDirection=rot)


def workload(name: str) -> Workload:
    """The named workloads (sizes as the benchmark configurations state them)."""
    if name == "sinmat_nogrid_128":
        return Workload(name, _geom(128, 128.0, 60, 256, 256, 1.0), ["water"], 80, 20, 2.0, None,
                        scint_mm=0.6, seed=1001)
    if name == "poly_grid_256":
        return Workload(name, _geom(256, 128.0, 360, 512, 384, 0.8), ["soft_tissue", "bone"], 120, 20, 2.0,
                        GridSpec(50, 200, 2.0, 1500.0), grid_layout=2, scint_mm=0.6, scint_err_mm=0.05, seed=1002)
    if name == "poly_grid_256_v36":
        # the same problem with every tenth view: the small case for profiling
        w = workload("poly_grid_256")
        w.name = name
        w.geometry["projNum"] = 36
        return w
    if name == "diff_3mat_256":
        return Workload(name, _geom(256, 128.0, 180, 384, 384, 1.0), ["soft_tissue", "bone", "iodine"], 120, 20,
                        2.0, GridSpec(50, 200, 2.0, 1500.0), grid_layout=2, scint_mm=0.6, seed=1003)
    if name == "large_4mat_512":
        return Workload(name, _geom(512, 204.8, 720, 1024, 768, 0.4), ["fat", "soft_tissue", "bone", "iodine"],
                        140, 15, 2.0, GridSpec(27, 140, 1.68, 1500.0), grid_layout=2, scint_mm=0.6, seed=1005)
    raise KeyError(name)


def scaled(w: Workload, n: int, views: int, U: int, V: int) -> Workload:
    """Same physics at a smaller geometry (keeps FOV and pitch ratios)."""
    g = dict(w.geometry)
    f = n / g["pNumX"]
    g.update(pNumX=n, pNumY=n, pNumZ=max(1, int(round(g["pNumZ"] * f))), projNum=views,
             dSize=g["dSize"] * g["dNumU"] / U, dNumU=U, dNumV=V)
    return Workload(w.name + f"_{n}", g, w.materials, w.kvp, w.e_min, w.al_mm, w.grid, w.grid_layout, w.scint_mm,
                    w.scint_err_mm, w.I0Val, w.seed)


# ---------------------------------------------------------------------------
# Seeded phantoms (torch on the given device; float32 [Z][Y][X] per material)

def _grid_coords(geom, device):
    import torch
    nx, ny, nz = geom["pNumX"], geom["pNumY"], geom["pNumZ"]
    # physical coordinates (mm) of voxel centres relative to the volume centre;
    # voxel j sits at j * pSize in the reference's sampling frame
    sx, sy, sz = geom["pLengthX"] / nx, geom["pLengthY"] / ny, geom["pLengthZ"] / nz
    x = (torch.arange(nx, device=device, dtype=torch.float32) * sx - geom["pLengthX"] / 2)
    y = (torch.arange(ny, device=device, dtype=torch.float32) * sy - geom["pLengthY"] / 2)
    z = (torch.arange(nz, device=device, dtype=torch.float32) * sz - geom["pLengthZ"] / 2)
    return x, y, z


def _rot(rng):
    a, b, c = rng.uniform(0, 2 * np.pi, 3)
    ca, sa, cb, sb, cc, sc = np.cos(a), np.sin(a), np.cos(b), np.sin(b), np.cos(c), np.sin(c)
    Rz = np.array([[ca, -sa, 0], [sa, ca, 0], [0, 0, 1]])
    Ry = np.array([[cb, 0, sb], [0, 1, 0], [-sb, 0, cb]])
    Rx = np.array([[1, 0, 0], [0, cc, -sc], [0, sc, cc]])
    return Rz @ Ry @ Rx


def _ellipsoid_mask(x, y, z, centre, axes, R):
    import torch
    X = x[None, None, :] - float(centre[0])
    Y = y[None, :, None] - float(centre[1])
    Z = z[:, None, None] - float(centre[2])
    Rt = torch.tensor(R.T, dtype=torch.float32, device=x.device)
    u = (Rt[0, 0] * X + Rt[0, 1] * Y + Rt[0, 2] * Z) / float(axes[0])
    v = (Rt[1, 0] * X + Rt[1, 1] * Y + Rt[1, 2] * Z) / float(axes[1])
    w = (Rt[2, 0] * X + Rt[2, 1] * Y + Rt[2, 2] * Z) / float(axes[2])
    return (u * u + v * v + w * w) <= 1.0


def _tube_mask(x, y, z, p0, d, radius):
    X = x[None, None, :] - float(p0[0])
    Y = y[None, :, None] - float(p0[1])
    Z = z[:, None, None] - float(p0[2])
    t = X * float(d[0]) + Y * float(d[1]) + Z * float(d[2])
    r2 = X * X + Y * Y + Z * Z - t * t
    return r2 <= radius * radius


def phantom(w: Workload, device="cpu") -> list:
    """Seeded density maps (g/cm^3), one float32 tensor [Z][Y][X] per material."""
    import torch
    g = w.geometry
    rng = np.random.RandomState(w.seed)
    x, y, z = _grid_coords(g, device)
    L = min(g["pLengthX"], g["pLengthY"])
    Lz = g["pLengthZ"]
    shape = (g["pNumZ"], g["pNumY"], g["pNumX"])
    mats = w.materials
    out = [torch.zeros(shape, dtype=torch.float32, device=device) for _ in mats]
    if mats == ["water"]:
        body = (x[None, None, :] ** 2 + y[None, :, None] ** 2 <= (0.4 * L) ** 2) & \
               (z[:, None, None].abs() <= 0.45 * Lz)
        out[0][body] = 1.0
        for _ in range(10):
            c = [rng.uniform(-0.2, 0.2) * L, rng.uniform(-0.2, 0.2) * L, rng.uniform(-0.3, 0.3) * Lz]
            ax = rng.uniform(0.04, 0.15, 3) * L
            m = _ellipsoid_mask(x, y, z, c, ax, _rot(rng))
            out[0][m & body] = float(rng.uniform(0.2, 1.8))
        return out
    body = ((x[None, None, :] / (0.45 * L)) ** 2 + (y[None, :, None] / (0.33 * L)) ** 2 <= 1.0) & \
           (z[:, None, None].abs() <= 0.46 * Lz)
    idx = {m: i for i, m in enumerate(mats)}
    bone = torch.zeros(shape, dtype=torch.bool, device=device)
    for _ in range(6):
        c = [rng.uniform(-0.25, 0.25) * L, rng.uniform(-0.18, 0.18) * L, rng.uniform(-0.3, 0.3) * Lz]
        ax = rng.uniform(0.05, 0.14, 3) * L
        R = _rot(rng)
        shell = _ellipsoid_mask(x, y, z, c, ax, R) & ~_ellipsoid_mask(x, y, z, c, ax * rng.uniform(0.55, 0.8), R)
        bone |= shell
    bone &= body
    soft = body & ~bone
    if "fat" in idx:
        fat = body & ~(((x[None, None, :] / (0.40 * L)) ** 2 + (y[None, :, None] / (0.28 * L)) ** 2) <= 1.0)
        soft &= ~fat
        out[idx["fat"]][fat] = 0.92
    iodine = None
    if "iodine" in idx:
        iodine = torch.zeros(shape, dtype=torch.float32, device=device)
        for _ in range(8):
            p0 = [rng.uniform(-0.2, 0.2) * L, rng.uniform(-0.15, 0.15) * L, rng.uniform(-0.2, 0.2) * Lz]
            d = rng.normal(size=3)
            d /= np.linalg.norm(d)
            m = _tube_mask(x, y, z, p0, d, float(rng.uniform(0.01, 0.03) * L)) & soft
            iodine[m] = float(rng.uniform(0.0, 0.020))
        out[idx["iodine"]] = iodine
    out[idx["soft_tissue"]][soft] = 1.06
    out[idx["bone"]][bone] = 1.92
    return out


def label_phantom(w: Workload, seed_offset: int = 0) -> np.ndarray:
    """uint8 label volume [Z][Y][X] (0 = air, m + 1 = material m), the
    reference's StructureMarkPath format (PhantomObject.cpp:75-91)."""
    import torch
    maps = phantom(Workload(w.name, w.geometry, w.materials, w.kvp, w.e_min, w.al_mm, w.grid, w.grid_layout,
                            w.scint_mm, w.scint_err_mm, w.I0Val, w.seed + seed_offset), "cpu")
    lab = torch.zeros(maps[0].shape, dtype=torch.uint8)
    for m, v in enumerate(maps):
        lab[v > 0] = m + 1
    return lab.numpy()


def batch_workloads(n: int = 48, seed: int = 4000) -> list:
    """The uneven batch: n seeded problems with volumes from 64^3 to
    320 x 320 x 200 (1-3 materials), SOD 900-1100 / SDD 1300-1600 mm, 30-720
    views, detectors 128^2 to 768 x 512, spectra 60-140 kVp in 1-keV bins from
    20 keV (41-121 bins).  The detector pitch makes the field of view cover the
    volume's diagonal; half the problems carry a focused grid."""
    rng = np.random.RandomState(seed)
    mats = {1: ["water"], 2: ["soft_tissue", "bone"], 3: ["soft_tissue", "bone", "iodine"]}
    out = []
    for k in range(n):
        nxy = int(rng.randint(64, 321))
        nz = int(rng.randint(64, 201))
        M = int(rng.randint(1, 4))
        views = int(rng.randint(30, 721))
        U = int(rng.randint(128, 769))
        V = int(rng.randint(128, 513))
        sod = float(rng.uniform(900.0, 1100.0))
        sdd = float(rng.uniform(1300.0, 1600.0))
        kvp = int(rng.randint(60, 141))
        vox = float(rng.uniform(0.4, 1.0))
        L = nxy * vox
        pitch = 1.5 * L * sdd / sod / U
        grid = GridSpec(50, 200, 2.0, sdd) if rng.uniform() < 0.5 else None
        g = _geom((nxy, nxy, nz), (L, L, nz * vox), views, U, V, pitch, sod=sod, sdd=sdd)
        out.append(Workload(f"batch_{k:02d}", g, mats[M], kvp, 20, 2.0, grid, grid_layout=2, scint_mm=0.6,
                            seed=seed + 1 + k))
    return out
