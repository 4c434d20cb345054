"""Seeded synthetic inputs for the Coulomb workloads.

KTT's own Coulomb examples draw atoms from unseeded ``std::random_device``
engines (``Examples/CoulombSum3d/CoulombSum3d.cpp:84-99``,
``Examples/CoulombSum2d/CoulombSum2d.cpp:61-76``); these generators keep the
same kinds of distributions at the sizes of the benchmark workloads, with a
seed so every run and every test sees the same atoms.  Atoms are returned as
``(n, 4)`` float32 arrays of (x, y, z, q) in Angstrom / elementary charge.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class Map3d:
    atoms: np.ndarray          # (n, 4) float32
    dims: tuple[int, int, int]  # (nx, ny, nz)
    spacing: float
    origin: tuple[float, float, float] = (0.0, 0.0, 0.0)

    @property
    def pairs(self) -> int:
        nx, ny, nz = self.dims
        return nx * ny * nz * self.atoms.shape[0]


@dataclass
class Slice2d:
    atoms: np.ndarray          # (n, 4) float32 (x, y, z, q)
    nx: int
    ny: int
    spacing: float
    z_slice: float

    def ktt_atoms(self) -> np.ndarray:
        """KTT's 2D argument convention: (x, y, (z_slice - z)^2, q) formed in FP32."""
        a = self.atoms.copy()
        dz = np.float32(self.z_slice) - a[:, 2]
        a[:, 2] = dz * dz
        return a

    @property
    def pairs(self) -> int:
        return self.nx * self.ny * self.atoms.shape[0]


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32))


def slice_2d(seed: int = 1, n_atoms: int = 4000, n: int = 256, spacing: float = 0.5,
             z_slice: float = 16.0) -> Slice2d:
    """Single slice at z = 16 A of a 256 x 256 grid (h = 0.5 A); 4,000 atoms with x, y ~ U[0, 128),
    z ~ U[0, 32), q ~ U[-1, 1]."""
    rng = np.random.default_rng(seed)
    a = np.empty((n_atoms, 4), dtype=np.float32)
    a[:, 0] = rng.uniform(0.0, 128.0, n_atoms)
    a[:, 1] = rng.uniform(0.0, 128.0, n_atoms)
    a[:, 2] = rng.uniform(0.0, 32.0, n_atoms)
    a[:, 3] = rng.uniform(-1.0, 1.0, n_atoms)
    return Slice2d(_f32(a), n, n, spacing, z_slice)


def uniform_map(seed: int = 2, n_atoms: int = 65536, n: int = 256, spacing: float = 0.5,
                box: float = 128.0) -> Map3d:
    """Full map: n^3 grid at h = 0.5 A; atoms uniform in the box^3 cube, q ~ U[-1, 1]."""
    rng = np.random.default_rng(seed)
    a = np.empty((n_atoms, 4), dtype=np.float32)
    a[:, :3] = rng.uniform(0.0, box, (n_atoms, 3))
    a[:, 3] = rng.uniform(-1.0, 1.0, n_atoms)
    return Map3d(_f32(a), (n, n, n), spacing)


def clustered_map(seed: int = 3, n_clusters: int = 64, per_cluster: int = 1024, n: int = 256,
                  spacing: float = 0.5, sigma: float = 2.0, box: float = 128.0) -> Map3d:
    """Precision stress: Gaussian clusters (sigma = 2 A, centres uniform in the cube), charges +1/-1
    alternating within each cluster plus N(0, 0.01) noise, total charge exactly zero (the last atom
    takes the remainder, summed in FP64 and rounded once)."""
    rng = np.random.default_rng(seed)
    centres = rng.uniform(0.0, box, (n_clusters, 3))
    pos = centres[:, None, :] + rng.normal(0.0, sigma, (n_clusters, per_cluster, 3))
    sign = np.where(np.arange(per_cluster) % 2 == 0, 1.0, -1.0)
    q = sign[None, :] + rng.normal(0.0, 0.01, (n_clusters, per_cluster))
    a = np.empty((n_clusters * per_cluster, 4), dtype=np.float32)
    a[:, :3] = pos.reshape(-1, 3)
    a[:, 3] = q.reshape(-1)
    a[-1, 3] = np.float32(-np.sum(a[:-1, 3].astype(np.float64)))
    return Map3d(_f32(a), (n, n, n), spacing)


@dataclass
class Molecule:
    atoms: np.ndarray
    dims: tuple[int, int, int]
    origin: tuple[float, float, float]
    spacing: float

    @property
    def pairs(self) -> int:
        nx, ny, nz = self.dims
        return nx * ny * nz * self.atoms.shape[0]


def molecule_batch(seed: int = 4, n_mol: int = 512, lo: int = 200, hi: int = 20000, density: float = 0.1,
                   margin: float = 8.0, spacing: float = 0.5) -> list[Molecule]:
    """Uneven batch: atom counts log-uniform in [lo, hi]; atoms uniform in a cube of side
    (n / density)^(1/3) A, q ~ U[-1, 1]; each grid is the atoms' bounding box plus `margin` A on every
    side at 0.5 A spacing, origin at the box corner."""
    rng = np.random.default_rng(seed)
    counts = np.exp(rng.uniform(np.log(lo), np.log(hi), n_mol)).astype(np.int64)
    mols = []
    for n in counts:
        side = (float(n) / density) ** (1.0 / 3.0)
        a = np.empty((int(n), 4), dtype=np.float32)
        a[:, :3] = rng.uniform(0.0, side, (int(n), 3))
        a[:, 3] = rng.uniform(-1.0, 1.0, int(n))
        lo_c = a[:, :3].min(axis=0).astype(np.float64) - margin
        hi_c = a[:, :3].max(axis=0).astype(np.float64) + margin
        dims = tuple(int(np.floor((hi_c[k] - lo_c[k]) / spacing)) + 1 for k in range(3))
        mols.append(Molecule(_f32(a), dims, tuple(float(np.float32(v)) for v in lo_c), spacing))
    return mols


def adjoint_problem(seed: int = 5, n_atoms: int = 8192, n: int = 128, spacing: float = 0.5, box: float = 64.0,
                    perturb: float = 0.1, exclusion: float = 1.5):
    """Charge fitting: atoms uniform in a 64 A cube on a 128^3 grid.  Returns (atoms, perturbed_charges,
    dims, spacing, exclusion): the target map is V computed with q + N(0, perturb); the loss weight is 1
    outside `exclusion` A of every atom and 0 inside."""
    rng = np.random.default_rng(seed)
    a = np.empty((n_atoms, 4), dtype=np.float32)
    a[:, :3] = rng.uniform(0.0, box, (n_atoms, 3))
    a[:, 3] = rng.uniform(-1.0, 1.0, n_atoms)
    q_target = (a[:, 3].astype(np.float64) + rng.normal(0.0, perturb, n_atoms)).astype(np.float32)
    return _f32(a), q_target, (n, n, n), spacing, exclusion


def exclusion_weights(atoms: np.ndarray, dims, spacing: float, radius: float,
                      origin=(0.0, 0.0, 0.0)) -> np.ndarray:
    """w = 0 at grid points within `radius` of any atom, 1 elsewhere; shape (nz, ny, nx) float32."""
    nx, ny, nz = dims
    w = np.ones((nz, ny, nx), dtype=np.float32)
    r_cells = int(np.ceil(radius / spacing))
    offs = np.arange(-r_cells, r_cells + 1)
    for a in atoms:
        c = [(a[k] - origin[k]) / spacing for k in range(3)]
        base = [int(np.floor(v)) for v in c]
        xs = np.clip(base[0] + offs, 0, nx - 1)
        ys = np.clip(base[1] + offs, 0, ny - 1)
        zs = np.clip(base[2] + offs, 0, nz - 1)
        gx = np.float32(origin[0]) + xs.astype(np.float32) * np.float32(spacing)
        gy = np.float32(origin[1]) + ys.astype(np.float32) * np.float32(spacing)
        gz = np.float32(origin[2]) + zs.astype(np.float32) * np.float32(spacing)
        d2 = ((gz[:, None, None] - a[2]) ** 2 + (gy[None, :, None] - a[1]) ** 2 + (gx[None, None, :] - a[0]) ** 2)
        m = d2 < radius * radius
        sub = w[np.ix_(zs, ys, xs)]
        sub[m] = 0.0
        w[np.ix_(zs, ys, xs)] = sub
    return w


def subset_indices(total: int, fraction: float, seed: int = 11) -> np.ndarray:
    """Seeded sorted subset of linear grid indices (e.g. the 1% check set of the full map)."""
    k = max(1, int(round(total * fraction)))
    rng = np.random.default_rng(seed)
    return np.sort(rng.choice(total, size=k, replace=False)).astype(np.int64)
