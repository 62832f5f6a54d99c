"""Seeded synthetic molecules for the benchmark and test workloads.

No public benchmark suite is involved: every geometry is built here from
idealised bond lengths and angles, then perturbed with a fixed seed.
Coordinates are returned in bohr (src/molecule/hfscf_constants.hpp:5).

Seeds: 20261203 + workload index (1..5), as the workload table fixes them.
"""
from __future__ import annotations

import numpy as np

from .basis import ANGSTROM_TO_BOHR as A2B

SEED_BASE = 20261203
TETRA = np.deg2rad(109.4712206)


def random_rotation(rng) -> np.ndarray:
    """Uniform random rotation matrix from a unit quaternion."""
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([
        [1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
        [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
        [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)],
    ])


def water(rng=None, orient=True):
    """One rigid water (O-H 0.9572 A, HOH 104.52 deg), angstrom, O first."""
    r, th = 0.9572, np.deg2rad(104.52)
    xyz = np.array([[0.0, 0.0, 0.0],
                    [0.0, r * np.sin(th / 2), r * np.cos(th / 2)],
                    [0.0, -r * np.sin(th / 2), r * np.cos(th / 2)]])
    if orient and rng is not None:
        xyz = xyz @ random_rotation(rng).T
    return [8, 1, 1], xyz


def h2o_ccpvdz():
    """H2O at O (0,0,0), H (0, +-1.4305, 1.1073) bohr."""
    return [8, 1, 1], np.array([[0.0, 0.0, 0.0], [0.0, 1.4305, 1.1073], [0.0, -1.4305, 1.1073]])


def _tetra_dirs(b, v):
    """Three unit vectors at the tetrahedral angle from bond b, the first in the b-v plane."""
    b = b / np.linalg.norm(b)
    v = v - np.dot(v, b) * b
    v /= np.linalg.norm(v)
    w = np.cross(b, v)
    return [np.cos(TETRA) * b + np.sin(TETRA) * (np.cos(p) * v + np.sin(p) * w)
            for p in (0.0, 2 * np.pi / 3, 4 * np.pi / 3)]


def n_alkane(nc: int, rng=None):
    """All-trans CnH(2n+2): C-C 1.53 A, C-H 1.09 A, tetrahedral angles, zigzag in xy."""
    cc, ch = 1.53, 1.09
    half = TETRA / 2
    C = np.array([[i * cc * np.sin(half), (i % 2) * cc * np.cos(half), 0.0] for i in range(nc)])
    H = []
    ez = np.array([0.0, 0.0, 1.0])
    for i in range(nc):
        nb = [C[j] for j in (i - 1, i + 1) if 0 <= j < nc]
        if len(nb) == 2:
            u = -((nb[0] - C[i]) / cc + (nb[1] - C[i]) / cc)
            u /= np.linalg.norm(u)
            a = TETRA / 2
            H += [C[i] + ch * (np.cos(a) * u + np.sin(a) * ez), C[i] + ch * (np.cos(a) * u - np.sin(a) * ez)]
        else:
            # terminal CH3: the in-plane H sits where the next zigzag carbon would be
            j = 1 if i == 0 else nc - 2
            step = C[1] - C[0] if i == 0 else C[nc - 1] - C[nc - 2]
            virtual = C[j] - 2 * np.array([step[0], 0.0, 0.0]) if i == 0 else C[j] + 2 * np.array([step[0], 0.0, 0.0])
            b = C[j] - C[i]
            for d in _tetra_dirs(b, virtual - C[i]):
                H.append(C[i] + ch * d)
    xyz = np.vstack([C, np.array(H)])
    xyz -= xyz.mean(axis=0)
    if rng is not None:
        xyz = xyz @ random_rotation(rng).T
    return [6] * nc + [1] * len(H), xyz


def methane(rng=None):
    d = np.array([[1, 1, 1], [1, -1, -1], [-1, 1, -1], [-1, -1, 1]], dtype=float) / np.sqrt(3)
    xyz = np.vstack([[0, 0, 0], 1.09 * d])
    return [6, 1, 1, 1, 1], xyz


def ammonia(rng=None):
    r, hnh = 1.012, np.deg2rad(106.7)
    # pyramid: H at angle t from the C3 axis with H-N-H = hnh
    t = np.arcsin(np.sin(hnh / 2) / np.sin(np.pi / 3))
    H = [[r * np.sin(t) * np.cos(p), r * np.sin(t) * np.sin(p), -r * np.cos(t)]
         for p in (0, 2 * np.pi / 3, 4 * np.pi / 3)]
    return [7, 1, 1, 1], np.vstack([[0, 0, 0], H])


def ethane(rng=None):
    return n_alkane(2)


def anthracene(rng=None):
    """C14H10: regular hexagons (C-C 1.40 A), C-H 1.08 A, planar in xy."""
    cc, ch = 1.40, 1.08
    dx = 2 * cc * np.cos(np.pi / 6)
    C = []
    for cx in (-dx, 0.0, dx):
        for k in range(6):
            a = np.pi / 6 + k * np.pi / 3
            p = np.array([cx + cc * np.cos(a), cc * np.sin(a), 0.0])
            if not any(np.linalg.norm(p - q) < 1e-6 for q in C):
                C.append(p)
    C = np.array(C)
    H = []
    for i, p in enumerate(C):
        nb = [q for q in C if 0 < np.linalg.norm(q - p) < cc + 1e-6]
        if len(nb) == 2:
            u = p - 0.5 * (nb[0] + nb[1])
            H.append(p + ch * u / np.linalg.norm(u))
    return [6] * len(C) + [1] * len(H), np.vstack([C, np.array(H)])


def water_cluster(n: int, spacing: float, rng, sigma: float):
    """n rigid waters on a 2x2x2 cubic lattice (first n sites), seeded orientation and displacement."""
    sites = [np.array([i, j, k], dtype=float) * spacing for i in (0, 1) for j in (0, 1) for k in (0, 1)]
    Z, xyz = [], []
    for m in range(n):
        z, w = water(rng, orient=True)
        w = w + sites[m] + rng.normal(scale=sigma, size=3)
        Z += z
        xyz.append(w)
    return Z, np.vstack(xyz)


def _jitter(xyz, rng, sigma):
    return xyz + rng.normal(scale=sigma, size=xyz.shape)


def workload(index: int):
    """(Z, coords_bohr, basis, pure) of workload 1..4."""
    rng = np.random.default_rng(SEED_BASE + index)
    if index == 1:
        Z, xyz = h2o_ccpvdz()
        return Z, xyz, "cc-pvdz", True
    if index == 2:
        Z, xyz = n_alkane(8, rng)
        return Z, xyz * A2B, "6-31g**", False
    if index == 3:
        Z, xyz = anthracene()
        return Z, _jitter(xyz, rng, 0.01) * A2B, "cc-pvdz", True
    if index == 4:
        Z, xyz = water_cluster(8, 2.9, rng, 0.1)
        return Z, xyz * A2B, "6-31g*", False
    raise ValueError(index)


def batch_molecules(count: int = 512, seed: int = SEED_BASE + 5):
    """Seeded mix of (H2O)n (n=1..6, 3.0 A lattice), CH4, C2H6 and NH3 with 0.05 A jitter,
    each in STO-3G or 6-31G* (50/50).  Returns a list of (Z, coords_bohr, basis, pure)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        kind = int(rng.integers(0, 9))
        if kind < 6:
            Z, xyz = water_cluster(kind + 1, 3.0, rng, 0.0)
        elif kind == 6:
            Z, xyz = methane()
        elif kind == 7:
            Z, xyz = ethane()
        else:
            Z, xyz = ammonia()
        xyz = _jitter(np.asarray(xyz, dtype=float), rng, 0.05)
        basis = "sto-3g" if rng.random() < 0.5 else "6-31g*"
        out.append((Z, xyz * A2B, basis, basis == "sto-3g"))
    return out
