"""Gaussian basis sets and shell lists, laid out as hfscf lays them out.

Shell order, offsets and the Cartesian/pure choice follow the reference:
  * atoms in input order; inside an atom, the .gbs shell order with SP split
    into S then P (src/basis/hfscf_basis.cpp:175-184, 244-274);
  * per-shell Cartesian offset ``idx`` and pure offset ``ids`` accumulate over
    all shells (src/basis/hfscf_basis.cpp:265-270);
  * the .gbs header picks cartesian/spherical, and ``pure`` overrides it
    (src/basis/hfscf_basis.cpp:53-60, src/molecule/hfscf_molecule.cpp:671-679).

Contraction coefficients are handed to the engine UNNORMALISED, exactly as read
from the basis file; the engine normalises them the way BASIS::Shell's
constructor does (src/integrals/hfscf_shell.cpp:44-54).
"""
from __future__ import annotations

import json
import os
from dataclasses import dataclass, field

import numpy as np

ANGSTROM_TO_BOHR = 1.8897261254535  # src/molecule/hfscf_constants.hpp:5
SYMBOL_TO_Z = {"H": 1, "He": 2, "C": 6, "N": 7, "O": 8}
Z_TO_SYMBOL = {v: k for k, v in SYMBOL_TO_Z.items()}

_DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "basis_data")
_ALIASES = {"sto-3g": "sto-3g", "6-31g*": "6-31gs", "6-31g(d)": "6-31gs",
            "6-31g**": "6-31gss", "6-31g(d,p)": "6-31gss", "cc-pvdz": "cc-pvdz"}


def ncart(L: int) -> int:
    return (L + 1) * (L + 2) // 2


def npure(L: int) -> int:
    return 2 * L + 1


def load_basis_table(name: str) -> dict:
    key = _ALIASES[name.lower()]
    with open(os.path.join(_DATA, key + ".json")) as f:
        return json.load(f)


@dataclass
class Shell:
    L: int
    atom: int
    center: np.ndarray
    exps: np.ndarray
    coefs: np.ndarray  # unnormalised, as in the basis file
    idx: int  # first Cartesian function
    ids: int  # first pure function


@dataclass
class Basis:
    """Shell list of one molecule in one basis set."""
    name: str
    pure: bool
    Z: np.ndarray
    coords: np.ndarray  # bohr, natoms x 3
    shells: list = field(default_factory=list)

    @property
    def nshell(self) -> int:
        return len(self.shells)

    @property
    def natoms(self) -> int:
        return len(self.Z)

    @property
    def ncart(self) -> int:
        return sum(ncart(s.L) for s in self.shells)

    @property
    def npure(self) -> int:
        return sum(npure(s.L) for s in self.shells)

    @property
    def nbf(self) -> int:
        return self.npure if self.pure else self.ncart

    @property
    def max_L(self) -> int:
        return max(s.L for s in self.shells)

    def shell_offsets(self) -> np.ndarray:
        return np.array([s.ids if self.pure else s.idx for s in self.shells], dtype=np.int64)

    def bf_atom(self) -> np.ndarray:
        """Atom index of every basis function."""
        out = []
        for s in self.shells:
            out += [s.atom] * (npure(s.L) if self.pure else ncart(s.L))
        return np.array(out, dtype=np.int64)

    def flat(self) -> dict:
        """Flat arrays in the layout the C ABI takes (hfgpu_basis)."""
        return {
            "L": np.array([s.L for s in self.shells], dtype=np.int32),
            "atom": np.array([s.atom for s in self.shells], dtype=np.int32),
            "nprim": np.array([len(s.exps) for s in self.shells], dtype=np.int32),
            "exps": np.concatenate([s.exps for s in self.shells]).astype(np.float64),
            "coefs": np.concatenate([s.coefs for s in self.shells]).astype(np.float64),
            "centers": np.array([s.center for s in self.shells], dtype=np.float64).reshape(-1, 3),
        }

    def with_coords(self, coords) -> "Basis":
        """The same shells on the atoms moved to `coords` (bohr)."""
        coords = np.asarray(coords, dtype=np.float64).reshape(-1, 3)
        out = Basis(self.name, self.pure, self.Z, coords)
        out.shells = [Shell(s.L, s.atom, coords[s.atom].copy(), s.exps, s.coefs, s.idx, s.ids) for s in self.shells]
        return out


def build_basis(name: str, Z, coords_bohr, pure: bool | None = None) -> Basis:
    table = load_basis_table(name)
    if pure is None:
        pure = table["coord_type"] != "cartesian"
    Z = np.asarray(Z, dtype=np.int64)
    coords = np.asarray(coords_bohr, dtype=np.float64).reshape(-1, 3)
    b = Basis(name=name, pure=bool(pure), Z=Z, coords=coords)
    idx = ids = 0
    for a, z in enumerate(Z):
        for sh in table["elements"][Z_TO_SYMBOL[int(z)]]:
            L = int(sh["L"])
            b.shells.append(Shell(L=L, atom=a, center=coords[a].copy(),
                                  exps=np.array(sh["exps"], dtype=np.float64),
                                  coefs=np.array(sh["coefs"], dtype=np.float64),
                                  idx=idx, ids=ids))
            idx += ncart(L)
            ids += npure(L)
    return b


def nuclear_repulsion(Z, coords) -> float:
    """sum_{a > b} Z_a Z_b / |R_a - R_b| (all pairs at once)."""
    Z = np.asarray(Z, dtype=np.float64)
    c = np.asarray(coords, dtype=np.float64)
    if len(Z) < 2:
        return 0.0
    i, j = np.tril_indices(len(Z), -1)
    r = np.sqrt(((c[i] - c[j]) ** 2).sum(axis=1))
    return float(np.sum(Z[i] * Z[j] / r))


def nuclear_repulsion_gradient(Z, coords) -> np.ndarray:
    """d/dR_a of the nuclear repulsion: -sum_{b != a} Z_a Z_b (R_a - R_b) / |R_a - R_b|^3."""
    Z = np.asarray(Z, dtype=np.float64)
    c = np.asarray(coords, dtype=np.float64)
    d = c[:, None, :] - c[None, :, :]
    r = np.sqrt((d * d).sum(axis=2))
    np.fill_diagonal(r, np.inf)
    return -np.sum((Z[:, None] * Z[None, :] / r ** 3)[:, :, None] * d, axis=1)
