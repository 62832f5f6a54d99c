"""Parity at the benchmark configurations, against an oracle SCF on the reference's own integrals.

The oracle side of every test runs on the host CPU: S, T, V and the packed ERIs from the
reference's code compiled in place (oracle/_ref), J/K from one pass over the packed ERIs
(or_jk_packed), the SCF
loop of oracle/scf.py (core guess, DIIS, the reference's convergence test), and for the
gradient the reference's nine derivative tensors contracted by or_grad2e_from_deriv1 plus the
reference's one-electron gradient routines.  The GPU side runs the engine's own SCF (scf.py).

The oracle ERIs are the reference's unscreened ones (do_screen = false).  With the reference's
default Schwarz screening (eri_screen, screen_tol 1e-12) single octane integrals move by up to
2.2e-7 and its SCF energy by 3.5e-7 Eh, so the screened vector cannot pin 1e-8; the engine's
own quartet screening (Q_ab Q_cd < 1e-12) is part of what these tests check.

Tolerances (the engine's stated targets): SCF total energy 1e-8 Eh (FP64), 1e-6 Eh (mixed
precision); J and K at the converged density 1e-10; RHF gradient 1e-7 Eh/bohr (FP64),
1e-5 Eh/bohr (mixed).  Oracle ERI generation takes seconds (octane, (H2O)8) to about a
minute (anthracene) on the host's cores.
"""
import numpy as np
import pytest

import oracle
from hfscf_b200 import basis as B
from hfscf_b200 import engine as E
from hfscf_b200 import molecules as M
from hfscf_b200 import scf

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not oracle.ref_available(), reason="reference library not built")]

E_TOL, E_TOL_MIXED = 1e-8, 1e-6
G_TOL, G_TOL_MIXED = 1e-7, 1e-5


def _workload(i):
    Z, x, name, pure = M.workload(i)
    return B.build_basis(name, Z, x, pure=pure)


def _oracle_rhf(bs, eri, rms_tol=1e-9):
    from oracle import scf as OS
    S, T, V = oracle.ref_onee(bs)

    def jk(D):
        J, K = oracle.jk_packed(eri, [D])
        return J[0], K[0]

    r = OS.rhf(S, T + V, int(sum(bs.Z)) // 2, jk, OS.nuclear_repulsion(bs.Z, bs.coords), rms_tol=rms_tol)
    assert r["converged"]
    return r


def test_octane_scf_energy_and_jk_match_oracle():
    """n-octane / 6-31G** (Cartesian d, 210 functions): FP64 SCF energy and J, K at the
    converged density."""
    bs = _workload(2)
    eri = oracle.ref_eri_packed(bs, do_screen=False)
    ref = _oracle_rhf(bs, eri)
    with E.Engine(bs) as eng:
        r = scf.rhf(bs, engine=eng, guess="sad")
        J, K = eng.jk(r.D, [r.D])
    assert r.converged
    assert abs(r.energy - ref["energy"]) < E_TOL, (r.energy, ref["energy"])
    J0, K0 = oracle.jk_packed(eri, [r.D])
    assert np.max(np.abs(J - J0[0])) < 1e-10
    assert np.max(np.abs(K[0] - K0[0])) < 1e-10


def test_anthracene_fp64_and_mixed_energies_match_oracle():
    """Anthracene / cc-pVDZ (pure d, 246 functions): the FP64 SCF energy to 1e-8 and the
    mixed-precision SCF (FP32 quartets below the Schwarz bound 1e-4, incremental Delta-D
    builds) to 1e-6, both against the oracle."""
    bs = _workload(3)
    eri = oracle.ref_eri_packed(bs, do_screen=False)
    ref = _oracle_rhf(bs, eri)
    del eri
    with E.Engine(bs) as eng:
        r64 = scf.rhf(bs, engine=eng, guess="sad")
        rmx = scf.rhf(bs, engine=eng, guess="sad", precision=E.MIXED, incremental=True)
    assert r64.converged and rmx.converged
    assert abs(r64.energy - ref["energy"]) < E_TOL, (r64.energy, ref["energy"])
    assert abs(rmx.energy - ref["energy"]) < E_TOL_MIXED, (rmx.energy, ref["energy"])


def _oracle_rhf_gradient(bs, r):
    from oracle import scf as OS
    D, F = r["D"], r["F"]
    d9 = oracle.ref_deriv1(bs)
    g = oracle.grad2e_packed_deriv1(d9, bs.bf_atom(), bs.natoms, D, 2.0, [D], 1.0)
    del d9
    g += oracle.ref_onee_grad(bs, D, D @ F @ D, 2.0, -2.0)
    g += OS.nuclear_repulsion_gradient(bs.Z, bs.coords)
    return g


def test_water_octamer_rhf_gradient_matches_oracle():
    """(H2O)8 / 6-31G* (Cartesian d, 152 functions): energy and full RHF gradient, FP64 and
    mixed precision, against the oracle SCF and the oracle gradient at its own density."""
    bs = _workload(4)
    eri = oracle.ref_eri_packed(bs, do_screen=False)
    ref = _oracle_rhf(bs, eri, rms_tol=1e-10)
    del eri
    g0 = _oracle_rhf_gradient(bs, ref)
    with E.Engine(bs) as eng:
        r64 = scf.rhf(bs, engine=eng, guess="sad", rms_tol=1e-10)
        g64 = scf.rhf_gradient(bs, r64, eng)
        rmx = scf.rhf(bs, engine=eng, guess="sad", rms_tol=1e-10, precision=E.MIXED, incremental=True)
        gmx = scf.rhf_gradient(bs, rmx, eng, E.MIXED)
    assert abs(r64.energy - ref["energy"]) < E_TOL
    assert abs(rmx.energy - ref["energy"]) < E_TOL_MIXED
    assert np.max(np.abs(g64 - g0)) < G_TOL, np.max(np.abs(g64 - g0))
    assert np.max(np.abs(gmx - g0)) < G_TOL_MIXED, np.max(np.abs(gmx - g0))


def _radical():
    """Methyl radical CH3 (planar, C-H 1.079 A) with a seeded 0.02 A jitter, 6-31G*."""
    rng = np.random.default_rng(20261209)
    r = 1.079
    xyz = np.array([[0.0, 0.0, 0.0], [r, 0.0, 0.0], [-r / 2, r * np.sqrt(3) / 2, 0.0],
                    [-r / 2, -r * np.sqrt(3) / 2, 0.0]]) + rng.normal(scale=0.02, size=(4, 3))
    return B.build_basis("6-31g*", [6, 1, 1, 1], xyz * B.ANGSTROM_TO_BOHR, pure=False)


def test_uhf_scf_and_gradient_match_oracle():
    """Open-shell UHF (doublet CH3): energy against the oracle UHF SCF, and the full UHF
    gradient at the GPU's density against the oracle's two-electron (C restatement) and
    one-electron (the reference's routines) terms at the same density."""
    from oracle import scf as OS
    bs = _radical()
    eri = oracle.ref_eri_packed(bs, do_screen=False)
    S, T, V = oracle.ref_onee(bs)

    def jk(D):
        J, K = oracle.jk_packed(eri, [D])
        return J[0], K[0]

    ref = OS.uhf(S, T + V, 5, 4, jk, OS.nuclear_repulsion(bs.Z, bs.coords))
    assert ref["converged"]
    with E.Engine(bs) as eng:
        r = scf.uhf(bs, eng, multiplicity=2)
        g = scf.uhf_gradient(bs, r, eng)
    assert r["converged"]
    assert abs(r["energy"] - ref["energy"]) < E_TOL, (r["energy"], ref["energy"])
    Da, Db, Fa, Fb = r["Da"], r["Db"], r["Fa"], r["Fb"]
    g0 = oracle.grad2e_uhf(bs, Da, Db)
    g0 += oracle.ref_onee_grad(bs, Da + Db, Da @ Fa @ Da + Db @ Fb @ Db, 1.0, -1.0)
    g0 += OS.nuclear_repulsion_gradient(bs.Z, bs.coords)
    assert np.max(np.abs(g - g0)) < 1e-10
