"""GPU parity of the two-electron engine against the oracle and the golden fixtures.

Tolerances (from the engine's stated targets):
  * ERIs: 1e-11 absolute (FP64);
  * J, K and Fock matrices: 1e-10 absolute (sums of up to ~1e5 ERI x density terms);
  * two-electron gradient at fixed density: 1e-10 absolute;
  * SCF total energy vs the oracle SCF: 1e-8 Eh; RHF gradient: 1e-7 Eh/bohr.
"""
import os

import numpy as np
import pytest

import oracle
from hfscf_b200 import basis as B
from hfscf_b200 import engine as E
from hfscf_b200 import molecules as M
from hfscf_b200 import scf

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
pytestmark = pytest.mark.gpu

ERI_TOL = 1e-11
MAT_TOL = 1e-10


def _golden_basis(name):
    g = np.load(os.path.join(GOLD, name), allow_pickle=False)
    return B.build_basis(str(g["basis"]), g["Z"], g["coords"], pure=bool(g["pure"])), g


def _small_molecules():
    rng = np.random.default_rng(7)
    out = []
    Z, x = M.water(rng)
    out.append(("h2o-631gss-cart", B.build_basis("6-31g**", Z, np.asarray(x) * B.ANGSTROM_TO_BOHR, pure=False)))
    Z, x = M.ammonia()
    x = np.asarray(x) * B.ANGSTROM_TO_BOHR + rng.normal(scale=0.05, size=(4, 3))
    out.append(("nh3-631gs-cart", B.build_basis("6-31g*", Z, x, pure=False)))
    out.append(("nh3-631gs-pure", B.build_basis("6-31g*", Z, x, pure=True)))
    Z, x = M.water(rng)
    out.append(("h2o-sto3g", B.build_basis("sto-3g", Z, np.asarray(x) * B.ANGSTROM_TO_BOHR)))
    Z, x = M.methane()
    x = np.asarray(x) * B.ANGSTROM_TO_BOHR + rng.normal(scale=0.05, size=(5, 3))
    out.append(("ch4-ccpvdz-pure", B.build_basis("cc-pvdz", Z, x, pure=True)))
    return out


SMALL = _small_molecules()


def _sym(rng, n, scale=1.0):
    A = rng.normal(size=(n, n))
    return scale * (A + A.T) / n


@pytest.mark.parametrize("fixture", ["h2o_ccpvdz_eri.npz", "ch4_ccpvdz_eri.npz"])
def test_packed_eris_match_reference_golden(fixture):
    bs, g = _golden_basis(fixture)
    with E.Engine(bs) as eng:
        eri = eng.eri_packed()
    assert np.max(np.abs(eri - g["eri"])) < ERI_TOL


@pytest.mark.parametrize("name,bs", SMALL, ids=[s[0] for s in SMALL])
def test_packed_eris_match_oracle(name, bs):
    ref = oracle.eri_packed(bs)
    with E.Engine(bs) as eng:
        eri = eng.eri_packed()
    assert np.max(np.abs(eri - ref)) < ERI_TOL


@pytest.mark.parametrize("name,bs", SMALL, ids=[s[0] for s in SMALL])
def test_jk_and_fock_match_oracle(name, bs):
    rng = np.random.default_rng(11)
    n = bs.nbf
    eri = oracle.eri_packed(bs)
    D, H = _sym(rng, n), _sym(rng, n)
    J0, K0 = oracle.jk(eri, D)
    with E.Engine(bs, density_tol=0.0) as eng:
        J, K = eng.jk(D, [D])
        F = eng.fock_rhf(D, H)
        Da, Db = _sym(rng, n), _sym(rng, n)
        Fa, Fb = eng.fock_uhf(Da, Db, H)
    assert np.max(np.abs(J - J0)) < MAT_TOL
    assert np.max(np.abs(K[0] - K0)) < MAT_TOL
    assert np.max(np.abs(F - oracle.fock_rhf(eri, D, H))) < MAT_TOL
    Fa0, Fb0 = oracle.fock_uhf(eri, Da, Db, H)
    assert np.max(np.abs(Fa - Fa0)) < MAT_TOL and np.max(np.abs(Fb - Fb0)) < MAT_TOL


@pytest.mark.parametrize("warp_max", [-1, 1 << 30], ids=["thread-per-quartet", "warp-per-quartet"])
@pytest.mark.parametrize("idx", [0, 4], ids=["h2o-631gss-cart", "ch4-ccpvdz-pure"])
def test_large_classes_both_kernel_forms_match_oracle(warp_max, idx):
    """The large classes have a thread-per-quartet and a warp-per-quartet kernel;
    each is forced in turn and checked (ERIs, J, K)."""
    name, bs = SMALL[idx]
    rng = np.random.default_rng(17)
    D = _sym(rng, bs.nbf)
    eri0 = oracle.eri_packed(bs)
    J0, K0 = oracle.jk(eri0, D)
    with E.Engine(bs, density_tol=0.0, warp_max_quartets=warp_max) as eng:
        eri = eng.eri_packed()
        J, K = eng.jk(D, [D])
    assert np.max(np.abs(eri - eri0)) < ERI_TOL
    assert np.max(np.abs(J - J0)) < MAT_TOL and np.max(np.abs(K[0] - K0)) < MAT_TOL


def test_density_screened_jk_stays_within_threshold():
    bs = SMALL[0][1]
    rng = np.random.default_rng(3)
    D = _sym(rng, bs.nbf, 1e-3)
    with E.Engine(bs, density_tol=0.0) as e0, E.Engine(bs, density_tol=1e-12) as e1:
        J0, K0 = e0.jk(D, [D])
        J1, K1 = e1.jk(D, [D])
    assert np.max(np.abs(J1 - J0)) < 1e-9 and np.max(np.abs(K1[0] - K0[0])) < 1e-9


def test_grad2e_matches_reference_golden():
    bs, g = _golden_basis("h2o_631gs_grad2e.npz")
    with E.Engine(bs) as eng:
        grad = eng.grad2e(g["D"])
    assert np.max(np.abs(grad - g["grad"])) < MAT_TOL


@pytest.mark.parametrize("name,bs", SMALL, ids=[s[0] for s in SMALL])
def test_grad2e_matches_oracle(name, bs):
    rng = np.random.default_rng(5)
    n = bs.nbf
    D, Da, Db = _sym(rng, n), _sym(rng, n), _sym(rng, n)
    with E.Engine(bs) as eng:
        g = eng.grad2e(D)
        gu = eng.grad2e_uhf(Da, Db)
    assert np.max(np.abs(g - oracle.grad2e_rhf(bs, D))) < MAT_TOL
    assert np.max(np.abs(gu - oracle.grad2e_uhf(bs, Da, Db))) < MAT_TOL
    assert np.max(np.abs(g.sum(axis=0))) < 1e-10  # translational invariance


def test_grad2e_central_differences():
    """Adjoint gradient vs central finite differences of E2 at fixed D (h = 1e-4 bohr)."""
    bs = SMALL[1][1]
    rng = np.random.default_rng(9)
    D = _sym(rng, bs.nbf, 0.5)
    h = 1e-4
    with E.Engine(bs, density_tol=0.0) as eng:
        g = eng.grad2e(D)
        fd = np.zeros_like(g)
        for a in range(bs.natoms):
            for d in range(3):
                x = bs.coords.copy()
                x[a, d] += h
                eng.set_geometry(x)
                ep = eng.energy2e(D)
                x[a, d] -= 2 * h
                eng.set_geometry(x)
                em = eng.energy2e(D)
                fd[a, d] = (ep - em) / (2 * h)
    assert np.max(np.abs(g - fd)) < 1e-6


def _oracle_scf(bs):
    eri = oracle.eri_packed(bs)
    return scf.rhf(bs, fock=lambda D, H: oracle.fock_rhf(eri, D, H))


def test_scf_energy_h2o_ccpvdz_matches_oracle():
    Z, x, name, pure = M.workload(1)
    bs = B.build_basis(name, Z, x, pure=pure)
    ref = _oracle_scf(bs)
    with E.Engine(bs) as eng:
        r = scf.rhf(bs, engine=eng)
    assert r.converged and ref.converged
    assert abs(r.energy - ref.energy) < 1e-8


def test_mixed_precision_energy_within_budget():
    Z, x = M.water_cluster(2, 2.9, np.random.default_rng(1), 0.1)
    bs = B.build_basis("6-31g*", Z, np.asarray(x) * B.ANGSTROM_TO_BOHR, pure=False)
    with E.Engine(bs) as eng:
        r64 = scf.rhf(bs, engine=eng)
        rmx = scf.rhf(bs, engine=eng, precision=E.MIXED)
    assert abs(rmx.energy - r64.energy) < 1e-6


def test_incremental_fock_energy_matches_full():
    Z, x = M.water_cluster(2, 2.9, np.random.default_rng(2), 0.1)
    bs = B.build_basis("6-31g*", Z, np.asarray(x) * B.ANGSTROM_TO_BOHR, pure=False)
    with E.Engine(bs) as eng:
        r0 = scf.rhf(bs, engine=eng)
        r1 = scf.rhf(bs, engine=eng, incremental=True)
    assert abs(r1.energy - r0.energy) < 1e-8


def test_rhf_gradient_central_differences():
    """Full RHF gradient vs central differences of the SCF energy (h = 1e-4 bohr)."""
    rng = np.random.default_rng(4)
    Z, x = M.water(rng)
    x = np.asarray(x) * B.ANGSTROM_TO_BOHR
    bs = B.build_basis("6-31g*", Z, x, pure=False)
    h = 1e-4
    with E.Engine(bs) as eng:
        r = scf.rhf(bs, engine=eng, e_tol=1e-12, rms_tol=1e-10)
        g = scf.rhf_gradient(bs, r, eng)
        fd = np.zeros_like(g)
        for a in range(bs.natoms):
            for d in range(3):
                e = []
                for s in (1, -1):
                    xx = x.copy()
                    xx[a, d] += s * h
                    b2 = bs.with_coords(xx)
                    eng.set_geometry(xx)
                    e.append(scf.rhf(b2, engine=eng, e_tol=1e-12, rms_tol=1e-10).energy)
                fd[a, d] = (e[0] - e[1]) / (2 * h)
    assert np.max(np.abs(g - fd)) < 1e-5
    assert np.max(np.abs(g.sum(axis=0))) < 1e-8


def test_grad2e_large_molecule_fd_and_invariance():
    """(H2O)8/6-31G* (152 functions): every gradient class runs at production sizes,
    including the table-mode classes with many quartets; checked against central
    differences of E2 for a few coordinates and against translational invariance."""
    Z, x, name, pure = M.workload(4)
    bs = B.build_basis(name, Z, x, pure=pure)
    rng = np.random.default_rng(12)
    D = _sym(rng, bs.nbf, 0.3)
    h = 1e-4
    with E.Engine(bs, density_tol=0.0) as eng:
        g = eng.grad2e(D)
        gm = eng.grad2e(D, precision=E.MIXED)
        assert np.max(np.abs(g.sum(axis=0))) < 1e-9
        assert np.max(np.abs(gm - g)) < 1e-5
        for a, d in ((0, 0), (5, 1), (17, 2)):
            vals = []
            for s in (1, -1):
                xx = bs.coords.copy()
                xx[a, d] += s * h
                eng.set_geometry(xx)
                vals.append(eng.energy2e(D))
            assert abs((vals[0] - vals[1]) / (2 * h) - g[a, d]) < 1e-6


def test_autograd_function_matches_adjoint_gradient():
    import torch

    from hfscf_b200.autograd import two_electron_energy
    bs = SMALL[0][1]
    rng = np.random.default_rng(31)
    D = _sym(rng, bs.nbf, 0.4)
    with E.Engine(bs) as eng:
        R = torch.tensor(bs.coords, dtype=torch.float64, requires_grad=True)
        e = two_electron_energy(R, torch.from_numpy(D), eng)
        (3.0 * e).backward()
        assert abs(float(e) - eng.energy2e(D)) < 1e-12
        assert np.max(np.abs(R.grad.numpy() - 3.0 * eng.grad2e(D))) < 1e-12


def _random_shells(seed, pure):
    """Three centres with s, p and d shells of random exponents (0.05..60) and contraction
    lengths 1..9, so that every one of the 21 quartet classes appears with long contractions."""
    rng = np.random.default_rng(seed)
    xyz = rng.normal(scale=1.2, size=(3, 3))
    bs = B.Basis("random", pure, np.array([1, 1, 1]), xyz)
    idx = ids = 0
    for atom in range(3):
        for L in (0, 1, 2, 0):
            k = int(rng.integers(1, 10))
            exps = np.sort(np.exp(rng.uniform(np.log(0.05), np.log(60.0), size=k)))[::-1]
            coefs = rng.uniform(0.1, 1.0, size=k) * rng.choice([-1.0, 1.0], size=k)
            bs.shells.append(B.Shell(L, atom, xyz[atom], exps, coefs, idx, ids))
            idx += B.ncart(L)
            ids += B.npure(L)
    return bs


@pytest.mark.skipif(not oracle.ref_available(), reason="reference library not built")
@pytest.mark.parametrize("pure", [False, True], ids=["cartesian", "pure"])
@pytest.mark.parametrize("seed", [101, 202])
def test_random_shells_every_class_matches_compiled_reference(seed, pure):
    """Per-class ERI parity against the reference's own Erios (compiled in place, not the
    restatement): random shells with contraction lengths up to 9 on three centres, every
    unique ERI to 1e-11 absolute (relative to the largest integral, which is O(1))."""
    bs = _random_shells(seed, pure)
    ref = oracle.ref_eri_packed(bs)
    with E.Engine(bs, schwarz_tol=0.0) as eng:
        eri = eng.eri_packed()
    scale = max(1.0, float(np.max(np.abs(ref))))
    assert np.max(np.abs(eri - ref)) < ERI_TOL * scale
