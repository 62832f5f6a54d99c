"""CPU tests of the oracle: the C restatement against the reference's own code
(oracle/_ref, when the reference sources were present at build time) and against
the committed golden fixtures."""
import os

import numpy as np
import pytest

import oracle
from hfscf_b200 import basis as B
from hfscf_b200 import molecules as M
from hfscf_b200 import engine as E

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="reference library not built here")


def _gold(name):
    g = np.load(os.path.join(GOLD, name), allow_pickle=False)
    return B.build_basis(str(g["basis"]), g["Z"], g["coords"], pure=bool(g["pure"])), g


@pytest.mark.parametrize("fixture", ["h2o_ccpvdz_eri.npz", "ch4_ccpvdz_eri.npz"])
def test_oracle_eris_match_golden(fixture):
    bs, g = _gold(fixture)
    assert np.max(np.abs(oracle.eri_packed(bs) - g["eri"])) < 1e-13


def test_oracle_grad2e_matches_golden():
    bs, g = _gold("h2o_631gs_grad2e.npz")
    assert np.max(np.abs(oracle.grad2e_rhf(bs, g["D"]) - g["grad"])) < 1e-12


@needs_ref
@pytest.mark.parametrize("name,pure", [("6-31g**", False), ("6-31g*", True), ("sto-3g", True)])
def test_oracle_eris_match_reference(name, pure):
    Z, x = M.water(np.random.default_rng(3))
    bs = B.build_basis(name, Z, np.asarray(x) * B.ANGSTROM_TO_BOHR, pure=pure)
    assert np.max(np.abs(oracle.eri_packed(bs) - oracle.ref_eri_packed(bs))) < 1e-13


@needs_ref
def test_oracle_grad2e_matches_reference_deriv_tensors():
    Z, x = M.water(np.random.default_rng(4))
    bs = B.build_basis("cc-pvdz", Z, np.asarray(x) * B.ANGSTROM_TO_BOHR, pure=True)
    rng = np.random.default_rng(1)
    A = rng.normal(size=(bs.nbf, bs.nbf))
    D = (A + A.T) / bs.nbf
    g_ref = oracle.grad2e_from_deriv1(oracle.ref_deriv1(bs), bs.bf_atom(), bs.natoms, D)
    assert np.max(np.abs(oracle.grad2e_rhf(bs, D) - g_ref)) < 1e-12


@needs_ref
def test_oracle_pieces_match_reference():
    for L in range(4):
        assert np.max(np.abs(oracle.ylm(L) - oracle.ref_ylm(L))) < 1e-15
    for m in range(12):
        for T in (1e-7, 0.05, 0.7, 3.3, 11.0, 29.5, 36.5, 80.0, 500.0):
            r = oracle.ref_boys(m, T)
            assert abs(oracle.boys(m, T) - r) <= 1e-13 * r
    rng = np.random.default_rng(0)
    for L in range(3):
        a = np.sort(rng.uniform(0.1, 50, size=4))[::-1]
        c = rng.uniform(-1, 1, size=4)
        assert np.allclose(oracle.shell_norm(L, a, c), oracle.ref_shell_coefs(L, a, c), rtol=1e-14, atol=0)


def test_boys_against_high_precision_series():
    """Oracle Boys values against an independent mpmath evaluation (50 digits).
    T starts at 1e-6: below 1e-8 the oracle keeps the reference's clamp of T
    (src/math/gamma.cpp:20-21)."""
    mp = pytest.importorskip("mpmath")
    mp.mp.dps = 50
    for m in (0, 3, 8, 13):
        for T in (1e-6, 0.4, 2.5, 9.0, 20.0, 35.9, 60.0):
            exact = mp.quad(lambda t: t ** (2 * m) * mp.e ** (-T * t * t), [0, 1])
            assert abs(oracle.boys(m, T) - float(exact)) <= 2e-14 * float(exact) + 1e-300


def test_packed_index_and_unpack_roundtrip():
    n = 5
    r = np.arange(n)
    i, j, k, l = np.meshgrid(r, r, r, r, indexing="ij")
    idx = oracle.index_ijkl(i, j, k, l)
    assert idx.max() == oracle.packed_len(n) - 1
    # 8-fold symmetry
    assert np.array_equal(idx, oracle.index_ijkl(j, i, k, l))
    assert np.array_equal(idx, oracle.index_ijkl(k, l, i, j))
    assert len(np.unique(idx)) == oracle.packed_len(n)


@pytest.mark.parametrize("name,pure", [("6-31g**", False), ("cc-pvdz", True), ("sto-3g", False)])
def test_host_one_electron_matches_reference(name, pure):
    """Host S, T, V and one-electron gradient against the reference's own one-electron
    routines (hfscf_osoverlap.cpp, hfscf_osnuclear.cpp and their _deriv1 forms)."""
    if not oracle.ref_available():
        pytest.skip("reference library not built")
    rng = np.random.default_rng(13)
    Z, x = M.water(rng)
    bs = B.build_basis(name, Z, np.asarray(x) * B.ANGSTROM_TO_BOHR, pure=pure)
    S0, T0, V0 = oracle.ref_onee(bs)
    S, T, V = E.one_electron(bs)
    assert max(np.abs(S - S0).max(), np.abs(T - T0).max(), np.abs(V - V0).max()) < 1e-12
    n = bs.nbf
    A = rng.normal(size=(n, n))
    D = (A + A.T) / n
    A = rng.normal(size=(n, n))
    Q = (A + A.T) / n
    g0 = oracle.ref_onee_grad(bs, D, Q, 2.0, -2.0)
    g = E.one_electron_grad(bs, D, Q, 2.0, -2.0)
    assert np.abs(g - g0).max() < 1e-11


def test_packed_digest_matches_row_contraction():
    """or_jk_packed (one pass over the unique ERIs, used for the oracle SCF at full size)
    gives the sums of the row-by-row contraction or_jk, for symmetric and general densities."""
    rng = np.random.default_rng(41)
    Z, x = M.water(rng)
    bs = B.build_basis("6-31g**", Z, np.asarray(x) * B.ANGSTROM_TO_BOHR, pure=False)
    eri = oracle.eri_packed(bs)
    n = bs.nbf
    A = rng.normal(size=(n, n))
    Ds = [(A + A.T) / n, rng.normal(size=(n, n)) / n]
    J, K = oracle.jk_packed(eri, Ds)
    for m, D in enumerate(Ds):
        J0, K0 = oracle.jk(eri, D)
        assert np.max(np.abs(J[m] - J0)) < 1e-13 and np.max(np.abs(K[m] - K0)) < 1e-13


@needs_ref
@pytest.mark.parametrize("name,pure", [("6-31g*", False), ("cc-pvdz", True)])
def test_packed_derivative_digest_matches_restatement(name, pure):
    """The gradient contracted from the reference's nine packed derivative tensors in one
    pass (or_grad2e_from_deriv1, used for the (H2O)8 oracle gradient) equals the C
    restatement over all ordered quartets (or_grad2e), RHF and UHF weights."""
    rng = np.random.default_rng(43)
    Z, x = M.water(rng)
    bs = B.build_basis(name, Z, np.asarray(x) * B.ANGSTROM_TO_BOHR, pure=pure)
    n = bs.nbf
    sym = lambda: (lambda A: (A + A.T) / n)(rng.normal(size=(n, n)))  # noqa: E731
    D, Da, Db = sym(), sym(), sym()
    d9 = oracle.ref_deriv1(bs)
    g = oracle.grad2e_packed_deriv1(d9, bs.bf_atom(), bs.natoms, D, 2.0, [D], 1.0)
    assert np.max(np.abs(g - oracle.grad2e_rhf(bs, D))) < 1e-13
    gu = oracle.grad2e_packed_deriv1(d9, bs.bf_atom(), bs.natoms, Da + Db, 0.5, [Da, Db], 0.5)
    assert np.max(np.abs(gu - oracle.grad2e_uhf(bs, Da, Db))) < 1e-13


@needs_ref
def test_oracle_scf_converges_to_a_stationary_density():
    """The oracle RHF driver (oracle/scf.py) on the reference's own integrals of H2O/cc-pVDZ:
    converged, idempotent D S D = D with tr(DS) = nocc, and a vanishing commutator FDS - SDF."""
    from oracle import scf as OS
    Z, x, name, pure = M.workload(1)
    bs = B.build_basis(name, Z, x, pure=pure)
    S, T, V = oracle.ref_onee(bs)
    eri = oracle.ref_eri_packed(bs)
    nocc = int(sum(Z)) // 2

    def jk(D):
        J, K = oracle.jk_packed(eri, [D])
        return J[0], K[0]

    r = OS.rhf(S, T + V, nocc, jk, OS.nuclear_repulsion(Z, bs.coords))
    D, F = r["D"], r["F"]
    assert r["converged"]
    assert np.max(np.abs(D @ S @ D - D)) < 1e-12
    assert abs(np.trace(D @ S) - nocc) < 1e-12
    assert np.max(np.abs(F @ D @ S - S @ D @ F)) < 1e-7
    assert abs(OS.nuclear_repulsion(Z, bs.coords) - B.nuclear_repulsion(Z, bs.coords)) < 1e-12


@needs_ref
@pytest.mark.parametrize("name,pure", [("6-31g*", False), ("cc-pvdz", True)])
def test_sad_host_logic_matches_oracle_sad(name, pure):
    """The engine's SAD host logic (scf.sad_atom_density, scf.atom_basis, scf.sad_populations)
    driven by the C restatement's J/K, against the oracle's SAD on the reference's integrals
    (oracle/scf.py: sad_guess), for H, C and O; both atomic UHF runs converged to rms 1e-10."""
    from oracle import scf as OS
    from hfscf_b200 import scf
    Z, x = M.water_cluster(2, 2.9, np.random.default_rng(8), 0.1)
    Z = np.concatenate([Z, [6]])
    x = np.vstack([np.asarray(x), [[4.0, 4.0, 4.0]]])
    bs = B.build_basis(name, Z, x * B.ANGSTROM_TO_BOHR, pure=pure)
    n = bs.nbf
    D = np.zeros((n, n))
    bf_atom = bs.bf_atom()
    done = {}
    for a, Zc in enumerate(bs.Z):
        Zc = int(Zc)
        if Zc not in done:
            ab = scf.atom_basis(bs, a)
            S, T, V = oracle.ref_onee(ab)
            eri = oracle.eri_packed(ab)

            def jk(DJ, DKs, eri=eri):
                return oracle.jk(eri, DJ)[0], [oracle.jk(eri, Dk)[1] for Dk in DKs]

            done[Zc] = scf.sad_atom_density(Zc, S, T, V, jk, rms_tol=1e-10, e_tol=1e-12, max_iter=200)
        f = np.nonzero(bf_atom == a)[0]
        D[np.ix_(f, f)] = done[Zc]
    D0 = OS.sad_guess(bs, rms_tol=1e-10, e_tol=1e-12, max_iter=200)
    # two runs stopped at DIIS rms < 1e-10 agree to about that; threaded BLAS moves last digits
    assert np.abs(D - D0).max() < 1e-8
    assert abs(np.trace(D0 @ oracle.ref_onee(bs)[0]) - float(np.sum(Z)) / 2) < 1e-8
