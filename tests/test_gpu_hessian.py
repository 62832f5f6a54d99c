"""GPU parity of the two-electron Hessian (adjoint second-derivative ERIs) against the oracle.

The oracle is the reference's own second-derivative shell routines compiled in place
(hfscf_oserideriv2qq.cpp, hfscf_oserideriv2pq.cpp) under a restatement of its contraction
driver, Mol::scf_hessian::calc_scf_hessian_tei (oracle.ref_hess2e = hessC + hessEx).

Tolerances:
  * Hessian at fixed density against the reference: 1e-9 Eh/bohr^2 absolute (entries up to
    ~1, each a sum over all quartets of second-derivative integrals times density products);
  * against central differences (h = 1e-4 bohr) of the GPU's own adjoint gradient: 1e-6;
  * symmetry and translational invariance (every row sums to zero over the atoms): 1e-10.
"""
import numpy as np
import pytest

import oracle
from hfscf_b200 import basis as B
from hfscf_b200 import engine as E
from hfscf_b200 import molecules as M

pytestmark = pytest.mark.gpu

HESS_TOL = 1e-9
FD_TOL = 1e-6


def _molecules():
    rng = np.random.default_rng(11)
    out = []
    Z, x = M.water(rng)
    x = np.asarray(x) * B.ANGSTROM_TO_BOHR + rng.normal(scale=0.05, size=(3, 3))
    out.append(("h2o-631gss-cart", B.build_basis("6-31g**", Z, x, pure=False)))
    out.append(("h2o-ccpvdz-pure", B.build_basis("cc-pvdz", Z, x, pure=True)))
    out.append(("h2o-sto3g", B.build_basis("sto-3g", Z, x)))
    Z, x = M.ammonia()
    x = np.asarray(x) * B.ANGSTROM_TO_BOHR + rng.normal(scale=0.05, size=(4, 3))
    out.append(("nh3-631gs-cart", B.build_basis("6-31g*", Z, x, pure=False)))
    out.append(("nh3-631gs-pure", B.build_basis("6-31g*", Z, x, pure=True)))
    return out


MOLS = _molecules()


def _sym(rng, n, scale=1.0):
    A = rng.normal(size=(n, n))
    return scale * (A + A.T) / n


def _ref_hessian(bs, D):
    if not oracle.ref_available():
        pytest.skip("compiled reference not built")
    hc, he = oracle.ref_hess2e(bs, D)
    return hc + he


FORMS = [(-1, "default"), (0, "thread"), (1, "block"), (2, "warp"), (3, "line")]


@pytest.mark.parametrize("form", [f for f, _ in FORMS], ids=[n for _, n in FORMS])
@pytest.mark.parametrize("name,bs", MOLS, ids=[m[0] for m in MOLS])
def test_hess2e_matches_reference(name, bs, form):
    """Every launch form (one thread per quartet on global scratch, one block or one warp per
    quartet over levelised tables, one thread per quartet on straight-line register code for the
    classes that have it, and the default mix) against the reference."""
    rng = np.random.default_rng(3)
    D = _sym(rng, bs.nbf)
    with E.Engine(bs) as eng:
        eng.set_hess_form(form)
        H = eng.hess2e(D)
    Href = _ref_hessian(bs, D)
    assert np.max(np.abs(H - Href)) < HESS_TOL, np.max(np.abs(H - Href))
    assert np.max(np.abs(H - H.T)) < 1e-10
    n3 = H.shape[0]
    # translational invariance: for each row, the sum over atoms of each direction vanishes
    rows = H.reshape(n3, -1, 3).sum(axis=1)
    assert np.max(np.abs(rows)) < 1e-10


def test_hess2e_uhf_matches_reference():
    """UHF: E2 = 1/2 [Dt J[Dt] - Da K[Da] - Db K[Db]], Dt = Da + Db, so its Hessian is
    hessC(Dt)/4 + hessEx(Da)/2 + hessEx(Db)/2 in terms of the reference's RHF Coulomb and
    exchange parts; with Da = Db = D it equals the RHF Hessian of D."""
    bs = MOLS[3][1]
    rng = np.random.default_rng(4)
    D = _sym(rng, bs.nbf)
    Da, Db = _sym(rng, bs.nbf), _sym(rng, bs.nbf)
    with E.Engine(bs) as eng:
        H = eng.hess2e(D)
        Hu = eng.hess2e_uhf(D, D)
        Hab = eng.hess2e_uhf(Da, Db)
    assert np.max(np.abs(Hu - H)) < 1e-10
    if not oracle.ref_available():
        pytest.skip("compiled reference not built")
    hc_t, _ = oracle.ref_hess2e(bs, Da + Db)
    _, he_a = oracle.ref_hess2e(bs, Da)
    _, he_b = oracle.ref_hess2e(bs, Db)
    Href = 0.25 * hc_t + 0.5 * he_a + 0.5 * he_b
    assert np.max(np.abs(Hab - Href)) < HESS_TOL, np.max(np.abs(Hab - Href))


def test_hess2e_uhf_central_differences():
    """UHF Hessian vs central differences of the UHF adjoint gradient at fixed Da, Db."""
    bs0 = MOLS[0][1]
    rng = np.random.default_rng(6)
    Da, Db = _sym(rng, bs0.nbf, 0.5), _sym(rng, bs0.nbf, 0.5)
    h = 1e-4
    with E.Engine(bs0, density_tol=0.0) as eng:
        H = eng.hess2e_uhf(Da, Db)
        fd = np.zeros_like(H)
        for a in range(bs0.natoms):
            for d in range(3):
                x = bs0.coords.copy()
                x[a, d] += h
                eng.set_geometry(x)
                gp = eng.grad2e_uhf(Da, Db)
                x[a, d] -= 2 * h
                eng.set_geometry(x)
                gm = eng.grad2e_uhf(Da, Db)
                fd[3 * a + d] = ((gp - gm) / (2 * h)).ravel()
    assert np.max(np.abs(H - fd)) < FD_TOL, np.max(np.abs(H - fd))


def test_hess2e_central_differences_large_molecule():
    """n-dodecane in STO-3G, 38 atoms: more than the per-block shared-memory Hessian holds, so
    the kernels add straight into the output.  Selected rows against central differences of
    the adjoint gradient; symmetry and translational invariance of every row."""
    rng = np.random.default_rng(21)
    Z, x = M.n_alkane(12, rng)
    bs = B.build_basis("sto-3g", Z, np.asarray(x) * B.ANGSTROM_TO_BOHR)
    assert bs.natoms > 36
    D = _sym(rng, bs.nbf, 0.2)
    h = 1e-4
    with E.Engine(bs, density_tol=0.0) as eng:
        H = eng.hess2e(D)
        for a, d in ((0, 0), (7, 1), (bs.natoms - 1, 2)):
            xx = bs.coords.copy()
            xx[a, d] += h
            eng.set_geometry(xx)
            gp = eng.grad2e(D)
            xx[a, d] -= 2 * h
            eng.set_geometry(xx)
            gm = eng.grad2e(D)
            row = ((gp - gm) / (2 * h)).ravel()
            assert np.max(np.abs(H[3 * a + d] - row)) < FD_TOL
            eng.set_geometry(bs.coords)
    n3 = H.shape[0]
    assert np.max(np.abs(H.reshape(n3, -1, 3).sum(axis=1))) < 1e-10
    assert np.max(np.abs(H - H.T)) < 1e-10


def test_hess2e_rejects_batched_handles():
    from hfscf_b200 import batch
    Z, x = M.water(np.random.default_rng(1))
    bs = B.build_basis("sto-3g", Z, np.asarray(x) * B.ANGSTROM_TO_BOHR, pure=False)
    be = batch.BatchEngine([bs, bs])
    try:
        n = 2 * bs.nbf
        H = np.zeros((18, 18))
        rc = E.lib().hfgpu_hess2e(be.h, E._p(np.zeros((n, n))), E.ctypes.c_double(1.0), E._p(H))
        assert rc == 6  # HFGPU_ERR_UNSUPPORTED
        assert not H.any()
    finally:
        be.close()


def test_hess2e_autotuned_forms_match_default():
    """hfgpu_autotune_hess times every class in each form it has (the straight-line form only
    where the class has one) and keeps the fastest; the Hessian with the chosen forms equals the
    default one to rounding, and a form set per class through hfgpu_set_hess_forms is reapplied."""
    Z, x = M.water_cluster(2, 2.9, np.random.default_rng(5), 0.1)
    bs = B.build_basis("6-31g*", Z, np.asarray(x) * B.ANGSTROM_TO_BOHR, pure=False)
    rng = np.random.default_rng(8)
    D = _sym(rng, bs.nbf, 0.3)
    # class order of a handle: (ss|ss), (ps|ss), (ps|ps), (pp|ss), (pp|ps), (pp|pp), (ds|ss),
    # (ds|ps), (ds|pp), (ds|ds), (dp|ss), ...; the classes with a straight-line form are
    # (ss|ss), (ps|ss), (ps|ps), (pp|ss), (pp|ps), (ds|ss), (ds|ps) and (dp|ss)
    line_classes = {0, 1, 2, 3, 4, 6, 7, 10}
    with E.Engine(bs, density_tol=0.0) as eng:
        H0 = eng.hess2e(D)
        forms = eng.autotune_hess(D, repeats=1)
        H1 = eng.hess2e(D)
        eng.set_hess_forms([3 if f == 3 else 1 for f in forms])
        H2 = eng.hess2e(D)
    assert len(forms) == E.NUM_CLASSES
    assert all(f in (0, 1, 2, 3) for f in forms)
    assert all(c in line_classes for c, f in enumerate(forms) if f == 3)
    assert np.max(np.abs(H1 - H0)) < 1e-11
    assert np.max(np.abs(H2 - H0)) < 1e-11
