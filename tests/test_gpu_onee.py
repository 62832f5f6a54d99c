"""One-electron integrals and gradient on the GPU against the reference's own
one-electron routines (oracle/_ref: hfscf_osoverlap.cpp, hfscf_osnuclear.cpp and
their _deriv1 forms, with the per-atom assembly of hfscf_grad_ints.cpp).

Tolerances: S, T, V 1e-12 absolute; gradient 1e-11 absolute (FP64 throughout).
"""
import numpy as np
import pytest

import oracle
from hfscf_b200 import basis as B
from hfscf_b200 import batch as BT
from hfscf_b200 import engine as E
from hfscf_b200 import molecules as M

pytestmark = pytest.mark.gpu


def _mols():
    rng = np.random.default_rng(41)
    out = []
    Z, x = M.water(rng)
    out.append(("h2o-631gss-cart", B.build_basis("6-31g**", Z, np.asarray(x) * B.ANGSTROM_TO_BOHR, pure=False)))
    Z, x = M.ammonia()
    x = np.asarray(x) * B.ANGSTROM_TO_BOHR + rng.normal(scale=0.05, size=(4, 3))
    out.append(("nh3-631gs-pure", B.build_basis("6-31g*", Z, x, pure=True)))
    Z, x = M.methane()
    x = np.asarray(x) * B.ANGSTROM_TO_BOHR + rng.normal(scale=0.05, size=(5, 3))
    out.append(("ch4-ccpvdz-pure", B.build_basis("cc-pvdz", Z, x, pure=True)))
    Z, x = M.water(rng)
    out.append(("h2o-sto3g", B.build_basis("sto-3g", Z, np.asarray(x) * B.ANGSTROM_TO_BOHR, pure=False)))
    return out


MOLS = _mols()


@pytest.mark.parametrize("name,bs", MOLS, ids=[m[0] for m in MOLS])
def test_one_electron_matrices_match_reference(name, bs):
    S0, T0, V0 = oracle.ref_onee(bs)
    with E.Engine(bs) as eng:
        S, T, V = eng.one_electron()
    assert np.abs(S - S0).max() < 1e-12
    assert np.abs(T - T0).max() < 1e-12
    assert np.abs(V - V0).max() < 1e-12


@pytest.mark.parametrize("name,bs", MOLS, ids=[m[0] for m in MOLS])
def test_one_electron_gradient_matches_reference(name, bs):
    rng = np.random.default_rng(43)
    n = bs.nbf
    A = rng.normal(size=(n, n))
    D = (A + A.T) / n
    A = rng.normal(size=(n, n))
    Q = (A + A.T) / n
    g0 = oracle.ref_onee_grad(bs, D, Q, 2.0, -2.0)
    with E.Engine(bs) as eng:
        g = eng.one_electron_grad(D, Q, 2.0, -2.0)
    assert np.abs(g - g0).max() < 1e-11
    assert np.abs(g.sum(axis=0)).max() < 1e-10  # translational invariance


def test_batched_one_electron_matches_per_molecule():
    import torch
    mols = M.batch_molecules(12, seed=5)
    bases = BT.batch_bases(mols)
    be = BT.BatchEngine(bases)
    dev = torch.device("cuda", 0)
    S = torch.empty(be.mat_total, dtype=torch.float64, device=dev)
    T = torch.empty_like(S)
    V = torch.empty_like(S)
    rng = np.random.default_rng(47)
    Dh = np.zeros(be.mat_total)
    Wh = np.zeros(be.mat_total)
    for k, b in enumerate(bases):
        n, off = int(be.nbf[k]), int(be.mat_off[k])
        A = rng.normal(size=(n, n))
        Dh[off:off + n * n] = ((A + A.T) / n).ravel()
        A = rng.normal(size=(n, n))
        Wh[off:off + n * n] = ((A + A.T) / n).ravel()
    D = torch.from_numpy(Dh).to(dev)
    W = torch.from_numpy(Wh).to(dev)
    g = torch.zeros((int(be.atom_off[-1]), 3), dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    be.one_electron_device(S, T, V)
    be.one_electron_grad_device(D, W, 2.0, -2.0, g)
    torch.cuda.synchronize()
    Sh, Th, Vh, gh = S.cpu().numpy(), T.cpu().numpy(), V.cpu().numpy(), g.cpu().numpy()
    be.close()
    for k, b in enumerate(bases):
        n, off = int(be.nbf[k]), int(be.mat_off[k])
        S0, T0, V0 = oracle.ref_onee(b)
        blk = slice(off, off + n * n)
        assert np.abs(Sh[blk].reshape(n, n) - S0).max() < 1e-12
        assert np.abs(Th[blk].reshape(n, n) - T0).max() < 1e-12
        assert np.abs(Vh[blk].reshape(n, n) - V0).max() < 1e-12
        g0 = oracle.ref_onee_grad(b, Dh[blk].reshape(n, n), Wh[blk].reshape(n, n), 2.0, -2.0)
        assert np.abs(gh[be.atom_off[k]:be.atom_off[k + 1]] - g0).max() < 1e-11
