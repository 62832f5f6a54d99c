"""Edge cases of the C ABI on the GPU: the smallest systems (one shell, one atom, s only),
ragged batches, and the error codes of bad calls (every call returns a status and leaves
the handle usable).  Tolerances as in test_gpu_parity: ERIs 1e-11, J/K 1e-10."""
import ctypes

import numpy as np
import pytest

import oracle
from hfscf_b200 import basis as B
from hfscf_b200 import batch
from hfscf_b200 import engine as E
from hfscf_b200 import molecules as M

pytestmark = pytest.mark.gpu


def _sym(rng, n):
    A = rng.normal(size=(n, n))
    return (A + A.T) / max(n, 1)


SMALL = [
    ("h-atom-sto3g", "sto-3g", [1], [[0.0, 0.0, 0.0]], False),   # one shell, one function
    ("h-atom-ccpvdz", "cc-pvdz", [1], [[0.1, -0.2, 0.3]], True),  # one atom, s and p
    ("h2-sto3g", "sto-3g", [1, 1], [[0.0, 0.0, 0.0], [0.0, 0.0, 1.4]], False),  # s only
    ("oh-631gs", "6-31g*", [8, 1], [[0.0, 0.0, 0.0], [0.0, 0.3, 1.8]], False),  # odd electrons: J/K only
]


@pytest.mark.parametrize("name,basis,Z,xyz,pure", SMALL, ids=[s[0] for s in SMALL])
def test_smallest_systems_match_oracle(name, basis, Z, xyz, pure):
    bs = B.build_basis(basis, np.array(Z), np.array(xyz, dtype=float), pure=pure)
    rng = np.random.default_rng(3)
    D = _sym(rng, bs.nbf)
    eri0 = oracle.eri_packed(bs)
    J0, K0 = oracle.jk(eri0, D)
    with E.Engine(bs, density_tol=0.0) as eng:
        eri = eng.eri_packed()
        J, K = eng.jk(D, [D])
        g = eng.grad2e(D)
    assert np.max(np.abs(eri - eri0)) < 1e-11
    assert np.max(np.abs(J - J0)) < 1e-10 and np.max(np.abs(K[0] - K0)) < 1e-10
    assert np.max(np.abs(g - oracle.grad2e_rhf(bs, D))) < 1e-10


def test_ragged_batch_matches_single_molecules():
    """One batch holding a one-function molecule, an s-only molecule and a 114-function
    water hexamer."""
    import torch
    mols = [(np.array([1]), np.zeros((1, 3)), "sto-3g", False),
            (np.array([1, 1]), np.array([[0.0, 0.0, 0.0], [0.0, 0.0, 1.4]]), "sto-3g", False)]
    Z, x = M.water_cluster(6, 3.0, np.random.default_rng(4), 0.05)
    mols.append((np.asarray(Z), np.asarray(x) * B.ANGSTROM_TO_BOHR, "6-31g*", False))
    bases = batch.batch_bases(mols)
    be = batch.BatchEngine(bases)
    rng = np.random.default_rng(6)
    Ds = [_sym(rng, b.nbf) for b in bases]
    dev = torch.device("cuda", 0)
    D = torch.from_numpy(np.concatenate([d.ravel() for d in Ds])).to(dev)
    J = torch.zeros_like(D)
    K = torch.zeros_like(D)
    torch.cuda.synchronize()
    be.jk_device(D, J, K)
    torch.cuda.synchronize()
    Jn, Kn = J.cpu().numpy(), K.cpu().numpy()
    for m, b in enumerate(bases):
        off, n = int(be.mat_off[m]), b.nbf
        with E.Engine(b, density_tol=0.0) as e1:
            J1, K1 = e1.jk(Ds[m], [Ds[m]])
        assert np.max(np.abs(Jn[off:off + n * n].reshape(n, n) - J1)) < 1e-10
        assert np.max(np.abs(Kn[off:off + n * n].reshape(n, n) - K1[0])) < 1e-10
    be.close()


def test_bad_calls_return_status_and_leave_the_handle_usable():
    rng = np.random.default_rng(8)
    Z, x = M.water(rng)
    bs = B.build_basis("6-31g*", Z, np.asarray(x) * B.ANGSTROM_TO_BOHR, pure=False)
    lib = E.lib()
    with E.Engine(bs) as eng:
        n = bs.nbf
        # packed ERI buffer of the wrong length
        buf = np.zeros(10)
        rc = lib.hfgpu_eri_packed(eng.h, buf.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                  ctypes.c_longlong(10))
        assert rc == 1
        assert b"eri_len" in lib.hfgpu_last_error(eng.h)
        # more exchange densities than the engine takes
        D = np.zeros((n, n))
        Ks = np.zeros((9, n, n))
        p = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))  # noqa: E731
        rc = lib.hfgpu_jk(eng.h, p(D), ctypes.c_int(9), p(Ks), p(D.copy()), p(Ks.copy()), ctypes.c_int(0))
        assert rc == 1
        # a non-finite density gives a non-finite energy, reported as such
        Dn = np.full((n, n), np.nan)
        E2 = ctypes.c_double()
        rc = lib.hfgpu_energy_forward(eng.h, p(Dn), ctypes.byref(E2), ctypes.c_int(0))
        assert rc == 5
        # the handle still works
        D = _sym(rng, n)
        J, K = eng.jk(D, [D])
        J0, K0 = oracle.jk(oracle.eri_packed(bs), D)
        assert np.max(np.abs(J - J0)) < 1e-10


def test_unsupported_basis_is_rejected():
    bs = B.build_basis("sto-3g", np.array([1]), np.zeros((1, 3)))
    bs.shells[0].L = 3  # f shells are beyond this engine (L <= 2)
    with pytest.raises(E.HfgpuError) as err:
        E.Engine(bs)
    assert err.value.code == 1


def test_batched_eigensolver_rejects_large_molecules():
    import torch
    Z, x, name, pure = M.workload(2)  # n-octane, 210 functions
    bases = batch.batch_bases([(np.asarray(Z), np.asarray(x), name, pure), (np.array([1]), np.zeros((1, 3)), "sto-3g", False)])
    be = batch.BatchEngine(bases)
    nmax = int(be.nbf.max())
    dev = torch.device("cuda", 0)
    A = torch.eye(nmax, dtype=torch.float64, device=dev).repeat(2, 1, 1)
    W = torch.empty((2, nmax), dtype=torch.float64, device=dev)
    V = torch.empty_like(A)
    with pytest.raises(E.HfgpuError) as err:
        be.eigh(A, W, V)
    assert err.value.code == 6
    be.close()


def test_setup_times_and_list_segments_cover_every_screened_quartet():
    """hfgpu_setup_times reports the four set-up phases; the quartet lists built in parallel
    chunks hold every quartet that passes the Schwarz test exactly once (class counts against
    a host count of the screened quartets from the pair Schwarz factors)."""
    rng = np.random.default_rng(12)
    Z, x = M.water_cluster(3, 3.0, rng, 0.05)
    bs = B.build_basis("6-31g*", Z, np.asarray(x) * B.ANGSTROM_TO_BOHR, pure=False)
    with E.Engine(bs) as eng:
        t = eng.setup_times()
        assert set(t) == {"pairs", "schwarz", "lists", "upload"}
        assert all(v >= 0.0 for v in t.values()) and t["lists"] > 0.0
        Q = eng.schwarz()
        listed = sum(eng.class_stats(c)["screened"] for c in range(E.NUM_CLASSES))
    # unique shell quartets (ab|cd), a >= b, c >= d, pair(ab) >= pair(cd) in the engine's
    # canonical sense: count unordered pairs of unordered shell pairs with Q_ab Q_cd >= 1e-12
    ns = len(bs.shells)
    q = np.array([Q[i, j] for i in range(ns) for j in range(i + 1)])
    prod = np.outer(q, q)
    iu = np.triu_indices(len(q))
    assert listed == int(np.count_nonzero(prod[iu] >= 1e-12))


@pytest.mark.parametrize("coop", [1, 0], ids=["cooperative", "two-launches-per-step"])
@pytest.mark.parametrize("n,nocc", [(7, 3), (152, 40), (210, 33), (700, 150)])
def test_purification_matches_the_diagonalisation_projector(n, nocc, coop):
    """hfgpu_purify_device: the projector onto the nocc lowest eigenvectors of a symmetric matrix
    with a gap, against numpy's eigh (1e-10), and a reported trace error below 1e-10; in the one
    cooperative launch and in the two-launches-per-step form (n = 700: more tiles than one wave
    of co-resident blocks, so the cooperative blocks loop over tiles)."""
    import torch
    rng = np.random.default_rng(n)
    Q, _ = np.linalg.qr(rng.normal(size=(n, n)))
    w = np.sort(np.concatenate([rng.uniform(-40.0, -0.3, nocc), rng.uniform(0.2, 6.0, n - nocc)]))
    Fo = (Q * w) @ Q.T
    Fo = 0.5 * (Fo + Fo.T)
    P0 = Q[:, :nocc] @ Q[:, :nocc].T
    Z, x = M.water(rng)
    bs = B.build_basis("sto-3g", Z, np.asarray(x) * B.ANGSTROM_TO_BOHR)
    dev = torch.device("cuda", 0)
    with E.Engine(bs) as eng:
        eng.set_purify_mode(coop)
        F = torch.from_numpy(Fo).to(dev)
        P = torch.empty_like(F)
        err = torch.zeros((), dtype=torch.float64, device=dev)
        eng.purify_device(F.data_ptr(), n, nocc, 64, P.data_ptr(), err.data_ptr())
        torch.cuda.synchronize()
        assert float(err) < 1e-10
        assert np.max(np.abs(P.cpu().numpy() - P0)) < 1e-10


@pytest.mark.parametrize("coop", [1, 0], ids=["cooperative", "two-launches-per-step"])
def test_purification_reports_a_missing_gap(coop):
    """Two equal eigenvalues at the Fermi level: no projector separates them, the purification
    does not converge and says so (err = 1), so the SCF diagonalises instead.  (24 steps: far
    more would let rounding split the pair, 2^-53 doubling each step.)"""
    import torch
    n, nocc = 12, 5
    rng = np.random.default_rng(3)
    Q, _ = np.linalg.qr(rng.normal(size=(n, n)))
    w = np.array([-9.0, -7.0, -5.0, -3.0, -1.0, -1.0, 1.0, 2.0, 3.0, 4.0, 5.0, 6.0])
    Fo = (Q * w) @ Q.T
    Fo = 0.5 * (Fo + Fo.T)
    Z, x = M.water(rng)
    bs = B.build_basis("sto-3g", Z, np.asarray(x) * B.ANGSTROM_TO_BOHR)
    dev = torch.device("cuda", 0)
    with E.Engine(bs) as eng:
        eng.set_purify_mode(coop)
        F = torch.from_numpy(Fo).to(dev)
        P = torch.empty_like(F)
        err = torch.zeros((), dtype=torch.float64, device=dev)
        eng.purify_device(F.data_ptr(), n, nocc, 24, P.data_ptr(), err.data_ptr())
        torch.cuda.synchronize()
        assert float(err) >= 1e-10
