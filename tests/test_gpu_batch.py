"""Batched many-molecule mode against the single-molecule engine (GPU)."""
import numpy as np
import pytest

from hfscf_b200 import basis as B
from hfscf_b200 import batch
from hfscf_b200 import engine as E
from hfscf_b200 import molecules as M
from hfscf_b200 import scf

pytestmark = pytest.mark.gpu


def _mols(n=10, seed=99):
    return batch.batch_bases(M.batch_molecules(n, seed=seed))


def test_batch_jk_matches_single_molecule_engine():
    import torch
    bases = _mols(8)
    be = batch.BatchEngine(bases)
    rng = np.random.default_rng(3)
    Ds = []
    for b in bases:
        A = rng.normal(size=(b.nbf, b.nbf))
        Ds.append((A + A.T) / b.nbf)
    dev = torch.device("cuda", 0)
    D = torch.from_numpy(np.concatenate([d.ravel() for d in Ds])).to(dev)
    J = torch.zeros_like(D)
    K = torch.zeros_like(D)
    be.jk_device(D, J, K)
    torch.cuda.synchronize()
    Jn, Kn = J.cpu().numpy(), K.cpu().numpy()
    for m, b in enumerate(bases):
        off, n = be.mat_off[m], b.nbf
        with E.Engine(b, density_tol=0.0) as e1:
            J1, K1 = e1.jk(Ds[m], [Ds[m]])
        assert np.max(np.abs(Jn[off:off + n * n].reshape(n, n) - J1)) < 1e-10
        assert np.max(np.abs(Kn[off:off + n * n].reshape(n, n) - K1[0])) < 1e-10
    be.close()


@pytest.mark.parametrize("use_graph,diag,freeze", [(True, "purify", False), (True, "purify", True),
                                                   (True, "gpu", False), (False, "gpu", False), (True, "host", False)],
                         ids=["cuda-graph-purify", "cuda-graph-purify-freeze", "cuda-graph", "eager", "host-diag"])
def test_batch_scf_and_gradients_match_single_molecule_runs(use_graph, diag, freeze):
    bases = _mols(10)
    # the eager case starts from the core-Hamiltonian guess, the others from the SAD guess
    out = batch.batch_rhf(bases, use_graph=use_graph, e_tol=1e-11, rms_tol=1e-9, diag=diag, freeze_converged=freeze,
                          guess="sad" if use_graph else "core")
    assert out["converged"].all()
    for m, b in enumerate(bases):
        with E.Engine(b) as e1:
            r = scf.rhf(b, engine=e1, e_tol=1e-11, rms_tol=1e-9)
            g = scf.rhf_gradient(b, r, e1)
        assert abs(out["energies"][m] - r.energy) < 1e-8
        assert np.max(np.abs(out["gradients"][m] - g)) < 1e-6


def test_batched_purification_matches_the_eigh_projector():
    """hfgpu_batch_purify_device: every molecule's projector onto its nocc lowest eigenvectors,
    for random symmetric blocks of uneven size with a gap at nocc (padded like the SCF's Fock
    batch), against numpy's eigh (1e-10), with each reported trace error below 1e-10."""
    import torch
    bases = _mols(9, seed=7)
    be = batch.BatchEngine(bases)
    nmol, nmax = len(bases), int(be.nbf.max())
    rng = np.random.default_rng(6)
    A = np.zeros((nmol, nmax, nmax))
    P0 = np.zeros_like(A)
    nocc = []
    for k in range(nmol):
        n = int(be.nbf[k])
        no = max(1, n // 3)
        nocc.append(no)
        Q, _ = np.linalg.qr(rng.normal(size=(n, n)))
        w = np.sort(np.concatenate([rng.uniform(-30.0, -0.4, no), rng.uniform(0.3, 5.0, n - no)]))
        A[k, :n, :n] = 0.5 * ((Q * w) @ Q.T + ((Q * w) @ Q.T).T)
        A[k, np.arange(n, nmax), np.arange(n, nmax)] = 1e3
        P0[k, :n, :n] = Q[:, :no] @ Q[:, :no].T
    dev = torch.device("cuda", 0)
    Ad = torch.from_numpy(A).to(dev)
    P = torch.full((nmol, nmax, nmax), 7.0, dtype=torch.float64, device=dev)
    err = torch.zeros(nmol, dtype=torch.float64, device=dev)
    nd = torch.tensor(nocc, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()
    be.purify(Ad, nd, P, err)
    torch.cuda.synchronize()
    assert float(err.max()) < 1e-10
    assert np.max(np.abs(P.cpu().numpy() - P0)) < 1e-10  # zero outside each block too
    be.close()


def test_batched_eigensolver_matches_lapack():
    """hfgpu_batch_eigh against numpy's LAPACK eigh on random symmetric blocks of uneven size."""
    import torch
    bases = _mols(9, seed=7)
    be = batch.BatchEngine(bases)
    nmol, nmax = len(bases), int(be.nbf.max())
    rng = np.random.default_rng(5)
    A = np.zeros((nmol, nmax, nmax))
    for k in range(nmol):
        n = int(be.nbf[k])
        R = rng.normal(size=(n, n))
        A[k, :n, :n] = (R + R.T) / 2
        A[k, np.arange(n, nmax), np.arange(n, nmax)] = 1e3
    dev = torch.device("cuda", 0)
    Ad = torch.from_numpy(A).to(dev)
    W = torch.empty((nmol, nmax), dtype=torch.float64, device=dev)
    V = torch.empty((nmol, nmax, nmax), dtype=torch.float64, device=dev)
    sw = torch.zeros(nmol, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()
    be.eigh(Ad, W, V, sw)
    torch.cuda.synchronize()
    Wn, Vn, swn = W.cpu().numpy(), V.cpu().numpy(), sw.cpu().numpy()
    be.close()
    for k in range(nmol):
        n = int(be.nbf[k])
        w0 = np.linalg.eigvalsh(A[k, :n, :n])
        assert np.abs(Wn[k, :n] - w0).max() < 1e-11 * max(1.0, np.abs(w0).max())
        Vk = Vn[k, :n, :n]
        assert np.abs(Vk.T @ Vk - np.eye(n)).max() < 1e-12
        assert np.abs(A[k, :n, :n] @ Vk - Vk * Wn[k, :n]).max() < 1e-11
        assert (Wn[k, n:] == 1e3).all() and swn[k] < 30


@pytest.mark.skipif(not __import__("oracle").ref_available(), reason="reference library not built")
def test_batch_energies_match_oracle_scf():
    """Six molecules of the batched workload's mix (both basis sets), solved together in one
    batched handle with the autotuned schedule, against an oracle SCF per molecule on the
    reference's own integrals (1e-8 Eh)."""
    import oracle
    from oracle import scf as OS
    bases = _mols(6, seed=1234)
    first = batch.batch_rhf(bases, autotune=True, gradient=False, max_iter=2)
    out = batch.batch_rhf(bases, e_tol=1e-11, rms_tol=1e-9, gradient=False, schedule=first["schedule"])
    assert out["converged"].all() and out["autotuned"]
    for m, b in enumerate(bases):
        S, T, V = oracle.ref_onee(b)
        eri = oracle.ref_eri_packed(b)

        def jk(D):
            J, K = oracle.jk_packed(eri, [D])
            return J[0], K[0]

        ref = OS.rhf(S, T + V, int(sum(b.Z)) // 2, jk, OS.nuclear_repulsion(b.Z, b.coords), rms_tol=1e-9)
        assert ref["converged"]
        assert abs(out["energies"][m] - ref["energy"]) < 1e-8, (m, out["energies"][m], ref["energy"])
