"""SCF caller around the GPU Fock builds, and gradient assembly.

This is the caller side of the hot path, restated in FP64 on the host:
  * symmetric orthogonalisation S^-1/2 (src/scfsolver/hfscf_hf_solver.cpp:184-204);
  * density D = C_occ C_occ^T without a factor 2 (:206-242), energy
    E = sum D (H + F) (:244-252), convergence test on the DIIS commutator RMS
    and |dE| (:389-423);
  * DIIS (src/scfsolver/hfscf_diis.cpp:9-123): error X^T (FDS - (FDS)^T) X,
    rms = sqrt(mean(e^2)); beyond diis_range vectors the LARGEST-error entry is
    dropped; the B matrix is rescaled when sum|B| < 1e-14; extrapolated F replaces F;
  * RHF gradient (src/gradient/hfscf_grad_rhf.cpp:7-178): two-electron term from
    the GPU adjoint kernel, one-electron terms 2 sum D.(dT + dV) - 2 sum Q.dS with
    Q = D F D, plus the nuclear repulsion gradient.

Only the Fock build (J/K) and the two-electron gradient run on the GPU; the
N x N linear algebra here is glue.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np

from . import engine as eng
from .basis import Basis, nuclear_repulsion, nuclear_repulsion_gradient

DIIS_EPS = 1.0e-14  # src/scfsolver/hfscf_diis.hpp:65


class Diis:
    """Restatement of DIIS_SOLVER::diis_solver::diis_extrapolate (RHF)."""

    def __init__(self, nvec=5):
        self.nvec = nvec
        self.F, self.E, self.rms_list = [], [], []
        self.rms = np.inf

    def extrapolate(self, F, D, S, X):
        if len(self.rms_list) > self.nvec:
            pos = int(np.argmax(self.rms_list))
            del self.F[pos], self.E[pos], self.rms_list[pos]
        FDS = F @ D @ S
        err = X.T @ (FDS - FDS.T) @ X
        self.F.append(F.copy())
        self.E.append(err)
        self.rms = float(np.sqrt(np.mean(err * err)))
        self.rms_list.append(self.rms)
        if len(self.rms_list) > 1:
            m = len(self.E)
            B = np.empty((m + 1, m + 1))
            for i in range(m):
                for j in range(m):
                    B[i, j] = np.sum(self.E[i] * self.E[j])
            if np.abs(B[:m, :m]).sum() < DIIS_EPS:
                B[:m, :m] /= B[:m, :m].max()
            B[m, :] = -1.0
            B[:, m] = -1.0
            B[m, m] = 0.0
            rhs = np.zeros(m + 1)
            rhs[m] = -1.0
            q, r = np.linalg.qr(B)
            c = np.linalg.solve(r, q.T @ rhs)
            F = sum(c[k] * self.F[k] for k in range(m))
        return F


@dataclass
class ScfResult:
    energy: float
    e_elec: float
    e_nuc: float
    D: np.ndarray
    F: np.ndarray
    C: np.ndarray
    eps: np.ndarray
    iterations: int
    converged: bool
    fock_times: list = field(default_factory=list)
    energies: list = field(default_factory=list)


def sym_orth(S):
    w, U = np.linalg.eigh(S)
    return (U / np.sqrt(w)) @ U.T


def rhf(basis: Basis, fock=None, *, H=None, S=None, e_tol=1e-10, rms_tol=1e-8, diis_range=5, max_iter=50,
        precision=eng.FP64, incremental=False, engine=None, D0=None) -> ScfResult:
    """Restricted HF to convergence.  ``fock(D, H) -> F`` builds the Fock matrix;
    by default the GPU engine's RHF Fock build.  With ``incremental`` the engine
    builds F_k = F_{k-1} + 2J[dD] - K[dD] (density screening on |dD|), with a full
    rebuild every 8 iterations."""
    nel = int(np.sum(basis.Z))
    if nel % 2:
        raise ValueError("RHF needs an even electron count")
    nocc = nel // 2
    if fock is None:
        engine = engine or eng.Engine(basis)
        fock = lambda D, H_: engine.fock_rhf(D, H_, precision)  # noqa: E731
    if H is None or S is None:
        # one-electron matrices on the GPU when there is an engine, on the host otherwise
        S_, T_, V_ = engine.one_electron() if engine is not None else eng.one_electron(basis)
        S, H = S_, T_ + V_
    X = sym_orth(S)
    # CORE guess (deterministic): diagonalise X^T H X
    if D0 is None:
        eps, Cp = np.linalg.eigh(X.T @ H @ X)
        C = X @ Cp
        D = C[:, :nocc] @ C[:, :nocc].T
    else:
        D = D0.copy()
        C = None
        eps = None
    E_prev, E = 0.0, float(np.sum(D * (H + H)))
    diis = Diis(diis_range)
    res = ScfResult(0, 0, 0, D, H, C, eps, 0, False)
    F_last, D_last = None, None
    it = 0
    while True:
        it += 1
        t = time.perf_counter()
        if incremental and engine is not None and F_last is not None and (it % 8) != 0:
            F = engine.fock_delta(D - D_last, F_last, precision)
        else:
            F = fock(D, H)
        res.fock_times.append(time.perf_counter() - t)
        F_last, D_last = F.copy(), D.copy()
        F = diis.extrapolate(F, D, S, X)
        eps, Cp = np.linalg.eigh(X.T @ F @ X)
        C = X @ Cp
        D = C[:, :nocc] @ C[:, :nocc].T
        E_prev, E = E, float(np.sum(D * (H + F)))
        res.energies.append(E)
        if diis.rms < rms_tol and abs(E - E_prev) < e_tol:
            res.converged = True
            break
        if it >= max_iter:
            break
    # final Fock matrix at the converged density, for energies/gradients
    F = fock(D, H)
    E = float(np.sum(D * (H + F)))
    enuc = nuclear_repulsion(basis.Z, basis.coords)
    res.energy, res.e_elec, res.e_nuc = E + enuc, E, enuc
    res.D, res.F, res.C, res.eps, res.iterations = D, F, C, eps, it
    return res


def rhf_gradient(basis: Basis, res: ScfResult, engine, precision=eng.FP64):
    """Full RHF gradient (natoms x 3), as Mol::scf_gradient::calc_scf_gradient_rhf
    (src/gradient/hfscf_grad_rhf.cpp:7-178) assembles it."""
    D, F = res.D, res.F
    Q = D @ F @ D
    g = engine.grad2e(D, 1.0, precision)
    g += engine.one_electron_grad(D, Q, 2.0, -2.0)
    g += nuclear_repulsion_gradient(basis.Z, basis.coords)
    return g


def uhf(basis: Basis, engine, *, multiplicity=1, e_tol=1e-10, rms_tol=1e-8, max_iter=100, precision=eng.FP64):
    """Unrestricted HF with the GPU UHF Fock build (src/scfsolver/hfscf_uhf_solver.cpp:155-191),
    DIIS on the stacked alpha/beta errors."""
    nel = int(np.sum(basis.Z))
    na = (nel + multiplicity - 1) // 2
    nb = nel - na
    S, T, V = engine.one_electron()
    H = T + V
    X = sym_orth(S)
    eps, Cp = np.linalg.eigh(X.T @ H @ X)
    C = X @ Cp
    Da, Db = C[:, :na] @ C[:, :na].T, C[:, :nb] @ C[:, :nb].T
    E = 0.5 * float(np.sum((Da + Db) * (H + H)))
    hist_F, hist_E = [], []
    it = 0
    converged = False
    while True:
        it += 1
        Fa, Fb = engine.fock_uhf(Da, Db, H, precision)
        ea = X.T @ (Fa @ Da @ S - S @ Da @ Fa) @ X
        eb = X.T @ (Fb @ Db @ S - S @ Db @ Fb) @ X
        rms = 0.5 * (np.sqrt(np.mean(ea ** 2)) + np.sqrt(np.mean(eb ** 2)))
        hist_F.append((Fa.copy(), Fb.copy()))
        hist_E.append(np.concatenate([ea.ravel(), eb.ravel()]))
        if len(hist_F) > 6:
            hist_F.pop(0)
            hist_E.pop(0)
        if len(hist_F) > 1:
            m = len(hist_F)
            B = -np.ones((m + 1, m + 1))
            B[m, m] = 0
            for i in range(m):
                for j in range(m):
                    B[i, j] = hist_E[i] @ hist_E[j]
            rhs = np.zeros(m + 1)
            rhs[m] = -1
            c = np.linalg.solve(B, rhs)
            Fa = sum(c[k] * hist_F[k][0] for k in range(m))
            Fb = sum(c[k] * hist_F[k][1] for k in range(m))
        _, Ca = np.linalg.eigh(X.T @ Fa @ X)
        _, Cb = np.linalg.eigh(X.T @ Fb @ X)
        Ca, Cb = X @ Ca, X @ Cb
        Da, Db = Ca[:, :na] @ Ca[:, :na].T, Cb[:, :nb] @ Cb[:, :nb].T
        E_prev = E
        E = 0.5 * float(np.sum((Da + Db) * H + Da * Fa + Db * Fb))
        if rms < rms_tol and abs(E - E_prev) < e_tol:
            converged = True
            break
        if it >= max_iter:
            break
    Fa, Fb = engine.fock_uhf(Da, Db, H, precision)
    E = 0.5 * float(np.sum((Da + Db) * H + Da * Fa + Db * Fb))
    return {"energy": E + nuclear_repulsion(basis.Z, basis.coords), "Da": Da, "Db": Db, "Fa": Fa, "Fb": Fb,
            "iterations": it, "converged": converged}


def uhf_gradient(basis: Basis, r, engine, precision=eng.FP64):
    Da, Db, Fa, Fb = r["Da"], r["Db"], r["Fa"], r["Fb"]
    W = Da @ Fa @ Da + Db @ Fb @ Db
    g = engine.grad2e_uhf(Da, Db, 1.0, precision)
    g += engine.one_electron_grad(Da + Db, W, 1.0, -1.0)
    g += nuclear_repulsion_gradient(basis.Z, basis.coords)
    return g
