"""Oracle SCF drivers and gradient assembly (TEST INFRASTRUCTURE ONLY).

A numpy restatement of the reference's conventional RHF/UHF SCF and RHF gradient, run on
integrals from the reference's own code (oracle/_ref) or the C restatement:
  * S^-1/2 by eigendecomposition (src/scfsolver/hfscf_hf_solver.cpp:184-204);
  * core guess: diagonalise X^T H X (same file, :206-242 at iteration 0);
  * density without a factor 2 (:221-231), energy sum D (H + F) (:244-252);
  * Fock build F = H + 2J - K from the packed ERIs (:254-286), UHF
    F_a = H + J[Da+Db] - K[Da] (src/scfsolver/hfscf_uhf_solver.cpp:155-191);
  * DIIS (src/scfsolver/hfscf_diis.cpp:9-123 RHF, :126-260 UHF): error X^T (FDS - SDF) X,
    the largest-error vector dropped beyond diis_size, B rescaled when sum|B| < 1e-14,
    solved by QR; convergence on the DIIS rms and |dE| (hfscf_hf_solver.cpp:389-423,
    hfscf_uhf_solver.cpp:198-225);
  * RHF gradient (src/gradient/hfscf_grad_rhf.cpp:7-178): 2 sum D.(dT + dV) - 2 sum Q.dS with
    Q = D F D, the two-electron term, and the nuclear repulsion gradient.
Only tests/ and bench.py's reference leg use this module.
"""
from __future__ import annotations

import numpy as np

DIIS_EPS = 1.0e-14


def nuclear_repulsion(Z, xyz) -> float:
    """sum_{A<B} Z_A Z_B / |R_A - R_B| (bohr)."""
    Z = np.asarray(Z, dtype=float)
    x = np.asarray(xyz, dtype=float)
    e = 0.0
    for a in range(len(Z)):
        for b in range(a):
            e += Z[a] * Z[b] / np.linalg.norm(x[a] - x[b])
    return e


def nuclear_repulsion_gradient(Z, xyz) -> np.ndarray:
    """d/dR_A of nuclear_repulsion: -sum_B Z_A Z_B (R_A - R_B) / |R_A - R_B|^3."""
    Z = np.asarray(Z, dtype=float)
    x = np.asarray(xyz, dtype=float)
    g = np.zeros_like(x)
    for a in range(len(Z)):
        for b in range(len(Z)):
            if a != b:
                d = x[a] - x[b]
                g[a] -= Z[a] * Z[b] * d / np.linalg.norm(d) ** 3
    return g


def _orthogonaliser(S):
    w, U = np.linalg.eigh(S)
    return (U / np.sqrt(w)) @ U.T


def _diis_solve(errs, rhs_vectors):
    m = len(errs)
    B = np.empty((m + 1, m + 1))
    for i in range(m):
        for j in range(m):
            B[i, j] = float(np.vdot(errs[i], errs[j]))
    if np.abs(B[:m, :m]).sum() < DIIS_EPS:
        B[:m, :m] /= B[:m, :m].max()
    B[m, :] = -1.0
    B[:, m] = -1.0
    B[m, m] = 0.0
    b = np.zeros(m + 1)
    b[m] = -1.0
    q, r = np.linalg.qr(B)
    c = np.linalg.solve(r, q.T @ b)
    return [sum(c[k] * v[k] for k in range(m)) for v in rhs_vectors]


def rhf(S, H, nocc, jk, e_nuc, *, e_tol=1e-10, rms_tol=1e-8, diis_size=5, max_iter=100):
    """Conventional RHF from the core guess.  jk(D) -> (J, K).  Returns a dict with the total
    energy, D, F (at the converged density), iterations and convergence flag."""
    X = _orthogonaliser(S)
    _, Cp = np.linalg.eigh(X.T @ H @ X)
    C = X @ Cp
    D = C[:, :nocc] @ C[:, :nocc].T
    E = float(np.sum(D * (H + H)))
    Fs, Es, rms_hist = [], [], []
    it, converged = 0, False
    while True:
        it += 1
        J, K = jk(D)
        F = H + 2.0 * J - K
        if len(rms_hist) > diis_size:
            pos = int(np.argmax(rms_hist))
            del Fs[pos], Es[pos], rms_hist[pos]
        FDS = F @ D @ S
        err = X.T @ (FDS - FDS.T) @ X
        Fs.append(F)
        Es.append(err)
        rms = float(np.sqrt(np.mean(err * err)))
        rms_hist.append(rms)
        if len(Es) > 1:
            (F,) = _diis_solve(Es, [Fs])
        _, Cp = np.linalg.eigh(X.T @ F @ X)
        C = X @ Cp
        D = C[:, :nocc] @ C[:, :nocc].T
        E_prev, E = E, float(np.sum(D * (H + F)))
        if rms < rms_tol and abs(E - E_prev) < e_tol:
            converged = True
            break
        if it >= max_iter:
            break
    J, K = jk(D)
    F = H + 2.0 * J - K
    E = float(np.sum(D * (H + F)))
    return {"energy": E + e_nuc, "D": D, "F": F, "iterations": it, "converged": converged}


def uhf(S, H, nalpha, nbeta, jk, e_nuc, *, e_tol=1e-10, rms_tol=1e-8, diis_size=5, max_iter=200):
    """Conventional UHF from the core guess (no HOMO/LUMO mixing, the reference's default).
    jk(D) -> (J, K) for one density."""
    X = _orthogonaliser(S)
    _, Cp = np.linalg.eigh(X.T @ H @ X)
    C = X @ Cp
    Da, Db = C[:, :nalpha] @ C[:, :nalpha].T, C[:, :nbeta] @ C[:, :nbeta].T
    E = float(np.sum(Da * (H + H)))
    Fa_h, Fb_h, Es, rms_hist = [], [], [], []
    it, converged = 0, False

    def fock(Da, Db):
        Ja, Ka = jk(Da)
        Jb, Kb = jk(Db)
        return H + Ja + Jb - Ka, H + Ja + Jb - Kb

    while True:
        it += 1
        Fa, Fb = fock(Da, Db)
        if len(rms_hist) > diis_size:
            pos = int(np.argmax(rms_hist))
            del Fa_h[pos], Fb_h[pos], Es[pos], rms_hist[pos]
        ga = X.T @ (Fa @ Da @ S - (Fa @ Da @ S).T) @ X
        gb = X.T @ (Fb @ Db @ S - (Fb @ Db @ S).T) @ X
        rms_a = 0.5 * float(np.sqrt(np.mean(ga * ga)))
        rms_b = 0.5 * float(np.sqrt(np.mean(gb * gb)))
        Es.append(np.concatenate([ga.ravel(), gb.ravel()]))
        Fa_h.append(Fa)
        Fb_h.append(Fb)
        rms_hist.append(rms_a + rms_b)
        if len(Es) > 1:
            Fa, Fb = _diis_solve(Es, [Fa_h, Fb_h])
        _, Ca = np.linalg.eigh(X.T @ Fa @ X)
        _, Cb = np.linalg.eigh(X.T @ Fb @ X)
        Ca, Cb = X @ Ca, X @ Cb
        Da, Db = Ca[:, :nalpha] @ Ca[:, :nalpha].T, Cb[:, :nbeta] @ Cb[:, :nbeta].T
        E_prev = E
        E = 0.5 * float(np.sum(Da * (H + Fa)) + np.sum(Db * (H + Fb)))
        if rms_a < rms_tol and rms_b < rms_tol and abs(E - E_prev) < e_tol:
            converged = True
            break
        if it >= max_iter:
            break
    Fa, Fb = fock(Da, Db)
    E = 0.5 * float(np.sum(Da * (H + Fa)) + np.sum(Db * (H + Fb)))
    return {"energy": E + e_nuc, "Da": Da, "Db": Db, "Fa": Fa, "Fb": Fb, "iterations": it,
            "converged": converged}
