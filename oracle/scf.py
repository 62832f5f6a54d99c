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
    Q = D F D, the two-electron term, and the nuclear repulsion gradient;
  * SAD guess (hfscf_hf_solver.cpp:478-553, src/scfsolver/hfscf_sad.cpp:13-400): atomic UHF
    per element on the element's one-atom integrals, fractional occupations, 6-vector DIIS.
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


def _atom_shells(basis, atom):
    """The shells of one atom as a one-atom basis (the atom's diagonal block of the molecule)."""
    from copy import copy
    sub = copy(basis)
    sub.Z = np.asarray([basis.Z[atom]])
    sub.coords = np.asarray(basis.coords[atom], dtype=float).reshape(1, 3)
    shells, idx, ids = [], 0, 0
    for s in basis.shells:
        if s.atom != atom:
            continue
        t = copy(s)
        t.atom, t.idx, t.ids = 0, idx, ids
        idx += (s.L + 1) * (s.L + 2) // 2
        ids += 2 * s.L + 1
        shells.append(t)
    sub.shells = shells
    return sub


def sad_guess(basis, rms_tol=1e-6, e_tol=1e-5, max_iter=25):
    """Superposition of atomic densities, restating Mol::hf_solver::get_sad_guess
    (src/scfsolver/hfscf_hf_solver.cpp:478-553) and Mol::sad_uhf_solver
    (src/scfsolver/hfscf_sad.cpp:13-400) on the reference's own integrals: per element (its first
    atom) an atomic UHF with H = T + V of the atom's own nucleus, the frozen-core / fractional
    valence weights of get_pop_numbers (:198-245) on the MO coefficients, Fock F_a = H + J[Da+Db]
    - K[Da] from the atom's ERIs, two-spin DIIS over 6 vectors, converged when both rms values are
    below rms_tol and |dE| < e_tol (or the rms sum < 1e-14); the atom density 0.5 (Da + Db)
    (hfscf_sad.hpp:44) copied onto every atom of the element."""
    import oracle
    n = basis.nbf
    D = np.zeros((n, n))
    bf_atom = basis.bf_atom()
    first = {}
    for a, Zc in enumerate(basis.Z):
        first.setdefault(int(Zc), a)
    zvalues = [0, 2, 10, 18, 36, 54, 86, 118]
    for Zc, a0 in first.items():
        ab = _atom_shells(basis, a0)
        S, T, V = oracle.ref_onee(ab)
        eri = oracle.ref_eri_packed(ab)
        H = T + V
        norb = S.shape[0]
        # populations (get_pop_numbers)
        k = max(i for i, z in enumerate(zvalues) if z <= Zc)
        if zvalues[k] == Zc:
            nfrozen, nactive = 0, zvalues[k] // 2
        else:
            nfrozen, nactive = zvalues[k] // 2, zvalues[k + 1] // 2 - zvalues[k] // 2
        nactive = min(nactive, norb - nfrozen)
        pop = np.zeros(norb)
        pop[:nfrozen] = 1.0
        pop[nfrozen:nfrozen + nactive] = np.sqrt((Zc - 2.0 * nfrozen) / (2.0 * nactive))
        occ = nfrozen + nactive
        X = _orthogonaliser(S)

        def dens(Fo):
            _, Cp = np.linalg.eigh(Fo)
            C = (X @ Cp) * pop[None, :]
            return C[:, :occ] @ C[:, :occ].T

        Da = dens(X.T @ H @ X)
        Db = Da.copy()
        E = float(np.sum(Da * H))
        Fa_h, Fb_h, Es, rms_hist = [], [], [], []
        it = 0
        while True:
            it += 1
            (Ja, Jb), (Ka, Kb) = oracle.jk_packed(eri, [Da, Db])
            Fa, Fb = H + Ja + Jb - Ka, H + Ja + Jb - Kb
            if len(rms_hist) > 6:
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
            Da, Db = dens(X.T @ Fa @ X), dens(X.T @ Fb @ X)
            E_prev, E = E, 0.5 * float(np.sum(Da * (H + Fa)) + np.sum(Db * (H + Fb)))
            if rms_a < rms_tol and rms_b < rms_tol and abs(E - E_prev) < e_tol:
                break
            if rms_a + rms_b < 1e-14:
                break
            if it >= max_iter:
                raise RuntimeError(f"oracle SAD atom Z={Zc} did not converge")
        Dat = 0.5 * (Da + Db)
        for a, Za in enumerate(basis.Z):
            if int(Za) == Zc:
                f = np.nonzero(bf_atom == a)[0]
                D[np.ix_(f, f)] = Dat
    return D
