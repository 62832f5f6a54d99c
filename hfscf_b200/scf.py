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
PURIFY_TOL = 1e-10  # largest tr P - tr P^2 accepted from the purification before the diagonalisation is used
PURIFY_STEPS = 64   # squarings of one purification (it stops changing P once converged)


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
    diag_fallbacks: int = 0  # device loop: iterations whose density came from the diagonalisation


class DiisUhf:
    """Restatement of the two-spin DIIS_SOLVER::diis_solver::diis_extrapolate
    (src/scfsolver/hfscf_diis.cpp:126-260): error vectors of both spins concatenated, the
    largest-error entry dropped when over the limit, rms per spin 0.5 sqrt(mean(e^2))."""

    def __init__(self, nvec=6):
        self.nvec = nvec
        self.Fa, self.Fb, self.E, self.rms_list = [], [], [], []
        self.rms_a = self.rms_b = np.inf

    def extrapolate(self, Fa, Fb, S, Da, Db, X):
        if len(self.rms_list) > self.nvec:
            pos = int(np.argmax(self.rms_list))
            del self.Fa[pos], self.Fb[pos], self.E[pos], self.rms_list[pos]
        ga = X.T @ (Fa @ Da @ S - (Fa @ Da @ S).T) @ X
        gb = X.T @ (Fb @ Db @ S - (Fb @ Db @ S).T) @ X
        self.rms_a = 0.5 * float(np.sqrt(np.mean(ga * ga)))
        self.rms_b = 0.5 * float(np.sqrt(np.mean(gb * gb)))
        self.E.append(np.concatenate([ga.ravel(), gb.ravel()]))
        self.Fa.append(Fa.copy())
        self.Fb.append(Fb.copy())
        self.rms_list.append(self.rms_a + self.rms_b)
        if len(self.rms_list) > 1:
            m = len(self.E)
            B = np.empty((m + 1, m + 1))
            for i in range(m):
                for j in range(m):
                    B[i, j] = float(self.E[i] @ self.E[j])
            if np.abs(B[:m, :m]).sum() < DIIS_EPS:
                B[:m, :m] /= B[:m, :m].max()
            B[m, :] = -1.0
            B[:, m] = -1.0
            B[m, m] = 0.0
            rhs = np.zeros(m + 1)
            rhs[m] = -1.0
            q, r = np.linalg.qr(B)
            c = np.linalg.solve(r, q.T @ rhs)
            Fa = sum(c[k] * self.Fa[k] for k in range(m))
            Fb = sum(c[k] * self.Fb[k] for k in range(m))
        return Fa, Fb


def sad_populations(Z: int, norb: int):
    """Frozen-core and fractional valence occupations of the SAD atom
    (Mol::sad_uhf_solver::get_pop_numbers, src/scfsolver/hfscf_sad.cpp:198-245): the noble-gas
    core below Z is frozen (weight 1), the next shell's orbitals share the remaining electrons
    (weight sqrt(n_valence / 2 n_active) on the MO coefficients).  Returns (weights, n_occupied)."""
    zvalues = [0, 2, 10, 18, 36, 54, 86, 118]
    k = next(i for i, z in enumerate(zvalues) if z >= Z)
    if zvalues[k] > Z:
        k -= 1
    if zvalues[k] == Z:
        nfrozen, nactive = 0, zvalues[k] // 2
    else:
        nfrozen = zvalues[k] // 2
        nactive = zvalues[k + 1] // 2 - nfrozen
    nactive = min(nactive, norb - nfrozen)
    w = np.zeros(norb)
    w[:nfrozen] = 1.0
    w[nfrozen:nfrozen + nactive] = np.sqrt((Z - 2.0 * nfrozen) / (2.0 * nactive))
    return w, nfrozen + nactive


def sad_atom_density(Z: int, S, T, V, jk, rms_tol=1e-6, e_tol=1e-5, max_iter=25):
    """Spin-averaged density of one atom from the SAD atomic UHF
    (Mol::sad_uhf_solver, src/scfsolver/hfscf_sad.cpp:13-476): H = T + V of the atom's own
    nucleus, S^-1/2 orthogonalisation, fractional occupations (sad_populations), Fock
    F_a = H + J[Da + Db] - K[Da] (and b) from ``jk(DJ, DK_list) -> (J, [K...])``, two-spin
    DIIS over 6 vectors, converged when both rms < rms_tol and |dE| < e_tol (or the rms sum
    < 1e-14).  Returns 0.5 (Da + Db)."""
    H = T + V
    w, U = np.linalg.eigh(S)
    X = U @ np.diag(1.0 / np.sqrt(w)) @ U.T
    pop, occ = sad_populations(Z, S.shape[0])

    def density(Fp):
        _, C = np.linalg.eigh(Fp)
        mo = X @ C * pop[None, :]
        return mo[:, :occ] @ mo[:, :occ].T

    Da = density(X.T @ H @ X)
    Db = Da.copy()
    E = float(np.sum(Da * H))
    diis = DiisUhf(6)
    it = 0
    while True:
        it += 1
        J, K = jk(Da + Db, [Da, Db])
        Fa = H + J - K[0]
        Fb = H + J - K[1]
        Fa, Fb = diis.extrapolate(Fa, Fb, S, Da, Db, X)
        Da, Db = density(X.T @ Fa @ X), density(X.T @ Fb @ X)
        E_prev, E = E, 0.5 * float(np.sum(Da * (H + Fa)) + np.sum(Db * (H + Fb)))
        if diis.rms_a < rms_tol and diis.rms_b < rms_tol and abs(E - E_prev) < e_tol:
            break
        if diis.rms_a + diis.rms_b < 1e-14:
            break
        if it >= max_iter:
            raise RuntimeError(f"SAD atom Z={Z} did not converge in {max_iter} iterations")
    return 0.5 * (Da + Db)


def atom_basis(basis: Basis, atom: int) -> Basis:
    """The shells of one atom as a basis of their own (the atom's block of the molecule's basis)."""
    shells, idx, ids = [], 0, 0
    for s in basis.shells:
        if s.atom != atom:
            continue
        shells.append(type(s)(L=s.L, atom=0, center=s.center, exps=s.exps, coefs=s.coefs, idx=idx, ids=ids))
        idx += (s.L + 1) * (s.L + 2) // 2
        ids += 2 * s.L + 1
    return Basis(name=basis.name, pure=basis.pure, Z=np.asarray([basis.Z[atom]]),
                 coords=np.asarray(basis.coords[atom]).reshape(1, 3), shells=shells)


def sad_guess(basis: Basis, engine_factory=None, rms_tol=1e-6, e_tol=1e-5, max_iter=25) -> np.ndarray:
    """Superposition-of-atomic-densities guess (Mol::hf_solver::get_sad_guess,
    src/scfsolver/hfscf_hf_solver.cpp:478-553): one atomic UHF per element (first atom of
    that element), its spin-averaged density copied onto the diagonal block of every atom of
    the element.  The atomic J/K builds run on the GPU engine of the atom's basis.  The
    tolerances default to the reference's SAD settings (src/settings/hfscf_settings.hpp:35-50)."""
    n = basis.nbf
    D = np.zeros((n, n))
    first = {}
    bf_atom = basis.bf_atom()
    for a, Zc in enumerate(basis.Z):
        first.setdefault(int(Zc), a)
    for Zc, a0 in first.items():
        ab = atom_basis(basis, a0)
        with (engine_factory or eng.Engine)(ab) as e:
            S, T, V = e.one_electron()
            Dat = sad_atom_density(Zc, S, T, V, lambda DJ, DKs: e.jk(DJ, DKs), rms_tol, e_tol, max_iter)
        for a, Za in enumerate(basis.Z):
            if int(Za) != Zc:
                continue
            f = np.nonzero(bf_atom == a)[0]
            D[np.ix_(f, f)] = Dat
    return D


def sym_orth(S):
    w, U = np.linalg.eigh(S)
    return (U / np.sqrt(w)) @ U.T


def rhf(basis: Basis, fock=None, *, H=None, S=None, e_tol=1e-10, rms_tol=1e-8, diis_range=5, max_iter=50,
        precision=eng.FP64, incremental=False, engine=None, D0=None, guess="core") -> ScfResult:
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
        if H is None and S is None:
            return _rhf_device(basis, engine, e_tol=e_tol, rms_tol=rms_tol, diis_range=diis_range,
                               max_iter=max_iter, precision=precision, incremental=incremental, D0=D0, guess=guess)
        fock = lambda D, H_: engine.fock_rhf(D, H_, precision)  # noqa: E731
    if H is None or S is None:
        # one-electron matrices on the GPU when there is an engine, on the host otherwise
        S_, T_, V_ = engine.one_electron() if engine is not None else eng.one_electron(basis)
        S, H = S_, T_ + V_
    X = sym_orth(S)
    if D0 is None and guess == "sad":
        D0 = sad_guess(basis)
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


def _rhf_device(basis: Basis, engine, *, e_tol, rms_tol, diis_range, max_iter, precision, incremental, D0,
                guess) -> ScfResult:
    """The loop of rhf() with every matrix on the GPU: J/K through hfgpu_jk_device, the
    one-electron matrices through hfgpu_one_electron_device, DIIS (as Diis) and the
    diagonalisations in torch on the device; per iteration only the DIIS matrix and two
    scalars come back to the host.  Same steps, order and convergence test as the host loop."""
    import torch
    dev = torch.device("cuda", engine._opts.device)
    cur = torch.cuda.current_stream(dev)
    # the engine's kernels and torch's ops must share one stream: the caller's, unless that is
    # the legacy default stream (which the engine's non-blocking stream does not wait for)
    private = cur.cuda_stream == 0
    stream = torch.cuda.Stream(dev) if private else cur
    engine.set_stream(stream.cuda_stream)
    try:
        with torch.cuda.stream(stream):
            return _rhf_device_loop(basis, engine, dev, e_tol=e_tol, rms_tol=rms_tol, diis_range=diis_range,
                                    max_iter=max_iter, precision=precision, incremental=incremental, D0=D0,
                                    guess=guess)
    finally:
        if private:
            torch.cuda.synchronize(dev)
            engine.set_stream(None)


def _rhf_device_loop(basis, engine, dev, *, e_tol, rms_tol, diis_range, max_iter, precision, incremental, D0,
                     guess) -> ScfResult:
    import torch
    n = basis.nbf
    nocc = int(np.sum(basis.Z)) // 2
    f64 = dict(dtype=torch.float64, device=dev)
    M = torch.empty((3, n, n), **f64)
    engine.one_electron_device(M[0].data_ptr(), M[1].data_ptr(), M[2].data_ptr())
    S = M[0]
    H = M[1] + M[2]
    w, U = torch.linalg.eigh(S)
    X = (U * w.rsqrt()) @ U.T
    J = torch.empty((n, n), **f64)
    K = torch.empty((n, n), **f64)

    def two_e(Dm):
        Dm = Dm.contiguous()
        engine.jk_device(Dm.data_ptr(), 1, Dm.data_ptr(), J.data_ptr(), K.data_ptr(), precision)
        return 2.0 * J - K

    if D0 is None and guess == "sad":
        D0 = sad_guess(basis)
    if D0 is None:
        eps, Cp = torch.linalg.eigh(X.T @ H @ X)
        C = X @ Cp
        D = C[:, :nocc] @ C[:, :nocc].T
    else:
        D = torch.from_numpy(np.ascontiguousarray(D0)).to(dev)
        C = eps = None
    E = float((D * (H + H)).sum())
    res = ScfResult(0, 0, 0, None, None, None, None, 0, False)
    # DIIS history in fixed device slots (no host round trip): diis_range + 1 slots; once all
    # are used, the new vector replaces the slot of the LARGEST rms, which is the reference's
    # "drop the largest-error entry, then append" (hfscf_diis.cpp:23-41) with the order of the
    # stored vectors, which the extrapolation does not depend on, left free.
    Pq = torch.empty((n, n), **f64)
    perr = torch.zeros((), **f64)
    cap = diis_range + 1
    Fs = torch.zeros((cap, n, n), **f64)
    Es = torch.zeros((cap, n * n), **f64)
    rms_d = torch.zeros(cap, **f64)
    used = 0
    F_last = D_last = None
    ev = []  # CUDA events around every Fock build, read once at the end
    it = 0
    while True:
        it += 1
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        if incremental and F_last is not None and (it % 8) != 0:
            F = F_last + two_e(D - D_last)
        else:
            F = H + two_e(D)
        e1.record()
        ev.append((e0, e1))
        F_last, D_last = F, D
        FDS = F @ D @ S
        err = X.T @ (FDS - FDS.T) @ X
        rms_t = err.square().mean().sqrt()
        if used < cap:
            slot = torch.tensor(used, device=dev)
            used += 1
        else:
            slot = torch.argmax(rms_d)
        Fs.index_copy_(0, slot.reshape(1), F.reshape(1, n, n))
        Es.index_copy_(0, slot.reshape(1), err.reshape(1, -1))
        rms_d.index_copy_(0, slot.reshape(1), rms_t.reshape(1))
        m = used
        if m > 1:
            Bm = Es[:m] @ Es[:m].T
            Bm = torch.where(Bm.abs().sum() < DIIS_EPS, Bm / Bm.max(), Bm)
            B = torch.full((m + 1, m + 1), -1.0, **f64)
            B[:m, :m] = Bm
            B[m, m] = 0.0
            rhs = torch.zeros(m + 1, **f64)
            rhs[m] = -1.0
            cvec = torch.linalg.solve_ex(B, rhs)[0][:m]  # no host check of the LU info
            F = torch.einsum("k,kij->ij", cvec, Fs[:m])
        # the new density: trace-correcting purification of X^T F X on the device
        # (hfgpu_purify_device; the same projector as C_occ C_occ^T of the diagonalisation of
        # src/scfsolver/hfscf_hf_solver.cpp:206-231), with the diagonalisation as the fallback
        # when the projector has not converged (no gap at nocc)
        Fo = (X.T @ F @ X).contiguous()
        engine.purify_device(Fo.data_ptr(), n, nocc, PURIFY_STEPS, Pq.data_ptr(), perr.data_ptr())
        D = X @ Pq @ X.T
        # one host round trip per iteration: the rms, the energy and the purification error
        rms, E_new, pe = (float(v) for v in torch.stack([rms_t, (D * (H + F)).sum(), perr]).cpu())
        if not pe < PURIFY_TOL:
            eps, Cp = torch.linalg.eigh(X.T @ F @ X)
            C = X @ Cp
            D = C[:, :nocc] @ C[:, :nocc].T
            E_new = float((D * (H + F)).sum())
            res.diag_fallbacks += 1
        E_prev, E = E, E_new
        res.energies.append(E)
        if rms < rms_tol and abs(E - E_prev) < e_tol:
            res.converged = True
            break
        if it >= max_iter:
            break
    res.fock_times = [a.elapsed_time(b) / 1e3 for a, b in ev]
    F = H + two_e(D)
    E = float((D * (H + F)).sum())
    # orbitals and orbital energies once, at the converged density's Fock matrix
    eps, Cp = torch.linalg.eigh(X.T @ F @ X)
    C = X @ Cp
    enuc = nuclear_repulsion(basis.Z, basis.coords)
    res.energy, res.e_elec, res.e_nuc = E + enuc, E, enuc
    res.D, res.F, res.C, res.eps = D.cpu().numpy(), F.cpu().numpy(), C.cpu().numpy(), eps.cpu().numpy()
    res.iterations = it
    return res


def rhf_gradient(basis: Basis, res: ScfResult, engine, precision=eng.FP64):
    """Full RHF gradient (natoms x 3), as Mol::scf_gradient::calc_scf_gradient_rhf
    (src/gradient/hfscf_grad_rhf.cpp:7-178) assembles it."""
    D, F = res.D, res.F
    if isinstance(engine, eng.Engine):
        return _rhf_gradient_device(basis, D, F, engine, precision)
    Q = D @ F @ D
    g = engine.grad2e(D, 1.0, precision)
    g += engine.one_electron_grad(D, Q, 2.0, -2.0)
    g += nuclear_repulsion_gradient(basis.Z, basis.coords)
    return g


def _rhf_gradient_device(basis: Basis, D, F, engine, precision):
    """rhf_gradient on the engine's GPU: Q = D F D there, and the two-electron term
    (hfgpu_grad2e_device, RHF weights) and the one-electron term (hfgpu_one_electron_grad_device)
    on two streams at once, so the one-electron kernel runs beside the tail of the two-electron
    classes; one host read of the summed gradient."""
    import torch
    dev = torch.device("cuda", engine._opts.device)
    prev = engine.stream_ptr
    s2, s1 = torch.cuda.Stream(dev), torch.cuda.Stream(dev)
    Dd = torch.from_numpy(np.ascontiguousarray(D)).to(dev)
    Fd = torch.from_numpy(np.ascontiguousarray(F)).to(dev)
    Qd = (Dd @ Fd @ Dd).contiguous()
    g2 = torch.zeros((basis.natoms, 3), dtype=torch.float64, device=dev)
    g1 = torch.zeros_like(g2)
    torch.cuda.synchronize(dev)  # inputs in place before either stream starts
    try:
        engine.set_stream(s2.cuda_stream)
        engine.grad2e_device(Dd.data_ptr(), 2.0, 1, Dd.data_ptr(), 1.0, g2.data_ptr(), precision)
        engine.set_stream(s1.cuda_stream)
        engine.one_electron_grad_device(Dd.data_ptr(), Qd.data_ptr(), 2.0, -2.0, g1.data_ptr())
        torch.cuda.synchronize(dev)
    finally:
        engine.set_stream(prev)
    g = (g2 + g1).cpu().numpy()
    if not np.all(np.isfinite(g)):
        raise eng.HfgpuError(5, "non-finite gradient")
    return g + nuclear_repulsion_gradient(basis.Z, basis.coords)


def uhf(basis: Basis, engine, *, multiplicity=1, e_tol=1e-10, rms_tol=1e-8, diis_range=5, max_iter=100,
        precision=eng.FP64):
    """Unrestricted HF with the GPU UHF Fock build, as Mol::uhf_solver runs it
    (src/scfsolver/hfscf_uhf_solver.cpp:155-225): F_a = H + J[Da+Db] - K[Da] from the engine,
    two-spin DIIS (DiisUhf, the reference's diis_extrapolate for UHF), core guess without
    HOMO/LUMO mixing (the default), energy 1/2 sum[Da (H + Fa) + Db (H + Fb)], converged when
    both spins' rms and |dE| are below the tolerances."""
    nel = int(np.sum(basis.Z))
    na = (nel + multiplicity - 1) // 2
    nb = nel - na
    S, T, V = engine.one_electron()
    H = T + V
    X = sym_orth(S)
    eps, Cp = np.linalg.eigh(X.T @ H @ X)
    C = X @ Cp
    Da, Db = C[:, :na] @ C[:, :na].T, C[:, :nb] @ C[:, :nb].T
    E = float(np.sum(Da * (H + H)))
    diis = DiisUhf(diis_range)
    it = 0
    converged = False
    while True:
        it += 1
        Fa, Fb = engine.fock_uhf(Da, Db, H, precision)
        Fa, Fb = diis.extrapolate(Fa, Fb, S, Da, Db, X)
        _, Ca = np.linalg.eigh(X.T @ Fa @ X)
        _, Cb = np.linalg.eigh(X.T @ Fb @ X)
        Ca, Cb = X @ Ca, X @ Cb
        Da, Db = Ca[:, :na] @ Ca[:, :na].T, Cb[:, :nb] @ Cb[:, :nb].T
        E_prev = E
        E = 0.5 * float(np.sum(Da * (H + Fa)) + np.sum(Db * (H + Fb)))
        if diis.rms_a < rms_tol and diis.rms_b < rms_tol and abs(E - E_prev) < e_tol:
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
