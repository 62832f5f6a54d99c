"""Batched RHF: hundreds of small molecules solved together on one GPU.

One batched engine handle holds every molecule (hfgpu_batch_create).  Each SCF
iteration is one J/K build for all molecules at once -- the per-class kernels
cover every molecule's quartets -- captured once as a CUDA graph and replayed.
DIIS and the Fock assembly run batched on the GPU in torch over matrices padded to
the largest molecule, and every molecule's Fock matrix is diagonalised in one launch
of the batched Jacobi eigensolver (hfgpu_batch_eigh), which also gives the
orthogonalisers S^-1/2.  S, T and V of every molecule come from one device launch.
After convergence, the two-electron gradient of every molecule comes from one
batched adjoint launch (hfgpu_batch_grad2e_device) and the one-electron part from
one more (hfgpu_one_electron_grad_device); only the nuclear repulsion term is added
on the host.  With diag="host" the diagonalisations run per molecule on a host
thread pool instead.

The SCF is the caller side, as in scf.py: symmetric orthogonalisation, D =
C_occ C_occ^T (no factor 2), E = sum D (H + F), DIIS on the orthogonalised
commutator.  Here DIIS keeps the last 6 vectors per molecule.
"""
from __future__ import annotations

import concurrent.futures as cf
import ctypes
import os
import time

import numpy as np
import torch

from . import engine as eng
from .basis import Basis, build_basis, nuclear_repulsion, nuclear_repulsion_gradient
from .scf import DIIS_EPS

PURIFY_TOL = 1e-10  # largest tr P - tr P^2 accepted from a molecule's purification
PURIFY_STEPS = 64   # squarings of one purification (each molecule stops at its converged step)
PAD_DIAG = 1.0e3  # padded diagonal of F: far above every occupied orbital energy


class BatchEngine:
    """A batched engine handle over many Cartesian molecules."""

    def __init__(self, bases: list[Basis], device: int = 0, schwarz_tol: float = 1e-12):
        self.bases = bases
        self.nmol = len(bases)
        self._views = [eng._BasisView(b) for b in bases]
        arr = (eng._Basis * self.nmol)(*[v.s for v in self._views])
        self._xyz = [np.ascontiguousarray(b.coords, dtype=np.float64) for b in bases]
        ptrs = (ctypes.POINTER(ctypes.c_double) * self.nmol)(*[eng._p(x) for x in self._xyz])
        o = eng._Opts()
        eng.lib().hfgpu_default_opts(ctypes.byref(o))
        o.schwarz_tol, o.device = schwarz_tol, device
        h = ctypes.c_void_p()
        rc = eng.lib().hfgpu_batch_create(ctypes.c_int(self.nmol), arr, ptrs, ctypes.byref(o), ctypes.byref(h))
        if rc:
            raise eng.HfgpuError(rc, "hfgpu_batch_create")
        self.h = h
        nbf = (ctypes.c_int * self.nmol)()
        off = (ctypes.c_longlong * self.nmol)()
        tot = ctypes.c_longlong()
        eng.lib().hfgpu_batch_layout(h, nbf, off, ctypes.byref(tot))
        self.nbf = np.array(list(nbf), dtype=np.int64)
        self.mat_off = np.array(list(off), dtype=np.int64)
        self.mat_total = int(tot.value)
        self.natoms = np.array([b.natoms for b in bases], dtype=np.int64)
        self.atom_off = np.concatenate([[0], np.cumsum(self.natoms)])

    def _check(self, rc):
        if rc:
            raise eng.HfgpuError(rc, eng.lib().hfgpu_last_error(self.h).decode())

    def setup_times(self):
        """Host wall time (s) of the handle's set-up: primitive pairs, Schwarz factors,
        quartet lists, list upload (hfgpu_setup_times)."""
        ms = (ctypes.c_double * 4)()
        self._check(eng.lib().hfgpu_setup_times(self.h, ms))
        return dict(zip(("pairs", "schwarz", "lists", "upload"), [v / 1e3 for v in ms]))

    def set_stream(self, stream_ptr):
        self._check(eng.lib().hfgpu_set_stream(self.h, ctypes.c_void_p(stream_ptr) if stream_ptr else None))

    def jk_device(self, D, J, K, precision=eng.FP64):
        self._check(eng.lib().hfgpu_batch_jk_device(self.h, ctypes.c_void_p(D.data_ptr()), ctypes.c_void_p(J.data_ptr()),
                                                    ctypes.c_void_p(K.data_ptr()), ctypes.c_int(precision)))

    def one_electron_device(self, S, T, V):
        """S, T, V of every molecule into block storage (device tensors), on the GPU."""
        Z = np.ascontiguousarray(np.concatenate([np.asarray(b.Z, dtype=np.float64) for b in self.bases]))
        self._check(eng.lib().hfgpu_one_electron_device(self.h, eng._p(Z), ctypes.c_void_p(S.data_ptr()),
                                                        ctypes.c_void_p(T.data_ptr()), ctypes.c_void_p(V.data_ptr())))

    def one_electron_grad_device(self, D, W, cH, cS, grad):
        """grad (device, total atoms x 3) += cH sum D d(T+V)/dX + cS sum W dS/dX, every molecule."""
        Z = np.ascontiguousarray(np.concatenate([np.asarray(b.Z, dtype=np.float64) for b in self.bases]))
        self._check(eng.lib().hfgpu_one_electron_grad_device(self.h, eng._p(Z), ctypes.c_void_p(D.data_ptr()),
                                                             ctypes.c_void_p(W.data_ptr()), ctypes.c_double(cH),
                                                             ctypes.c_double(cS), ctypes.c_void_p(grad.data_ptr())))

    def autotune(self, D, precision=eng.FP64, repeats=2):
        """hfgpu_autotune on the batched handle (D in block storage, on the device)."""
        out = np.zeros((eng.NUM_CLASSES, 4), dtype=np.int32)
        self._check(eng.lib().hfgpu_autotune(self.h, ctypes.c_void_p(D.data_ptr()), ctypes.c_int(precision),
                                             ctypes.c_int(repeats), out.ctypes.data_as(eng._ip)))
        return out

    def set_schedule(self, schedule):
        """hfgpu_set_schedule on the batched handle (HFGPU_NUM_CLASSES x 4 ints)."""
        sched = np.ascontiguousarray(schedule, dtype=np.int32)
        self._check(eng.lib().hfgpu_set_schedule(self.h, sched.ctypes.data_as(eng._ip)))

    def eigh(self, A, W, V, sweeps=None):
        """hfgpu_batch_eigh: eigenvalues (ascending) and eigenvectors of every molecule's block of
        the padded batch A [nmol, nmax, nmax] (device tensors)."""
        self._check(eng.lib().hfgpu_batch_eigh(self.h, ctypes.c_void_p(A.data_ptr()), ctypes.c_void_p(W.data_ptr()),
                                               ctypes.c_void_p(V.data_ptr()),
                                               ctypes.c_void_p(sweeps.data_ptr() if sweeps is not None else 0)))

    def purify(self, Fo, nocc, P, err, max_steps=64):
        """hfgpu_batch_purify_device: P = projector onto the nocc lowest eigenvectors of every
        molecule's block of the padded Fo [nmol, nmax, nmax]; err [nmol] (device tensors; nocc int32)."""
        self._check(eng.lib().hfgpu_batch_purify_device(self.h, ctypes.c_void_p(Fo.data_ptr()),
                                                        ctypes.c_void_p(nocc.data_ptr()), ctypes.c_int(max_steps),
                                                        ctypes.c_void_p(P.data_ptr()), ctypes.c_void_p(err.data_ptr())))

    def grad2e_device(self, D, grad, precision=eng.FP64):
        self._check(eng.lib().hfgpu_batch_grad2e_device(self.h, ctypes.c_void_p(D.data_ptr()),
                                                        ctypes.c_void_p(grad.data_ptr()), ctypes.c_int(precision)))

    def close(self):
        if getattr(self, "h", None) is not None:
            eng.lib().hfgpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class _Layout:
    """Index maps between block storage (molecule m: n_m x n_m at mat_off[m]) and
    padded batched matrices [nmol, nmax, nmax]."""

    def __init__(self, nbf, mat_off, device):
        self.nmol = len(nbf)
        self.nmax = int(nbf.max())
        idx = []
        for m, (n, off) in enumerate(zip(nbf, mat_off)):
            i, j = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
            idx.append(m * self.nmax * self.nmax + i.ravel() * self.nmax + j.ravel())
        self.pad_index = torch.from_numpy(np.concatenate(idx)).to(device)
        mask = np.zeros((self.nmol, self.nmax), dtype=bool)
        for m, n in enumerate(nbf):
            mask[m, :n] = True
        self.mask = torch.from_numpy(mask).to(device)

    def to_block(self, Mp):
        return Mp.reshape(-1)[self.pad_index]

    def to_pad(self, Mb, fill_diag=0.0):
        out = torch.zeros((self.nmol * self.nmax * self.nmax,), dtype=Mb.dtype, device=Mb.device)
        out[self.pad_index] = Mb
        out = out.view(self.nmol, self.nmax, self.nmax)
        if fill_diag:
            d = torch.diagonal(out, dim1=1, dim2=2)
            d += (~self.mask).to(out.dtype) * fill_diag
        return out


def batch_sad_guess(bases: list[Basis], nmax: int, engine_factory=None) -> np.ndarray:
    """SAD guess of every molecule, padded to nmax (the reference's default guess,
    Mol::hf_solver::get_sad_guess, src/scfsolver/hfscf_hf_solver.cpp:478-553): the atomic UHF of
    each (basis set, element) pair runs once (scf.sad_atom_density on a GPU engine of that atom's
    shells) and its spin-averaged density is copied onto every atom of that element in every
    molecule with that basis set.  ``engine_factory(atom_basis)`` makes the context-managed engine
    of an atom (default: eng.Engine)."""
    from . import scf as _scf
    factory = engine_factory or eng.Engine
    cache = {}
    D = np.zeros((len(bases), nmax, nmax))
    for k, b in enumerate(bases):
        # an atom's functions are contiguous, atoms in order
        off = np.concatenate([[0], np.cumsum(np.bincount(b.bf_atom(), minlength=len(b.Z)))])
        for a, Zc in enumerate(b.Z.tolist()):
            key = (b.name, bool(b.pure), int(Zc))
            if key not in cache:
                with factory(_scf.atom_basis(b, a)) as e:
                    S, T, V = e.one_electron()
                    cache[key] = _scf.sad_atom_density(int(Zc), S, T, V, lambda DJ, DKs: e.jk(DJ, DKs))
            D[k, off[a]:off[a + 1], off[a]:off[a + 1]] = cache[key]
    return D


def batch_rhf(bases: list[Basis], device: int = 0, precision=eng.FP64, e_tol=1e-10, rms_tol=1e-8,
              max_iter=60, use_graph=True, gradient=True, autotune=False, diag="purify", diis_range=5,
              schedule=None, freeze_converged=False, guess="sad"):
    """Converged RHF energies (and gradients) of every molecule of the batch.  ``diag``:
    "purify" (default) takes every molecule's density from one launch of the batched
    trace-correcting purification (hfgpu_batch_purify_device, molecules of up to 116 functions),
    diagonalising with the batched Jacobi kernel instead in an iteration where some molecule's
    purification did not converge; "gpu" diagonalises every iteration with the batched Jacobi
    kernel (hfgpu_batch_eigh, molecules of up to 118 functions); "host" runs LAPACK per
    molecule on a host thread pool.  ``autotune`` runs hfgpu_autotune on the first density
    before the graph is captured (off by default: for 512 small molecules it cost 2.4 s and
    bought nothing over the default schedule).  ``schedule``: a launch schedule to use instead
    (e.g. one the autotuner returned for the same batch in an earlier, untimed run); the result
    dict's "schedule" is the schedule the run used.  ``guess``: "sad" (default, the
    reference's default: superposition of atomic densities, batch_sad_guess) or "core" (the
    orbitals of the core Hamiltonian).  ``freeze_converged``: a molecule that has
    met the convergence test stops iterating, as its own SCF would (its density and energy are
    kept, its quartets are skipped by the density screening of the later builds); without it
    every molecule iterates until the last one converges (the default: the frozen molecules' quartets
    are still launched and skipped one by one, so freezing saved no time on the 512-molecule
    batch, 0.64 against 0.65 s of SCF, and moved no energy by more than 3e-13 Eh)."""
    dev = torch.device("cuda", device)
    t0 = time.perf_counter()
    stages = {}

    def stage(name, t_start):
        torch.cuda.synchronize()
        stages[name] = time.perf_counter() - t_start
        return time.perf_counter()

    be = BatchEngine(bases, device)
    tt = stage("handle", t0)
    for k, v in be.setup_times().items():
        stages["handle_" + k] = v
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    be.set_stream(stream.cuda_stream)
    lay = _Layout(be.nbf, be.mat_off, dev)
    nmol, nmax = lay.nmol, lay.nmax
    # one-electron matrices of every molecule, on the GPU, into block storage
    Sblk = torch.empty(be.mat_total, dtype=torch.float64, device=dev)
    Tblk = torch.empty_like(Sblk)
    Vblk = torch.empty_like(Sblk)
    be.one_electron_device(Sblk, Tblk, Vblk)
    Hblk = Tblk + Vblk
    del Tblk, Vblk
    S = lay.to_pad(Sblk, fill_diag=1.0)
    H = lay.to_pad(Hblk, fill_diag=PAD_DIAG)
    tt = stage("one_electron", tt)
    Wev = torch.empty((nmol, nmax), dtype=torch.float64, device=dev)
    Vev = torch.empty((nmol, nmax, nmax), dtype=torch.float64, device=dev)
    # symmetric orthogonalisers X = S^-1/2 (padding: identity)
    Xh = []
    if diag == "purify" and nmax > 116:
        diag = "gpu"  # the purification keeps a molecule's matrix in one block's shared memory
    if diag in ("gpu", "purify"):
        be.eigh(S, Wev, Vev)
        X = (Vev * Wev.rsqrt()[:, None, :]) @ Vev.transpose(1, 2)
    else:
        # per-molecule LAPACK on the host; the diagonalisations of the SCF run there too,
        # on a thread pool over the unpadded blocks (LAPACK releases the GIL)
        Sh_all = Sblk.cpu().numpy()
        Xpad = np.zeros((nmol, nmax, nmax))
        for k, b in enumerate(bases):
            n, o = b.nbf, int(be.mat_off[k])
            w, U = np.linalg.eigh(Sh_all[o:o + n * n].reshape(n, n))
            Xh.append((U / np.sqrt(w)) @ U.T)
            Xpad[k, :n, :n] = Xh[-1]
            Xpad[k, np.arange(n, nmax), np.arange(n, nmax)] = 1.0
        X = torch.from_numpy(Xpad).to(dev)
    nocc_h = [int(np.sum(b.Z)) // 2 for b in bases]
    pool = cf.ThreadPoolExecutor(max_workers=max(1, min(32, os.cpu_count() or 1)))
    Dh = np.zeros(be.mat_total)

    occ = (torch.arange(nmax, device=dev)[None, :] <
           torch.tensor(nocc_h, device=dev)[:, None]).to(torch.float64)
    tt = stage("orthogonaliser", tt)

    def density_gpu(F):
        Fp = X.transpose(1, 2) @ F @ X
        Fp = 0.5 * (Fp + Fp.transpose(1, 2))
        be.eigh(Fp, Wev, Vev)
        C = X @ Vev
        return (C * occ[:, None, :]) @ C.transpose(1, 2)

    nocc_d = torch.tensor(nocc_h, dtype=torch.int32, device=dev)
    Ppur = torch.empty((nmol, nmax, nmax), dtype=torch.float64, device=dev)
    perr = torch.empty(nmol, dtype=torch.float64, device=dev)
    fallbacks = [0]

    def density_purify(F):
        Fp = X.transpose(1, 2) @ F @ X
        Fp = (0.5 * (Fp + Fp.transpose(1, 2))).contiguous()
        be.purify(Fp, nocc_d, Ppur, perr, PURIFY_STEPS)
        return X @ Ppur @ X.transpose(1, 2)

    def density(F):
        if diag == "purify":
            return density_purify(F)
        if diag == "gpu":
            return density_gpu(F)
        Fh = lay.to_block(F).cpu().numpy()

        def one(k):
            n, off = int(be.nbf[k]), int(be.mat_off[k])
            Fk = Fh[off:off + n * n].reshape(n, n)
            _, Cp = np.linalg.eigh(Xh[k].T @ Fk @ Xh[k])
            C = Xh[k] @ Cp[:, :nocc_h[k]]
            Dh[off:off + n * n] = (C @ C.T).ravel()

        list(pool.map(one, range(nmol)))
        return lay.to_pad(torch.from_numpy(Dh).to(dev))

    if guess == "sad":
        D = torch.from_numpy(batch_sad_guess(bases, nmax)).to(dev)
    else:
        D = density(H)
        if diag == "purify" and bool((perr >= PURIFY_TOL).any()):
            D = density_gpu(H)
            fallbacks[0] += 1
    Dblk = lay.to_block(D).contiguous()
    Jblk = torch.zeros_like(Dblk)
    Kblk = torch.zeros_like(Dblk)
    Fblk = torch.zeros_like(Dblk)

    def build():
        be.jk_device(Dblk, Jblk, Kblk, precision)
        torch.add(Hblk, Jblk, alpha=2.0, out=Fblk)
        Fblk.sub_(Kblk)

    tuned = False
    if schedule is not None:
        be.set_schedule(schedule)
        tuned = True
    build()  # warm-up: loads every kernel before any capture
    tt = stage("guess_and_first_build", tt)
    if autotune:
        schedule = be.autotune(Dblk, precision)
        tuned = True
    tt = stage("autotune", tt)
    graph = None
    if use_graph:
        try:
            graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(graph, stream=stream):
                build()
            torch.cuda.synchronize()
        except Exception:
            graph = None
            torch.cuda.synchronize()
    tt = stage("graph_capture", tt)
    t_setup = time.perf_counter() - t0
    # DIIS history per molecule (the reference's diis_extrapolate, src/scfsolver/hfscf_diis.cpp:9-123):
    # beyond diis_range vectors each molecule drops its own LARGEST-error entry before the new
    # one is added; the B matrix is rescaled where sum|B| < 1e-14
    hF = hE = hR = None  # [nmol, m, n, n], [nmol, m, n*n], [nmol, m]
    E_prev = torch.zeros(nmol, dtype=torch.float64, device=dev)
    converged = torch.zeros(nmol, dtype=torch.bool, device=dev)
    n_per = torch.from_numpy(be.nbf).to(dev).to(torch.float64)
    it = 0
    build_events = []
    t1 = time.perf_counter()
    while it < max_iter:
        it += 1
        if freeze_converged and it > 1:
            # a converged molecule stops, as its own SCF would: its block of the density is zeroed
            # for the build (density screening then skips its quartets) and its D is kept
            Dblk.copy_(lay.to_block(D * (~converged).to(D.dtype)[:, None, None]))
        else:
            Dblk.copy_(lay.to_block(D))
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        if graph is not None:
            graph.replay()
        else:
            build()
        ev1.record(stream)
        build_events.append((ev0, ev1))
        F = lay.to_pad(Fblk, fill_diag=PAD_DIAG)
        FDS = F @ D @ S
        err = X.transpose(1, 2) @ (FDS - FDS.transpose(1, 2)) @ X
        rms = torch.sqrt((err * err).sum(dim=(1, 2)) / (n_per * n_per))
        if hF is not None and hF.shape[1] > diis_range:
            keep = torch.arange(hF.shape[1], device=dev)[None, :] != hR.argmax(dim=1)[:, None]
            m1 = hF.shape[1] - 1
            hF = hF[keep].reshape(nmol, m1, *hF.shape[2:])
            hE = hE[keep].reshape(nmol, m1, -1)
            hR = hR[keep].reshape(nmol, m1)
        if hF is None:
            hF, hE, hR = F[:, None], err.reshape(nmol, 1, -1), rms[:, None]
        else:
            hF = torch.cat([hF, F[:, None]], dim=1)
            hE = torch.cat([hE, err.reshape(nmol, 1, -1)], dim=1)
            hR = torch.cat([hR, rms[:, None]], dim=1)
        m = hF.shape[1]
        if m > 1:
            Bm = hE @ hE.transpose(1, 2)
            small = Bm.abs().sum(dim=(1, 2)) < DIIS_EPS
            Bm = torch.where(small[:, None, None], Bm / Bm.amax(dim=(1, 2), keepdim=True), Bm)
            B = -torch.ones((nmol, m + 1, m + 1), dtype=torch.float64, device=dev)
            B[:, :m, :m] = Bm
            B[:, m, m] = 0.0
            rhs = torch.zeros((nmol, m + 1), dtype=torch.float64, device=dev)
            rhs[:, m] = -1.0
            c = torch.linalg.solve(B, rhs)[:, :m]
            F = torch.einsum("bk,bkij->bij", c, hF)
        D_prev = D
        D = density(F)
        E = ((D * (H + F)).sum(dim=(1, 2)) - PAD_DIAG * 0)  # padded entries of D are zero
        conv = (rms < rms_tol) & ((E - E_prev).abs() < e_tol)
        if freeze_converged:
            # molecules converged at an earlier iteration keep their density and energy (their
            # F of this iteration was built from a zero density block and is not used)
            D = torch.where(converged[:, None, None], D_prev, D)
            E = torch.where(converged, E_prev, E)
            conv = conv | converged
        if diag == "purify":
            # one host read per iteration: whether every molecule converged, and whether some
            # molecule's purification did not (then this iteration diagonalises instead)
            flags = torch.stack([(perr >= PURIFY_TOL).any(), (converged | conv).all()]).cpu()
            if bool(flags[0]):
                fallbacks[0] += 1
                D = density_gpu(F)
                E = (D * (H + F)).sum(dim=(1, 2))
                conv = (rms < rms_tol) & ((E - E_prev).abs() < e_tol)
                if freeze_converged:
                    D = torch.where(converged[:, None, None], D_prev, D)
                    E = torch.where(converged, E_prev, E)
                    conv = conv | converged
                done = bool((converged | conv).all())
            else:
                done = bool(flags[1])
        else:
            done = bool((converged | conv).all())
        converged |= conv
        E_prev = E
        if done:
            break
    torch.cuda.synchronize()
    t_scf = time.perf_counter() - t1
    t_fin = time.perf_counter()
    # final Fock matrices at the converged densities
    Dblk.copy_(lay.to_block(D))
    build()
    F = lay.to_pad(Fblk, fill_diag=0.0)
    Dz = D
    E_el = (Dz * (lay.to_pad(Hblk) + F)).sum(dim=(1, 2)).cpu().numpy()
    enuc = np.array([nuclear_repulsion(b.Z, b.coords) for b in bases])
    out = {"energies": E_el + enuc, "iterations": it, "converged": converged.cpu().numpy(),
           "setup_s": t_setup, "setup_stages_s": stages, "scf_s": t_scf, "graph": graph is not None,
           "autotuned": tuned, "schedule": schedule, "density": diag, "diag_fallbacks": fallbacks[0],
           "build_ms_mean": float(np.mean([a.elapsed_time(b) for a, b in build_events])), "nmol": nmol,
           "final_s": time.perf_counter() - t_fin}
    if gradient:
        t2 = time.perf_counter()
        g = torch.zeros((int(be.atom_off[-1]), 3), dtype=torch.float64, device=dev)
        be.grad2e_device(Dblk, g, precision)
        # one-electron part on the GPU: 2 sum D d(T+V)/dX - 2 sum Q dS/dX with Q = D F D
        Qblk = lay.to_block(D @ F @ D).contiguous()
        be.one_electron_grad_device(Dblk, Qblk, 2.0, -2.0, g)
        torch.cuda.synchronize()
        g2 = g.cpu().numpy()
        grads = [g2[be.atom_off[k]:be.atom_off[k + 1]] + nuclear_repulsion_gradient(b.Z, b.coords)
                 for k, b in enumerate(bases)]
        out["gradients"] = grads
        out["grad_s"] = time.perf_counter() - t2
    t3 = time.perf_counter()
    pool.shutdown()
    be.close()
    torch.cuda.set_stream(torch.cuda.default_stream(dev))
    out["close_s"] = time.perf_counter() - t3
    return out


def batch_bases(molecules):
    """Cartesian bases for (Z, coords_bohr, basis_name, pure) tuples (s/p pure == Cartesian)."""
    return [build_basis(name, Z, x, pure=False) for Z, x, name, _ in molecules]
