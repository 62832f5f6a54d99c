"""Python mirror of the engine's C ABI (include/hfgpu.h).

``Erios`` mirrors the reference's integral-engine interface
(ERIOS::Erios, src/integrals/hfscf_oseri.hpp:27-123) and ``FockBuilder`` the
Fock hooks of Mol::hf_solver / Mol::uhf_solver
(src/scfsolver/hfscf_hf_solver.cpp:254-286, hfscf_uhf_solver.cpp:155-191).  Both
sit on one ``Engine`` handle.  Every call goes to the CUDA library
``libhfgpu.so``; there is no CPU fallback, and a missing library raises.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from .basis import Basis

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libhfgpu.so")

FP64, MIXED = 0, 1
STATUS = {0: "ok", 1: "invalid argument", 2: "out of memory", 3: "CUDA error", 4: "bad call order",
          5: "non-finite result", 6: "unsupported"}

_lib = None
_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


class HfgpuError(RuntimeError):
    def __init__(self, code, msg=""):
        super().__init__(f"hfgpu error {code} ({STATUS.get(code, '?')}): {msg}")
        self.code = code


class _Basis(ctypes.Structure):
    _fields_ = [("nshell", ctypes.c_int), ("natoms", ctypes.c_int), ("pure", ctypes.c_int),
                ("L", _ip), ("shell_atom", _ip), ("nprim", _ip), ("exps", _dp), ("coefs", _dp)]


class _Opts(ctypes.Structure):
    _fields_ = [("schwarz_tol", ctypes.c_double), ("density_tol", ctypes.c_double),
                ("mixed_fp32_bound", ctypes.c_double), ("mixed_density_tol", ctypes.c_double), ("device", ctypes.c_int),
                ("warp_max_quartets", ctypes.c_int), ("grad_warp_max_waves", ctypes.c_int),
                ("reserved", ctypes.c_int * 5)]


def lib():
    """The CUDA engine library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m hfscf_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        L.hfgpu_last_error.restype = ctypes.c_char_p
        _lib = L
    return _lib


def exported_symbols():
    """Names declared in include/hfgpu.h (checked against the library by the tests)."""
    import re
    hdr = os.path.join(os.path.dirname(HERE), "include", "hfgpu.h")
    text = open(hdr).read()
    return sorted(set(re.findall(r"^(?:int|long long|const char\*)\s+(hfgpu_[a-z0-9_]+)\s*\(", text, re.M)))


def _p(a, ct=ctypes.c_double):
    return a.ctypes.data_as(ctypes.POINTER(ct))


def _c(a, dtype=np.float64):
    return np.ascontiguousarray(a, dtype=dtype)


class _BasisView:
    """Keeps the flat basis arrays alive while the C struct points at them."""

    def __init__(self, basis: Basis):
        f = basis.flat()
        self.L = _c(f["L"], np.int32)
        self.atom = _c(f["atom"], np.int32)
        self.nprim = _c(f["nprim"], np.int32)
        self.exps = _c(f["exps"])
        self.coefs = _c(f["coefs"])
        self.s = _Basis(basis.nshell, basis.natoms, int(basis.pure), _p(self.L, ctypes.c_int),
                        _p(self.atom, ctypes.c_int), _p(self.nprim, ctypes.c_int), _p(self.exps), _p(self.coefs))


class Engine:
    """One engine handle: a basis on one GPU, with the current geometry."""

    def __init__(self, basis: Basis, schwarz_tol=1e-12, density_tol=1e-12, mixed_fp32_bound=1e-4, device=0,
                 warp_max_quartets=None, grad_warp_max_waves=None, stage_wait_test=False, grad_max_blocks=None):
        self.basis = basis
        self.n = basis.nbf
        self._bv = _BasisView(basis)
        o = _Opts()
        lib().hfgpu_default_opts(ctypes.byref(o))
        o.schwarz_tol, o.density_tol, o.mixed_fp32_bound, o.device = schwarz_tol, density_tol, mixed_fp32_bound, device
        if warp_max_quartets is not None:
            o.warp_max_quartets = warp_max_quartets
        if grad_warp_max_waves is not None:
            o.grad_warp_max_waves = grad_warp_max_waves
        if stage_wait_test:
            o.reserved[0] = 1  # staging waits run out on purpose (tests the bounded wait)
        if grad_max_blocks is not None:
            o.reserved[1] = grad_max_blocks
        self._opts = o
        self.stream_ptr = None  # the handle's own stream until set_stream
        h = ctypes.c_void_p()
        self._check(lib().hfgpu_create(ctypes.byref(self._bv.s), ctypes.byref(o), ctypes.byref(h)), None)
        self.h = h
        self.coords = None
        self.set_geometry(basis.coords)

    def _check(self, rc, h="self"):
        if rc != 0:
            msg = ""
            hh = self.h if h == "self" else h
            if hh is not None:
                msg = lib().hfgpu_last_error(hh).decode()
            raise HfgpuError(rc, msg)

    def close(self):
        if getattr(self, "h", None) is not None:
            lib().hfgpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # --- geometry / integrals -------------------------------------------------
    def set_geometry(self, coords_bohr):
        c = _c(coords_bohr).reshape(-1, 3)
        self._check(lib().hfgpu_set_geometry(self.h, _p(c), ctypes.c_int(len(c))))
        self.coords = c.copy()
        self.basis = self.basis.with_coords(c)

    def schwarz(self) -> np.ndarray:
        ns = self.basis.nshell
        Q = np.zeros((ns, ns))
        self._check(lib().hfgpu_schwarz(self.h, _p(Q)))
        return Q

    def boys(self, m, T, precision=FP64) -> np.ndarray:
        """F_0..F_m at the points T through the engine's Boys evaluation (hfgpu_boys):
        shape (len(T), m + 1)."""
        T = _c(np.atleast_1d(T))
        F = np.zeros((len(T), m + 1))
        self._check(lib().hfgpu_boys(self.h, ctypes.c_int(precision), ctypes.c_int(m), _p(T),
                                     ctypes.c_longlong(len(T)), _p(F)))
        return F

    def eri_packed(self) -> np.ndarray:
        n = self.n
        ln = n * (n + 1) * (n * n + n + 2) // 8
        out = np.zeros(ln)
        self._check(lib().hfgpu_eri_packed(self.h, _p(out), ctypes.c_longlong(ln)))
        return out

    # --- Fock builds -----------------------------------------------------------
    def jk(self, DJ=None, DKs=(), precision=FP64):
        n = self.n
        DJc = _c(DJ) if DJ is not None else None
        DK = _c(np.stack(DKs)) if len(DKs) else np.zeros((0, n, n))
        J = np.zeros((n, n))
        K = np.zeros((len(DKs), n, n))
        self._check(lib().hfgpu_jk(self.h, _p(DJc) if DJc is not None else None, ctypes.c_int(len(DKs)),
                                   _p(DK) if len(DKs) else None, _p(J), _p(K) if len(DKs) else None,
                                   ctypes.c_int(precision)))
        return (J if DJ is not None else None), K

    def fock_rhf(self, D, H, precision=FP64) -> np.ndarray:
        F = np.zeros((self.n, self.n))
        self._check(lib().hfgpu_fock_rhf(self.h, _p(_c(D)), _p(_c(H)), _p(F), ctypes.c_int(precision)))
        return F

    def fock_uhf(self, Da, Db, H, precision=FP64):
        Fa, Fb = np.zeros((self.n, self.n)), np.zeros((self.n, self.n))
        self._check(lib().hfgpu_fock_uhf(self.h, _p(_c(Da)), _p(_c(Db)), _p(_c(H)), _p(Fa), _p(Fb),
                                         ctypes.c_int(precision)))
        return Fa, Fb

    def fock_delta(self, dD, F, precision=FP64) -> np.ndarray:
        F = _c(F).copy()
        self._check(lib().hfgpu_fock_delta(self.h, _p(_c(dD)), _p(F), ctypes.c_int(precision)))
        return F

    # --- device-pointer calls (torch tensors or raw addresses) -----------------
    def set_stream(self, stream_ptr: int | None):
        self._check(lib().hfgpu_set_stream(self.h, ctypes.c_void_p(stream_ptr) if stream_ptr else None))
        self.stream_ptr = stream_ptr or None

    def jk_device(self, DJ_ptr, nK, DK_ptr, J_ptr, K_ptr, precision=FP64):
        self._check(lib().hfgpu_jk_device(self.h, ctypes.c_void_p(DJ_ptr), ctypes.c_int(nK), ctypes.c_void_p(DK_ptr),
                                          ctypes.c_void_p(J_ptr), ctypes.c_void_p(K_ptr), ctypes.c_int(precision)))

    def grad2e_device(self, DJ_ptr, cJ, nK, DK_ptr, cK, grad_ptr, precision=FP64):
        self._check(lib().hfgpu_grad2e_device(self.h, ctypes.c_void_p(DJ_ptr), ctypes.c_double(cJ), ctypes.c_int(nK),
                                              ctypes.c_void_p(DK_ptr), ctypes.c_double(cK), ctypes.c_void_p(grad_ptr),
                                              ctypes.c_int(precision)))

    def fock_rhf_ptr(self, D_ptr, H_ptr, F_ptr, precision=FP64):
        """hfgpu_fock_rhf on raw host pointers (e.g. pinned buffers)."""
        self._check(lib().hfgpu_fock_rhf(self.h, ctypes.c_void_p(D_ptr), ctypes.c_void_p(H_ptr),
                                         ctypes.c_void_p(F_ptr), ctypes.c_int(precision)))

    # --- measurement hooks ------------------------------------------------------
    def set_timing(self, on: bool):
        self._check(lib().hfgpu_set_timing(self.h, ctypes.c_int(int(on))))

    def class_stats(self, cls: int):
        out = (ctypes.c_longlong * 9)()
        self._check(lib().hfgpu_class_stats(self.h, ctypes.c_int(cls), out))
        keys = ("la", "lb", "lc", "ld", "screened", "high_bound", "computed", "skipped", "prim_quartets")
        return dict(zip(keys, list(out)))

    def set_partition(self, part: int, nparts: int):
        """hfgpu_set_partition: later J/K builds and gradients compute only quartets part,
        part + nparts, ... of every class list (partial outputs, summed over the parts)."""
        self._check(lib().hfgpu_set_partition(self.h, ctypes.c_int(part), ctypes.c_int(nparts)))

    def class_work(self, cls: int):
        """hfgpu_class_work: Schwarz-screened quartets of class cls and their primitive quartets."""
        out = (ctypes.c_longlong * 2)()
        self._check(lib().hfgpu_class_work(self.h, ctypes.c_int(cls), out))
        return {"quartets": out[0], "prim_quartets": out[1]}

    def setup_times(self):
        """Host wall time (s) of the last geometry set-up: primitive pairs, Schwarz factors,
        quartet lists, list upload (hfgpu_setup_times)."""
        ms = (ctypes.c_double * 4)()
        self._check(lib().hfgpu_setup_times(self.h, ms))
        return dict(zip(("pairs", "schwarz", "lists", "upload"), [v / 1e3 for v in ms]))

    def class_time_ms(self, cls: int) -> float:
        ms = ctypes.c_float()
        self._check(lib().hfgpu_class_time(self.h, ctypes.c_int(cls), ctypes.byref(ms)))
        return ms.value

    # --- one-electron integrals on the device -----------------------------------------
    def one_electron_device(self, S_ptr, T_ptr, V_ptr):
        """hfgpu_one_electron_device into device buffers (n x n each)."""
        Z = _c(self.basis.Z)
        self._check(lib().hfgpu_one_electron_device(self.h, _p(Z), ctypes.c_void_p(S_ptr), ctypes.c_void_p(T_ptr),
                                                    ctypes.c_void_p(V_ptr)))

    def one_electron_grad_device(self, D_ptr, W_ptr, cH, cS, grad_ptr):
        """grad (device, natoms x 3) += cH sum D d(T+V)/dX + cS sum W dS/dX."""
        Z = _c(self.basis.Z)
        self._check(lib().hfgpu_one_electron_grad_device(self.h, _p(Z), ctypes.c_void_p(D_ptr), ctypes.c_void_p(W_ptr),
                                                         ctypes.c_double(cH), ctypes.c_double(cS),
                                                         ctypes.c_void_p(grad_ptr)))

    def one_electron(self):
        """S, T, V (host arrays) computed on the GPU."""
        import torch
        dev = torch.device("cuda", self._opts.device)
        n = self.n
        M = torch.empty((3, n, n), dtype=torch.float64, device=dev)
        torch.cuda.synchronize(dev)  # the handle's stream need not be torch's
        self.one_electron_device(M[0].data_ptr(), M[1].data_ptr(), M[2].data_ptr())
        torch.cuda.synchronize(dev)
        out = M.cpu().numpy()
        return out[0], out[1], out[2]

    def one_electron_grad(self, D, W, cH, cS) -> np.ndarray:
        """cH sum D d(T+V)/dX + cS sum W dS/dX (natoms x 3, host) computed on the GPU."""
        import torch
        dev = torch.device("cuda", self._opts.device)
        Dd = torch.from_numpy(_c(D)).to(dev)
        Wd = torch.from_numpy(_c(W)).to(dev)
        g = torch.zeros((self.basis.natoms, 3), dtype=torch.float64, device=dev)
        torch.cuda.synchronize(dev)
        self.one_electron_grad_device(Dd.data_ptr(), Wd.data_ptr(), cH, cS, g.data_ptr())
        torch.cuda.synchronize(dev)
        return g.cpu().numpy()

    # --- launch schedule ----------------------------------------------------------
    def autotune(self, D, precision=FP64, repeats=3) -> np.ndarray:
        """hfgpu_autotune: per class, the fastest launch form on this geometry and density.
        ``D`` is a CUDA tensor (n x n, float64) or a host array (copied to the device).
        Returns the schedule, HFGPU_NUM_CLASSES x 4 ints (block, primwarp, warp, capped)."""
        import torch
        if isinstance(D, torch.Tensor) and D.is_cuda:
            Dd = D.contiguous()
        else:
            Dd = torch.from_numpy(_c(D)).to(torch.device("cuda", self._opts.device))
        out = np.zeros((NUM_CLASSES, 4), dtype=np.int32)
        self._check(lib().hfgpu_autotune(self.h, ctypes.c_void_p(Dd.data_ptr()), ctypes.c_int(precision),
                                         ctypes.c_int(repeats), out.ctypes.data_as(_ip)))
        return out

    def autotune_grad(self, D, precision=FP64, repeats=2) -> np.ndarray:
        """hfgpu_autotune_grad on density D (host array or device tensor): the gradient form per
        class (0 thread, 1 warp, 2 warp split per accumulator set, 3 block of four warps, 4 block
        split per set, 5 and 6 the same with eight warps, -1 no choice)."""
        import torch
        Dd = D if isinstance(D, torch.Tensor) else torch.from_numpy(_c(D)).to(torch.device("cuda", self._opts.device))
        forms = np.zeros(NUM_CLASSES, dtype=np.int32)
        self._check(lib().hfgpu_autotune_grad(self.h, ctypes.c_void_p(Dd.data_ptr()), ctypes.c_int(precision),
                                              ctypes.c_int(repeats), forms.ctypes.data_as(_ip)))
        return forms

    def set_grad_forms(self, forms):
        """hfgpu_set_grad_forms: the gradient form per class (-1, 0 thread, 1 warp, 2 warp split,
        3 block, 4 block split, 5 block of eight warps, 6 its split)."""
        f = np.ascontiguousarray(np.broadcast_to(np.asarray(forms, dtype=np.int32), (NUM_CLASSES,)))
        self._check(lib().hfgpu_set_grad_forms(self.h, f.ctypes.data_as(_ip)))

    def get_schedule(self) -> np.ndarray:
        out = np.zeros((NUM_CLASSES, 4), dtype=np.int32)
        self._check(lib().hfgpu_get_schedule(self.h, out.ctypes.data_as(_ip)))
        return out

    def set_schedule(self, sched):
        s = np.ascontiguousarray(np.asarray(sched, dtype=np.int32).reshape(NUM_CLASSES, 4))
        self._check(lib().hfgpu_set_schedule(self.h, s.ctypes.data_as(_ip)))

    def device_status(self) -> int:
        """hfgpu_device_status: the kernels' status word since the last call (then cleared)."""
        st = ctypes.c_int()
        self._check(lib().hfgpu_device_status(self.h, ctypes.byref(st)))
        return st.value

    def purify_device(self, Fo_ptr, n, nocc, max_steps, P_ptr, err_ptr):
        """hfgpu_purify_device: P = projector onto the nocc lowest eigenvectors of Fo (device)."""
        self._check(lib().hfgpu_purify_device(self.h, ctypes.c_void_p(Fo_ptr), ctypes.c_int(n), ctypes.c_int(nocc),
                                              ctypes.c_int(max_steps), ctypes.c_void_p(P_ptr),
                                              ctypes.c_void_p(err_ptr)))

    def set_purify_mode(self, cooperative: int):
        """hfgpu_set_purify_mode: 1 one cooperative launch per purification, 0 two launches per step."""
        self._check(lib().hfgpu_set_purify_mode(self.h, ctypes.c_int(cooperative)))

    def request_abort(self, on=True):
        """hfgpu_request_abort: set (or reset) the host abort flag of the persistent launches."""
        self._check(lib().hfgpu_request_abort(self.h, ctypes.c_int(int(on))))

    def last_launches(self) -> int:
        k = ctypes.c_int()
        self._check(lib().hfgpu_last_launches(self.h, ctypes.byref(k)))
        return k.value

    def last_counts(self):
        a, b = ctypes.c_longlong(), ctypes.c_longlong()
        self._check(lib().hfgpu_last_counts(self.h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    # --- autograd-shaped pair ---------------------------------------------------
    def energy2e(self, D, precision=FP64) -> float:
        e = ctypes.c_double()
        self._check(lib().hfgpu_energy_forward(self.h, _p(_c(D)), ctypes.byref(e), ctypes.c_int(precision)))
        return e.value

    def grad2e(self, D, scale=1.0, precision=FP64) -> np.ndarray:
        g = np.zeros((self.basis.natoms, 3))
        self._check(lib().hfgpu_grad2e_backward(self.h, _p(_c(D)), ctypes.c_double(scale), _p(g),
                                                ctypes.c_int(precision)))
        return g

    def grad2e_uhf(self, Da, Db, scale=1.0, precision=FP64) -> np.ndarray:
        g = np.zeros((self.basis.natoms, 3))
        self._check(lib().hfgpu_grad2e_uhf_backward(self.h, _p(_c(Da)), _p(_c(Db)), ctypes.c_double(scale), _p(g),
                                                    ctypes.c_int(precision)))
        return g

    def hess2e(self, D, scale=1.0) -> np.ndarray:
        """Two-electron part of the RHF Hessian at fixed D, (3 natoms, 3 natoms): the reference's
        m_hessianC + m_hessianEx (Mol::scf_hessian::calc_scf_hessian_tei), by hfgpu_hess2e."""
        n3 = 3 * self.basis.natoms
        H = np.zeros((n3, n3))
        self._check(lib().hfgpu_hess2e(self.h, _p(_c(D)), ctypes.c_double(scale), _p(H)))
        return H

    def set_hess_form(self, form: int):
        """hfgpu_set_hess_form: -1 by class (default), 0 thread (global scratch), 1 block, 2 warp per
        quartet, 3 thread on straight-line register code where the class has it."""
        self._check(lib().hfgpu_set_hess_form(self.h, ctypes.c_int(form)))

    def autotune_hess(self, D, repeats=2):
        """hfgpu_autotune_hess on density D (host array, device tensor or device pointer): per
        class the fastest of the thread, block, warp and straight-line forms; returns the chosen
        forms (0 thread, 1 block, 2 warp, 3 straight-line)."""
        import torch
        if isinstance(D, int):
            ptr = D
        else:
            Dd = D if isinstance(D, torch.Tensor) else torch.from_numpy(_c(D)).to(torch.device("cuda", self._opts.device))
            ptr = Dd.data_ptr()
        forms = (ctypes.c_int * NUM_CLASSES)()
        self._check(lib().hfgpu_autotune_hess(self.h, ctypes.c_void_p(ptr), ctypes.c_int(repeats), forms))
        return list(forms)

    def set_hess_forms(self, forms):
        arr = (ctypes.c_int * NUM_CLASSES)(*forms)
        self._check(lib().hfgpu_set_hess_forms(self.h, arr))

    def hess2e_uhf(self, Da, Db, scale=1.0) -> np.ndarray:
        n3 = 3 * self.basis.natoms
        H = np.zeros((n3, n3))
        self._check(lib().hfgpu_hess2e_uhf(self.h, _p(_c(Da)), _p(_c(Db)), ctypes.c_double(scale), _p(H)))
        return H

    def hess2e_device(self, DJ_ptr, cJ, nK, DK_ptr, cK, hess_ptr):
        self._check(lib().hfgpu_hess2e_device(self.h, ctypes.c_void_p(DJ_ptr), ctypes.c_double(cJ), ctypes.c_int(nK),
                                              ctypes.c_void_p(DK_ptr), ctypes.c_double(cK), ctypes.c_void_p(hess_ptr)))


NUM_CLASSES = 21


def fp64_peak_tflops(device=0) -> float:
    t = ctypes.c_double()
    rc = lib().hfgpu_fp64_peak(ctypes.c_int(device), ctypes.byref(t))
    if rc:
        raise HfgpuError(rc)
    return t.value


# --- one-electron integrals (host CPU, no handle) ---------------------------------
def one_electron(basis: Basis):
    bv = _BasisView(basis)
    n = basis.nbf
    S, T, V = np.zeros((n, n)), np.zeros((n, n)), np.zeros((n, n))
    Z = _c(basis.Z)
    xyz = _c(basis.coords)
    rc = lib().hfgpu_one_electron(ctypes.byref(bv.s), _p(xyz), _p(Z), _p(S), _p(T), _p(V))
    if rc:
        raise HfgpuError(rc)
    return S, T, V


def one_electron_grad(basis: Basis, D, W, cH, cS) -> np.ndarray:
    bv = _BasisView(basis)
    g = np.zeros((basis.natoms, 3))
    rc = lib().hfgpu_one_electron_grad(ctypes.byref(bv.s), _p(_c(basis.coords)), _p(_c(basis.Z)), _p(_c(D)),
                                       _p(_c(W)), ctypes.c_double(cH), ctypes.c_double(cS), _p(g))
    if rc:
        raise HfgpuError(rc)
    return g


class Erios:
    """Interface of the reference's ERIOS::Erios over the GPU engine
    (src/integrals/hfscf_oseri.hpp:27-123): packed ERIs and the Schwarz diagonal."""

    def __init__(self, engine: Engine):
        self.engine = engine

    def compute_repulsion_packed(self):
        return self.engine.eri_packed()

    def compute_screen_matrix(self):
        return self.engine.schwarz()


class FockBuilder:
    """The Fock hooks of Mol::hf_solver / Mol::uhf_solver over the GPU engine."""

    def __init__(self, engine: Engine, precision=FP64):
        self.engine = engine
        self.precision = precision

    def update_fock_matrix(self, D, H):
        return self.engine.fock_rhf(D, H, self.precision)

    def update_fock_matrix_uhf(self, Da, Db, H):
        return self.engine.fock_uhf(Da, Db, H, self.precision)
