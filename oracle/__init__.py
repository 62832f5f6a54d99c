"""Python access to the test oracle (TEST INFRASTRUCTURE ONLY).

Two CPU libraries sit behind this module:
  * ``liboracle.so``: the C restatement of the reference's two-electron
    algorithms (hfscf_oracle.c);
  * ``_ref/libhfref.so``: the reference's own integral code compiled in place
    (Makefile target ``ref``).  It exists only where the reference sources were
    present at build time.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_REF = None

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def _p(a, ct=ctypes.c_double):
    return a.ctypes.data_as(ctypes.POINTER(ct))


def build(ref: bool = False) -> None:
    target = ["all"] if ref else ["liboracle.so"]
    subprocess.run(["make", "-s", "-C", HERE] + target, check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build(ref=False)
        L = ctypes.CDLL(path)
        L.or_boys.restype = ctypes.c_double
        L.or_boys.argtypes = [ctypes.c_int, ctypes.c_double]
        L.or_index_ijkl.restype = ctypes.c_longlong
        L.or_packed_len.restype = ctypes.c_longlong
        L.or_packed_len.argtypes = [ctypes.c_longlong]
        L.or_nbf.restype = ctypes.c_longlong
        _LIB = L
    return _LIB


def ref_available() -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", "libhfref.so"))


def ref():
    global _REF
    if _REF is None:
        L = ctypes.CDLL(os.path.join(HERE, "_ref", "libhfref.so"))
        L.hfref_boys.restype = ctypes.c_double
        L.hfref_boys.argtypes = [ctypes.c_double, ctypes.c_double]
        L.hfref_nbf.restype = ctypes.c_longlong
        _REF = L
    return _REF


def packed_len(n: int) -> int:
    return n * (n + 1) * (n * n + n + 2) // 8


def _flat(basis):
    f = basis.flat()
    return (ctypes.c_int(basis.nshell), _p(f["L"], ctypes.c_int), _p(np.ascontiguousarray(f["centers"])),
            _p(f["nprim"], ctypes.c_int), _p(f["exps"]), _p(f["coefs"]), ctypes.c_int(int(basis.pure))), f


# ---- C restatement -------------------------------------------------------
def boys(m: int, T: float) -> float:
    return lib().or_boys(int(m), float(T))


def ylm(L: int) -> np.ndarray:
    out = np.zeros(((L + 1) * (L + 2) // 2, 2 * L + 1))
    lib().or_ylm(ctypes.c_int(L), _p(out))
    return out


def shell_norm(L, exps, coefs) -> np.ndarray:
    exps = np.ascontiguousarray(exps, dtype=np.float64)
    coefs = np.ascontiguousarray(coefs, dtype=np.float64)
    out = np.zeros_like(coefs)
    lib().or_shell_norm(ctypes.c_int(L), ctypes.c_int(len(exps)), _p(exps), _p(coefs), _p(out))
    return out


def eri_packed(basis) -> np.ndarray:
    args, keep = _flat(basis)
    out = np.zeros(packed_len(basis.nbf))
    rc = lib().or_eri_packed(*args, _p(out))
    assert rc == 0
    return out


def shell_quartet(basis, i, j, k, l) -> np.ndarray:
    args, keep = _flat(basis)
    dims = [(2 * basis.shells[s].L + 1) if basis.pure else (basis.shells[s].L + 1) * (basis.shells[s].L + 2) // 2
            for s in (i, j, k, l)]
    out = np.zeros(int(np.prod(dims)))
    rc = lib().or_shell_quartet(*args, ctypes.c_int(i), ctypes.c_int(j), ctypes.c_int(k), ctypes.c_int(l), _p(out))
    assert rc == 0
    return out.reshape(dims)


def fock_rhf(eri, D, H) -> np.ndarray:
    n = D.shape[0]
    F = np.zeros((n, n))
    lib().or_fock_rhf(ctypes.c_longlong(n), _p(eri), _p(np.ascontiguousarray(D)), _p(np.ascontiguousarray(H)), _p(F))
    return F


def fock_uhf(eri, Da, Db, H):
    n = Da.shape[0]
    Fa, Fb = np.zeros((n, n)), np.zeros((n, n))
    lib().or_fock_uhf(ctypes.c_longlong(n), _p(eri), _p(np.ascontiguousarray(Da)), _p(np.ascontiguousarray(Db)),
                      _p(np.ascontiguousarray(H)), _p(Fa), _p(Fb))
    return Fa, Fb


def jk(eri, D):
    n = D.shape[0]
    J, K = np.zeros((n, n)), np.zeros((n, n))
    lib().or_jk(ctypes.c_longlong(n), _p(eri), _p(np.ascontiguousarray(D)), _p(J), _p(K))
    return J, K


def jk_packed(eri, Ds):
    """J[D_m], K[D_m] for a list of densities, from the packed ERI vector in one pass over the
    unique integrals (or_jk_packed): the sums of or_jk, fast enough for N = 250."""
    Ds = [np.ascontiguousarray(D, dtype=np.float64) for D in Ds]
    n = Ds[0].shape[0]
    Dst = np.ascontiguousarray(np.stack(Ds))
    J, K = np.zeros_like(Dst), np.zeros_like(Dst)
    rc = lib().or_jk_packed(ctypes.c_longlong(n), _p(eri), ctypes.c_int(len(Ds)), _p(Dst), _p(J), _p(K))
    assert rc == 0
    return J, K


def grad2e(basis, DJ, cJ, DKs, cK) -> np.ndarray:
    args, keep = _flat(basis)
    sa = keep["atom"]
    DK = np.ascontiguousarray(np.stack(DKs)) if len(DKs) else np.zeros((0,))
    g = np.zeros((basis.natoms, 3))
    rc = lib().or_grad2e(*args, _p(sa, ctypes.c_int), ctypes.c_int(basis.natoms), _p(np.ascontiguousarray(DJ)),
                         ctypes.c_double(cJ), ctypes.c_int(len(DKs)), _p(DK), ctypes.c_double(cK), _p(g))
    assert rc == 0
    return g


def grad2e_rhf(basis, D) -> np.ndarray:
    return grad2e(basis, D, 2.0, [D], 1.0)


def grad2e_uhf(basis, Da, Db) -> np.ndarray:
    return grad2e(basis, Da + Db, 0.5, [Da, Db], 0.5)


# ---- the reference's own code (oracle/_ref) ------------------------------
def ref_eri_packed(basis, cutoff=1e-14, do_screen=False) -> np.ndarray:
    args, keep = _flat(basis)
    out = np.zeros(packed_len(basis.nbf))
    rc = ref().hfref_eri_packed(*args, ctypes.c_double(cutoff), ctypes.c_int(int(do_screen)), _p(out))
    assert rc == 0
    return out


def ref_deriv1(basis, coords=(1, 1, 1), cutoff=1e-14) -> np.ndarray:
    args, keep = _flat(basis)
    c = np.array(coords, dtype=np.int32)
    out = np.zeros((9, packed_len(basis.nbf)))
    rc = ref().hfref_deriv1(*args, ctypes.c_double(cutoff), _p(c, ctypes.c_int), _p(out))
    assert rc == 0
    return out


def ref_hess2e(basis, D, cutoff=1e-14):
    """Two-electron part of the RHF Hessian at a fixed density D, (3 natoms, 3 natoms), as
    hessC + hessEx of Mol::scf_hessian::calc_scf_hessian_tei (src/hessian/hfscf_hessian_ints.cpp:20-303),
    from the reference's second-derivative shell routines (hfscf_oserideriv2qq.cpp, _pq.cpp).
    Returns (hessC, hessEx)."""
    args, f = _flat(basis)
    na3 = 3 * basis.natoms
    hc, he = np.zeros((na3, na3)), np.zeros((na3, na3))
    rc = ref().hfref_hess2e(*args, ctypes.c_double(cutoff), _p(f["atom"], ctypes.c_int), ctypes.c_int(basis.natoms),
                            _p(np.ascontiguousarray(D, dtype=np.float64)), _p(hc), _p(he))
    assert rc == 0
    return hc, he


def ref_time_hess_sample(basis, stride=20, cutoff=1e-14):
    """Seconds of the reference's Hessian two-electron part (hfref_time_hess_sample): per direction
    pair the sampled second-derivative shell routines (qq, pq) scaled to their whole loops, and
    the assembly + contraction of one atom pair of each kind; total = 3 (qq + pq) +
    3 natoms (natoms + 1) / 2 pair_qq + 3 natoms^2 pair_pq."""
    args, f = _flat(basis)
    t = [ctypes.c_double() for _ in range(4)]
    rc = ref().hfref_time_hess_sample(*args, ctypes.c_double(cutoff), _p(f["atom"], ctypes.c_int),
                                      ctypes.c_int(basis.natoms), ctypes.c_int(stride), *[ctypes.byref(x) for x in t])
    assert rc == 0
    qq, pq, pqq, ppq = (x.value for x in t)
    na = basis.natoms
    return {"t_qq_ints_s": qq, "t_pq_ints_s": pq, "t_pair_qq_s": pqq, "t_pair_pq_s": ppq,
            "t_hess2e_s": 3 * (qq + pq) + 3 * na * (na + 1) / 2 * pqq + 3 * na * na * ppq}


def ref_onee(basis):
    """S, T, V from the reference's one-electron shell routines (hfscf_osoverlap.cpp,
    hfscf_osnuclear.cpp) over the driver loop of hfscf_hf_hamiltonian.cpp:14-37."""
    args, f = _flat(basis)
    n = basis.nbf
    Z = np.ascontiguousarray(np.asarray(basis.Z), dtype=np.int32)
    xyz = np.ascontiguousarray(basis.coords, dtype=np.float64)
    S, T, V = np.zeros((n, n)), np.zeros((n, n)), np.zeros((n, n))
    rc = ref().hfref_onee(*args, ctypes.c_int(basis.natoms), _p(Z, ctypes.c_int), _p(xyz), _p(S), _p(T), _p(V))
    assert rc == 0
    return S, T, V


def ref_onee_grad(basis, D, Q, cD=2.0, cQ=-2.0) -> np.ndarray:
    """cD sum D.(dT + dV) + cQ sum Q.dS per atom and direction, from the reference's
    first-derivative shell routines and its per-atom assembly (hfscf_grad_ints.cpp:14-77,153-199)."""
    args, f = _flat(basis)
    Z = np.ascontiguousarray(np.asarray(basis.Z), dtype=np.int32)
    xyz = np.ascontiguousarray(basis.coords, dtype=np.float64)
    Dc = np.ascontiguousarray(D, dtype=np.float64)
    Qc = np.ascontiguousarray(Q, dtype=np.float64)
    g = np.zeros((basis.natoms, 3))
    rc = ref().hfref_onee_grad(*args, ctypes.c_int(basis.natoms), _p(Z, ctypes.c_int), _p(xyz),
                               _p(f["atom"], ctypes.c_int), _p(Dc), _p(Qc), ctypes.c_double(cD),
                               ctypes.c_double(cQ), _p(g))
    assert rc == 0
    return g


def ref_screen_diagonal(basis, cutoff=1e-14) -> np.ndarray:
    """(pq|pq) over Cartesian functions as the reference's Schwarz screen matrix holds it
    (Erios::compute_screen_matrix, src/integrals/hfscf_oseri_screen.cpp:22-181); entries of
    shell pairs that the reference's block test skips are -1.  Cartesian bases only."""
    assert not basis.pure
    args, keep = _flat(basis)
    n = basis.nbf
    out = np.zeros((n, n))
    rc = ref().hfref_screen_diagonal(*args[:6], ctypes.c_double(cutoff), _p(out))
    assert rc == 0
    return out


def ref_boys(m, T) -> float:
    return ref().hfref_boys(float(m), float(T))


def ref_ylm(L) -> np.ndarray:
    out = np.zeros(((L + 1) * (L + 2) // 2, 2 * L + 1))
    ref().hfref_ylm(ctypes.c_int(L), _p(out))
    return out


def ref_shell_coefs(L, exps, coefs) -> np.ndarray:
    exps = np.ascontiguousarray(exps, dtype=np.float64)
    coefs = np.ascontiguousarray(coefs, dtype=np.float64)
    out = np.zeros_like(coefs)
    ref().hfref_shell_coefs(ctypes.c_int(L), ctypes.c_int(len(exps)), _p(exps), _p(coefs), _p(out))
    return out


# ---- restatement of the reference gradient contraction on packed tensors ----
def index_ijkl(i, j, k, l):
    i, j, k, l = (np.asarray(x, dtype=np.int64) for x in (i, j, k, l))
    ij = np.where(i > j, i * (i + 1) // 2 + j, j * (j + 1) // 2 + i)
    kl = np.where(k > l, k * (k + 1) // 2 + l, l * (l + 1) // 2 + k)
    return np.where(ij > kl, ij * (ij + 1) // 2 + kl, kl * (kl + 1) // 2 + ij)


def unpack(packed, n) -> np.ndarray:
    """Full n^4 tensor from a packed 8-fold vector."""
    r = np.arange(n)
    i, j, k, l = np.meshgrid(r, r, r, r, indexing="ij")
    return packed[index_ijkl(i, j, k, l)]


def grad2e_packed_deriv1(deriv9, bf_atom, natoms, DJ, cJ, DKs, cK) -> np.ndarray:
    """Two-electron gradient from the reference's nine packed derivative tensors in one pass
    over the unique slots (or_grad2e_from_deriv1, C); RHF: DJ = D, cJ = 2, DKs = [D], cK = 1."""
    n = DJ.shape[0]
    d9 = np.ascontiguousarray(deriv9, dtype=np.float64)
    at = np.ascontiguousarray(bf_atom, dtype=np.int32)
    DK = np.ascontiguousarray(np.stack(DKs)) if len(DKs) else np.zeros((0,))
    g = np.zeros((natoms, 3))
    rc = lib().or_grad2e_from_deriv1(ctypes.c_longlong(n), _p(d9), _p(at, ctypes.c_int), ctypes.c_int(natoms),
                                     _p(np.ascontiguousarray(DJ)), ctypes.c_double(cJ), ctypes.c_int(len(DKs)),
                                     _p(DK), ctypes.c_double(cK), _p(g))
    assert rc == 0
    return g


def grad2e_from_deriv1(deriv9, bf_atom, natoms, D) -> np.ndarray:
    """RHF two-electron gradient from the reference's nine packed derivative tensors,
    restating src/gradient/hfscf_grad_ints.cpp:79-108 (dV/dX assembly over the
    canonical slot order i>=j, k>=l, ij<=kl) and hfscf_grad_rhf.cpp:121-141."""
    n = D.shape[0]
    r = np.arange(n)
    i, j, k, l = np.meshgrid(r, r, r, r, indexing="ij")
    canon = (i >= j) & (k >= l) & ((i * (i + 1) // 2 + j) <= (k * (k + 1) // 2 + l))
    ci, cj, ck, cl = i[canon], j[canon], k[canon], l[canon]
    slots = index_ijkl(ci, cj, ck, cl)
    g = np.zeros((natoms, 3))
    for d in range(3):
        A, B, C = (deriv9[3 * d + q] for q in range(3))
        for atom in range(natoms):
            m = (bf_atom == atom)
            dV = np.zeros(len(A))
            dV[slots] += np.where(m[ci], A[slots], 0.0) + np.where(m[cj], B[slots], 0.0) + \
                np.where(m[ck], C[slots], 0.0) - np.where(m[cl], A[slots] + B[slots] + C[slots], 0.0)
            full = unpack(dV, n)
            G = 2.0 * np.einsum("kl,ijkl->ij", D, full) - np.einsum("kl,ikjl->ij", D, full)
            g[atom, d] = np.sum(D * G)
    return g
