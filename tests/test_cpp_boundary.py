"""The C++ boundary (include/hfgpu.hpp) compiled with g++ as a maintainer's C++ translation
unit would be, linked against libhfgpu.so, and run.

CPU: the program compiles and links against the header and the library (no GPU needed).
GPU: the program fills the packed ERI vector quartet by quartet through GpuErios (the
reference's create_repulsion_matrix loop, screening on), one Fock build through GpuJK and the
two-electron gradient through GpuGradient and the two-electron Hessian through GpuHessian; each
is checked against the oracle (ERIs 1e-11, F 1e-10, gradient 1e-10, Hessian 1e-9 against the
reference's own second-derivative code; screened slots below the reference's screen_tol 1e-12
may be zero).
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

import oracle
from hfscf_b200 import basis as B
from hfscf_b200 import engine as E
from hfscf_b200 import molecules as M

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "boundary_check.cpp")
LIBDIR = os.path.join(ROOT, "hfscf_b200")


def _compile(out_dir):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    if not os.path.exists(E.LIB_PATH):
        pytest.skip("libhfgpu.so not built")
    exe = os.path.join(out_dir, "boundary_check")
    cmd = [gxx, "-std=c++17", "-O2", "-Wall", "-Wextra", "-I", os.path.join(ROOT, "include"), SRC, "-o", exe,
           "-L", LIBDIR, "-lhfgpu", f"-Wl,-rpath,{LIBDIR}", "-L/usr/local/cuda/lib64",
           "-Wl,-rpath-link,/usr/local/cuda/lib64"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]
    return exe


def test_cpp_boundary_compiles_and_links(tmp_path):
    exe = _compile(str(tmp_path))
    assert os.access(exe, os.X_OK)


@pytest.mark.gpu
@pytest.mark.parametrize("pure", [False, True], ids=["cartesian", "pure"])
def test_cpp_boundary_matches_oracle(tmp_path, pure):
    exe = _compile(str(tmp_path))
    rng = np.random.default_rng(51)
    Z, x = M.water(rng)
    bs = B.build_basis("cc-pvdz" if pure else "6-31g*", Z, np.asarray(x) * B.ANGSTROM_TO_BOHR, pure=pure)
    n = bs.nbf
    A = rng.normal(size=(n, n))
    D = (A + A.T) / n
    A = rng.normal(size=(n, n))
    H = (A + A.T) / n
    f = bs.flat()
    vals = [bs.nshell, bs.natoms, int(pure)] + list(f["L"]) + list(f["atom"]) + list(f["nprim"])
    nums = list(f["exps"]) + list(f["coefs"]) + list(np.asarray(bs.coords).ravel()) + list(D.ravel()) + list(H.ravel())
    inp = tmp_path / "in.txt"
    inp.write_text(" ".join(str(int(v)) for v in vals) + "\n" + " ".join(repr(float(v)) for v in nums) + "\n")
    out = tmp_path / "out.bin"
    r = subprocess.run([exe, str(inp), str(out)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    data = np.fromfile(out, dtype=np.float64)
    nl = oracle.packed_len(n)
    na = bs.natoms
    eri, F = data[:nl], data[nl:nl + n * n].reshape(n, n)
    g = data[nl + n * n:nl + n * n + 3 * na].reshape(na, 3)
    hess = data[nl + n * n + 3 * na:].reshape(3 * na, 3 * na)
    eri0 = oracle.eri_packed(bs)
    err = np.abs(eri - eri0)
    screened = (eri == 0.0) & (np.abs(eri0) < 1e-12)
    assert np.max(np.where(screened, 0.0, err)) < 1e-11
    assert np.max(np.abs(F - oracle.fock_rhf(eri0, D, H))) < 1e-10
    assert np.max(np.abs(g - oracle.grad2e_rhf(bs, D))) < 1e-10
    if oracle.ref_available():
        hc, he = oracle.ref_hess2e(bs, D)
        assert np.max(np.abs(hess - (hc + he))) < 1e-9
