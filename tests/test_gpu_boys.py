"""Direct tests of the GPU Boys function and the GPU Schwarz factors.

Boys function (hfgpu_boys, the evaluation every quartet kernel runs) against 40-digit
mpmath values (tests/golden/boys_mpmath.npz, made by tests/golden/make_boys.py) for
m = 0..10 over T in [0, 1e3]:
  * FP64: the Taylor step about the nearest grid point T_k = k/10 drops the term
    F_{M+7}(T_k) d^7 / 7! with |d| <= 0.05, at most 1.6e-13 F_M; the tolerance is
    2e-13 relative (measured error below it on every point);
  * FP32 (the mixed-precision kernels): four Taylor terms (remainder <= 2.6e-7 F_M), FP32
    table values, Horner steps, expf and the recursions; the tolerance is 3e-6 relative,
    against values taken at T rounded to float32;
  * below T = 1e-8 the reference evaluates F_m(1e-8) (src/math/gamma.cpp:20-21) and the
    GPU the exact F_m(T); the two differ by at most 1e-8 / (2m + 3).
Schwarz factors (hfgpu_schwarz) against the reference's own screen matrix
(Erios::compute_screen_matrix, src/integrals/hfscf_oseri_screen.cpp:22-181), as (ab|ab) to
1e-10 relative + 1e-13 absolute.
"""
import os

import numpy as np
import pytest

import oracle
from hfscf_b200 import basis as B
from hfscf_b200 import engine as E
from hfscf_b200 import molecules as M

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FP64_REL = 2e-13
FP32_REL = 3e-6


def _engine():
    Z, x = M.water(np.random.default_rng(1))
    return E.Engine(B.build_basis("sto-3g", Z, np.asarray(x) * B.ANGSTROM_TO_BOHR))


@pytest.mark.parametrize("m", range(11))
def test_gpu_boys_fp64_against_high_precision(m):
    g = np.load(os.path.join(GOLD, "boys_mpmath.npz"))
    T, F = g["T"], g["F"]
    with _engine() as eng:
        Fg = eng.boys(m, T, E.FP64)
    rel = np.abs(Fg - F[:, : m + 1]) / F[:, : m + 1]
    assert rel.max() < FP64_REL, (rel.max(), T[np.argmax(rel.max(axis=1))])


@pytest.mark.parametrize("m", range(11))
def test_gpu_boys_fp32_within_stated_bound(m):
    g = np.load(os.path.join(GOLD, "boys_mpmath.npz"))
    T, F = g["T32"], g["F32"]
    with _engine() as eng:
        Fg = eng.boys(m, T, E.MIXED)
    rel = np.abs(Fg - F[:, : m + 1]) / F[:, : m + 1]
    assert rel.max() < FP32_REL, (rel.max(), T[np.argmax(rel.max(axis=1))])


@pytest.mark.skipif(not oracle.ref_available(), reason="reference library not built")
def test_gpu_boys_below_the_reference_clamp():
    """Where the reference clamps (T < 1e-8) the GPU value differs from the reference's by at
    most 1e-8 / (2m + 3); above the clamp the two agree to the FP64 tolerance."""
    T = np.array([0.0, 1e-14, 1e-11, 3e-9, 9.99e-9, 1e-8, 2e-8, 1e-6, 0.3, 7.7, 36.0, 250.0])
    with _engine() as eng:
        Fg = eng.boys(10, T, E.FP64)
    for i, t in enumerate(T):
        for m in range(11):
            r = oracle.ref_boys(m, t)
            if t < 1e-8:
                # F_m(0) - F_m(1e-8) = 1e-8 / (2m + 3) + O(1e-16); 1e-13 covers the reference's rounding
                assert abs(Fg[i, m] - r) <= 1e-8 / (2 * m + 3) + 1e-13
            else:
                assert abs(Fg[i, m] - r) <= 1e-13 * r


def test_gpu_boys_rejects_bad_arguments():
    with _engine() as eng:
        with pytest.raises(E.HfgpuError):
            eng.boys(11, [1.0])
        with pytest.raises(E.HfgpuError):
            eng.boys(2, [-1.0])
        with pytest.raises(E.HfgpuError):
            eng.boys(2, [np.nan])


@pytest.mark.skipif(not oracle.ref_available(), reason="reference library not built")
def test_schwarz_factors_match_reference_screen_matrix():
    """(H2O)8 / 6-31G* (Cartesian d, 80 shells): the GPU's sqrt(max |(ab|ab)|) per shell pair
    against the square root of the largest (pq|pq) of the pair's block of the reference's
    screen matrix.  Pairs whose whole block the reference's block test skips must have a
    negligible factor on the GPU too."""
    Z, x, name, pure = M.workload(4)
    bs = B.build_basis(name, Z, x, pure=pure)
    Qref_f = oracle.ref_screen_diagonal(bs)
    with E.Engine(bs) as eng:
        Q = eng.schwarz()
    first = np.concatenate([[0], np.cumsum([(s.L + 1) * (s.L + 2) // 2 for s in bs.shells])])
    ns = bs.nshell
    checked = 0
    for a in range(ns):
        for b in range(ns):
            blk = Qref_f[first[a]:first[a + 1], first[b]:first[b + 1]]
            if np.all(blk < 0):
                assert Q[a, b] < 1e-5
                continue
            # compared as (ab|ab): the reference drops intermediates below 1e-12 while it builds
            # the screen matrix (hfscf_oseri_screen.cpp:140,155), which moves the smallest diagonal
            # integrals at the 1e-15 level
            q2 = np.max(np.abs(blk))
            assert abs(Q[a, b] ** 2 - q2) <= 1e-10 * q2 + 1e-13, (a, b, Q[a, b] ** 2, q2)
            checked += 1
    assert checked > ns * ns // 2
