"""SAD guess (Mol::hf_solver::get_sad_guess, src/scfsolver/hfscf_hf_solver.cpp:478-553)
on the GPU engine against the oracle's restatement of the atomic UHF on the reference's own
integrals, and SCF from
it against SCF from the core guess.  The guess comparison converges both atomic UHF runs
tightly (rms 1e-10): at the reference's loose SAD tolerance (rms 1e-6) the stopping point
depends on last-digit differences between two J/K builds, which the DIIS solves amplify.
Tolerances: guess density 1e-8; SCF energy 1e-8 Eh."""
import numpy as np
import pytest

import oracle.scf as OS
from hfscf_b200 import basis as B
from hfscf_b200 import engine as E
from hfscf_b200 import molecules as M
from hfscf_b200 import scf

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,pure", [("6-31g*", False), ("cc-pvdz", True)])
def test_sad_guess_matches_oracle_restatement(name, pure):
    Z, x = M.water_cluster(2, 2.9, np.random.default_rng(8), 0.1)
    Z = np.concatenate([Z, [6]])
    x = np.vstack([np.asarray(x), [[4.0, 4.0, 4.0]]])
    bs = B.build_basis(name, Z, x * B.ANGSTROM_TO_BOHR, pure=pure)
    D = scf.sad_guess(bs, rms_tol=1e-10, e_tol=1e-12, max_iter=200)
    D0 = OS.sad_guess(bs, rms_tol=1e-10, e_tol=1e-12, max_iter=200)
    assert np.abs(D - D0).max() < 1e-8


def test_scf_from_sad_reaches_the_core_guess_energy_in_fewer_iterations():
    Z, x = M.water_cluster(3, 2.9, np.random.default_rng(9), 0.1)
    bs = B.build_basis("6-31g*", Z, np.asarray(x) * B.ANGSTROM_TO_BOHR, pure=False)
    with E.Engine(bs) as eng:
        r_core = scf.rhf(bs, engine=eng)
        r_sad = scf.rhf(bs, engine=eng, guess="sad")
    assert r_core.converged and r_sad.converged
    assert abs(r_sad.energy - r_core.energy) < 1e-8
    assert r_sad.iterations < r_core.iterations
