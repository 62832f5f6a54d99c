"""Generate the golden fixtures from the reference's own integral code.

The reference (hfscf) is compiled in place by oracle/Makefile into
oracle/_ref/libhfref.so; this script calls it through oracle/__init__.py and
stores small fixtures next to itself:

  h2o_ccpvdz_eri.npz    every unique ERI of H2O/cc-pVDZ (pure d, 24 functions,
                        O (0,0,0), H (0, +-1.4305, 1.1073) bohr), packed 8-fold,
                        from Erios::compute_contracted_shell_quartet.
  h2o_631gs_grad2e.npz  two-electron gradient of a water (6-31G*, Cartesian d)
                        at a fixed seeded density, contracted from the
                        reference's nine derivative-ERI tensors
                        (Erios::compute_contracted_shell_quartet_deriv1).
  ch4_ccpvdz_eri.npz    methane/cc-pVDZ packed ERIs (34 functions, pure d).

Usage: python tests/golden/make_golden.py   (needs the reference sources)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402
from hfscf_b200 import basis as B, molecules as M  # noqa: E402


def main():
    oracle.build(ref=True)
    Z, x, name, pure = M.workload(1)
    bs = B.build_basis(name, Z, x, pure=pure)
    np.savez_compressed(os.path.join(HERE, "h2o_ccpvdz_eri.npz"), Z=np.array(Z), coords=x, basis=name, pure=pure,
                        eri=oracle.ref_eri_packed(bs))
    Z, xa = M.methane()
    x = np.asarray(xa) * B.ANGSTROM_TO_BOHR + np.array([0.011, -0.007, 0.003])
    bs = B.build_basis("cc-pvdz", Z, x, pure=True)
    np.savez_compressed(os.path.join(HERE, "ch4_ccpvdz_eri.npz"), Z=np.array(Z), coords=x, basis="cc-pvdz",
                        pure=True, eri=oracle.ref_eri_packed(bs))
    rng = np.random.default_rng(20261203)
    Z, xa = M.water(rng)
    x = np.asarray(xa) * B.ANGSTROM_TO_BOHR
    bs = B.build_basis("6-31g*", Z, x, pure=False)
    n = bs.nbf
    A = rng.normal(size=(n, n))
    D = (A + A.T) / n
    d9 = oracle.ref_deriv1(bs)
    g = oracle.grad2e_from_deriv1(d9, bs.bf_atom(), bs.natoms, D)
    np.savez_compressed(os.path.join(HERE, "h2o_631gs_grad2e.npz"), Z=np.array(Z), coords=x, basis="6-31g*",
                        pure=False, D=D, grad=g)
    print("ok")


if __name__ == "__main__":
    main()
