"""Generate config_oracle.json: oracle SCF energies (and gradients where affordable) of the
four single-molecule benchmark configurations, from the reference's own integral code.

For each configuration (the seeded geometries of hfscf_b200.molecules.workload):
  * S, T, V and the unscreened packed ERIs from the reference compiled in place (oracle/_ref);
  * RHF to rms 1e-10 / dE 1e-11 with oracle/scf.py (core guess, the reference's DIIS);
  * the full RHF gradient (two-electron term from the reference's nine derivative tensors,
    contracted by or_grad2e_from_deriv1; the reference's one-electron gradient routines; the
    nuclear repulsion gradient) for H2O/cc-pVDZ, (H2O)8/6-31G* and n-octane/6-31G** (the
    anthracene derivative tensors would take 9 x 3.4 GiB and are left out).
bench.py reports the engine's energies and gradients against these values.

Usage: python tests/golden/make_config_refs.py   (needs the reference sources; ~10 min on
8 cores and ~20 GB of host memory for the octane derivative tensors)
"""
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402
from oracle import scf as OS  # noqa: E402
from hfscf_b200 import basis as B, molecules as M  # noqa: E402

GRADIENT_CONFIGS = (1, 2, 4)


def main():
    oracle.build(ref=True)
    out = {"method": "oracle RHF on the reference's unscreened integrals (oracle/_ref), rms 1e-10, dE 1e-11",
           "configs": {}}
    for idx in (1, 2, 3, 4):
        t0 = time.time()
        Z, x, name, pure = M.workload(idx)
        bs = B.build_basis(name, Z, x, pure=pure)
        S, T, V = oracle.ref_onee(bs)
        eri = oracle.ref_eri_packed(bs, do_screen=False)

        def jk(D):
            J, K = oracle.jk_packed(eri, [D])
            return J[0], K[0]

        r = OS.rhf(S, T + V, int(sum(Z)) // 2, jk, OS.nuclear_repulsion(Z, bs.coords), e_tol=1e-11, rms_tol=1e-10)
        assert r["converged"]
        del eri
        entry = {"basis": name, "pure": bool(pure), "nbf": bs.nbf, "natoms": bs.natoms, "energy": r["energy"],
                 "iterations": r["iterations"]}
        if idx in GRADIENT_CONFIGS:
            D, F = r["D"], r["F"]
            d9 = oracle.ref_deriv1(bs)
            g = oracle.grad2e_packed_deriv1(d9, bs.bf_atom(), bs.natoms, D, 2.0, [D], 1.0)
            del d9
            g += oracle.ref_onee_grad(bs, D, D @ F @ D, 2.0, -2.0)
            g += OS.nuclear_repulsion_gradient(Z, bs.coords)
            entry["gradient"] = g.tolist()
        out["configs"][str(idx)] = entry
        print(idx, name, bs.nbf, r["energy"], f"{time.time() - t0:.1f}s", flush=True)
    with open(os.path.join(HERE, "config_oracle.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
