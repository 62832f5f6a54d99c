"""Frozen algorithmic FLOP model of the two-electron kernels.

Work is counted from the generated class code (csrc/generated/ops.json, written
by gen_eri.py with the operation counts of the straight-line VRR/HRR it emits),
so it is the algorithm's arithmetic, not a hardware counter:

  F(class launch) = sum over computed primitive quartets [C_prim + C_boys(L)]
                  + sum over computed contracted quartets [C_hrr + C_sph + C_dig * n_out]

  C_prim   VRR operations + primitive scalars (p+q, rho, W-P, W-Q, T, prefactor:
           29 flops) + one add per contracted target (from ops.json "prim_flops");
  C_boys   Boys function: 6-term Taylor (13 flops), downward recursion (3 per
           order) and the prefactor scaling (1 per order): 14 + 4 L;
  C_hrr    horizontal recurrence on the contracted set (2 flops per step);
  C_sph    Cartesian -> pure transform when the basis is pure (0 for Cartesian);
  C_dig    J/K digestion: 12 flops per final-basis integral (J_ab, J_cd and the
           four K blocks, one FMA each).
The gradient uses the same form with the gradient class counts and
C_dig_grad = 2 flops per Cartesian weight per derivative component (9).
"""
from __future__ import annotations

import json
import os

HERE = os.path.dirname(os.path.abspath(__file__))
OPS = os.path.join(HERE, "csrc", "generated", "ops.json")

C_DIG = 12


def c_boys(L: int) -> int:
    return 14 + 4 * L


def _ops():
    with open(OPS) as f:
        return json.load(f)


def class_block_size(cls_index: int, pure: bool) -> int:
    """Integrals in one contracted block of the class in the final basis."""
    la, lb, lc, ld = _ops()["eri"][cls_index]["class"]
    if pure:
        return (2 * la + 1) * (2 * lb + 1) * (2 * lc + 1) * (2 * ld + 1)
    return ((la + 1) * (la + 2) // 2) * ((lb + 1) * (lb + 2) // 2) * ((lc + 1) * (lc + 2) // 2) * \
        ((ld + 1) * (ld + 2) // 2)


def class_integrals(cls_index: int, computed_quartets: int, pure: bool) -> int:
    """Contracted integrals a launch computes (model-independent count: blocks x block size)."""
    return int(computed_quartets) * class_block_size(cls_index, pure)


def class_flops(cls_index: int, computed_quartets: int, prim_quartets: int, pure: bool) -> float:
    m = _ops()["eri"][cls_index]
    nout = class_block_size(cls_index, pure)
    per_prim = m["prim_flops"] + c_boys(m["boys_m"])
    per_q = m["hrr_flops"] + (m["pure_flops"] if pure else 0) + C_DIG * nout
    return float(prim_quartets) * per_prim + float(computed_quartets) * per_q


def class_name(cls_index: int) -> str:
    la, lb, lc, ld = _ops()["eri"][cls_index]["class"]
    s = "spdf"
    return f"({s[la]}{s[lb]}|{s[lc]}{s[ld]})"
