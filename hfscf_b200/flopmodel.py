"""Frozen algorithmic FLOP model of the two-electron work (the roofline's numerator).

The count is fixed by the Head-Gordon-Pople scheme (J. Chem. Phys. 89, 5777 (1988)) and
is enumerated here, from the class's angular momenta alone; it does not read the engine's
generated code, so a more wasteful kernel cannot raise the "achieved" rate.  One flop is
one multiply or one add (an FMA is two).

  F_build = sum over surviving primitive quartets [C_prim + C_boys(L) + C_vrr + n_targets]
          + sum over surviving contracted quartets [C_hrr + C_sph + C_dig * n_out]

  C_prim   primitive-quartet scalars: p+q, 1/sqrt(p+q), rho, P-Q, T, W-P, W-Q and the
           [00|00] prefactor: 25;
  C_boys   one Boys evaluation F_0..F_L: 30 + 4 L (a Taylor step and e^-T, then the
           downward recursion and the prefactor scaling per order);
  C_vrr    Obara-Saika vertical recurrence building every [e0|f0]^(m) needed for the
           targets la <= |e| <= la+lb, lc <= |f| <= lc+ld, each intermediate built along
           its largest Cartesian component (ties: x, then y, then z):
             electron 1: PA_i x + WP_i y (3), + e_i/2p (x' - rho/p y') (4) when e_i > 1;
             electron 2: QC_i x + WQ_i y (3), + f_i/2q (x' - rho/q y') (4) when f_i > 1,
                         + e_i/2(p+q) z (2) when e_i > 0;
  n_targets  one add per contracted target (the primitive sum);
  C_hrr    horizontal recurrence on the contracted set, ket then bra,
           (a b+1_i| = (a+1_i b| + AB_i (a b|: 2 per intermediate;
  C_sph    Cartesian -> pure transform, one index at a time: 2 per non-zero solid-harmonic
           coefficient applied (0 in a Cartesian basis);
  C_dig    J/K digestion: 12 per integral of the final basis (J_ab, J_cd and the four K
           blocks, one FMA each).

Gradient (adjoint or not, the same frozen count): the derivative classes with L + 1 on three
centres, d/dA_i (ab|cd) = 2 alpha (a+1_i b|cd) - a_i (a-1_i b|cd) and likewise for B and C
(D by translational invariance), per primitive quartet the Boys function to order L + 1, the
VRR of every [e0|f0] the raised and lowered classes need, one add per unweighted target and two
(a product and an add) per exponent-weighted target (2 alpha, 2 beta, 2 gamma sets); per
contracted quartet the HRR of the six raised and lowered classes, two flops per derivative
integral that has a lowered term, the pure transform of the nine derivative blocks and
C_DIG_GRAD = 4 per derivative integral per centre component (grad_class_flops).

Classes are numbered as the engine numbers them (hfgpu_class_stats): pair classes
ss ps pp ds dp dd = 0..5 (la >= lb), quartet class cp (cp + 1) / 2 + cq for cp >= cq.
The count of the engine's own generated code (csrc/generated/ops.json) is kept as a second
number (generated_class_flops).
"""
from __future__ import annotations

import json
import math
import os
from functools import lru_cache

HERE = os.path.dirname(os.path.abspath(__file__))
OPS = os.path.join(HERE, "csrc", "generated", "ops.json")

C_PRIM = 25
C_DIG = 12
C_DIG_GRAD = 4
PAIRS = [(0, 0), (1, 0), (1, 1), (2, 0), (2, 1), (2, 2)]


def c_boys(L: int) -> int:
    return 30 + 4 * L


def ncart(L: int) -> int:
    return (L + 1) * (L + 2) // 2


def npure(L: int) -> int:
    return 2 * L + 1


def cart(L: int):
    return [(L - i, i - j, j) for i in range(L + 1) for j in range(i + 1)]


def class_am(cls_index: int):
    """(la, lb, lc, ld) of quartet class cls_index."""
    cp = int((math.isqrt(8 * cls_index + 1) - 1) // 2)
    cq = cls_index - cp * (cp + 1) // 2
    return PAIRS[cp] + PAIRS[cq]


def class_name(cls_index: int) -> str:
    la, lb, lc, ld = class_am(cls_index)
    s = "spdf"
    return f"({s[la]}{s[lb]}|{s[lc]}{s[ld]})"


def _dir(v):
    return max(range(3), key=lambda d: (v[d], -d))


def _dec(v, i):
    w = list(v)
    w[i] -= 1
    return tuple(w)


def _target_set(e_lo, e_hi, f_lo, f_hi):
    return {(e, f) for le in range(max(e_lo, 0), e_hi + 1) for e in cart(le)
            for lf in range(max(f_lo, 0), f_hi + 1) for f in cart(lf)}


@lru_cache(maxsize=None)
def _vrr_count(la, lb, lc, ld):
    """(flops, targets) of the vertical recurrence of one primitive quartet."""
    return _vrr_enumerate(frozenset(_target_set(la, la + lb, lc, lc + ld)))


def _vrr_enumerate(targets):
    """(flops, number of targets) of building every [e0|f0]^(0) in targets by the VRR."""
    built = set()
    flops = 0
    stack = []
    for e, f in targets:
        stack.append((e, f, 0))
    while stack:
        e, f, m = stack.pop()
        if (e, f, m) in built or (sum(e) == 0 and sum(f) == 0):
            continue
        built.add((e, f, m))
        if sum(f) > 0:
            i = _dir(f)
            f1 = _dec(f, i)
            deps = [(e, f1, m), (e, f1, m + 1)]
            flops += 3
            if f1[i] > 0:
                f2 = _dec(f1, i)
                deps += [(e, f2, m), (e, f2, m + 1)]
                flops += 4
            if e[i] > 0:
                deps.append((_dec(e, i), f1, m + 1))
                flops += 2
        else:
            i = _dir(e)
            e1 = _dec(e, i)
            deps = [(e1, f, m), (e1, f, m + 1)]
            flops += 3
            if e1[i] > 0:
                deps += [(_dec(e1, i), f, m), (_dec(e1, i), f, m + 1)]
                flops += 4
        stack.extend(deps)
    return flops, len(targets)


@lru_cache(maxsize=None)
def _hrr_count(la, lb, lc, ld):
    """Flops of the horizontal recurrence of one contracted quartet (ket first, then bra)."""
    ket, bra = set(), set()

    def k(e, c, d):
        if sum(d) == 0 or (e, c, d) in ket:
            return
        ket.add((e, c, d))
        i = _dir(d)
        d1 = _dec(d, i)
        c1 = list(c)
        c1[i] += 1
        k(e, tuple(c1), d1)
        k(e, c, d1)

    def b(a, bb, c, d):
        if sum(bb) == 0:
            k(a, c, d)
            return
        if (a, bb, c, d) in bra:
            return
        bra.add((a, bb, c, d))
        i = _dir(bb)
        b1 = _dec(bb, i)
        a1 = list(a)
        a1[i] += 1
        b(tuple(a1), b1, c, d)
        b(a, b1, c, d)

    for a in cart(la):
        for bb in cart(lb):
            for c in cart(lc):
                for d in cart(ld):
                    b(a, bb, c, d)
    return 2 * (len(ket) + len(bra))


# Non-zero coefficients of one shell's Cartesian -> pure matrix: the identity for s and p;
# for d the five real solid harmonics xy, yz, 2zz - xx - yy, xz, xx - yy hold 1+1+3+1+2.
_YLM_NNZ = {0: 1, 1: 3, 2: 8}


@lru_cache(maxsize=None)
def _sph_count(la, lb, lc, ld) -> int:
    Ls = (la, lb, lc, ld)
    dims = [ncart(L) for L in Ls]
    flops = 0
    for st, L in enumerate(Ls):
        if L >= 2:
            other = 1
            for q in range(4):
                if q != st:
                    other *= dims[q]
            flops += 2 * _YLM_NNZ[L] * other
        dims[st] = npure(L)
    return flops


def class_block_size(cls_index: int, pure: bool) -> int:
    """Integrals in one contracted block of the class in the final basis."""
    Ls = class_am(cls_index)
    out = 1
    for L in Ls:
        out *= npure(L) if pure else ncart(L)
    return out


def class_integrals(cls_index: int, computed_quartets: int, pure: bool) -> int:
    """Contracted integrals a launch computes (model-independent count: blocks x block size)."""
    return int(computed_quartets) * class_block_size(cls_index, pure)


def per_prim_flops(cls_index: int) -> int:
    la, lb, lc, ld = class_am(cls_index)
    v, nt = _vrr_count(la, lb, lc, ld)
    return C_PRIM + c_boys(la + lb + lc + ld) + v + nt


def per_quartet_flops(cls_index: int, pure: bool) -> int:
    la, lb, lc, ld = class_am(cls_index)
    return _hrr_count(la, lb, lc, ld) + (_sph_count(la, lb, lc, ld) if pure else 0) + \
        C_DIG * class_block_size(cls_index, pure)


def class_flops(cls_index: int, computed_quartets: int, prim_quartets: int, pure: bool) -> float:
    """Frozen-model FLOPs of computed_quartets contracted quartets holding prim_quartets
    primitive quartets."""
    return float(prim_quartets) * per_prim_flops(cls_index) + \
        float(computed_quartets) * per_quartet_flops(cls_index, pure)


# ---- gradient ------------------------------------------------------------------------------
@lru_cache(maxsize=None)
def _grad_sets(la, lb, lc, ld):
    """[e0|f0] target sets of the derivative classes: unweighted (lowered classes) and the
    2 alpha, 2 beta, 2 gamma weighted sets (raised on A, B, C)."""
    U = set()
    if la > 0:
        U |= _target_set(la - 1, la - 1 + lb, lc, lc + ld)
    if lb > 0:
        U |= _target_set(la, la + lb - 1, lc, lc + ld)
    if lc > 0:
        U |= _target_set(la, la + lb, lc - 1, lc - 1 + ld)
    A = _target_set(la + 1, la + 1 + lb, lc, lc + ld)
    B = _target_set(la, la + lb + 1, lc, lc + ld)
    C = _target_set(la, la + lb, lc + 1, lc + 1 + ld)
    return U, A, B, C


def grad_per_prim_flops(cls_index: int) -> int:
    la, lb, lc, ld = class_am(cls_index)
    U, A, B, C = _grad_sets(la, lb, lc, ld)
    v, _ = _vrr_enumerate(frozenset(U | A | B | C))
    return C_PRIM + c_boys(la + lb + lc + ld + 1) + v + len(U) + 2 * (len(A) + len(B) + len(C))


def _lowered_terms(la, lb, lc, ld) -> int:
    """Derivative integrals (per Cartesian block, over the nine centre components) that have
    a lowered term: sum over A, B, C and i of the Cartesian functions with a nonzero i index."""
    blk = ncart(la) * ncart(lb) * ncart(lc) * ncart(ld)
    n = 0
    for L in (la, lb, lc):
        with_i = sum(1 for c in cart(L) for i in range(3) if c[i] > 0)
        n += with_i * blk // ncart(L)
    return n


def grad_per_quartet_flops(cls_index: int, pure: bool) -> int:
    la, lb, lc, ld = class_am(cls_index)
    h = _hrr_count(la + 1, lb, lc, ld) + _hrr_count(la, lb + 1, lc, ld) + _hrr_count(la, lb, lc + 1, ld)
    if la > 0:
        h += _hrr_count(la - 1, lb, lc, ld)
    if lb > 0:
        h += _hrr_count(la, lb - 1, lc, ld)
    if lc > 0:
        h += _hrr_count(la, lb, lc - 1, ld)
    sph = 9 * _sph_count(la, lb, lc, ld) if pure else 0
    return h + 2 * _lowered_terms(la, lb, lc, ld) + sph + C_DIG_GRAD * 9 * class_block_size(cls_index, pure)


def grad_class_flops(cls_index: int, quartets: int, prim_quartets: int, pure: bool) -> float:
    """Frozen-model FLOPs of the first derivatives of `quartets` contracted quartets holding
    `prim_quartets` primitive quartets, contracted with their density weights."""
    return float(prim_quartets) * grad_per_prim_flops(cls_index) + \
        float(quartets) * grad_per_quartet_flops(cls_index, pure)


# ---- second number: the operation count of the engine's generated code ---------------------
def _ops():
    with open(OPS) as f:
        return json.load(f)


def generated_class_flops(cls_index: int, computed_quartets: int, prim_quartets: int, pure: bool) -> float:
    """FLOPs of the engine's own generated straight-line code (csrc/generated/ops.json)."""
    m = _ops()["eri"][cls_index]
    assert tuple(m["class"]) == class_am(cls_index)
    per_prim = m["prim_flops"] + (14 + 4 * m["boys_m"])
    per_q = m["hrr_flops"] + (m["pure_flops"] if pure else 0) + C_DIG * class_block_size(cls_index, pure)
    return float(prim_quartets) * per_prim + float(computed_quartets) * per_q
