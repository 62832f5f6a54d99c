"""Generator of the per-class ERI device code (straight-line CUDA).

For every shell-quartet class (la lb|lc ld) with la >= lb, lc >= ld, L <= 2 it
emits a device function that computes one contracted Cartesian block by the
Head-Gordon-Pople scheme:

  * Obara-Saika vertical recurrence (VRR) per primitive quartet, building
    [e0|f0]^(0) for la <= |e| <= la+lb, lc <= |f| <= lc+ld from
    [00|00]^(m) = K_ab K_cd 2 pi^2.5 / (p q sqrt(p+q)) F_m(T);
  * contraction over primitive pairs into register accumulators;
  * horizontal recurrence (HRR) on the contracted set,
    (a b+1_i| = (a+1_i b| + AB_i (a b|, then the same on the ket;
  * optionally the Cartesian -> pure transform with the solid-harmonic
    coefficients of src/math/solid_harmonics.cpp:30-108.

It also emits, per class, the adjoint gradient function: the same VRR run one
order higher, accumulated four ways (unweighted and weighted by 2 alpha of
centres A, B, C), HRR to the shifted classes, and contraction with a
Cartesian weight block W, giving dE/dA, dE/dB, dE/dC (dE/dD by translational
invariance).  The rule d/dA_i g_a = 2 alpha g_{a+1_i} - a_i g_{a-1_i} is the
one the reference applies (src/integrals/hfscf_oserideriv1.cpp:227-231).

Cartesian components are ordered as the reference orders them,
l = L-i, m = i-j, n = j (src/integrals/hfscf_shell.cpp:27-40).

Usage: python gen_eri.py OUT.cuh   (prints per-class operation counts)
"""
from __future__ import annotations

import json
import math
import sys
from fractions import Fraction

LMAX = 2
XYZ = "xyz"


def cart(L):
    return [(L - i, i - j, j) for i in range(L + 1) for j in range(i + 1)]


def cidx(c):
    L = sum(c)
    return cart(L).index(tuple(c))


def add(v, i, k=1):
    w = list(v)
    w[i] += k
    return tuple(w)


def tag(v):
    return "".join(str(x) for x in v)


# ---------------------------------------------------------------------------
# Real solid harmonics in the reference's convention (Cartesian x^L normalised,
# columns m = -L..L, prefactor 2^-L sqrt(2 (L-|m|)!/(L+|m|)!) for m != 0).
# ---------------------------------------------------------------------------
def ylm(L):
    nc = (L + 1) * (L + 2) // 2
    out = [[0.0] * (2 * L + 1) for _ in range(nc)]
    for mval in range(-L, L + 1):
        m = abs(mval)
        prefac = 2.0 ** (-L)
        if m:
            prefac *= math.sqrt(math.factorial(L - m) * 2.0 / math.factorial(L + m))
        for k in range((L - m) // 2 + 1):
            ffac = (-1) ** k * math.comb(L, k) * math.comb(2 * (L - k), L)
            if m:
                ffac *= math.factorial(L - 2 * k) / math.factorial(L - 2 * k - m)
            ffac *= prefac
            for a in range(k + 1):
                afac = math.comb(k, a) * ffac
                for b in range(a + 1):
                    fac = math.comb(a, b) * afac
                    zexp = 2 * (b - k) + L - m
                    yexp = 2 * (a - b)
                    if m == 0:
                        ii = yexp + zexp
                        out[ii * (ii + 1) // 2 + zexp][L + mval] += fac
                        continue
                    for p in range(m + 1):
                        r = (m - p) % 4
                        f = ({0: 1, 2: -1}.get(r, 0)) if mval > 0 else ({1: 1, 3: -1}.get(r, 0))
                        if f:
                            ii = yexp + m - p + zexp
                            out[ii * (ii + 1) // 2 + zexp][L + mval] += f * math.comb(m, p) * fac
    return out


class Emitter:
    """Collects straight-line statements and counts floating-point operations."""

    def __init__(self, indent="  "):
        self.lines = []
        self.indent = indent
        self.flops = 0

    def emit(self, s, flops=0):
        self.lines.append(self.indent + s)
        self.flops += flops


def lit(x):
    """A floating literal typed by the template parameter R."""
    if float(x).is_integer():
        return f"R({int(x)})"
    return f"R({repr(float(x))})"


# ---------------------------------------------------------------------------
# VRR: [e0|f0]^(m)
# ---------------------------------------------------------------------------
class VRR:
    def __init__(self, em: Emitter, prefix="v"):
        self.em = em
        self.memo = {}
        self.prefix = prefix
        self.consts = {}

    def kconst(self, base, k):
        """k * base as a named constant (base is inv2p, inv2q or inv2pq)."""
        if k == 1:
            return base
        key = (base, k)
        if key not in self.consts:
            name = f"{base}_{k}"
            self.em.emit(f"const R {name} = R({k}) * {base};", 1)
            self.consts[key] = name
        return self.consts[key]

    def get(self, e, f, m):
        key = (e, f, m)
        if key in self.memo:
            return self.memo[key]
        name = f"{self.prefix}_{tag(e)}_{tag(f)}_{m}"
        if sum(f) > 0:
            # ket vertical step on the direction with the largest f_i
            i = max(range(3), key=lambda d: (f[d], -d))
            f1 = add(f, i, -1)
            a = self.get(e, f1, m)
            b = self.get(e, f1, m + 1)
            expr = f"QC{XYZ[i]} * {a} + WQ{XYZ[i]} * {b}"
            fl = 3
            if f1[i] > 0:
                f2 = add(f1, i, -1)
                c = self.get(e, f2, m)
                d = self.get(e, f2, m + 1)
                expr += f" + {self.kconst('inv2q', f1[i])} * ({c} - rq * {d})"
                fl += 3
            if e[i] > 0:
                e1 = add(e, i, -1)
                g = self.get(e1, f1, m + 1)
                expr += f" + {self.kconst('inv2pq', e[i])} * {g}"
                fl += 2
        elif sum(e) > 0:
            i = max(range(3), key=lambda d: (e[d], -d))
            e1 = add(e, i, -1)
            a = self.get(e1, f, m)
            b = self.get(e1, f, m + 1)
            expr = f"PA{XYZ[i]} * {a} + WP{XYZ[i]} * {b}"
            fl = 3
            if e1[i] > 0:
                e2 = add(e1, i, -1)
                c = self.get(e2, f, m)
                d = self.get(e2, f, m + 1)
                expr += f" + {self.kconst('inv2p', e1[i])} * ({c} - rp * {d})"
                fl += 3
        else:
            expr = f"F[{m}]"
            fl = 0
            name = f"F[{m}]"
            self.memo[key] = name
            return name
        self.em.emit(f"const R {name} = {expr};", fl)
        self.memo[key] = name
        return name


def interleave_accumulation(body, adds):
    """Places every accumulation statement right after the statement that defines its VRR value
    (`adds`: (value name, statement) pairs), instead of after the whole recurrence: a target
    value then dies as soon as its last use in the recurrence has passed, rather than living to
    the end of the primitive-quartet body next to every accumulator.  Statements of values that
    are not defined in `body` (the Boys values F[m]) go first."""
    where = {}
    for i, line in enumerate(body):
        st = line.strip()
        if st.startswith("const R "):
            where[st[len("const R "):].split(" =", 1)[0]] = i
    after = {}
    head = []
    for name, stmt in adds:
        if name in where:
            after.setdefault(where[name], []).append(stmt)
        else:
            head.append(stmt)
    out = list(head)
    for i, line in enumerate(body):
        out.append(line)
        out.extend(after.get(i, []))
    return out


def vrr_targets(lo_e, hi_e, lo_f, hi_f):
    out = []
    for le in range(lo_e, hi_e + 1):
        for e in cart(le):
            for lf in range(lo_f, hi_f + 1):
                for f in cart(lf):
                    out.append((e, f))
    return out


# ---------------------------------------------------------------------------
# HRR on contracted [e0|f0] -> (a b|c d)
# ---------------------------------------------------------------------------
class HRR:
    def __init__(self, em: Emitter, acc, prefix="h"):
        self.em = em
        self.acc = acc  # function (e, f) -> accumulator expression
        self.kmemo = {}
        self.bmemo = {}
        self.prefix = prefix

    def ket(self, e, c, d):
        key = (e, c, d)
        if key in self.kmemo:
            return self.kmemo[key]
        if sum(d) == 0:
            name = self.acc(e, c)
        else:
            i = max(range(3), key=lambda k: (d[k], -k))
            d1 = add(d, i, -1)
            a = self.ket(e, add(c, i), d1)
            b = self.ket(e, c, d1)
            name = f"{self.prefix}k_{tag(e)}_{tag(c)}_{tag(d)}"
            self.em.emit(f"const R {name} = {a} + CD{XYZ[i]} * {b};", 2)
        self.kmemo[key] = name
        return name

    def bra(self, a, b, c, d):
        key = (a, b, c, d)
        if key in self.bmemo:
            return self.bmemo[key]
        if sum(b) == 0:
            name = self.ket(a, c, d)
        else:
            i = max(range(3), key=lambda k: (b[k], -k))
            b1 = add(b, i, -1)
            x = self.bra(add(a, i), b1, c, d)
            y = self.bra(a, b1, c, d)
            name = f"{self.prefix}b_{tag(a)}_{tag(b)}_{tag(c)}_{tag(d)}"
            self.em.emit(f"const R {name} = {x} + AB{XYZ[i]} * {y};", 2)
        self.bmemo[key] = name
        return name


PRIM_HEADER = """\
      // primitive-quartet scalars
      const R pq = p + q;
      const R rs = rsqrt_t(pq);      // 1 / sqrt(p + q)
      const R ipq = rs * rs;
      const R rho = p * q * ipq;
      const R rp = q * ipq;          // rho / p
      const R rq = p * ipq;          // rho / q
      const R inv2p = R(0.5) * ip;
      const R inv2q = R(0.5) * iq;
      const R inv2pq = R(0.5) * ipq;
      const R PQx = Px - Qx, PQy = Py - Qy, PQz = Pz - Qz;
      const R WPx = -rp * PQx, WPy = -rp * PQy, WPz = -rp * PQz;
      const R WQx = rq * PQx, WQy = rq * PQy, WQz = rq * PQz;
      const R T = rho * (PQx * PQx + PQy * PQy + PQz * PQz);
      const R pre = Kab * Kcd * rs;
"""
PRIM_HEADER_FLOPS = 1 + 1 + 1 + 2 + 1 + 1 + 1 + 1 + 1 + 3 + 3 + 3 + 6 + 2

def ncart(L):
    return (L + 1) * (L + 2) // 2


UNROLL2_MAX_VRR = 50
PRIMWARP_MAX_VRR = 150   # classes that also get a warp-over-primitives variant


def gen_eri_primwarp(la, lb, lc, ld):
    """Same integral block as gen_eri_class, for a group of G lanes (G = 4 ... 32, aligned
    inside the warp): the lanes split the primitive quartets, then the accumulators are
    summed with shuffles inside the group and every lane of it runs the HRR (the block is
    valid in all G lanes).  Every lane of the warp must call it (full-mask shuffles)."""
    L = la + lb + lc + ld
    em = Emitter("    ")
    vrr = VRR(em)
    targets = vrr_targets(la, la + lb, lc, lc + ld)
    names = [vrr.get(e, f, 0) for e, f in targets]
    prim_body = list(em.lines)
    acc_index = {t: n for n, t in enumerate(targets)}
    em2 = Emitter("  ")
    hrr = HRR(em2, lambda e, f: f"acc[{acc_index[(e, f)]}]")
    outs = [hrr.bra(a, b, c, d) for a in cart(la) for b in cart(lb) for c in cart(lc) for d in cart(ld)]
    nt = len(targets)
    s = [f"template <typename R, int G>",
         f"__device__ __forceinline__ void eri_{la}{lb}{lc}{ld}_pw(const PrimPair<R>* __restrict__ bp, int nbp, "
         f"const PrimPair<R>* __restrict__ kp, int nkp, R ABx, R ABy, R ABz, R CDx, R CDy, R CDz, "
         f"const BoysTable<R>& boys, R* __restrict__ out, int lane) {{",
         f"  R acc[{nt}];", "#pragma unroll", f"  for (int t = 0; t < {nt}; ++t) acc[t] = R(0);",
         "  const int npq = nbp * nkp;",
         "  for (int x = lane; x < npq; x += G) {",
         "    const int ib = x / nkp, ik = x - ib * nkp;",
         "    const R p = bp[ib].p, ip = bp[ib].ip, Px = bp[ib].Px, Py = bp[ib].Py, Pz = bp[ib].Pz;",
         "    const R PAx = bp[ib].PAx, PAy = bp[ib].PAy, PAz = bp[ib].PAz, Kab = bp[ib].Kp;",
         "    const R q = kp[ik].p, iq = kp[ik].ip, Qx = kp[ik].Px, Qy = kp[ik].Py, Qz = kp[ik].Pz;",
         "    const R QCx = kp[ik].PAx, QCy = kp[ik].PAy, QCz = kp[ik].PAz, Kcd = kp[ik].Kp;"]
    s.append("\n".join("  " + l[6:] if l.startswith("      ") else l for l in PRIM_HEADER.rstrip("\n").split("\n")))
    s.append(f"    R F[{L + 1}];")
    s.append(f"    boys.template eval<{L}>(T, pre, F);")
    s += interleave_accumulation(prim_body, [(nme, f"    acc[{t}] += {nme};") for t, nme in enumerate(names)])
    s.append("  }")
    s.append("#pragma unroll")
    s.append(f"  for (int t = 0; t < {nt}; ++t)")
    s.append("#pragma unroll")
    s.append("    for (int off = G / 2; off > 0; off >>= 1) acc[t] += __shfl_xor_sync(0xffffffffu, acc[t], off, G);")
    s += em2.lines
    for o, nme in enumerate(outs):
        s.append(f"  out[{o}] = {nme};")
    s.append("}")
    return "\n".join(s)


def gen_eri_class(la, lb, lc, ld):
    """Device function computing the contracted Cartesian block of class (la lb|lc ld)."""
    L = la + lb + lc + ld
    em = Emitter("      ")
    vrr = VRR(em)
    targets = vrr_targets(la, la + lb, lc, lc + ld)
    names = [vrr.get(e, f, 0) for e, f in targets]
    prim_body = list(em.lines)
    prim_flops = em.flops + PRIM_HEADER_FLOPS + len(targets)  # + accumulation
    acc_index = {t: n for n, t in enumerate(targets)}
    em2 = Emitter("  ")
    hrr = HRR(em2, lambda e, f: f"acc[{acc_index[(e, f)]}]")
    outs = []
    for a in cart(la):
        for b in cart(lb):
            for c in cart(lc):
                for d in cart(ld):
                    outs.append(hrr.bra(a, b, c, d))
    nout = len(outs)
    s = []
    fn = f"eri_{la}{lb}{lc}{ld}"
    s.append(f"// ({'spdf'[la]}{'spdf'[lb]}|{'spdf'[lc]}{'spdf'[ld]}): {len(targets)} contracted VRR targets, "
             f"{len(vrr.memo)} VRR values, {nout} outputs")
    # BT: the Boys table in global memory (BoysTable) or staged in shared memory (BoysShared)
    s.append("template <typename R, typename BT>")
    s.append(f"__device__ __forceinline__ void {fn}(const PrimPair<R>* __restrict__ bp, int nbp, "
             f"const PrimPair<R>* __restrict__ kp, int nkp, R ABx, R ABy, R ABz, R CDx, R CDy, R CDz, "
             f"const BT& boys, R* __restrict__ out) {{")
    s.append(f"  R acc[{len(targets)}];")
    s.append(f"#pragma unroll")
    s.append(f"  for (int t = 0; t < {len(targets)}; ++t) acc[t] = R(0);")
    # Ket primitives outside, bra primitives inside: the lanes of a warp mostly hold
    # quartets of one bra pair (the lists are bra-major), so the inner loads are broadcasts
    # and the gathers of the lanes' different ket pairs happen once per ket primitive.
    s.append("  for (int ik = 0; ik < nkp; ++ik) {")
    s.append("    const R q = kp[ik].p, iq = kp[ik].ip, Qx = kp[ik].Px, Qy = kp[ik].Py, Qz = kp[ik].Pz;")
    s.append("    const R QCx = kp[ik].PAx, QCy = kp[ik].PAy, QCz = kp[ik].PAz, Kcd = kp[ik].Kp;")
    if len(vrr.memo) <= UNROLL2_MAX_VRR:
        # small classes: two primitive quartets in flight hide the load latency
        s.append("#pragma unroll 2")
    s.append("    for (int ib = 0; ib < nbp; ++ib) {")
    s.append("      const R p = bp[ib].p, ip = bp[ib].ip, Px = bp[ib].Px, Py = bp[ib].Py, Pz = bp[ib].Pz;")
    s.append("      const R PAx = bp[ib].PAx, PAy = bp[ib].PAy, PAz = bp[ib].PAz, Kab = bp[ib].Kp;")
    s.append(PRIM_HEADER.rstrip("\n"))
    s.append(f"      R F[{L + 1}];")
    s.append(f"      boys.template eval<{L}>(T, pre, F);")
    s += interleave_accumulation(prim_body, [(n, f"      acc[{t}] += {n};") for t, n in enumerate(names)])
    s.append("    }")
    s.append("  }")
    s += em2.lines
    for o, n in enumerate(outs):
        s.append(f"  out[{o}] = {n};")
    s.append("}")
    meta = {"class": [la, lb, lc, ld], "vrr_targets": len(targets), "vrr_values": len(vrr.memo),
            "prim_flops": prim_flops, "hrr_flops": em2.flops, "nout": nout, "boys_m": L}
    return "\n".join(s), meta


def gen_pure(la, lb, lc, ld):
    """Cartesian -> pure transform of one block, index by index (as TRANSFORM::transform,
    src/integrals/hfscf_transform.cpp:80-154), skipping zero coefficients."""
    Ls = (la, lb, lc, ld)
    ncs = [ncart(x) for x in Ls]
    nps = [2 * x + 1 for x in Ls]
    Y = [ylm(x) for x in Ls]
    em = Emitter("  ")
    cur = {}
    dims = list(ncs)
    # current[(i0,i1,i2,i3)] -> expression name
    import itertools
    for idx in itertools.product(*[range(n) for n in ncs]):
        flat = ((idx[0] * ncs[1] + idx[1]) * ncs[2] + idx[2]) * ncs[3] + idx[3]
        cur[idx] = f"in[{flat}]"
    for stage in range(4):
        if Ls[stage] < 2:
            # L = 0: identity; L = 1: a permutation (pure p = y, z, x) -- no arithmetic
            new = {}
            newdims = list(dims)
            newdims[stage] = nps[stage]
            for idx in itertools.product(*[range(n) for n in newdims]):
                col = idx[stage]
                src = [r for r in range(ncs[stage]) if Y[stage][r][col] != 0.0]
                assert len(src) == 1 and Y[stage][src[0]][col] == 1.0
                j = list(idx)
                j[stage] = src[0]
                new[idx] = cur[tuple(j)]
            cur, dims = new, newdims
            continue
        new = {}
        newdims = list(dims)
        newdims[stage] = nps[stage]
        for idx in itertools.product(*[range(n) for n in newdims]):
            col = idx[stage]
            terms = []
            for r in range(ncs[stage]):
                c = Y[stage][r][col]
                if c != 0.0:
                    j = list(idx)
                    j[stage] = r
                    terms.append((c, cur[tuple(j)]))
            name = f"t{stage}_{''.join(map(str, idx))}"
            expr = " + ".join(f"{lit(c)} * {v}" if c != 1.0 else v for c, v in terms)
            em.emit(f"const R {name} = {expr};", 2 * len(terms) - 1)
            new[idx] = name
        cur, dims = new, newdims
    body = list(em.lines)
    nout = nps[0] * nps[1] * nps[2] * nps[3]
    for idx in itertools.product(*[range(n) for n in nps]):
        flat = ((idx[0] * nps[1] + idx[1]) * nps[2] + idx[2]) * nps[3] + idx[3]
        body.append(f"  out[{flat}] = {cur[idx]};")
    fn = f"to_pure_{la}{lb}{lc}{ld}"
    s = ["template <typename R>",
         f"__device__ __forceinline__ void {fn}(const R* __restrict__ in, R* __restrict__ out) {{"]
    s += body
    s.append("}")
    return "\n".join(s), em.flops


def gen_pure_T(la, lb, lc, ld):
    """Transpose transform: Cartesian weights from pure weights (for the gradient),
    W_cart[abcd] = sum_ijkl Y[a][i] Y[b][j] Y[c][k] Y[d][l] W_pure[ijkl]."""
    import itertools
    Ls = (la, lb, lc, ld)
    ncs = [ncart(x) for x in Ls]
    nps = [2 * x + 1 for x in Ls]
    Y = [ylm(x) for x in Ls]
    em = Emitter("  ")
    cur = {}
    for idx in itertools.product(*[range(n) for n in nps]):
        flat = ((idx[0] * nps[1] + idx[1]) * nps[2] + idx[2]) * nps[3] + idx[3]
        cur[idx] = f"in[{flat}]"
    dims = list(nps)
    for stage in range(4):
        new = {}
        newdims = list(dims)
        newdims[stage] = ncs[stage]
        for idx in itertools.product(*[range(n) for n in newdims]):
            row = idx[stage]
            terms = []
            for col in range(nps[stage]):
                c = Y[stage][row][col]
                if c != 0.0:
                    j = list(idx)
                    j[stage] = col
                    terms.append((c, cur[tuple(j)]))
            if not terms:
                new[idx] = "R(0)"
                continue
            if len(terms) == 1 and terms[0][0] == 1.0:
                new[idx] = terms[0][1]
                continue
            name = f"u{stage}_{''.join(map(str, idx))}"
            expr = " + ".join(f"{lit(c)} * {v}" if c != 1.0 else v for c, v in terms)
            em.emit(f"const R {name} = {expr};", 2 * len(terms) - 1)
            new[idx] = name
        cur, dims = new, newdims
    body = list(em.lines)
    for idx in itertools.product(*[range(n) for n in ncs]):
        flat = ((idx[0] * ncs[1] + idx[1]) * ncs[2] + idx[2]) * ncs[3] + idx[3]
        body.append(f"  out[{flat}] = {cur[idx]};")
    fn = f"from_pure_{la}{lb}{lc}{ld}"
    s = ["template <typename R>",
         f"__device__ __forceinline__ void {fn}(const R* __restrict__ in, R* __restrict__ out) {{"]
    s += body
    s.append("}")
    return "\n".join(s)


# ---------------------------------------------------------------------------
# Adjoint gradient: contraction of W with d(ab|cd)/dA, dB, dC.
# ---------------------------------------------------------------------------
def grad_sets(la, lb, lc, ld):
    """Contracted [e0|f0] sets the adjoint gradient needs, by weight."""
    em = Emitter("      ")
    vrr = VRR(em)
    # Which contracted [e0|f0] sets are needed, by weight.
    need = {"U": set(), "A": set(), "B": set(), "C": set()}
    for le in range(max(la - 1, 0), la + lb):          # (a-1 b|cd) and (a b-1|cd): |e| <= la+lb-1
        for lf in range(lc, lc + ld + 1):
            for e in cart(le):
                for f in cart(lf):
                    need["U"].add((e, f))
    for le in range(la, la + lb + 1):                   # (ab|c-1 d), (ab|c d-1): |f| <= lc+ld-1
        for lf in range(max(lc - 1, 0), lc + ld):
            for e in cart(le):
                for f in cart(lf):
                    need["U"].add((e, f))
    for le in range(la + 1, la + lb + 2):
        for lf in range(lc, lc + ld + 1):
            for e in cart(le):
                for f in cart(lf):
                    need["A"].add((e, f))
    for le in range(la, la + lb + 2):
        for lf in range(lc, lc + ld + 1):
            for e in cart(le):
                for f in cart(lf):
                    need["B"].add((e, f))
    for le in range(la, la + lb + 1):
        for lf in range(lc + 1, lc + ld + 2):
            for e in cart(le):
                for f in cart(lf):
                    need["C"].add((e, f))
    order = {k: sorted(v, key=lambda t: (sum(t[0]), cidx(t[0]), sum(t[1]), cidx(t[1]))) for k, v in need.items()}
    return order


def grad_terms(la, lb, lc, ld):
    """For every (centre, direction): list of (W index, [(coef, set, a, b, c, d), ...])."""
    gsum = {(c, d): [] for c in "ABC" for d in range(3)}
    w = 0
    for a in cart(la):
        for b in cart(lb):
            for c in cart(lc):
                for d in cart(ld):
                    for dr in range(3):
                        t = [(1, "A", add(a, dr), b, c, d)]
                        if a[dr] > 0:
                            t.append((-a[dr], "U", add(a, dr, -1), b, c, d))
                        gsum[("A", dr)].append((w, t))
                        t = [(1, "B", a, add(b, dr), c, d)]
                        if b[dr] > 0:
                            t.append((-b[dr], "U", a, add(b, dr, -1), c, d))
                        gsum[("B", dr)].append((w, t))
                        t = [(1, "C", a, b, add(c, dr), d)]
                        if c[dr] > 0:
                            t.append((-c[dr], "U", a, b, add(c, dr, -1), d))
                        gsum[("C", dr)].append((w, t))
                    w += 1
    return gsum


def gen_grad_class(la, lb, lc, ld):
    L = la + lb + lc + ld + 1
    em = Emitter("      ")
    vrr = VRR(em)
    order = grad_sets(la, lb, lc, ld)
    allt = sorted(set().union(*[set(v) for v in order.values()]),
                  key=lambda t: (sum(t[0]), cidx(t[0]), sum(t[1]), cidx(t[1])))
    vals = {t: vrr.get(t[0], t[1], 0) for t in allt}
    prim_body = list(em.lines)
    idx = {}
    n = 0
    for k in ("U", "A", "B", "C"):
        for t in order[k]:
            idx[(k, t)] = n
            n += 1
    nacc = n
    # HRR + contraction
    em2 = Emitter("  ")
    hr = {k: HRR(em2, (lambda kk: (lambda e, f: f"acc[{idx[(kk, (e, f))]}]"))(k), prefix=f"h{k}")
          for k in ("U", "A", "B", "C")}
    gt = grad_terms(la, lb, lc, ld)
    gsum = {}
    for key, items in gt.items():
        gsum[key] = []
        for wi, terms in items:
            t = [hr[terms[0][1]].bra(*terms[0][2:])]
            if len(terms) > 1:
                t.append((-terms[1][0], hr["U"].bra(*terms[1][2:])))
            gsum[key].append((wi, t))
    for (cen, dr), items in gsum.items():
        terms = []
        for wi, t in items:
            e = t[0]
            if len(t) > 1:
                k, u = t[1]
                e = f"({e} - {lit(k)} * {u})"
            terms.append(f"W[{wi}] * {e}")
        em2.emit(f"g{cen}[{dr}] = " + " + ".join(terms) + ";", 2 * len(terms) + sum(2 for _, t in items if len(t) > 1))
    fn = f"grad_{la}{lb}{lc}{ld}"
    s = [f"// adjoint gradient of ({'spdf'[la]}{'spdf'[lb]}|{'spdf'[lc]}{'spdf'[ld]}): {nacc} accumulators, "
         f"{len(vrr.memo)} VRR values"]
    s.append("template <typename R>")
    s.append(f"__device__ __forceinline__ void {fn}(const PrimPair<R>* __restrict__ bp, const R* __restrict__ ea, "
             f"const R* __restrict__ eb, int nbp, const PrimPair<R>* __restrict__ kp, const R* __restrict__ ec, int nkp, "
             f"R ABx, R ABy, R ABz, R CDx, R CDy, R CDz, const BoysTable<R>& boys, const R* __restrict__ W, "
             f"R* __restrict__ gA, R* __restrict__ gB, R* __restrict__ gC) {{")
    s.append(f"  R acc[{nacc}];")
    s.append("#pragma unroll")
    s.append(f"  for (int t = 0; t < {nacc}; ++t) acc[t] = R(0);")
    s.append("  for (int ib = 0; ib < nbp; ++ib) {")
    s.append("    const R p = bp[ib].p, ip = bp[ib].ip, Px = bp[ib].Px, Py = bp[ib].Py, Pz = bp[ib].Pz;")
    s.append("    const R PAx = bp[ib].PAx, PAy = bp[ib].PAy, PAz = bp[ib].PAz, Kab = bp[ib].Kp;")
    s.append("    const R wa = R(2) * ea[ib], wb = R(2) * eb[ib];")
    s.append("    for (int ik = 0; ik < nkp; ++ik) {")
    s.append("      const R q = kp[ik].p, iq = kp[ik].ip, Qx = kp[ik].Px, Qy = kp[ik].Py, Qz = kp[ik].Pz;")
    s.append("      const R QCx = kp[ik].PAx, QCy = kp[ik].PAy, QCz = kp[ik].PAz, Kcd = kp[ik].Kp;")
    s.append("      const R wc = R(2) * ec[ik];")
    s.append(PRIM_HEADER.rstrip("\n"))
    s.append(f"      R F[{L + 1}];")
    s.append(f"      boys.template eval<{L}>(T, pre, F);")
    adds = []
    for k, wname in (("U", None), ("A", "wa"), ("B", "wb"), ("C", "wc")):
        for t in order[k]:
            v = vals[t]
            adds.append((v, f"      acc[{idx[(k, t)]}] += {v};" if wname is None else
                         f"      acc[{idx[(k, t)]}] += {wname} * {v};"))
    s += interleave_accumulation(prim_body, adds)
    s.append("    }")
    s.append("  }")
    s += em2.lines
    s.append("}")
    meta = {"class": [la, lb, lc, ld], "accumulators": nacc, "vrr_values": len(vrr.memo),
            "prim_flops": em.flops + PRIM_HEADER_FLOPS + 2 * nacc, "hrr_flops": em2.flops, "boys_m": L}
    return "\n".join(s), meta


GRAD_SETS = ("U", "A", "B", "C")


def gen_grad_class_pass(la, lb, lc, ld, psets):
    """The part of gen_grad_class that some of the accumulator sets carry (psets: one set name or
    a tuple of them): the VRR (one order higher) of those sets' targets only, their accumulation
    (weight 1, 2 alpha_a, 2 alpha_b or 2 alpha_c), their HRR, and the gradient terms that read
    them -- for A, B, C the 2 alpha (a+1_i b|cd)-type terms of that centre; for U the
    -a_i (a-1_i b|cd)-type terms of all three centres.  Passes whose sets cover U, A, B, C once
    add up to the whole gradient; each keeps a share of the accumulators of the one-pass form, at
    the price of recomputing the shared part of the recurrence."""
    if isinstance(psets, str):
        psets = (psets,)
    L = la + lb + lc + ld + 1
    em = Emitter("      ")
    vrr = VRR(em)
    allsets = grad_sets(la, lb, lc, ld)
    idx, adds_src, nacc = {}, [], 0
    for k in psets:
        for t in allsets[k]:
            idx[(k, t)] = nacc
            adds_src.append((k, t))
            nacc += 1
    targets = sorted({t for _, t in adds_src}, key=lambda t: (sum(t[0]), cidx(t[0]), sum(t[1]), cidx(t[1])))
    vals = {t: vrr.get(t[0], t[1], 0) for t in targets}
    prim_body = list(em.lines)
    em2 = Emitter("  ")
    hr = {k: HRR(em2, (lambda kk: (lambda e, f: f"acc[{idx[(kk, (e, f))]}]"))(k), prefix=f"h{k}") for k in psets}
    gt = grad_terms(la, lb, lc, ld)
    outs = {}
    for (cen, dr), items in gt.items():
        terms = []
        for wi, tl in items:
            for coef, st, a, b, c, d in tl:
                if st not in psets:
                    continue
                v = hr[st].bra(a, b, c, d)
                terms.append(f"W[{wi}] * {v}" if coef == 1 else f"{lit(coef)} * W[{wi}] * {v}")
        outs[(cen, dr)] = terms
    for (cen, dr), terms in outs.items():
        em2.emit(f"g{cen}[{dr}] = " + (" + ".join(terms) if terms else "R(0)") + ";", 3 * len(terms))
    wname = {"U": None, "A": "wa", "B": "wb", "C": "wc"}
    tag_sets = "".join(psets)
    fn = f"grad_{la}{lb}{lc}{ld}_{tag_sets}"
    s = [f"// adjoint gradient of ({'spdf'[la]}{'spdf'[lb]}|{'spdf'[lc]}{'spdf'[ld]}), sets {tag_sets} only: {nacc} "
         f"accumulators, {len(vrr.memo)} VRR values"]
    s.append("template <typename R>")
    s.append(f"__device__ __forceinline__ void {fn}({GRAD_SIG}) {{")
    s.append(f"  R acc[{nacc}];")
    s.append("#pragma unroll")
    s.append(f"  for (int t = 0; t < {nacc}; ++t) acc[t] = R(0);")
    s.append("  for (int ib = 0; ib < nbp; ++ib) {")
    s.append("    const R p = bp[ib].p, ip = bp[ib].ip, Px = bp[ib].Px, Py = bp[ib].Py, Pz = bp[ib].Pz;")
    s.append("    const R PAx = bp[ib].PAx, PAy = bp[ib].PAy, PAz = bp[ib].PAz, Kab = bp[ib].Kp;")
    s.append("    const R wa = R(2) * ea[ib], wb = R(2) * eb[ib];")
    s.append("    (void)wa; (void)wb;")
    s.append("    for (int ik = 0; ik < nkp; ++ik) {")
    s.append("      const R q = kp[ik].p, iq = kp[ik].ip, Qx = kp[ik].Px, Qy = kp[ik].Py, Qz = kp[ik].Pz;")
    s.append("      const R QCx = kp[ik].PAx, QCy = kp[ik].PAy, QCz = kp[ik].PAz, Kcd = kp[ik].Kp;")
    s.append("      const R wc = R(2) * ec[ik];")
    s.append("      (void)wc;")
    s.append(PRIM_HEADER.rstrip("\n"))
    s.append(f"      R F[{L + 1}];")
    s.append(f"      boys.template eval<{L}>(T, pre, F);")
    adds = [(vals[t], f"      acc[{idx[(k, t)]}] += {vals[t]};" if wname[k] is None else
             f"      acc[{idx[(k, t)]}] += {wname[k]} * {vals[t]};") for k, t in adds_src]
    s += interleave_accumulation(prim_body, adds)
    s.append("    }")
    s.append("  }")
    s += em2.lines
    s.append("}")
    return "\n".join(s), {"accumulators": nacc, "vrr_values": len(vrr.memo), "prim_flops": em.flops,
                          "hrr_flops": em2.flops}


def classes():
    pairs = [(a, b) for a in range(LMAX + 1) for b in range(a + 1)]  # ss ps pp ds dp dd
    out = []
    for i, (la, lb) in enumerate(pairs):
        for j, (lc, ld) in enumerate(pairs):
            if j <= i:
                out.append((la, lb, lc, ld))
    return pairs, out


GRAD_STRAIGHT_MAX_VRR = 900   # larger gradient classes run in table mode
GRAD_SPLIT_MIN_ACC = 150      # straight-line gradient classes with this many accumulators run as 4 passes
GRAD_PAIR_MAX_ACC = 160       # ... or as 2 passes of two sets each when both halves stay below this


def class_args_sig():
    return ("const PrimPair<R>* __restrict__ bp, int nbp, const PrimPair<R>* __restrict__ kp, int nkp, "
            "R ABx, R ABy, R ABz, R CDx, R CDy, R CDz, const BoysTable<R>& boys, R* __restrict__ out")


GRAD_SIG = ("const PrimPair<R>* __restrict__ bp, const R* __restrict__ ea, const R* __restrict__ eb, int nbp, "
            "const PrimPair<R>* __restrict__ kp, const R* __restrict__ ec, int nkp, R ABx, R ABy, R ABz, "
            "R CDx, R CDy, R CDz, const BoysTable<R>& boys, const R* __restrict__ W, R* __restrict__ gA, "
            "R* __restrict__ gB, R* __restrict__ gC")
GRAD_ARGS = "bp, ea, eb, nbp, kp, ec, nkp, ABx, ABy, ABz, CDx, CDy, CDz, boys, W, gA, gB, gC"


def common_header():
    out = ["// GENERATED by gen_eri.py -- do not edit.", "#pragma once", '#include "../hfgpu_common.cuh"', "",
           "// Cartesian -> pure coefficients for L = 0, 1, 2 (ncart x npure, row-major),",
           "// hfscfmath::Ylm_transmat (src/math/solid_harmonics.cpp:16-27).",
           "static __constant__ double c_ylm[3][30] = {"]
    for L in range(3):
        Y = ylm(L)
        flat = [Y[r][c] for r in range(len(Y)) for c in range(2 * L + 1)]
        flat += [0.0] * (30 - len(flat))
        out.append("  {" + ", ".join(repr(float(x)) for x in flat) + "},")
    out.append("};")
    out.append("")
    out.append("template <int LA, int LB, int LC, int LD>")
    out.append("struct ClassCode;")
    return "\n".join(out) + "\n"


def cap_blocks(vrr_values):
    """Blocks of 128 threads per SM the register-capped thread variant asks for (0: no such
    variant): 8 (64 registers) for the smallest classes, 5 (about 100) for the next ones."""
    if vrr_values <= 1:
        return 0  # (ss|ss) already fits in 64 registers
    if vrr_values <= 20:
        return 8
    if vrr_values <= 60:
        return 5
    return 0


STAGED_MAX_L = 4          # classes that also get the persistent form with the Boys table in shared memory
LOWRES_MIN_VRR = 250      # classes that also get the low-residency thread variant (their registers spill)
WARP_MIN_VRR = 250        # classes that also get a warp-per-quartet form (hfgpu_autotune picks)
WARP_DEFAULT_MIN_VRR = 1000  # (dd|dp) and (dd|dd): measured faster as one warp per quartet by default


def class_header(c):
    la, lb, lc, ld = c
    t = f"{la}{lb}{lc}{ld}"
    parts = ["// GENERATED by gen_eri.py -- do not edit.", "#pragma once", '#include "common.cuh"', ""]
    code, m = gen_eri_class(*c)
    warp = m["vrr_values"] >= WARP_MIN_VRR
    m["warp"] = warp
    parts += [code, ""]
    primwarp = m["vrr_values"] <= PRIMWARP_MAX_VRR
    m["primwarp"] = primwarp
    if primwarp:
        parts += [gen_eri_primwarp(*c), ""]
    if warp:
        wcode, wm = gen_warp_class(*c)
        parts += [wcode, ""]
        m.update({"warp_" + k: v for k, v in wm.items() if k != "class"})
    pc, pf = gen_pure(*c)
    parts += [pc, ""]
    parts += [gen_pure_T(*c), ""]
    m["pure_flops"] = pf
    # the adjoint gradient: straight-line for small classes, op tables for large ones
    code_g, mg = gen_grad_class(*c)
    straight = mg["vrr_values"] <= GRAD_STRAIGHT_MAX_VRR
    if not straight:
        code_g, mg = gen_grad_table(*c)
    parts += [code_g, ""]
    mg["table"] = not straight
    # the op-table classes also get the warp-per-quartet form (measured faster than one thread
    # per quartet on global scratch for every one of them).  The straight-line classes keep one
    # thread per quartet: warp forms generated for those with more than 150 accumulators measured
    # slower at n-octane and anthracene sizes (29.6 against 25.7 ms and 216 against 189 ms per
    # gradient), and with the block forms offered to the autotuner as well it kept the four-pass
    # thread form for all but one of them (octane 17.9 -> 17.0 ms, anthracene 135 -> 121 ms, for
    # 3-8x the tuning time)
    gwarp = not straight
    if gwarp:
        gwcode, gwmeta = gen_grad_warp(*c)
        parts += [gwcode, ""]
        mg["grad_warp"] = gwmeta
        # and the per-set split of the warp form: four one-set tables, four launches
        for ps in GRAD_SETS:
            pcode, pmeta = gen_grad_warp(*c, sets=(ps,), suffix="_" + ps)
            parts += [pcode, ""]
            mg["grad_warp_" + ps] = pmeta
    parts.append(f"template <>")
    parts.append(f"struct ClassCode<{la}, {lb}, {lc}, {ld}> {{")
    parts.append(f"  static constexpr bool kGradTable = {'false' if straight else 'true'};")
    parts.append(f"  static constexpr bool kWarp = {'true' if warp else 'false'};")
    parts.append(f"  static constexpr bool kWarpDefault = {'true' if m['vrr_values'] >= WARP_DEFAULT_MIN_VRR else 'false'};")
    parts.append(f"  using WarpTab = {'WarpTab' + t if warp else 'void'};")
    parts.append(f"  using GradTab = {'void' if straight else 'GradTable' + t};")
    parts.append(f"  static constexpr bool kGradWarp = {'true' if gwarp else 'false'};")
    parts.append(f"  using GradWarpTab = {'GradWarpTab' + t if gwarp else 'void'};")
    for pi, ps in enumerate(GRAD_SETS):
        parts.append(f"  using GradWarpTabP{pi} = {'GradWarpTab' + t + '_' + ps if gwarp else 'void'};")
    parts.append(f"  static constexpr bool kPrimWarp = {'true' if primwarp else 'false'};")
    parts.append(f"  static constexpr int kCapBlocks = {cap_blocks(m['vrr_values'])};")
    # the persistent form with the Boys table in shared memory: classes of total L <= STAGED_MAX_L
    parts.append(f"  static constexpr bool kStaged = {'true' if la + lb + lc + ld <= STAGED_MAX_L else 'false'};")
    # the low-residency variant of the thread form: the classes whose register code spills
    parts.append(f"  static constexpr bool kLowRes = {'true' if m['vrr_values'] >= LOWRES_MIN_VRR else 'false'};")
    if primwarp:
        parts.append(f"  template <typename R, int G>")
        parts.append(f"  static __device__ __forceinline__ void eri_pw({class_args_sig()}, int lane) {{")
        parts.append(f"    eri_{t}_pw<R, G>(bp, nbp, kp, nkp, ABx, ABy, ABz, CDx, CDy, CDz, boys, out, lane);")
        parts.append("  }")
    parts.append(f"  template <typename R, typename BT>")
    parts.append(f"  static __device__ __forceinline__ void eri({class_args_sig().replace('const BoysTable<R>&', 'const BT&')}) {{")
    parts.append(f"    eri_{t}<R, BT>(bp, nbp, kp, nkp, ABx, ABy, ABz, CDx, CDy, CDz, boys, out);")
    parts.append("  }")
    parts.append("  template <typename R>")
    parts.append(f"  static __device__ __forceinline__ void to_pure(const R* __restrict__ in, R* __restrict__ out) {{ to_pure_{t}<R>(in, out); }}")
    parts.append("  template <typename R>")
    parts.append(f"  static __device__ __forceinline__ void from_pure(const R* __restrict__ in, R* __restrict__ out) {{ from_pure_{t}<R>(in, out); }}")
    # the straight-line classes whose one-pass accumulators spill run as four passes, one
    # accumulator set each (gen_grad_class_pass), or as two passes (sets U and A, sets B and C)
    # when each half stays below GRAD_PAIR_MAX_ACC accumulators: the recurrence is then
    # recomputed once instead of three times
    npass = 4 if straight and mg["accumulators"] >= GRAD_SPLIT_MIN_ACC else 1
    pass_sets = [(ps,) for ps in GRAD_SETS]
    if npass == 4:
        nset = {k: len(v) for k, v in grad_sets(*c).items()}
        if max(nset["U"] + nset["A"], nset["B"] + nset["C"]) < GRAD_PAIR_MAX_ACC:
            npass = 2
            pass_sets = [("U", "A"), ("B", "C")]
    mg["passes"] = npass
    parts.append(f"  static constexpr int kGradPasses = {npass};")
    if straight:
        parts.append("  template <typename R>")
        parts.append(f"  static __device__ __forceinline__ void grad({GRAD_SIG}) {{ grad_{t}<R>({GRAD_ARGS}); }}")
    if npass > 1:
        pcodes = []
        for pi, ps in enumerate(pass_sets):
            pcode, pm = gen_grad_class_pass(la, lb, lc, ld, ps)
            pcodes += [pcode, ""]
            mg["pass_" + "".join(ps)] = pm
        at = parts.index("template <>")  # the pass functions go before the ClassCode specialisation
        parts[at:at] = pcodes
        parts.append("  template <typename R, int PASS>")
        parts.append(f"  static __device__ __forceinline__ void grad_pass({GRAD_SIG}) {{")
        for pi, ps in enumerate(pass_sets):
            parts.append(f"    if constexpr (PASS == {pi}) grad_{t}_{''.join(ps)}<R>({GRAD_ARGS});")
        parts.append("  }")
    parts.append("};")
    return "\n".join(parts) + "\n", m, mg


INST_TEMPLATE = """// GENERATED by gen_eri.py -- do not edit.
#include <algorithm>

#include "../hfgpu_kernels.cuh"
#include "class_{t}.cuh"
#include "../hfgpu_launch.h"

namespace hfgpu {{
// Large classes: one warp per quartet when the class has too few quartets to keep
// the GPU busy with one (spilling, latency-bound) thread per quartet; one thread
// per quartet otherwise.
template <typename CC, typename R>
static void launch_quartet_impl(const QuartetArgs<R>& a, const int2* q, int nq, cudaStream_t s) {{
  if constexpr (CC::kStaged) {{
    if (a.staged) {{
      // persistent: about as many blocks as the GPU holds at once (each stages the Boys table once)
      auto k = quartet_staged_kernel<{la}, {lb}, {lc}, {ld}, R>;
      const int bs = a.block > 0 ? a.block : 64;
      const int smem = boys_plane_bytes<R>();
      int dev = 0, sms = 148, per_sm = 1;
      cudaGetDevice(&dev);
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, bs, smem);
      const int grid = std::min((nq + bs - 1) / bs, std::max(per_sm, 1) * sms);
      k<<<grid, bs, smem, s>>>(a, q, nq);
      return;
    }}
  }}
  bool warp = false;
  if constexpr (CC::kWarp) warp = nq <= a.warp_max;
  if (!warp && a.capped == 3) {{
    // low residency: the launch reserves (unused) shared memory so that at most two blocks share
    // an SM; the spilled stacks of the large-register classes then stay inside L2
    const int bs = a.block > 0 ? a.block : 64;
    const int pad = 100 * 1024;
    auto k = quartet_kernel<{la}, {lb}, {lc}, {ld}, R>;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, pad);
    k<<<(nq + bs - 1) / bs, bs, pad, s>>>(a, q, nq);
    return;
  }}
  if (!warp) {{
    const int bs = a.block > 0 ? a.block : 64;
    if constexpr (CC::kCapBlocks > 0) {{
      if (a.capped) {{
        quartet_kernel<{la}, {lb}, {lc}, {ld}, R, CC::kCapBlocks><<<(nq + bs - 1) / bs, bs, 0, s>>>(a, q, nq);
        return;
      }}
    }}
    quartet_kernel<{la}, {lb}, {lc}, {ld}, R><<<(nq + bs - 1) / bs, bs, 0, s>>>(a, q, nq);
    return;
  }}
  if constexpr (CC::kWarp) {{
    using Tab = typename CC::WarpTab;
    constexpr int per = warp_slots<Tab, R>();
    if (a.warp_threads == 128) {{
      // one block of four warps per quartet
      const int bytes = per * (int)sizeof(R);
      auto k = quartet_warp_kernel<{la}, {lb}, {lc}, {ld}, R, Tab, 128>;
      cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
      k<<<nq, 128, bytes, s>>>(a, q, nq);
    }} else {{
      const int bytes = 4 * per * (int)sizeof(R);
      auto k = quartet_warp_kernel<{la}, {lb}, {lc}, {ld}, R, Tab>;
      cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
      k<<<(nq + 3) / 4, 128, bytes, s>>>(a, q, nq);
    }}
  }}
}}
template <typename R>
static void launch_quartet(const QuartetArgs<R>& a, const int2* q, int nq, cudaStream_t s) {{
  if (nq <= 0) return;
  launch_quartet_impl<ClassCode<{la}, {lb}, {lc}, {ld}>, R>(a, q, nq, s);
}}
template <typename CC, typename R>
static bool launch_primwarp_impl(const QuartetArgs<R>& a, const int2* q, int nq, cudaStream_t s) {{
  if constexpr (CC::kPrimWarp) {{
    // a.group lanes per quartet, 128-thread blocks
    switch (a.group) {{
      case 4: quartet_primwarp_kernel<{la}, {lb}, {lc}, {ld}, R, 4><<<(nq + 31) / 32, 128, 0, s>>>(a, q, nq); break;
      case 8: quartet_primwarp_kernel<{la}, {lb}, {lc}, {ld}, R, 8><<<(nq + 15) / 16, 128, 0, s>>>(a, q, nq); break;
      case 16: quartet_primwarp_kernel<{la}, {lb}, {lc}, {ld}, R, 16><<<(nq + 7) / 8, 128, 0, s>>>(a, q, nq); break;
      default: quartet_primwarp_kernel<{la}, {lb}, {lc}, {ld}, R, 32><<<(nq + 3) / 4, 128, 0, s>>>(a, q, nq); break;
    }}
    return true;
  }} else {{
    return false;
  }}
}}
template <typename R>
static bool launch_primwarp(const QuartetArgs<R>& a, const int2* q, int nq, cudaStream_t s) {{
  if (nq <= 0) return true;
  return launch_primwarp_impl<ClassCode<{la}, {lb}, {lc}, {ld}>, R>(a, q, nq, s);
}}
template <typename R>
static void launch_grad(const GradArgs<R>& a, int pure, const int2* q, int nq, int grid, cudaStream_t s) {{
  if (nq <= 0) return;
  const size_t sm = sizeof(double) * 3 * a.smem_atoms;
  if constexpr (ClassCode<{la}, {lb}, {lc}, {ld}>::kGradPasses == 4) {{
    // one launch per accumulator set, one after the other on the stream; each adds its part
    grad_kernel<{la}, {lb}, {lc}, {ld}, R, 0><<<grid, 128, sm, s>>>(a, pure, q, nq);
    grad_kernel<{la}, {lb}, {lc}, {ld}, R, 1><<<grid, 128, sm, s>>>(a, pure, q, nq);
    grad_kernel<{la}, {lb}, {lc}, {ld}, R, 2><<<grid, 128, sm, s>>>(a, pure, q, nq);
    grad_kernel<{la}, {lb}, {lc}, {ld}, R, 3><<<grid, 128, sm, s>>>(a, pure, q, nq);
  }} else if constexpr (ClassCode<{la}, {lb}, {lc}, {ld}>::kGradPasses == 2) {{
    // one launch per pair of accumulator sets (U with A, B with C)
    grad_kernel<{la}, {lb}, {lc}, {ld}, R, 0><<<grid, 128, sm, s>>>(a, pure, q, nq);
    grad_kernel<{la}, {lb}, {lc}, {ld}, R, 1><<<grid, 128, sm, s>>>(a, pure, q, nq);
  }} else {{
    grad_kernel<{la}, {lb}, {lc}, {ld}, R><<<grid, 128, sm, s>>>(a, pure, q, nq);
  }}
}}
template <typename Tab, typename R, int NT>
static bool launch_grad_warp_nt(const GradArgs<R>& a, int pure, const int2* q, int nq, cudaStream_t s) {{
  constexpr size_t bytes = sizeof(R) * (size_t)grad_warp_slots<Tab, R>();
  if (bytes > 232448) return false;  // more shared memory than one block may have
  auto k = grad_warp_kernel<{la}, {lb}, {lc}, {ld}, R, Tab, NT>;
  cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  k<<<nq, NT, bytes, s>>>(a, pure, q, nq);
  return true;
}}
template <typename Tab, typename R>
static bool launch_grad_warp_tab(const GradArgs<R>& a, int pure, const int2* q, int nq, cudaStream_t s) {{
  // one warp per quartet, or one block of four or eight warps per quartet
  if (a.warp_threads == 256) return launch_grad_warp_nt<Tab, R, 256>(a, pure, q, nq, s);
  if (a.warp_threads == 128) return launch_grad_warp_nt<Tab, R, 128>(a, pure, q, nq, s);
  return launch_grad_warp_nt<Tab, R, 32>(a, pure, q, nq, s);
}}
template <typename CC, typename R>
static bool launch_grad_warp_impl(const GradArgs<R>& a, int pure, const int2* q, int nq, cudaStream_t s) {{
  if constexpr (CC::kGradWarp) {{
    if (a.warp_split) {{
      // one launch per accumulator set (smaller tables: more warps per SM); each adds its part
      return launch_grad_warp_tab<typename CC::GradWarpTabP0, R>(a, pure, q, nq, s) &&
             launch_grad_warp_tab<typename CC::GradWarpTabP1, R>(a, pure, q, nq, s) &&
             launch_grad_warp_tab<typename CC::GradWarpTabP2, R>(a, pure, q, nq, s) &&
             launch_grad_warp_tab<typename CC::GradWarpTabP3, R>(a, pure, q, nq, s);
    }}
    return launch_grad_warp_tab<typename CC::GradWarpTab, R>(a, pure, q, nq, s);
  }} else {{
    return false;
  }}
}}
template <typename CC, typename R>
static int grad_warp_bytes_impl() {{
  if constexpr (CC::kGradWarp) {{
    return (int)(sizeof(R) * (size_t)grad_warp_slots<typename CC::GradWarpTab, R>());
  }} else {{
    return 0;
  }}
}}
static int grad_warp_bytes(int fp32) {{
  return fp32 ? grad_warp_bytes_impl<ClassCode<{la}, {lb}, {lc}, {ld}>, float>()
              : grad_warp_bytes_impl<ClassCode<{la}, {lb}, {lc}, {ld}>, double>();
}}
template <typename R>
static bool launch_grad_warp(const GradArgs<R>& a, int pure, const int2* q, int nq, cudaStream_t s) {{
  if (nq <= 0) return true;
  return launch_grad_warp_impl<ClassCode<{la}, {lb}, {lc}, {ld}>, R>(a, pure, q, nq, s);
}}
template <typename CC, int NCART>
static int grad_scratch_slots_impl() {{
  if constexpr (CC::kGradTable) {{
    using Tab = typename CC::GradTab;
    return Tab::NVSLOT + Tab::NHSLOT + 3 * NCART;
  }} else {{
    return 0;
  }}
}}
static int grad_scratch_slots(int) {{
  return grad_scratch_slots_impl<ClassCode<{la}, {lb}, {lc}, {ld}>, BlockDims<{la}, {lb}, {lc}, {ld}, false>::NCART>();
}}
extern const ClassLaunchers launchers_{t};
const ClassLaunchers launchers_{t} = {{{la}, {lb}, {lc}, {ld}, &launch_quartet<double>, &launch_quartet<float>,
                                      &launch_grad<double>, &launch_grad<float>, &grad_scratch_slots,
                                      ClassCode<{la}, {lb}, {lc}, {ld}>::kPrimWarp,
                                      &launch_primwarp<double>, &launch_primwarp<float>,
                                      ClassCode<{la}, {lb}, {lc}, {ld}>::kWarp,
                                      ClassCode<{la}, {lb}, {lc}, {ld}>::kWarpDefault,
                                      ClassCode<{la}, {lb}, {lc}, {ld}>::kGradWarp,
                                      &launch_grad_warp<double>, &launch_grad_warp<float>, &grad_warp_bytes,
                                      ClassCode<{la}, {lb}, {lc}, {ld}>::kCapBlocks > 0,
                                      ClassCode<{la}, {lb}, {lc}, {ld}>::kStaged,
                                      ClassCode<{la}, {lb}, {lc}, {ld}>::kLowRes}};
}}  // namespace hfgpu
"""


HESS_INST_TEMPLATE = """// GENERATED by gen_eri.py -- do not edit.
#include "../hfgpu_hess_kernels.cuh"
{line_include}#include "hess_{t}.cuh"
#include "../hfgpu_hess_launch.h"

namespace hfgpu {{
static void launch_hess(const GradArgs<double>& a, const HessOut& o, int pure, const int2* q, int nq, int grid,
                        int smem, cudaStream_t s) {{
  if (nq <= 0) return;
  auto k = hess_kernel<{la}, {lb}, {lc}, {ld}, HessTable{t}>;
  if (smem > 48 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  k<<<grid, 128, smem, s>>>(a, o, pure, q, nq);
}}
static int hess_scratch_slots(int) {{
  return HessTable{t}::NVSLOT + HessTable{t}::NHSLOT + 45 +
         3 * BlockDims<{la}, {lb}, {lc}, {ld}, false>::NCART;
}}
// block form: the whole table in shared memory when it fits, else the HRR slots in global scratch
constexpr size_t kSmAll = sizeof(double) * hess_block_shared_doubles<HessBlockTab{t}>(false);
constexpr size_t kSmPart = sizeof(double) * hess_block_shared_doubles<HessBlockTab{t}>(true);
constexpr size_t kSmMax = 227 * 1024;
static int hess_block_global_slots() {{ return kSmAll <= kSmMax ? 0 : HessBlockTab{t}::NHSLOT + 1; }}
static bool launch_hess_block(const GradArgs<double>& a, const HessOut& o, int pure, const int2* q, int nq, int grid,
                              cudaStream_t s) {{
  if (nq <= 0) return true;
  if constexpr (kSmAll <= kSmMax) {{
    auto k = hess_block_kernel<{la}, {lb}, {lc}, {ld}, HessBlockTab{t}, false>;
    if (kSmAll > 48 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmAll);
    k<<<grid, 128, kSmAll, s>>>(a, o, pure, q, nq);
    return true;
  }} else if constexpr (kSmPart <= kSmMax) {{
    auto k = hess_block_kernel<{la}, {lb}, {lc}, {ld}, HessBlockTab{t}, true>;
    if (kSmPart > 48 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmPart);
    k<<<grid, 128, kSmPart, s>>>(a, o, pure, q, nq);
    return true;
  }} else {{
    return false;
  }}
}}
// warp form: four quartets per 128-thread block, one warp each, every warp's tables in shared memory
static bool launch_hess_warp(const GradArgs<double>& a, const HessOut& o, int pure, const int2* q, int nq,
                             cudaStream_t s) {{
  if (nq <= 0) return true;
  if constexpr (4 * kSmAll <= kSmMax) {{
    auto k = hess_block_kernel<{la}, {lb}, {lc}, {ld}, HessBlockTab{t}, false, 32>;
    if (4 * kSmAll > 48 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(4 * kSmAll));
    k<<<(nq + 3) / 4, 128, 4 * kSmAll, s>>>(a, o, pure, q, nq);
    return true;
  }} else {{
    return false;
  }}
}}
{line_fn}
extern const HessLaunchers hess_launchers_{t};
const HessLaunchers hess_launchers_{t} = {{{la}, {lb}, {lc}, {ld}, &launch_hess, &hess_scratch_slots,
                                          &launch_hess_block, &hess_block_global_slots, &launch_hess_warp,
                                          {has_line}, &launch_hess_line}};
}}  // namespace hfgpu
"""

# straight-line form (gen_hess_line): one thread per quartet, grid-stride over grid blocks
HESS_LINE_LAUNCH = """// straight-line form: one thread per quartet on register code, grid blocks of 128 threads
static bool launch_hess_line(const GradArgs<double>& a, const HessOut& o, int pure, const int2* q, int nq, int grid,
                             int smem, cudaStream_t s) {{
  if (nq <= 0) return true;
  auto k = hess_line_kernel<{la}, {lb}, {lc}, {ld}, HessLine{t}>;
  const int bytes = smem + kHessLineH45Bytes;  // the block's Hessian (smem > 0) and the h45 slices
  if (bytes > 48 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  k<<<grid, kHessLineThreads, bytes, s>>>(a, o, pure, q, nq);
  return true;
}}"""
HESS_LINE_NONE = """// no straight-line form: the class's passes would spill or be too many (gen_hess_line)
static bool launch_hess_line(const GradArgs<double>&, const HessOut&, int, const int2*, int, int, int, cudaStream_t) {
  return false;
}"""


def main(outdir):
    import os
    os.makedirs(outdir, exist_ok=True)
    pairs, cls = classes()
    meta = {"pair_classes": pairs, "eri": [], "grad": []}

    def write_if_changed(path, text):
        if os.path.exists(path) and open(path).read() == text:
            return
        with open(path, "w") as f:
            f.write(text)

    write_if_changed(os.path.join(outdir, "common.cuh"), common_header())
    names = []
    for c in cls:
        t = "".join(map(str, c))
        text, m, mg = class_header(c)
        meta["eri"].append(m)
        meta["grad"].append(mg)
        write_if_changed(os.path.join(outdir, f"class_{t}.cuh"), text)
        la, lb, lc, ld = c
        write_if_changed(os.path.join(outdir, f"inst_{t}.cu"), INST_TEMPLATE.format(t=t, la=la, lb=lb, lc=lc, ld=ld))
        names.append(t)
    # the adjoint Hessian: one table header and one launcher unit per class
    hnames = []
    meta["hess"] = []
    for c in cls:
        t = "".join(map(str, c))
        code_h, mh = gen_hess_table(*c)
        meta["hess"].append(mh)
        code_b, mb = gen_hess_block(*c)
        mh["block"] = mb
        code_l, ml = gen_hess_line(*c)
        mh["line"] = ml
        write_if_changed(os.path.join(outdir, f"hess_{t}.cuh"),
                         "// GENERATED by gen_eri.py -- do not edit.\n#pragma once\n#include \"common.cuh\"\n\n" +
                         code_h + "\n\n" + code_b + "\n" + ("\n" + code_l + "\n" if code_l else ""))
        la, lb, lc, ld = c
        line = code_l is not None
        write_if_changed(os.path.join(outdir, f"hess_{t}.cu"), HESS_INST_TEMPLATE.format(
            t=t, la=la, lb=lb, lc=lc, ld=ld,
            line_include=f'#include "class_{t}.cuh"  // ClassCode::from_pure of the straight-line form\n' if line else "",
            line_fn=(HESS_LINE_LAUNCH.format(t=t, la=la, lb=lb, lc=lc, ld=ld) if line else HESS_LINE_NONE),
            has_line="true" if line else "false"))
        hnames.append(t)
    hd = ["// GENERATED by gen_eri.py -- do not edit.", '#include "../hfgpu_hess_launch.h"', "namespace hfgpu {"]
    hd += [f"extern const HessLaunchers hess_launchers_{t};" for t in hnames]
    hd.append(f"const HessLaunchers* const kHessLaunchers[{len(hnames)}] = {{")
    hd += [f"  &hess_launchers_{t}," for t in hnames]
    hd.append("};")
    hd.append(f"const int kNumHessClasses = {len(hnames)};")
    hd.append("}  // namespace hfgpu")
    write_if_changed(os.path.join(outdir, "hess_dispatch.cu"), "\n".join(hd) + "\n")
    disp = ["// GENERATED by gen_eri.py -- do not edit.", '#include "../hfgpu_launch.h"', "namespace hfgpu {"]
    for t in names:
        disp.append(f"extern const ClassLaunchers launchers_{t};")
    disp.append(f"const ClassLaunchers* const kClassLaunchers[{len(names)}] = {{")
    disp += [f"  &launchers_{t}," for t in names]
    disp.append("};")
    disp.append(f"const int kNumClasses = {len(names)};")
    disp.append("}  // namespace hfgpu")
    write_if_changed(os.path.join(outdir, "dispatch.cu"), "\n".join(disp) + "\n")
    write_if_changed(os.path.join(outdir, "ops.json"), json.dumps(meta, indent=1))
    for m in meta["eri"]:
        print("eri ", m["class"], "vrr", m["vrr_values"], "acc", m["vrr_targets"], "prim_fl", m["prim_flops"],
              "hrr_fl", m["hrr_flops"], "pure_fl", m["pure_flops"])
    for m in meta["grad"]:
        print("grad", m["class"], "table" if m.get("table") else "straight", "prim_fl", m["prim_flops"],
              "hrr_fl", m["hrr_flops"])




# ---------------------------------------------------------------------------
# Table mode: the large gradient classes run as op lists through a generic
# executor (hfgpu_table.cuh) on thread-interleaved scratch, because their
# straight-line form does not fit the register file and takes ptxas far too long.
# ---------------------------------------------------------------------------
class Dag:
    """VRR as a DAG of ops: node = (kind, dir, a, b, c, d, g, k1, k2)."""

    def __init__(self, L):
        self.nodes = []   # list of tuples
        self.memo = {}
        self.L = L
        for m in range(L + 1):
            self.memo[((0, 0, 0), (0, 0, 0), m)] = len(self.nodes)
            self.nodes.append(("F", m))

    def get(self, e, f, m):
        key = (e, f, m)
        if key in self.memo:
            return self.memo[key]
        Z = -1
        if sum(f) > 0:
            i = max(range(3), key=lambda d: (f[d], -d))
            f1 = add(f, i, -1)
            a = self.get(e, f1, m)
            b = self.get(e, f1, m + 1)
            c = d = Z
            k1 = k2 = 0
            g = Z
            if f1[i] > 0:
                f2 = add(f1, i, -1)
                c = self.get(e, f2, m)
                d = self.get(e, f2, m + 1)
                k1 = f1[i]
            if e[i] > 0:
                g = self.get(add(e, i, -1), f1, m + 1)
                k2 = e[i]
            node = ("K", i, a, b, c, d, g, k1, k2)
        else:
            i = max(range(3), key=lambda d: (e[d], -d))
            e1 = add(e, i, -1)
            a = self.get(e1, f, m)
            b = self.get(e1, f, m + 1)
            c = d = Z
            k1 = 0
            if e1[i] > 0:
                e2 = add(e1, i, -1)
                c = self.get(e2, f, m)
                d = self.get(e2, f, m + 1)
                k1 = e1[i]
            node = ("B", i, a, b, c, d, Z, k1, 0)
        self.memo[key] = len(self.nodes)
        self.nodes.append(node)
        return self.memo[key]


def linear_scan(n_values, uses_per_op, defs_per_op, preassigned):
    """Slot allocation.  uses_per_op[i] / defs_per_op[i]: value ids used / defined by op i.
    preassigned: value id -> slot for values that exist before op 0.  Slot 0 stays zero."""
    last = {}
    for i, us in enumerate(uses_per_op):
        for u in us:
            last[u] = i
    slot = dict(preassigned)
    free = []
    top = max(list(preassigned.values()) + [0]) + 1
    for v, s in preassigned.items():
        if v not in last:
            free.append(s)
    for i in range(len(uses_per_op)):
        for v in defs_per_op[i]:
            if free:
                slot[v] = free.pop()
            else:
                slot[v] = top
                top += 1
        for u in set(uses_per_op[i]):
            if last.get(u) == i:
                free.append(slot[u])
        for v in defs_per_op[i]:
            if v not in last:  # dead store (should not happen)
                free.append(slot[v])
    return slot, top


def _u16(x):
    assert 0 <= x < 65536, x
    return x


def _i32(u):
    """A 32-bit pattern as a C int literal."""
    u &= 0xFFFFFFFF
    return u - (1 << 32) if u >= (1 << 31) else u


def pack_grad_vrr(r):
    kind, i, dst, sa, sb, sc, sd, sg, k1, k2 = r
    assert 0 <= kind < 16 and 0 <= i < 16 and 0 <= k1 < 256 and 0 <= k2 < 256
    return (_i32(_u16(dst) | _u16(sa) << 16), _i32(_u16(sb) | _u16(sc) << 16), _i32(_u16(sd) | _u16(sg) << 16),
            _i32(kind | i << 4 | k1 << 8 | k2 << 16))


def pack_grad_hrr(r):
    kind, i, dst, x, y, kk = r[:6]
    assert 0 <= kind < 16 and 0 <= i < 16 and 0 <= kk < 128 and y < 65536
    return (_i32(_u16(dst) | _u16(x) << 16), _i32(_u16(y) | kind << 16 | i << 20 | kk << 24))


def pack_warp_vrr(r):
    kd, dst, sa, sb, sc, sd, sg, k12 = r
    assert 0 <= kd < 256 and 0 <= k12 < (1 << 16)
    return (_i32(_u16(dst) | _u16(sa) << 16), _i32(_u16(sb) | _u16(sc) << 16), _i32(_u16(sd) | _u16(sg) << 16),
            _i32(kd | k12 << 8))


def pack_warp_hrr(r):
    kd, dst, x, y = r
    assert 0 <= kd < (1 << 15)
    return (_i32(_u16(dst) | _u16(x) << 16), _i32(_u16(y) | kd << 16))


def gen_grad_table(la, lb, lc, ld):
    L = la + lb + lc + ld + 1
    order = grad_sets(la, lb, lc, ld)
    dag = Dag(L)
    setoff = {}
    nacc = 0
    for k in ("U", "A", "B", "C"):
        setoff[k] = nacc
        nacc += len(order[k])
    tgt_nodes = {}
    for k in ("U", "A", "B", "C"):
        for j, (e, f) in enumerate(order[k]):
            n = dag.get(e, f, 0)
            tgt_nodes.setdefault(n, []).append((k, setoff[k] + j))
    # ---- VRR op list: (kind, dir, dst, a, b, c, d, g, k1, k2) in value ids; acc ops after targets
    ops, uses, defs = [], [], []
    for nid, node in enumerate(dag.nodes):
        if node[0] == "F":
            continue
        kind, i, a, b, c, d, g, k1, k2 = node
        ops.append(["K" if kind == "K" else "B", i, nid, a, b, c, d, g, k1, k2])
        uses.append([x for x in (a, b, c, d, g) if x >= 0])
        defs.append([nid])
        for (k, ai) in tgt_nodes.get(nid, []):
            ops.append(["A", "UABC".index(k), ai, nid, -1, -1, -1, -1, 0, 0])
            uses.append([nid])
            defs.append([])
    # F[m] seeds that are targets themselves (only for the all-s class)
    pre_ops = []
    for nid, node in enumerate(dag.nodes):
        if node[0] == "F" and nid in tgt_nodes:
            for (k, ai) in tgt_nodes[nid]:
                pre_ops.append(["A", "UABC".index(k), ai, nid, -1, -1, -1, -1, 0, 0])
    ops = pre_ops + ops
    uses = [[o[3]] for o in pre_ops] + uses
    defs = [[] for _ in pre_ops] + defs
    pre = {m: 1 + m for m in range(L + 1)}  # F[m] lives in slot 1+m
    slot, nvslot = linear_scan(len(dag.nodes), uses, defs, pre)
    kinds = {"B": 0, "K": 1, "A": 2}
    vrr_rows = []
    for o in ops:
        k, i, dst, a, b, c, d, g, k1, k2 = o
        if k == "A":
            vrr_rows.append((2, i, dst, slot[a], 0, 0, 0, 0, 0, 0))
        else:
            sl = lambda x: slot[x] if x >= 0 else 0
            vrr_rows.append((kinds[k], i, slot[dst], sl(a), sl(b), sl(c), sl(d), sl(g), k1, k2))
    # ---- HRR + contraction list on the second region: slot 0 zero, acc j at slot 1+j
    hnodes = {}
    hops, huses, hdefs = [], [], []
    counter = [nacc + 1]

    def acc_id(k, e, f):
        return 1 + setoff[k] + order[k].index((e, f))

    def new_id():
        counter[0] += 1
        return counter[0] - 1

    def ket(k, e, c, d):
        key = ("k", k, e, c, d)
        if key in hnodes:
            return hnodes[key]
        if sum(d) == 0:
            v = acc_id(k, e, c)
        else:
            i = max(range(3), key=lambda q: (d[q], -q))
            d1 = add(d, i, -1)
            x = ket(k, e, add(c, i), d1)
            y = ket(k, e, c, d1)
            v = new_id()
            hops.append((1, i, v, x, y, 0, 0))
            huses.append([x, y])
            hdefs.append([v])
        hnodes[key] = v
        return v

    def bra(k, a, b, c, d):
        key = ("b", k, a, b, c, d)
        if key in hnodes:
            return hnodes[key]
        if sum(b) == 0:
            v = ket(k, a, c, d)
        else:
            i = max(range(3), key=lambda q: (b[q], -q))
            b1 = add(b, i, -1)
            x = bra(k, add(a, i), b1, c, d)
            y = bra(k, a, b1, c, d)
            v = new_id()
            hops.append((0, i, v, x, y, 0, 0))
            huses.append([x, y])
            hdefs.append([v])
        hnodes[key] = v
        return v

    gt = grad_terms(la, lb, lc, ld)
    for (cen, dr), items in gt.items():
        gi = "ABC".index(cen) * 3 + dr
        for wi, terms in items:
            x = bra(terms[0][1], *terms[0][2:])
            if len(terms) > 1:
                y = bra("U", *terms[1][2:])
                kk = -terms[1][0]
            else:
                y, kk = -1, 0
            hops.append((2, gi, wi, x, y, kk, 0))
            huses.append([x] + ([y] if y >= 0 else []))
            hdefs.append([])
    hpre = {1 + j: 1 + j for j in range(nacc)}
    hslot, nhslot = linear_scan(counter[0], huses, hdefs, hpre)
    hrows = []
    for o in hops:
        kind, i, dst, x, y, kk, _ = o
        if kind == 2:
            hrows.append((2, i, dst, hslot[x], hslot[y] if y >= 0 else 0, kk, 0, 0))
        else:
            hrows.append((kind, i, hslot[dst], hslot[x], hslot[y], 0, 0, 0))
    tagc = f"{la}{lb}{lc}{ld}"
    s = [f"// table-mode adjoint gradient of class {tagc}: {len(vrr_rows)} VRR ops over {nvslot} slots, "
         f"{nacc} accumulators, {len(hrows)} HRR/contraction ops over {nhslot} slots"]
    # one 16-byte row per VRR op and one 8-byte row per HRR op (a single vector load each):
    # VRR {dst | sa<<16, sb | sc<<16, sd | sg<<16, kind | dir<<4 | k1<<8 | k2<<16}
    # HRR {dst | x<<16, y | kind<<16 | dir<<20 | k<<24}
    s.append(f"__device__ const int4 gvrr_{tagc}[{len(vrr_rows)}] = {{")
    s += ["  {" + ",".join(map(str, pack_grad_vrr(r))) + "}," for r in vrr_rows]
    s.append("};")
    s.append(f"__device__ const int2 ghrr_{tagc}[{len(hrows)}] = {{")
    s += ["  {" + ",".join(map(str, pack_grad_hrr(r))) + "}," for r in hrows]
    s.append("};")
    s.append(f"struct GradTable{tagc} {{ static constexpr int L = {L}, NVOPS = {len(vrr_rows)}, NVSLOT = {nvslot}, "
             f"NACC = {nacc}, NHOPS = {len(hrows)}, NHSLOT = {nhslot}; "
             f"static __device__ const int4* vrr() {{ return gvrr_{tagc}; }} "
             f"static __device__ const int2* hrr() {{ return ghrr_{tagc}; }} }};")
    flops = sum(3 + (3 if r[8] else 0) + (2 if r[9] else 0) for r in vrr_rows if r[0] < 2) + \
        2 * sum(1 for r in vrr_rows if r[0] == 2)
    hfl = sum(2 if r[0] < 2 else 4 for r in hrows)
    meta = {"class": [la, lb, lc, ld], "table": True, "vrr_ops": len(vrr_rows), "vrr_slots": nvslot,
            "accumulators": nacc, "hrr_ops": len(hrows), "hrr_slots": nhslot,
            "prim_flops": flops + PRIM_HEADER_FLOPS, "hrr_flops": hfl, "boys_m": L}
    return "\n".join(s), meta




# ---------------------------------------------------------------------------
# Warp mode: the large energy classes run one warp per quartet.  The VRR and
# HRR are levelised (an op's inputs come from earlier levels only), so the 32
# lanes execute one level's ops in parallel out of shared memory, with a
# __syncwarp between levels.  Slots are reused once their last reader's level
# has completed.
# ---------------------------------------------------------------------------
def _levelise(nodes_deps, n_pre):
    """nodes_deps: list of (node id, [dep ids]) in topological order; ids < n_pre are inputs (level 0)."""
    lev = {i: 0 for i in range(n_pre)}
    for nid, deps in nodes_deps:
        lev[nid] = 1 + max([lev[d] for d in deps] + [0])
    return lev


def _alloc_levels(order_by_level, deps_of, lev, pre_slots, live_to_end):
    """Slot allocation with level granularity.  Returns (slot map, number of slots)."""
    last = {}
    for nid in order_by_level:
        for d in deps_of[nid]:
            last[d] = max(last.get(d, -1), lev[nid])
    END = 10 ** 9
    for v in live_to_end:
        last[v] = END
    slot = dict(pre_slots)
    top = max(list(pre_slots.values()) + [-1]) + 1
    free = []
    # inputs never read are free from the start
    for v, s in pre_slots.items():
        if v not in last:
            free.append(s)
    maxlev = max([lev[n] for n in order_by_level] + [0])
    by_level = {}
    for nid in order_by_level:
        by_level.setdefault(lev[nid], []).append(nid)
    freed_at = {}
    for v, l in last.items():
        if l != END:
            freed_at.setdefault(l, []).append(v)
    for v in pre_slots:
        if v in last and last[v] == 0:
            pass
    for l in range(1, maxlev + 1):
        for nid in by_level.get(l, []):
            if free:
                slot[nid] = free.pop()
            else:
                slot[nid] = top
                top += 1
        for v in freed_at.get(l, []):
            if v in slot:
                free.append(slot[v])
    return slot, top


def _alloc_levels_with_readers(order_by_level, deps_of, lev, pre_slots, live_to_end, readers):
    """_alloc_levels where `readers` (level, [dep ids]) read values but produce none."""
    last = {}
    for nid in order_by_level:
        for d in deps_of[nid]:
            last[d] = max(last.get(d, -1), lev[nid])
    for l, deps in readers:
        for d in deps:
            last[d] = max(last.get(d, -1), l)
    END = 10 ** 9
    for v in live_to_end:
        last[v] = END
    slot = dict(pre_slots)
    top = max(list(pre_slots.values()) + [-1]) + 1
    free = [s for v, s in pre_slots.items() if v not in last]
    maxlev = max([lev[n] for n in order_by_level] + [l for l, _ in readers] + [0])
    by_level = {}
    for nid in order_by_level:
        by_level.setdefault(lev[nid], []).append(nid)
    freed_at = {}
    for v, l in last.items():
        if l != END:
            freed_at.setdefault(l, []).append(v)
    for l in range(1, maxlev + 1):
        for nid in by_level.get(l, []):
            if free:
                slot[nid] = free.pop()
            else:
                slot[nid] = top
                top += 1
        for v in freed_at.get(l, []):
            if v in slot:
                free.append(slot[v])
    return slot, top


def gen_grad_warp(la, lb, lc, ld, sets=("U", "A", "B", "C"), suffix=""):
    """Adjoint gradient of one quartet by one warp: the VRR one order higher and the HRR of
    the weighted sets are levelised (an op's inputs come from earlier levels), so the
    32 lanes run one level's ops in parallel out of shared memory; the contractions with
    the weight block W are ops of the HRR levels that only read.  `sets` restricts the table to
    some of the four accumulator sets (one pass of the per-set split: the terms that read those
    sets only, so the four one-set tables add up to the whole gradient)."""
    L = la + lb + lc + ld + 1
    order = grad_sets(la, lb, lc, ld)
    dag = Dag(L)
    setoff, nacc = {}, 0
    for k in sets:
        setoff[k] = nacc
        nacc += len(order[k])
    acc_src, acc_set = [], []
    for k in sets:
        for (e, f) in order[k]:
            acc_src.append(dag.get(e, f, 0))
            acc_set.append(("U", "A", "B", "C").index(k))
    ops = [(nid, nd) for nid, nd in enumerate(dag.nodes) if nd[0] != "F"]
    deps = {nid: [x for x in nd[2:7] if x >= 0] for nid, nd in ops}
    lev = _levelise([(nid, deps[nid]) for nid, _ in ops], L + 1)
    vorder = sorted([nid for nid, _ in ops], key=lambda n: (lev[n], n))
    pre = {m: m for m in range(L + 1)}
    slot, nvs = _alloc_levels(vorder, deps, lev, pre, set(acc_src))
    ZV = nvs
    nodes = dict(ops)
    vrows, vlev, cur = [], [0], 1
    for nid in vorder:
        while lev[nid] > cur:
            vlev.append(len(vrows))
            cur += 1
        kind, i, a, b, c, d, g, k1, k2 = nodes[nid]
        s_ = lambda x: slot[x] if x >= 0 else ZV
        vrows.append(((1 if kind == "K" else 0) | (i << 2), slot[nid], s_(a), s_(b), s_(c), s_(d), s_(g),
                      k1 | (k2 << 8)))
    vlev.append(len(vrows))
    # HRR of the four sets (accumulator j is value j) and the contractions
    hnodes, hinfo, hdeps = {}, {}, {}
    counter = [nacc]

    def new_id():
        counter[0] += 1
        return counter[0] - 1

    def ket(k, e, c, d):
        key = ("k", k, e, c, d)
        if key in hnodes:
            return hnodes[key]
        if sum(d) == 0:
            v = setoff[k] + order[k].index((e, c))
        else:
            i = max(range(3), key=lambda q: (d[q], -q))
            d1 = add(d, i, -1)
            x, y = ket(k, e, add(c, i), d1), ket(k, e, c, d1)
            v = new_id()
            hinfo[v], hdeps[v] = (1, i, x, y), [x, y]
        hnodes[key] = v
        return v

    def bra(k, a, b, c, d):
        key = ("b", k, a, b, c, d)
        if key in hnodes:
            return hnodes[key]
        if sum(b) == 0:
            v = ket(k, a, c, d)
        else:
            i = max(range(3), key=lambda q: (b[q], -q))
            b1 = add(b, i, -1)
            x, y = bra(k, add(a, i), b1, c, d), bra(k, a, b1, c, d)
            v = new_id()
            hinfo[v], hdeps[v] = (0, i, x, y), [x, y]
        hnodes[key] = v
        return v

    cops = []
    for (cen, dr), items in grad_terms(la, lb, lc, ld).items():
        gi = "ABC".index(cen) * 3 + dr
        for wi, terms in items:
            x = bra(terms[0][1], *terms[0][2:]) if terms[0][1] in sets else -1
            if len(terms) > 1 and "U" in sets:
                y, kk = bra("U", *terms[1][2:]), -terms[1][0]
            else:
                y, kk = -1, 0
            if x < 0 and y < 0:
                continue
            cops.append((gi, wi, x, y, kk))
    hord = sorted(hinfo)
    hlev = _levelise([(v, hdeps[v]) for v in hord], nacc)
    clev = [1 + max(hlev[x] if x >= 0 else 0, hlev[y] if y >= 0 else 0) for (_, _, x, y, _) in cops]
    readers = [(l, ([x] if x >= 0 else []) + ([y] if y >= 0 else [])) for l, (_, _, x, y, _) in zip(clev, cops)]
    hpre = {j: j for j in range(nacc)}
    hslot, nhs = _alloc_levels_with_readers(sorted(hord, key=lambda v: (hlev[v], v)), hdeps, hlev, hpre, set(),
                                            readers)
    ZH = nhs
    items = [(hlev[v], 0, v) for v in hord] + [(l, 1, j) for j, l in enumerate(clev)]
    items.sort()
    hrows, hlv, cur = [], [0], 1
    for l, is_c, v in items:
        while l > cur:
            hlv.append(len(hrows))
            cur += 1
        if is_c:
            gi, wi, x, y, kk = cops[v]
            hrows.append((2 | (gi << 2) | (kk << 6), wi, hslot[x] if x >= 0 else ZH, hslot[y] if y >= 0 else ZH))
        else:
            kind, i, x, y = hinfo[v]
            hrows.append((kind | (i << 2), hslot[v], hslot[x], hslot[y]))
    hlv.append(len(hrows))
    t = f"{la}{lb}{lc}{ld}{suffix}"
    ncart_blk = ncart(la) * ncart(lb) * ncart(lc) * ncart(ld)
    s = [f"// warp-mode adjoint gradient of class {t}: {len(vrows)} VRR ops in {len(vlev) - 1} levels over "
         f"{nvs} slots, {nacc} accumulators, {len(hrows)} HRR/contraction ops in {len(hlv) - 1} levels over "
         f"{nhs} slots"]
    s.append(f"__device__ const int4 gwv_{t}[{max(len(vrows), 1)}] = {{")
    s += ["  {" + ",".join(map(str, pack_warp_vrr(r))) + "}," for r in vrows]
    s.append("};")
    s.append(f"__device__ const int gwv_lv_{t}[{len(vlev)}] = {{{','.join(map(str, vlev))}}};")
    s.append(f"__device__ const int2 gwa_{t}[{nacc}] = {{" +
             ",".join("{%d,%d}" % (slot[n], k) for n, k in zip(acc_src, acc_set)) + "};")
    s.append(f"__device__ const int2 gwh_{t}[{max(len(hrows), 1)}] = {{")
    s += ["  {" + ",".join(map(str, pack_warp_hrr(r))) + "}," for r in hrows]
    s.append("};")
    s.append(f"__device__ const int gwh_lv_{t}[{len(hlv)}] = {{{','.join(map(str, hlv))}}};")
    s.append(f"struct GradWarpTab{t} {{ static constexpr int L = {L}, NVLEV = {len(vlev) - 1}, NVSLOT = {nvs}, "
             f"NACC = {nacc}, NHLEV = {len(hlv) - 1}, NHSLOT = {nhs}, NCART = {ncart_blk}; "
             f"static __device__ const int4* vrr() {{ return gwv_{t}; }} "
             f"static __device__ const int* vlev() {{ return gwv_lv_{t}; }} "
             f"static __device__ const int2* acc() {{ return gwa_{t}; }} "
             f"static __device__ const int2* hrr() {{ return gwh_{t}; }} "
             f"static __device__ const int* hlev() {{ return gwh_lv_{t}; }} }};")
    meta = {"class": [la, lb, lc, ld], "grad_warp": True, "vrr_ops": len(vrows), "vrr_levels": len(vlev) - 1,
            "vrr_slots": nvs, "acc": nacc, "hrr_ops": len(hrows), "hrr_levels": len(hlv) - 1, "hrr_slots": nhs,
            "smem_doubles_per_warp": nvs + 1 + nhs + 1 + 3 * ncart_blk}
    return "\n".join(s), meta


def gen_warp_class(la, lb, lc, ld):
    L = la + lb + lc + ld
    dag = Dag(L)
    targets = vrr_targets(la, la + lb, lc, lc + ld)
    tnodes = [dag.get(e, f, 0) for e, f in targets]
    ops = [(nid, nd) for nid, nd in enumerate(dag.nodes) if nd[0] != "F"]
    deps = {nid: [x for x in nd[2:7] if x >= 0] for nid, nd in ops}
    lev = _levelise([(nid, deps[nid]) for nid, _ in ops], L + 1)
    order = sorted([nid for nid, _ in ops], key=lambda n: (lev[n], n))
    pre = {m: m for m in range(L + 1)}
    slot, nvs = _alloc_levels(order, deps, lev, pre, set(tnodes))
    ZV = nvs  # zero slot
    nodes = dict(ops)
    vrows, vlev = [], [0]
    cur = 1
    for nid in order:
        while lev[nid] > cur:
            vlev.append(len(vrows))
            cur += 1
        kind, i, a, b, c, d, g, k1, k2 = nodes[nid]
        s_ = lambda x: slot[x] if x >= 0 else ZV
        vrows.append(((1 if kind == "K" else 0) | (i << 2), slot[nid], s_(a), s_(b), s_(c), s_(d), s_(g),
                      k1 | (k2 << 8)))
    vlev.append(len(vrows))
    acc_rows = [slot[n] for n in tnodes]
    nacc = len(targets)
    # HRR DAG on the accumulators
    acc_of = {t: j for j, t in enumerate(targets)}
    hnodes, hdeps, hinfo = {}, {}, {}
    counter = [nacc]

    def ket(e, c, d):
        key = ("k", e, c, d)
        if key in hnodes:
            return hnodes[key]
        if sum(d) == 0:
            v = acc_of[(e, c)]
        else:
            i = max(range(3), key=lambda q: (d[q], -q))
            d1 = add(d, i, -1)
            x = ket(e, add(c, i), d1)
            y = ket(e, c, d1)
            v = counter[0]
            counter[0] += 1
            hdeps[v] = [x, y]
            hinfo[v] = (1, i, x, y)
        hnodes[key] = v
        return v

    def bra(a, b, c, d):
        key = ("b", a, b, c, d)
        if key in hnodes:
            return hnodes[key]
        if sum(b) == 0:
            v = ket(a, c, d)
        else:
            i = max(range(3), key=lambda q: (b[q], -q))
            b1 = add(b, i, -1)
            x = bra(add(a, i), b1, c, d)
            y = bra(a, b1, c, d)
            v = counter[0]
            counter[0] += 1
            hdeps[v] = [x, y]
            hinfo[v] = (0, i, x, y)
        hnodes[key] = v
        return v

    outs = [bra(a, b, c, d) for a in cart(la) for b in cart(lb) for c in cart(lc) for d in cart(ld)]
    hord = sorted(hinfo, key=lambda v: v)
    hlev = _levelise([(v, hdeps[v]) for v in hord], nacc)
    hord = sorted(hord, key=lambda v: (hlev[v], v))
    hpre = {j: j for j in range(nacc)}
    hslot, nhs = _alloc_levels(hord, hdeps, hlev, hpre, set(outs))
    hrows, hlv = [], [0]
    cur = 1
    for v in hord:
        while hlev[v] > cur:
            hlv.append(len(hrows))
            cur += 1
        kind, i, x, y = hinfo[v]
        hrows.append((kind | (i << 2), hslot[v], hslot[x], hslot[y]))
    hlv.append(len(hrows))
    wout = [hslot[o] for o in outs]
    t = f"{la}{lb}{lc}{ld}"
    ncart_blk = len(outs)
    s = [f"// warp-mode J/K of class {t}: {len(vrows)} VRR ops in {len(vlev) - 1} levels over {nvs} slots, "
         f"{nacc} accumulators, {len(hrows)} HRR ops in {len(hlv) - 1} levels over {nhs} slots"]
    # VRR row {dst | sa<<16, sb | sc<<16, sd | sg<<16, kd | k12<<8}; HRR row {dst | x<<16, y | kd<<16}
    s.append(f"__device__ const int4 wvrr_{t}[{max(len(vrows), 1)}] = {{")
    s += ["  {" + ",".join(map(str, pack_warp_vrr(r))) + "}," for r in vrows]
    s.append("};")
    s.append(f"__device__ const int wvrr_lv_{t}[{len(vlev)}] = {{{','.join(map(str, vlev))}}};")
    s.append(f"__device__ const int wacc_{t}[{nacc}] = {{{','.join(map(str, acc_rows))}}};")
    s.append(f"__device__ const int2 whrr_{t}[{max(len(hrows), 1)}] = {{")
    s += ["  {" + ",".join(map(str, pack_warp_hrr(r))) + "}," for r in hrows] or ["  {0,0},"]
    s.append("};")
    s.append(f"__device__ const int whrr_lv_{t}[{len(hlv)}] = {{{','.join(map(str, hlv))}}};")
    s.append(f"__device__ const int wout_{t}[{ncart_blk}] = {{{','.join(map(str, wout))}}};")
    s.append(f"struct WarpTab{t} {{ static constexpr int L = {L}, NVLEV = {len(vlev) - 1}, NVSLOT = {nvs}, "
             f"NACC = {nacc}, NHLEV = {len(hlv) - 1}, NHSLOT = {nhs}, NCART = {ncart_blk}; "
             f"static __device__ const int4* vrr() {{ return wvrr_{t}; }} "
             f"static __device__ const int* vlev() {{ return wvrr_lv_{t}; }} "
             f"static __device__ const int* acc() {{ return wacc_{t}; }} "
             f"static __device__ const int2* hrr() {{ return whrr_{t}; }} "
             f"static __device__ const int* hlev() {{ return whrr_lv_{t}; }} "
             f"static __device__ const int* out() {{ return wout_{t}; }} }};")
    meta = {"class": [la, lb, lc, ld], "vrr_ops": len(vrows), "vrr_levels": len(vlev) - 1, "vrr_slots": nvs,
            "acc": nacc, "hrr_ops": len(hrows), "hrr_levels": len(hlv) - 1, "hrr_slots": nhs,
            "smem_doubles_per_warp": nvs + 1 + nhs + 1 + 2 * ncart_blk}
    return "\n".join(s), meta



# ---------------------------------------------------------------------------
# Adjoint second derivatives (the two-electron part of the Hessian at a fixed density):
# H[X][Y] += sum_abcd W_abcd d2(ab|cd)/dX dY for X, Y in {A, B, C} x {x, y, z}; centre D
# follows from translational invariance on the host side of the kernel.  A derivative by
# centre P in direction i acts on a primitive as 2 alpha_P (p + 1_i) - p_i (p - 1_i); applying
# it twice gives integrals with the angular momentum of up to two centres shifted by one or two,
# weighted by one of ten exponent products (HESS_SETS; the factors 2 alpha are in the weights).
# ---------------------------------------------------------------------------
HESS_SETS = [(), ("A",), ("B",), ("C",), ("A", "A"), ("B", "B"), ("C", "C"), ("A", "B"), ("A", "C"), ("B", "C")]
HESS_COORDS = [(P, i) for P in range(3) for i in range(3)]
HESS_PAIRS = [(r, s) for r in range(9) for s in range(r, 9)]   # 45 outputs, upper triangle


def _d1(P, i, comps):
    """First derivative by centre P (0, 1, 2 = A, B, C) in direction i of the Cartesian
    components comps = (a, b, c, d): [(coefficient, weight centres, shifted components)]."""
    up = list(comps)
    up[P] = add(comps[P], i)
    out = [(1, ("ABC"[P],), tuple(up))]
    v = comps[P][i]
    if v > 0:
        dn = list(comps)
        dn[P] = add(comps[P], i, -1)
        out.append((-v, (), tuple(dn)))
    return out


def hess_terms(la, lb, lc, ld):
    """[(output index, W index, coefficient, set index, a, b, c, d)]: the second derivative
    of (ab|cd) by coordinates r <= s of HESS_PAIRS as integer combinations of shifted
    integrals of the ten weight sets."""
    terms = []
    w = 0
    for a in cart(la):
        for b in cart(lb):
            for c in cart(lc):
                for d in cart(ld):
                    comps = (a, b, c, d)
                    for hi, (r, s) in enumerate(HESS_PAIRS):
                        (P, i), (Q, j) = HESS_COORDS[r], HESS_COORDS[s]
                        acc = {}
                        for c1, w1, comps1 in _d1(Q, j, comps):
                            for c2, w2, comps2 in _d1(P, i, comps1):
                                key = (tuple(sorted(w1 + w2)), comps2)
                                acc[key] = acc.get(key, 0) + c1 * c2
                        for (ws, cs), k in sorted(acc.items()):
                            if k:
                                terms.append((hi, w, k, HESS_SETS.index(ws)) + cs)
                    w += 1
    return terms


def pack_hess_hrr(r):
    """HRR op {dst | x<<16, y | kind<<16 | dir<<20} (kind 0 bra, 1 ket) or contraction
    {W index | x<<16, (coef + 128) | 2<<16 | out<<20}."""
    kind = r[0]
    if kind == 2:
        _, hi, wi, x, k = r
        assert -128 <= k < 128 and 0 <= hi < 45
        return (_i32(_u16(wi) | _u16(x) << 16), _i32((k + 128) | 2 << 16 | hi << 20))
    _, i, dst, x, y = r
    return (_i32(_u16(dst) | _u16(x) << 16), _i32(_u16(y) | kind << 16 | i << 20))


def gen_hess_table(la, lb, lc, ld):
    """Op tables of the adjoint Hessian of one class, run by hess_table() (one thread per
    quartet on thread-interleaved scratch): the VRR two orders higher with every target
    accumulated into the weight sets that need it, the HRR of each set to the shifted
    classes, and one contraction row per term of hess_terms."""
    L = la + lb + lc + ld + 2
    terms = hess_terms(la, lb, lc, ld)
    # HRR over lazily numbered values: accumulators ("acc", set, e, f) first discovered, the
    # intermediate values after; both renumbered below
    acc_ids, hnodes, hops = {}, {}, []
    counter = [0]

    def new_id():
        counter[0] += 1
        return ("h", counter[0] - 1)

    def ket(k, e, c, d):
        key = ("k", k, e, c, d)
        if key in hnodes:
            return hnodes[key]
        if sum(d) == 0:
            v = ("acc", k, e, c)
            acc_ids.setdefault(v, len(acc_ids))
        else:
            i = max(range(3), key=lambda q: (d[q], -q))
            d1 = add(d, i, -1)
            x, y = ket(k, e, add(c, i), d1), ket(k, e, c, d1)
            v = new_id()
            hops.append((1, i, v, x, y))
        hnodes[key] = v
        return v

    def bra(k, a, b, c, d):
        key = ("b", k, a, b, c, d)
        if key in hnodes:
            return hnodes[key]
        if sum(b) == 0:
            v = ket(k, a, c, d)
        else:
            i = max(range(3), key=lambda q: (b[q], -q))
            b1 = add(b, i, -1)
            x, y = bra(k, add(a, i), b1, c, d), bra(k, a, b1, c, d)
            v = new_id()
            hops.append((0, i, v, x, y))
        hnodes[key] = v
        return v

    for hi, wi, k, si, a, b, c, d in terms:
        x = bra(si, a, b, c, d)
        hops.append((2, hi, wi, x, k))
    nacc = len(acc_ids)
    # value numbering for the HRR region: slot 0 = zero, accumulator j at 1 + j, then the rest
    vid = {v: 1 + j for v, j in acc_ids.items()}
    nxt = [1 + nacc]

    def num(v):
        if v not in vid:
            vid[v] = nxt[0]
            nxt[0] += 1
        return vid[v]

    huses, hdefs = [], []
    for o in hops:
        if o[0] == 2:
            huses.append([num(o[3])])
            hdefs.append([])
        else:
            huses.append([num(o[3]), num(o[4])])
            hdefs.append([num(o[2])])
    hpre = {1 + j: 1 + j for j in range(nacc)}
    hslot, nhslot = linear_scan(nxt[0], huses, hdefs, hpre)
    hrows = []
    for o in hops:
        if o[0] == 2:
            _, hi, wi, x, k = o
            hrows.append((2, hi, wi, hslot[vid[x]], k))
        else:
            kind, i, v, x, y = o
            hrows.append((kind, i, hslot[vid[v]], hslot[vid[x]], hslot[vid[y]]))
    # VRR: every accumulator is [e0|f0]^(0) of its set
    dag = Dag(L)
    tgt_nodes = {}
    for (_, k, e, f), j in acc_ids.items():
        tgt_nodes.setdefault(dag.get(e, f, 0), []).append((k, j))
    ops, uses, defs = [], [], []
    for nid, node in enumerate(dag.nodes):
        if node[0] != "F":
            kind, i, a, b, c, d, g, k1, k2 = node
            ops.append(["K" if kind == "K" else "B", i, nid, a, b, c, d, g, k1, k2])
            uses.append([x for x in (a, b, c, d, g) if x >= 0])
            defs.append([nid])
        for (k, j) in tgt_nodes.get(nid, []):
            ops.append(["A", k, j, nid, -1, -1, -1, -1, 0, 0])
            uses.append([nid])
            defs.append([])
    pre = {m: 1 + m for m in range(L + 1)}  # F[m] lives in slot 1+m
    slot, nvslot = linear_scan(len(dag.nodes), uses, defs, pre)
    kinds = {"B": 0, "K": 1, "A": 2}
    vrows = []
    for o in ops:
        k, i, dst, a, b, c, d, g, k1, k2 = o
        if k == "A":
            vrows.append((2, i, dst, slot[a], 0, 0, 0, 0, 0, 0))
        else:
            sl = lambda x: slot[x] if x >= 0 else 0
            vrows.append((kinds[k], i, slot[dst], sl(a), sl(b), sl(c), sl(d), sl(g), k1, k2))
    t = f"{la}{lb}{lc}{ld}"
    s = [f"// table-mode adjoint Hessian of class {t}: {len(vrows)} VRR ops over {nvslot} slots, {nacc} "
         f"accumulators in {len(HESS_SETS)} weight sets, {len(hrows)} HRR/contraction ops over {nhslot} slots"]
    s.append(f"__device__ const int4 hvrr_{t}[{len(vrows)}] = {{")
    s += ["  {" + ",".join(map(str, pack_grad_vrr(r))) + "}," for r in vrows]
    s.append("};")
    s.append(f"__device__ const int2 hhrr_{t}[{len(hrows)}] = {{")
    s += ["  {" + ",".join(map(str, pack_hess_hrr(r))) + "}," for r in hrows]
    s.append("};")
    s.append(f"struct HessTable{t} {{ static constexpr int L = {L}, NVOPS = {len(vrows)}, NVSLOT = {nvslot}, "
             f"NACC = {nacc}, NHOPS = {len(hrows)}, NHSLOT = {nhslot}; "
             f"static __device__ const int4* vrr() {{ return hvrr_{t}; }} "
             f"static __device__ const int2* hrr() {{ return hhrr_{t}; }} }};")
    meta = {"class": [la, lb, lc, ld], "vrr_ops": len(vrows), "vrr_slots": nvslot, "accumulators": nacc,
            "hrr_ops": len(hrows), "hrr_slots": nhslot, "terms": len(terms)}
    return "\n".join(s), meta



def pack_hess_block_hrr(r):
    """Block-form HRR row {dst, x, y, kind | dir<<2} (kind 0 bra, 1 ket) or contraction row
    {W index, x, 0, 2 | out<<4 | (coef + 128)<<10}: full 32-bit slot numbers (the level-wise
    slot allocation of the large classes needs more than 2^16)."""
    if r[0] == 2:
        _, hi, wi, x, k = r
        assert -128 <= k < 128 and 0 <= hi < 45
        return (wi, x, 0, 2 | hi << 4 | (k + 128) << 10)
    kind, i, dst, x, y = r
    return (dst, x, y, kind | i << 2)


def gen_hess_block(la, lb, lc, ld):
    """Levelised op tables of the adjoint Hessian of one class for one block of threads per
    quartet (hess_block_kernel): the VRR two orders higher and the HRR of the ten weight sets
    are levelised (an op reads only values of earlier levels), so a level's ops run
    thread-parallel; each HRR level ends with its contraction rows, sorted by output entry,
    which the threads take in contiguous chunks (one register sum per run of equal entries)."""
    L = la + lb + lc + ld + 2
    terms = hess_terms(la, lb, lc, ld)
    hnodes, hinfo, hdeps, acc_key = {}, {}, {}, {}
    nxt = [0]

    def new_id():
        nxt[0] += 1
        return ("h", nxt[0] - 1)

    def ket(k, e, c, d):
        key = ("k", k, e, c, d)
        if key in hnodes:
            return hnodes[key]
        if sum(d) == 0:
            v = ("acc", k, e, c)
            acc_key.setdefault(v, len(acc_key))
        else:
            i = max(range(3), key=lambda q: (d[q], -q))
            d1 = add(d, i, -1)
            x, y = ket(k, e, add(c, i), d1), ket(k, e, c, d1)
            v = new_id()
            hinfo[v], hdeps[v] = (1, i, x, y), [x, y]
        hnodes[key] = v
        return v

    def bra(k, a, b, c, d):
        key = ("b", k, a, b, c, d)
        if key in hnodes:
            return hnodes[key]
        if sum(b) == 0:
            v = ket(k, a, c, d)
        else:
            i = max(range(3), key=lambda q: (b[q], -q))
            b1 = add(b, i, -1)
            x, y = bra(k, add(a, i), b1, c, d), bra(k, a, b1, c, d)
            v = new_id()
            hinfo[v], hdeps[v] = (0, i, x, y), [x, y]
        hnodes[key] = v
        return v

    cops = [(hi, wi, bra(si, a, b, c, d), k) for hi, wi, k, si, a, b, c, d in terms]
    nacc = len(acc_key)
    # number every HRR value: accumulators 0 .. nacc-1 (the inputs), the rest after
    num = {v: j for v, j in acc_key.items()}
    for v in hinfo:
        num[v] = len(num)
    hord = [num[v] for v in hinfo]  # creation order is topological
    hdeps_n = {num[v]: [num[x] for x in hdeps[v]] for v in hinfo}
    hlev = _levelise([(v, hdeps_n[v]) for v in hord], nacc)
    clev = [1 + hlev[num[x]] for (_, _, x, _) in cops]
    readers = [(l, [num[x]]) for l, (_, _, x, _) in zip(clev, cops)]
    hpre = {j: j for j in range(nacc)}
    hslot, nhs = _alloc_levels_with_readers(sorted(hord, key=lambda v: (hlev[v], v)), hdeps_n, hlev, hpre, set(),
                                            readers)
    inv = {num[v]: v for v in hinfo}
    maxl = max([hlev[v] for v in hord] + clev + [0])
    hrows, hlv = [], []
    by_l = {}
    for v in hord:
        by_l.setdefault(hlev[v], [[], []])[0].append(v)
    for j, l in enumerate(clev):
        by_l.setdefault(l, [[], []])[1].append(j)
    for l in range(1, maxl + 1):
        ops_l, con_l = by_l.get(l, [[], []])
        start = len(hrows)
        for v in ops_l:
            kind, i, x, y = hinfo[inv[v]]
            hrows.append((kind, i, hslot[v], hslot[num[x]], hslot[num[y]]))
        mid = len(hrows)
        for j in sorted(con_l, key=lambda j: (cops[j][0], cops[j][1])):
            hi, wi, x, k = cops[j]
            hrows.append((2, hi, wi, hslot[num[x]], k))
        hlv.append((start, mid))
    hlv.append((len(hrows), len(hrows)))
    # VRR, levelised; accumulator j <- weight(set) * value at slot
    dag = Dag(L)
    acc_src, acc_set = [0] * nacc, [0] * nacc
    for (_, k, e, f), j in acc_key.items():
        acc_src[j] = dag.get(e, f, 0)
        acc_set[j] = k
    ops = [(nid, nd) for nid, nd in enumerate(dag.nodes) if nd[0] != "F"]
    deps = {nid: [x for x in nd[2:7] if x >= 0] for nid, nd in ops}
    lev = _levelise([(nid, deps[nid]) for nid, _ in ops], L + 1)
    vorder = sorted([nid for nid, _ in ops], key=lambda n: (lev[n], n))
    pre = {m: m for m in range(L + 1)}
    slot, nvs = _alloc_levels(vorder, deps, lev, pre, set(acc_src))
    ZV = nvs
    nodes = dict(ops)
    vrows, vlev, cur = [], [0], 1
    for nid in vorder:
        while lev[nid] > cur:
            vlev.append(len(vrows))
            cur += 1
        kind, i, a, b, c, d, g, k1, k2 = nodes[nid]
        s_ = lambda x: slot[x] if x >= 0 else ZV
        vrows.append(((1 if kind == "K" else 0) | (i << 2), slot[nid], s_(a), s_(b), s_(c), s_(d), s_(g),
                      k1 | (k2 << 8)))
    vlev.append(len(vrows))
    t = f"{la}{lb}{lc}{ld}"
    ncart_blk = ncart(la) * ncart(lb) * ncart(lc) * ncart(ld)
    s = [f"// block-mode adjoint Hessian of class {t}: {len(vrows)} VRR ops in {len(vlev) - 1} levels over "
         f"{nvs} slots, {nacc} accumulators, {len(hrows)} HRR/contraction ops in {len(hlv) - 1} levels over "
         f"{nhs} slots"]
    s.append(f"__device__ const int4 hbv_{t}[{max(len(vrows), 1)}] = {{")
    s += ["  {" + ",".join(map(str, pack_warp_vrr(r))) + "}," for r in vrows]
    s.append("};")
    s.append(f"__device__ const int hbv_lv_{t}[{len(vlev)}] = {{{','.join(map(str, vlev))}}};")
    s.append(f"__device__ const int2 hba_{t}[{nacc}] = {{" +
             ",".join("{%d,%d}" % (slot[n], k) for n, k in zip(acc_src, acc_set)) + "};")
    s.append(f"__device__ const int4 hbh_{t}[{max(len(hrows), 1)}] = {{")
    s += ["  {" + ",".join(map(str, pack_hess_block_hrr(r))) + "}," for r in hrows]
    s.append("};")
    s.append(f"__device__ const int2 hbh_lv_{t}[{len(hlv)}] = {{" + ",".join("{%d,%d}" % p for p in hlv) + "};")
    s.append(f"struct HessBlockTab{t} {{ static constexpr int L = {L}, NVLEV = {len(vlev) - 1}, NVSLOT = {nvs}, "
             f"NACC = {nacc}, NHLEV = {len(hlv) - 1}, NHSLOT = {nhs}, NCART = {ncart_blk}; "
             f"static __device__ const int4* vrr() {{ return hbv_{t}; }} "
             f"static __device__ const int* vlev() {{ return hbv_lv_{t}; }} "
             f"static __device__ const int2* acc() {{ return hba_{t}; }} "
             f"static __device__ const int4* hrr() {{ return hbh_{t}; }} "
             f"static __device__ const int2* hlev() {{ return hbh_lv_{t}; }} }};")
    meta = {"class": [la, lb, lc, ld], "vrr_ops": len(vrows), "vrr_levels": len(vlev) - 1, "vrr_slots": nvs,
            "acc": nacc, "hrr_ops": len(hrows), "hrr_levels": len(hlv) - 1, "hrr_slots": nhs,
            "slots": nvs + 1 + nhs + 1 + 45 + 3 * ncart_blk}
    return "\n".join(s), meta


HESS_LINE_PASS_ACC = 64   # accumulators of one pass of the straight-line Hessian form
HESS_LINE_MAX_PASSES = 24  # classes that need more passes keep the table forms only
# weight of each set of HESS_SETS as a named register, and its definition in the bra or ket
# primitive loop; set 0 has weight 1
HESS_WEIGHT = [None, "wa", "wb", "wc", "waa", "wbb", "wcc", "wab", "wac", "wbc"]
HESS_WEIGHT_DEF = {"waa": "wa * wa", "wbb": "wb * wb", "wab": "wa * wb",
                   "wcc": "wc * wc", "wac": "wa * wc", "wbc": "wb * wc"}
HESS_LINE_SIG = ("const PrimPair<R>* __restrict__ bp, const R* __restrict__ ea, const R* __restrict__ eb, int nbp, "
                 "const PrimPair<R>* __restrict__ kp, const R* __restrict__ ec, int nkp, R ABx, R ABy, R ABz, "
                 "R CDx, R CDy, R CDz, const BoysTable<R>& boys, WF&& weights, H h45")
HESS_LINE_ARGS = "bp, ea, eb, nbp, kp, ec, nkp, ABx, ABy, ABz, CDx, CDy, CDz, boys, weights, h45"


def hess_term_needs(terms):
    """The contracted [e0|f0] values the HRR of the given terms (one weight set) reads."""
    need = {}

    def record(e, f):
        need.setdefault((e, f), len(need))
        return "x"

    hr = HRR(Emitter(), record, prefix="h")
    for hi, wi, kk, si, a, b, c, d in terms:
        hr.bra(a, b, c, d)
    return list(need)


def hess_line_units(la, lb, lc, ld, terms):
    """The contraction terms cut into units [(set, terms, needed [e0|f0] values)] of at most
    HESS_LINE_PASS_ACC accumulators where possible: a weight set whole, or split by the bra
    component a of the differentiated integral (its W index), else by the ket component c, else
    by both -- the HRR of each part then reads only the values near its own components."""
    nb, nc, nd = ncart(lb), ncart(lc), ncart(ld)
    keys = [lambda t: t[1] // (nb * nc * nd), lambda t: (t[1] // nd) % nc,
            lambda t: (t[1] // (nb * nc * nd), (t[1] // nd) % nc)]
    units = []
    for k in range(len(HESS_SETS)):
        tk = [t for t in terms if t[3] == k]
        if not tk:
            continue
        whole = hess_term_needs(tk)
        if len(whole) <= HESS_LINE_PASS_ACC:
            units.append((k, tk, whole))
            continue
        best = None
        for key in keys:
            groups = {}
            for t in tk:
                groups.setdefault(key(t), []).append(t)
            parts = [(k, g, hess_term_needs(g)) for _, g in sorted(groups.items())]
            worst = max(len(u[2]) for u in parts)
            if best is None or worst < best[0]:
                best = (worst, parts)
            if worst <= HESS_LINE_PASS_ACC:
                break
        units += best[1]
    return units


def hess_line_passes(la, lb, lc, ld, terms=None):
    """Units packed, in order, into passes of at most HESS_LINE_PASS_ACC distinct accumulators
    (a unit larger than that runs alone): [[(set, terms, needs), ...], ...]."""
    terms = hess_terms(la, lb, lc, ld) if terms is None else terms
    passes, cur, keys = [], [], set()
    for u in hess_line_units(la, lb, lc, ld, terms):
        ukeys = {(u[0],) + ef for ef in u[2]}
        if cur and len(keys | ukeys) > HESS_LINE_PASS_ACC:
            passes.append(cur)
            cur, keys = [], set()
        cur.append(u)
        keys |= ukeys
    if cur:
        passes.append(cur)
    return passes


def gen_hess_line(la, lb, lc, ld):
    """Straight-line adjoint Hessian of one class for one thread per quartet, every value in
    registers (the many-quartet classes, which the table forms run slowly: a level barrier or a
    global-scratch round trip per handful of ops).  The contraction terms are cut into passes of
    at most HESS_LINE_PASS_ACC accumulators (hess_line_passes).  A pass runs the primitive loops
    with the VRR of its targets only, then fetches the quartet's weight block (weights(W),
    Cartesian), runs the HRR its terms read and adds them into the 45 entries h45 of the 9 x 9
    block (an accessor to the thread's slice of shared memory), so that nothing but a pass's
    accumulators lives through its primitive loops.  None when a unit still needs more than
    HESS_LINE_PASS_ACC accumulators or the class more than HESS_LINE_MAX_PASSES passes."""
    terms = hess_terms(la, lb, lc, ld)
    # the sets share no accumulators, so the passes number at least their total over the pass size
    total = sum(len(hess_term_needs([t for t in terms if t[3] == k])) for k in range(len(HESS_SETS)))
    if total > HESS_LINE_MAX_PASSES * HESS_LINE_PASS_ACC:
        return None, None
    passes = hess_line_passes(la, lb, lc, ld, terms)
    if len(passes) > HESS_LINE_MAX_PASSES or max(len(u[2]) for p in passes for u in p) > HESS_LINE_PASS_ACC:
        return None, None
    t = f"{la}{lb}{lc}{ld}"
    ncw = ncart(la) * ncart(lb) * ncart(lc) * ncart(ld)
    s = []
    pmeta = []
    for pi, units in enumerate(passes):
        idx = {}
        for k, _, need in units:
            for ef in need:
                idx.setdefault((k,) + ef, len(idx))
        psets = sorted({u[0] for u in units})
        nacc = len(idx)
        em2 = Emitter("    ")
        hr = {k: HRR(em2, (lambda kk: (lambda e, f: f"acc[{idx[(kk, e, f)]}]"))(k), prefix=f"h{pi}_{k}")
              for k in psets}
        out = {}
        for k, tl, _ in units:
            for hi, wi, kk, si, a, b, c, d in tl:
                v = hr[si].bra(a, b, c, d)
                out.setdefault(hi, []).append(f"W[{wi}] * {v}" if kk == 1 else f"{lit(kk)} * W[{wi}] * {v}")
        for hi in sorted(out):
            em2.emit(f"h45[{hi}] += " + " + ".join(out[hi]) + ";", 3 * len(out[hi]))
        em = Emitter("        ")
        vrr = VRR(em)
        targets = sorted({(e, f) for (_, e, f) in idx}, key=lambda q: (sum(q[0]), cidx(q[0]), sum(q[1]), cidx(q[1])))
        vals = {q: vrr.get(q[0], q[1], 0) for q in targets}
        Lp = max(sum(e) + sum(f) for e, f in targets)
        used = {HESS_WEIGHT[k] for k in psets if HESS_WEIGHT[k]}
        s.append(f"  {{  // pass {pi}: weight sets {psets}, {nacc} accumulators, {len(vrr.memo)} VRR values")
        s.append(f"    R acc[{nacc}];")
        s.append("#pragma unroll")
        s.append(f"    for (int t = 0; t < {nacc}; ++t) acc[t] = R(0);")
        s.append("    for (int ib = 0; ib < nbp; ++ib) {")
        s.append("      const R p = bp[ib].p, ip = bp[ib].ip, Px = bp[ib].Px, Py = bp[ib].Py, Pz = bp[ib].Pz;")
        s.append("      const R PAx = bp[ib].PAx, PAy = bp[ib].PAy, PAz = bp[ib].PAz, Kab = bp[ib].Kp;")
        s.append("      const R wa = R(2) * ea[ib], wb = R(2) * eb[ib];")
        s.append("      (void)wa; (void)wb;")
        for w in ("waa", "wbb", "wab"):
            if w in used:
                s.append(f"      const R {w} = {HESS_WEIGHT_DEF[w]};")
        s.append("      for (int ik = 0; ik < nkp; ++ik) {")
        s.append("        const R q = kp[ik].p, iq = kp[ik].ip, Qx = kp[ik].Px, Qy = kp[ik].Py, Qz = kp[ik].Pz;")
        s.append("        const R QCx = kp[ik].PAx, QCy = kp[ik].PAy, QCz = kp[ik].PAz, Kcd = kp[ik].Kp;")
        s.append("        const R wc = R(2) * ec[ik];")
        s.append("        (void)wc;")
        for w in ("wcc", "wac", "wbc"):
            if w in used:
                s.append(f"        const R {w} = {HESS_WEIGHT_DEF[w]};")
        s += ["  " + line for line in PRIM_HEADER.rstrip("\n").split("\n")]
        s.append(f"        R F[{Lp + 1}];")
        s.append(f"        boys.template eval<{Lp}>(T, pre, F);")
        adds = []
        for (k, e, f), j in idx.items():
            v = vals[(e, f)]
            w = HESS_WEIGHT[k]
            adds.append((v, f"        acc[{j}] += {v};" if w is None else f"        acc[{j}] += {w} * {v};"))
        s += interleave_accumulation(list(em.lines), adds)
        s.append("      }")
        s.append("    }")
        s.append(f"    R W[{ncw}];")
        s.append("    weights(W);")
        s += em2.lines
        s.append("  }")
        pmeta.append({"sets": psets, "accumulators": nacc, "vrr_values": len(vrr.memo), "boys_m": Lp})
    head = [f"// straight-line adjoint Hessian of ({'spdf'[la]}{'spdf'[lb]}|{'spdf'[lc]}{'spdf'[ld]}): "
            f"{len(passes)} passes, {sum(m['accumulators'] for m in pmeta)} accumulators, "
            f"{sum(m['vrr_values'] for m in pmeta)} VRR values",
            "template <typename R, typename WF, typename H>",
            f"__device__ __forceinline__ void hess_line_{t}({HESS_LINE_SIG}) {{"]
    s = head + s + ["}", f"struct HessLine{t} {{",
                    "  template <typename R, typename WF, typename H>",
                    f"  static __device__ __forceinline__ void run({HESS_LINE_SIG}) {{ hess_line_{t}<R>({HESS_LINE_ARGS}); }}",
                    "};"]
    return "\n".join(s), {"class": [la, lb, lc, ld], "passes": pmeta}


if __name__ == "__main__":
    main(sys.argv[1])
