"""CPU tests of the host side: the C-ABI library, basis handling, molecules."""
import ctypes
import os

import numpy as np
import pytest

from hfscf_b200 import basis as B
from hfscf_b200 import engine as E
from hfscf_b200 import molecules as M


def test_library_exports_every_declared_symbol():
    lib = E.lib()
    names = E.exported_symbols()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_default_options():
    o = E._Opts()
    assert E.lib().hfgpu_default_opts(ctypes.byref(o)) == 0
    assert o.schwarz_tol == 1e-12 and o.mixed_fp32_bound == 1e-4
    assert o.density_tol == 1e-12 and o.mixed_density_tol == 1e-12
    assert o.warp_max_quartets == 1 << 30 and o.grad_warp_max_waves == 48


def test_flop_model_counts():
    """The counting model of the roofline: block sizes in the final basis, FLOPs linear in the
    computed quartets and primitive quartets, classes named in the order of hfgpu_class_stats."""
    from hfscf_b200 import flopmodel as F
    names = [F.class_name(c) for c in range(E.NUM_CLASSES)]
    assert names[0] == "(ss|ss)" and names[-1] == "(dd|dd)" and len(set(names)) == E.NUM_CLASSES
    assert F.class_block_size(E.NUM_CLASSES - 1, False) == 6 ** 4
    assert F.class_block_size(E.NUM_CLASSES - 1, True) == 5 ** 4
    assert F.class_block_size(0, False) == 1
    assert F.class_integrals(E.NUM_CLASSES - 1, 7, True) == 7 * 625
    for c in range(E.NUM_CLASSES):
        f1 = F.class_flops(c, 10, 100, False)
        assert F.class_flops(c, 20, 200, False) == pytest.approx(2 * f1)
        assert F.class_flops(c, 0, 0, False) == 0.0
        if c < 6:  # s and p only: the pure and Cartesian bases are the same
            assert F.class_flops(c, 10, 100, True) == F.class_flops(c, 10, 100, False)


def test_gradient_flop_model_hand_counts_and_scaling():
    """The frozen gradient count of (ss|ss), by hand: per primitive quartet 25 scalars, Boys
    F_0..F_1 (34), VRR of [p0|s0] and [s0|p0] (6 x 3) and the weighted sums of the raised sets
    (2 alpha: 3 targets, 2 beta: 4, 2 gamma: 3; two flops each) = 97; per contracted quartet the
    HRR of (sp|ss) (3 x 2) and 4 flops for each of the nine derivative integrals = 42.  Every
    class costs more than its energy count and scales linearly in its work."""
    from hfscf_b200 import flopmodel as F
    assert F.grad_per_prim_flops(0) == 97
    assert F.grad_per_quartet_flops(0, False) == 42
    for c in range(E.NUM_CLASSES):
        assert F.grad_per_prim_flops(c) > F.per_prim_flops(c)
        assert F.grad_per_quartet_flops(c, False) > F.per_quartet_flops(c, False)
        g1 = F.grad_class_flops(c, 10, 100, True)
        assert F.grad_class_flops(c, 20, 200, True) == pytest.approx(2 * g1)


def test_basis_sizes_of_the_workloads():
    sizes = {}
    for w in (1, 2, 3, 4):
        Z, x, name, pure = M.workload(w)
        sizes[w] = B.build_basis(name, Z, x, pure=pure).nbf
    assert sizes == {1: 24, 2: 210, 3: 246, 4: 152}


def test_shell_order_and_offsets_follow_the_reference():
    bs = B.build_basis("6-31g*", [8, 1], [[0, 0, 0], [0, 0, 1.8]], pure=False)
    Ls = [s.L for s in bs.shells]
    assert Ls == [0, 0, 1, 0, 1, 2, 0, 0]  # O: S, SP->S,P, SP->S,P, D ; H: S, S
    assert [s.idx for s in bs.shells] == [0, 1, 2, 5, 6, 9, 15, 16]


def test_batch_molecules_are_seeded_and_mixed():
    a = M.batch_molecules(64)
    b = M.batch_molecules(64)
    assert all(np.array_equal(x[1], y[1]) for x, y in zip(a, b))
    assert {m[2] for m in a} == {"sto-3g", "6-31g*"}


def _md_overlap_kinetic(bs):
    """Independent S and T by numerical quadrature-free closed forms for s/p/d (MD Hermite E)."""
    from math import comb, factorial
    shells = bs.shells

    def norm_c(sh):
        import oracle
        return oracle.shell_norm(sh.L, sh.exps, sh.coefs)

    def E1(i, j, t, Qx, a, b):
        p = a + b
        q = a * b / p
        if t < 0 or t > i + j:
            return 0.0
        if i == j == t == 0:
            return np.exp(-q * Qx * Qx)
        if j == 0:
            return (1 / (2 * p)) * E1(i - 1, j, t - 1, Qx, a, b) - (q * Qx / a) * E1(i - 1, j, t, Qx, a, b) + \
                (t + 1) * E1(i - 1, j, t + 1, Qx, a, b)
        return (1 / (2 * p)) * E1(i, j - 1, t - 1, Qx, a, b) + (q * Qx / b) * E1(i, j - 1, t, Qx, a, b) + \
            (t + 1) * E1(i, j - 1, t + 1, Qx, a, b)

    def s1(i, j, A, Bc, a, b):
        return E1(i, j, 0, A - Bc, a, b) * np.sqrt(np.pi / (a + b))

    def comps(L):
        return [(L - i, i - j, j) for i in range(L + 1) for j in range(i + 1)]

    n = bs.ncart
    S = np.zeros((n, n))
    T = np.zeros((n, n))
    for sa in shells:
        ca = norm_c(sa)
        for sb in shells:
            cb = norm_c(sb)
            for x, la in enumerate(comps(sa.L)):
                for y, lb in enumerate(comps(sb.L)):
                    sv = tv = 0.0
                    for a, c1 in zip(sa.exps, ca):
                        for b, c2 in zip(sb.exps, cb):
                            s = [s1(la[d], lb[d], sa.center[d], sb.center[d], a, b) for d in range(3)]
                            t = 0.0
                            for d in range(3):
                                l2 = lb[d]
                                td = -2 * b * b * s1(la[d], l2 + 2, sa.center[d], sb.center[d], a, b) + \
                                    b * (2 * l2 + 1) * s1(la[d], l2, sa.center[d], sb.center[d], a, b)
                                if l2 > 1:
                                    td -= 0.5 * l2 * (l2 - 1) * s1(la[d], l2 - 2, sa.center[d], sb.center[d], a, b)
                                others = [s[e] for e in range(3) if e != d]
                                t += td * others[0] * others[1]
                            sv += c1 * c2 * s[0] * s[1] * s[2]
                            tv += c1 * c2 * t
                    S[sa.idx + x, sb.idx + y] = sv
                    T[sa.idx + x, sb.idx + y] = tv
    return S, T


def test_one_electron_overlap_kinetic_against_independent_hermite_forms():
    Z, x = M.water(np.random.default_rng(2))
    bs = B.build_basis("6-31g*", Z, np.asarray(x) * B.ANGSTROM_TO_BOHR, pure=False)
    S, T, V = E.one_electron(bs)
    S0, T0 = _md_overlap_kinetic(bs)
    assert np.max(np.abs(S - S0)) < 1e-12 and np.max(np.abs(T - T0)) < 1e-11
    assert np.allclose(V, V.T) and np.all(np.diag(V) < 0)


def test_one_electron_gradient_translational_invariance():
    Z, x = M.water(np.random.default_rng(3))
    bs = B.build_basis("cc-pvdz", Z, np.asarray(x) * B.ANGSTROM_TO_BOHR, pure=True)
    n = bs.nbf
    rng = np.random.default_rng(0)
    A = rng.normal(size=(n, n))
    D = (A + A.T) / n
    g = E.one_electron_grad(bs, D, D, 2.0, -2.0)
    assert np.max(np.abs(g.sum(axis=0))) < 1e-10


def test_one_electron_gradient_matches_finite_differences():
    Z, x = M.water(np.random.default_rng(4))
    x = np.asarray(x) * B.ANGSTROM_TO_BOHR
    bs = B.build_basis("6-31g*", Z, x, pure=False)
    n = bs.nbf
    rng = np.random.default_rng(1)
    A = rng.normal(size=(n, n))
    D = (A + A.T) / n
    W = D @ D
    g = E.one_electron_grad(bs, D, W, 2.0, -2.0)
    h = 1e-5
    for a in range(3):
        for d in range(3):
            vals = []
            for s in (1, -1):
                xx = x.copy()
                xx[a, d] += s * h
                S, T, V = E.one_electron(bs.with_coords(xx))
                vals.append(2 * np.sum(D * (T + V)) - 2 * np.sum(W * S))
            assert abs((vals[0] - vals[1]) / (2 * h) - g[a, d]) < 1e-6


def test_sad_populations_follow_the_reference():
    """Frozen-core / fractional valence weights of get_pop_numbers (hfscf_sad.cpp:198-245)."""
    from hfscf_b200 import scf
    w, occ = scf.sad_populations(1, 2)
    assert occ == 1 and np.allclose(w, [np.sqrt(0.5), 0.0])
    w, occ = scf.sad_populations(6, 14)
    assert occ == 5 and w[0] == 1.0 and np.allclose(w[1:5], np.sqrt(0.5)) and (w[5:] == 0).all()
    w, occ = scf.sad_populations(8, 14)
    assert occ == 5 and np.allclose(w[1:5], np.sqrt(6 / 8))
    w, occ = scf.sad_populations(2, 5)
    assert occ == 1 and w[0] == 1.0


def test_sad_atom_density_with_oracle_jk_holds_the_atom_electrons():
    """The SAD atomic UHF run with the oracle's J/K (CPU): the spin-averaged density
    carries Z/2 electrons in the atom's overlap metric."""
    import oracle
    from hfscf_b200 import scf
    Z, x = M.water(np.random.default_rng(2))
    bs = B.build_basis("6-31g*", Z, np.asarray(x) * B.ANGSTROM_TO_BOHR, pure=False)
    for a in (0, 1):
        ab = scf.atom_basis(bs, a)
        S, T, V = E.one_electron(ab)
        eri = oracle.eri_packed(ab)

        def jk(DJ, DKs):
            J = oracle.jk(eri, DJ)[0]
            return J, [oracle.jk(eri, Dk)[1] for Dk in DKs]

        D = scf.sad_atom_density(int(ab.Z[0]), S, T, V, jk)
        assert abs(np.sum(D * S) - ab.Z[0] / 2) < 1e-10


def test_batched_layout_round_trip_and_padding():
    """Block storage (molecule m: n_m x n_m at its offset) <-> padded [nmol, nmax, nmax]
    matrices of the batched SCF: a round trip is exact, the padding is zero off the
    diagonal and carries the fill value on it (it keeps padded orbitals out of the
    occupied set)."""
    import torch

    from hfscf_b200.batch import _Layout
    nbf = np.array([1, 4, 2])
    off = np.concatenate([[0], np.cumsum(nbf * nbf)[:-1]])
    lay = _Layout(nbf, off, torch.device("cpu"))
    rng = np.random.default_rng(2)
    blocks = torch.from_numpy(rng.normal(size=int((nbf * nbf).sum())))
    P = lay.to_pad(blocks, fill_diag=7.0)
    assert P.shape == (3, 4, 4)
    assert torch.equal(lay.to_block(P), blocks)
    for m, (n, o) in enumerate(zip(nbf, off)):
        assert torch.equal(P[m, :n, :n].reshape(-1), blocks[o:o + n * n])
        pad = P[m].clone()
        pad[:n, :n] = 0.0
        assert torch.equal(pad, torch.diag(torch.tensor([0.0] * n + [7.0] * (4 - n), dtype=pad.dtype)))


def _gen_eri():
    import importlib.util
    path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "hfscf_b200", "csrc", "gen_eri.py")
    spec = importlib.util.spec_from_file_location("gen_eri_for_tests", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_hessian_generator_second_derivative_rule_pointwise():
    """The adjoint Hessian's term lists (gen_eri.hess_terms) restate the second derivative of a
    product of four Cartesian Gaussians by their centres as shifted Gaussians times exponent
    weights.  Integrals are linear in the product, so the rule holds pointwise: checked at
    random points against central differences in the centre coordinates (h = 1e-3)."""
    g = _gen_eri()
    rng = np.random.default_rng(2)
    la, lb, lc, ld = 2, 1, 1, 0
    alpha = rng.uniform(0.3, 1.2, size=4)
    cen = rng.normal(size=(4, 3))
    r1, r2 = rng.normal(size=3), rng.normal(size=3)

    def prod(comps, cc):
        v = 1.0
        for P in range(4):
            r = r1 if P < 2 else r2
            d = r - cc[P]
            v *= np.prod(d ** np.array(comps[P])) * np.exp(-alpha[P] * d @ d)
        return v

    weights = {(): 1.0}
    for s in g.HESS_SETS:
        weights[s] = np.prod([2 * alpha["ABC".index(c)] for c in s]) if s else 1.0
    comps_of = [(a, b, c, d) for a in g.cart(la) for b in g.cart(lb) for c in g.cart(lc) for d in g.cart(ld)]
    rule = np.zeros((len(comps_of), 45))
    for hi, wi, k, si, a, b, c, d in g.hess_terms(la, lb, lc, ld):
        rule[wi, hi] += k * weights[g.HESS_SETS[si]] * prod((a, b, c, d), cen)
    h = 1e-3
    for wi, comps in enumerate(comps_of):
        for hi, (r, s) in enumerate(g.HESS_PAIRS):
            (P, i), (Q, j) = g.HESS_COORDS[r], g.HESS_COORDS[s]
            fd = 0.0
            for sp, sq, sgn in ((1, 1, 1), (1, -1, -1), (-1, 1, -1), (-1, -1, 1)):
                cc = cen.copy()
                cc[P, i] += sp * h
                cc[Q, j] += sq * h
                fd += sgn * prod(comps, cc)
            fd /= 4 * h * h
            assert abs(rule[wi, hi] - fd) < 1e-5 * max(1.0, abs(fd)), (comps, r, s, rule[wi, hi], fd)


def test_hessian_line_form_passes_cover_every_term_once():
    """The straight-line Hessian form (gen_eri.gen_hess_line) cuts the contraction terms into
    units and packs them into passes; together the passes must hold every term of hess_terms
    exactly once, each pass at most HESS_LINE_PASS_ACC accumulators, each unit's accumulators
    exactly the [e0|f0] values its own HRR reads.  The classes that get the form are the eight
    many-quartet classes the C header names."""
    g = _gen_eri()
    _, cls = g.classes()
    with_line = []
    for c in cls:
        terms = g.hess_terms(*c)
        code, meta = g.gen_hess_line(*c)
        if code is None:
            continue
        with_line.append(tuple(c))
        passes = g.hess_line_passes(*c, terms)
        assert len(passes) == len(meta["passes"]) <= g.HESS_LINE_MAX_PASSES
        seen = sorted(t for p in passes for _, tl, _ in p for t in tl)
        assert seen == sorted(terms)
        for p, m in zip(passes, meta["passes"]):
            keys = {(k,) + ef for k, _, need in p for ef in need}
            assert len(keys) == m["accumulators"] <= g.HESS_LINE_PASS_ACC
            for k, tl, need in p:
                assert all(t[3] == k for t in tl)
                assert sorted(need) == sorted(g.hess_term_needs(tl))
    assert with_line == [(0, 0, 0, 0), (1, 0, 0, 0), (1, 0, 1, 0), (1, 1, 0, 0), (1, 1, 1, 0),
                         (2, 0, 0, 0), (2, 0, 1, 0), (2, 1, 0, 0)]


class _OracleAtomEngine:
    """Stand-in for an atom's GPU engine in the SAD guess: S, T, V from the reference's own
    one-electron routines and J/K from the C restatement's packed ERIs (host only)."""

    def __init__(self, bs):
        import oracle
        self.bs = bs
        self.eri = oracle.eri_packed(bs)

    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False

    def one_electron(self):
        import oracle
        return oracle.ref_onee(self.bs)

    def jk(self, DJ, DKs):
        import oracle
        return oracle.jk(self.eri, DJ)[0], [oracle.jk(self.eri, Dk)[1] for Dk in DKs]


def test_batched_sad_guess_equals_the_per_molecule_guess():
    """batch_sad_guess runs the atomic UHF once per (basis set, element) and copies it onto every
    atom: each molecule's padded block equals scf.sad_guess of that molecule with the same atomic
    engines (host J/K) to 1e-8 (the atomic density is the same wherever the atom sits; the
    atomic runs, stopped at the SAD tolerances of rms 1e-6, differ in the last digits with the
    atom's position), and the padding is zero."""
    import oracle
    from hfscf_b200 import batch as BT
    from hfscf_b200 import scf
    if not oracle.ref_available():
        pytest.skip("reference library not built here")
    mols = M.batch_molecules(512)[:8]
    bases = BT.batch_bases(mols)
    assert len({b.name for b in bases}) == 2  # both basis sets of the mix
    nmax = max(b.nbf for b in bases)
    D = BT.batch_sad_guess(bases, nmax, engine_factory=_OracleAtomEngine)
    for k, b in enumerate(bases):
        Dk = scf.sad_guess(b, engine_factory=_OracleAtomEngine)
        n = b.nbf
        assert np.abs(D[k, :n, :n] - Dk).max() < 1e-8
        assert not D[k, n:, :].any() and not D[k, :, n:].any()
