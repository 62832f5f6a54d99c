"""The straight-line Hessian code (gen_eri.gen_hess_line) against the one-thread op tables of
the same class (gen_eri.gen_hess_table), both compiled with g++ and run on the host.

The table form is pinned to the reference's second-derivative routines by the GPU tests.  This
test checks the line form's generator on the CPU: its cut of the terms into passes, its VRR per
pass, HRR and contraction.  Both are generated here for the classes with a line form and written
into pytest's temporary directory after a small host stand-in for PrimPair, the Boys values and
the int2/int4 rows.  For every class with a line form, each of three random primitive
quartet sets (two bra and two ket primitives, random centres, exponents and weights) gives the 45
block entries both ways; they agree to 1e-12 relative to the largest entry.
"""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

STUB = r"""
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <algorithm>
#define __device__
#define __forceinline__ inline
#define __restrict__
#define __constant__
struct int2 { int x, y; };
struct int4 { int x, y, z, w; };
template <typename R> struct PrimPair { R p, ip, Px, Py, Pz, PAx, PAy, PAz, Kp, eb2; };
template <typename R> inline R rsqrt_t(R x) { return R(1) / std::sqrt(x); }
// F[m] = pre * F_m(T), F_m from its power series (T below 40 here)
template <typename R> struct BoysTable {
  template <int M> void eval(R T, R pre, R* F) const {
    for (int m = 0; m <= M; ++m) {
      double term = 1.0 / (2 * m + 1), sum = term;
      for (int k = 1; k < 400 && term > 1e-18 * sum; ++k) {
        term *= 2.0 * T / (2 * m + 2 * k + 1);
        sum += term;
      }
      F[m] = pre * std::exp(-T) * sum;
    }
  }
};
"""

# host copy of the one-thread table executor (the row formats of gen_eri.pack_grad_vrr and
# pack_hess_hrr)
EXEC = r"""
template <typename Tab>
void run_table(const PrimPair<double>* bp, const double* ea, const double* eb, int nbp,
               const PrimPair<double>* kp, const double* ec, int nkp, const double* AB, const double* CD,
               const double* W, double* h45) {
  std::vector<double> vs(Tab::NVSLOT + 1, 0.0), hs(Tab::NHSLOT + Tab::NACC + 2, 0.0);
  BoysTable<double> boys;
  for (int ib = 0; ib < nbp; ++ib)
    for (int ik = 0; ik < nkp; ++ik) {
      const PrimPair<double>& P = bp[ib];
      const PrimPair<double>& Q = kp[ik];
      const double wa = 2 * ea[ib], wb = 2 * eb[ib], wc = 2 * ec[ik];
      const double pq = P.p + Q.p, rs = 1.0 / std::sqrt(pq), ipq = rs * rs;
      const double rho = P.p * Q.p * ipq, rp = Q.p * ipq, rq = P.p * ipq;
      const double PQ[3] = {P.Px - Q.Px, P.Py - Q.Py, P.Pz - Q.Pz};
      const double PA[3] = {P.PAx, P.PAy, P.PAz}, QC[3] = {Q.PAx, Q.PAy, Q.PAz};
      const double T = rho * (PQ[0] * PQ[0] + PQ[1] * PQ[1] + PQ[2] * PQ[2]);
      double F[Tab::L + 1];
      boys.template eval<Tab::L>(T, P.Kp * Q.Kp * rs, F);
      vs[0] = 0.0;
      for (int m = 0; m <= Tab::L; ++m) vs[1 + m] = F[m];
      const double wt[10] = {1, wa, wb, wc, wa * wa, wb * wb, wc * wc, wa * wb, wa * wc, wb * wc};
      for (int o = 0; o < Tab::NVOPS; ++o) {
        const int4 op = Tab::vrr()[o];
        const int kind = op.w & 15, dir = (op.w >> 4) & 15, dst = op.x & 0xffff;
        const int sa = (unsigned)op.x >> 16, sb = op.y & 0xffff, sc = (unsigned)op.y >> 16, sd = op.z & 0xffff;
        if (kind == 2) { hs[1 + dst] += wt[dir] * vs[sa]; continue; }
        const int k1 = (op.w >> 8) & 255;
        if (kind == 0) {
          vs[dst] = PA[dir] * vs[sa] - rp * PQ[dir] * vs[sb] + k1 * 0.5 * P.ip * (vs[sc] - rp * vs[sd]);
        } else {
          const int sg = (unsigned)op.z >> 16, k2 = (unsigned)op.w >> 16;
          vs[dst] = QC[dir] * vs[sa] + rq * PQ[dir] * vs[sb] + k1 * 0.5 * Q.ip * (vs[sc] - rq * vs[sd]) +
                    k2 * 0.5 * ipq * vs[sg];
        }
      }
    }
  for (int x = 0; x < 45; ++x) h45[x] = 0.0;
  for (int o = 0; o < Tab::NHOPS; ++o) {
    const int2 op = Tab::hrr()[o];
    const int kind = (op.y >> 16) & 15, sx = (unsigned)op.x >> 16;
    if (kind == 2) {
      const int wi = op.x & 0xffff, k = (op.y & 0xffff) - 128, hi = (op.y >> 20) & 63;
      h45[hi] += k * W[wi] * hs[sx];
    } else {
      const int dst = op.x & 0xffff, sy = op.y & 0xffff, dir = (op.y >> 20) & 15;
      hs[dst] = hs[sx] + (kind == 0 ? AB[dir] : CD[dir]) * hs[sy];
    }
  }
}

// one class: random shells, both forms, the largest difference relative to the largest entry
template <typename Tab, typename Line>
double check(int ncw, unsigned seed) {
  std::srand(seed);
  auto u = [](double lo, double hi) { return lo + (hi - lo) * (std::rand() / (double)RAND_MAX); };
  double A[3], B[3], C[3], D[3];
  for (int i = 0; i < 3; ++i) { A[i] = u(-1, 1); B[i] = u(-1, 1); C[i] = u(-1, 1); D[i] = u(-1, 1); }
  PrimPair<double> bp[2], kp[2];
  double ea[2], eb[2], ec[2], ed[2];
  auto make = [](PrimPair<double>& P, double a, double b, const double* X, const double* Y) {
    P.p = a + b; P.ip = 1.0 / P.p;
    const double Pc[3] = {(a * X[0] + b * Y[0]) / P.p, (a * X[1] + b * Y[1]) / P.p, (a * X[2] + b * Y[2]) / P.p};
    P.Px = Pc[0]; P.Py = Pc[1]; P.Pz = Pc[2];
    P.PAx = Pc[0] - X[0]; P.PAy = Pc[1] - X[1]; P.PAz = Pc[2] - X[2];
    double r2 = 0; for (int i = 0; i < 3; ++i) r2 += (X[i] - Y[i]) * (X[i] - Y[i]);
    P.Kp = std::exp(-a * b / P.p * r2) * std::sqrt(2 * std::pow(M_PI, 2.5)) / P.p;
    P.eb2 = b * b;
  };
  for (int i = 0; i < 2; ++i) {
    ea[i] = u(0.2, 3.0); eb[i] = u(0.2, 3.0); ec[i] = u(0.2, 3.0); ed[i] = u(0.2, 3.0);
    make(bp[i], ea[i], eb[i], A, B);
    make(kp[i], ec[i], ed[i], C, D);
  }
  std::vector<double> W(ncw);
  for (auto& w : W) w = u(-1, 1);
  const double AB[3] = {A[0] - B[0], A[1] - B[1], A[2] - B[2]}, CD[3] = {C[0] - D[0], C[1] - D[1], C[2] - D[2]};
  double ht[45], hl[45];
  run_table<Tab>(bp, ea, eb, 2, kp, ec, 2, AB, CD, W.data(), ht);
  for (int x = 0; x < 45; ++x) hl[x] = 0.0;
  BoysTable<double> boys;
  auto weights = [&](double* Wc) { for (int i = 0; i < ncw; ++i) Wc[i] = W[i]; };
  Line::template run<double>(bp, ea, eb, 2, kp, ec, 2, AB[0], AB[1], AB[2], CD[0], CD[1], CD[2], boys, weights,
                             (double*)hl);
  double mx = 0, diff = 0;
  for (int x = 0; x < 45; ++x) { mx = std::max(mx, std::fabs(ht[x])); diff = std::max(diff, std::fabs(ht[x] - hl[x])); }
  return mx > 0 ? diff / mx : diff;
}
"""


def _gen_eri():
    import importlib.util
    spec = importlib.util.spec_from_file_location("gen_eri_for_line_test",
                                                  os.path.join(ROOT, "hfscf_b200", "csrc", "gen_eri.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_line_form_matches_table_form_on_the_host(tmp_path):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    g = _gen_eri()
    _, cls = g.classes()
    parts = [STUB, "#include <vector>"]
    classes = []
    for c in cls:
        if sum(c) > 3:  # every class with a line form has total angular momentum 3 or less
            continue
        code_l, _ = g.gen_hess_line(*c)
        if code_l is None:
            continue
        code_t, _ = g.gen_hess_table(*c)
        classes.append("".join(map(str, c)))
        parts += [code_t, code_l]
    assert classes == ["0000", "1000", "1010", "1100", "1110", "2000", "2010", "2100"]
    parts.append(EXEC)
    body = ["int main() {", "  double worst = 0;"]
    for t in classes:
        la, lb, lc, ld = (int(ch) for ch in t)
        ncw = 1
        for L in (la, lb, lc, ld):
            ncw *= (L + 1) * (L + 2) // 2
        for seed in (1, 2, 3):
            body.append(f"  {{ double d = check<HessTable{t}, HessLine{t}>({ncw}, {seed}u);")
            body.append(f'    std::printf("{t} {seed} %.3e\\n", d); worst = std::max(worst, d); }}')
    body += ['  std::printf("worst %.3e\\n", worst);', "  return worst < 1e-12 ? 0 : 1;", "}"]
    src = tmp_path / "hess_line_check.cpp"
    src.write_text("\n".join(parts + body) + "\n")
    exe = tmp_path / "hess_line_check"
    r = subprocess.run([gxx, "-std=c++17", "-O1", "-w", str(src), "-o", str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout[-3000:]
