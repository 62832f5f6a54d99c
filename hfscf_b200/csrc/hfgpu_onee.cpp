// One-electron integrals on the host CPU: overlap, kinetic, nuclear attraction
// and their contributions to the SCF gradient.  These are O(N^2) and stay on the
// CPU in this engine; they exist so that the SCF caller and the full gradient can
// be assembled around the two-electron GPU kernels.  Obara-Saika recurrences
// (Helgaker, Jorgensen, Olsen, "Molecular Electronic-Structure Theory", 9.3, 9.10),
// the same scheme as the reference's OSOverlap/OSKinetic/OSNuclear
// (src/integrals/hfscf_osoverlap.cpp, hfscf_oskineticderiv1.cpp, hfscf_osnuclear.cpp).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "hfgpu_onee.h"

namespace {

constexpr double kPi = 3.14159265358979323846;

int ncart(int L) { return (L + 1) * (L + 2) / 2; }

void cart_comps(int L, int (*c)[3]) {
  int k = 0;
  for (int i = 0; i <= L; ++i)
    for (int j = 0; j <= i; ++j, ++k) {
      c[k][0] = L - i;
      c[k][1] = i - j;
      c[k][2] = j;
    }
}

double fact(int n) {
  double r = 1;
  for (int i = 2; i <= n; ++i) r *= i;
  return r;
}

double binom(int n, int k) {
  if (k < 0 || k > n) return 0;
  double r = 1;
  for (int i = 1; i <= k; ++i) r = r * (n - k + i) / i;
  return r;
}

// Cartesian -> pure coefficients (ncart x (2L+1)), the reference's Ylm_transmat
// convention (src/math/solid_harmonics.cpp:16-108).
void ylm(int L, double* out) {
  const int nc = ncart(L), np = 2 * L + 1;
  std::fill(out, out + nc * np, 0.0);
  for (int mval = -L; mval <= L; ++mval) {
    const int m = std::abs(mval);
    double prefac = std::pow(2.0, -L);
    if (m) prefac *= std::sqrt(fact(L - m) * 2.0 / fact(L + m));
    for (int k = 0; k <= (L - m) / 2; ++k) {
      double ffac = ((k % 2) ? -1.0 : 1.0) * binom(L, k) * binom(2 * (L - k), L);
      if (m) ffac *= fact(L - 2 * k) / fact(L - 2 * k - m);
      ffac *= prefac;
      for (int a = 0; a <= k; ++a)
        for (int b = 0; b <= a; ++b) {
          const double fac = binom(a, b) * binom(k, a) * ffac;
          const int zexp = 2 * (b - k) + L - m, yexp = 2 * (a - b);
          if (m == 0) {
            const int ii = yexp + zexp;
            out[(ii * (ii + 1) / 2 + zexp) * np + L + mval] += fac;
            continue;
          }
          for (int p = 0; p <= m; ++p) {
            const int r = (m - p) % 4;
            const int f = mval > 0 ? (r == 0 ? 1 : (r == 2 ? -1 : 0)) : (r == 1 ? 1 : (r == 3 ? -1 : 0));
            if (!f) continue;
            const int ii = yexp + m - p + zexp;
            out[(ii * (ii + 1) / 2 + zexp) * np + L + mval] += f * binom(m, p) * fac;
          }
        }
    }
  }
}

// Boys F_m(T), m = 0..M: series for F_M then downward recursion; asymptotic + upward for large T.
void boys(int M, double T, double* F) {
  if (T < 35.0) {
    double term = 1.0 / (2 * M + 1), sum = term;
    for (int i = 0; i < 400; ++i) {
      term *= 2.0 * T / (2 * M + 2 * i + 3);
      sum += term;
      if (term < sum * 1e-17) break;
    }
    const double e = std::exp(-T);
    F[M] = e * sum;
    for (int m = M; m > 0; --m) F[m - 1] = (2.0 * T * F[m] + e) / (2 * m - 1);
  } else {
    const double e = std::exp(-T);
    F[0] = 0.5 * std::sqrt(kPi / T);
    for (int m = 0; m < M; ++m) F[m + 1] = ((2 * m + 1) * F[m] - e) / (2.0 * T);
  }
}

struct Shell1e {
  int L, atom, np, first;
  const double* a;
  const double* c;
  const double* R;
};

constexpr int LM = 6;  // index bound for 1-D tables (L + 2 + 1)

// 1-D overlap table S[i][j], i <= imax, j <= jmax (without the exp prefactor).
void overlap1d(double PA, double PB, double p, int imax, int jmax, double S[LM][LM]) {
  const double i2p = 0.5 / p;
  S[0][0] = std::sqrt(kPi / p);
  for (int i = 0; i <= imax; ++i)
    for (int j = 0; j <= jmax; ++j) {
      if (i == 0 && j == 0) continue;
      double v;
      if (i > 0) {
        v = PA * S[i - 1][j];
        if (i > 1) v += (i - 1) * i2p * S[i - 2][j];
        if (j > 0) v += j * i2p * S[i - 1][j - 1];
      } else {
        v = PB * S[i][j - 1];
        if (j > 1) v += (j - 1) * i2p * S[i][j - 2];
      }
      S[i][j] = v;
    }
}

// Cartesian blocks of one primitive pair, for the requested derivative order on
// centre A (da = 0 or 1, direction dir) of S and T.
struct Blocks {
  double S[36], T[36];
};

double kin1d(const double S[LM][LM], double b, int i, int j) {
  // -1/2 d^2/dx^2 acting on the right function x^j e^{-b x^2}
  double v = -2.0 * b * b * S[i][j + 2] + b * (2 * j + 1) * S[i][j];
  if (j > 1) v -= 0.5 * j * (j - 1) * S[i][j - 2];
  return v;
}

// value of S or T for exponents e1 (on A) and e2 (on B)
void st_value(const double Sx[LM][LM], const double Sy[LM][LM], const double Sz[LM][LM], double b, const int* e1,
              const int* e2, double& s, double& t) {
  const double sx = Sx[e1[0]][e2[0]], sy = Sy[e1[1]][e2[1]], sz = Sz[e1[2]][e2[2]];
  s = sx * sy * sz;
  t = kin1d(Sx, b, e1[0], e2[0]) * sy * sz + sx * kin1d(Sy, b, e1[1], e2[1]) * sz + sx * sy * kin1d(Sz, b, e1[2], e2[2]);
}

// Nuclear attraction primitive table V[a][b] (Cartesian) for one nucleus via 3-D OS VRR on a+b,
// then HRR.  Returns values for the requested bra/ket momenta (la, lb) up to la<=3, lb<=3.
struct NucTab {
  // index by (lx,ly,lz) of total e up to emax with auxiliary m
  double v[8][8][8][10];
};

void nuc_vrr(double PAx, double PAy, double PAz, double PCx, double PCy, double PCz, double p, int emax, const double* F,
             double pre, NucTab& t) {
  const double i2p = 0.5 / p;
  for (int m = 0; m <= emax; ++m) t.v[0][0][0][m] = pre * F[m];
  for (int e = 1; e <= emax; ++e)
    for (int x = e; x >= 0; --x)
      for (int y = e - x; y >= 0; --y) {
        const int z = e - x - y;
        int d = x > 0 ? 0 : (y > 0 ? 1 : 2);
        int c[3] = {x, y, z};
        c[d] -= 1;
        const double PA = d == 0 ? PAx : (d == 1 ? PAy : PAz);
        const double PC = d == 0 ? PCx : (d == 1 ? PCy : PCz);
        for (int m = 0; m <= emax - e; ++m) {
          double v = PA * t.v[c[0]][c[1]][c[2]][m] - PC * t.v[c[0]][c[1]][c[2]][m + 1];
          if (c[d] > 0) {
            int c2[3] = {c[0], c[1], c[2]};
            c2[d] -= 1;
            v += c[d] * i2p * (t.v[c2[0]][c2[1]][c2[2]][m] - t.v[c2[0]][c2[1]][c2[2]][m + 1]);
          }
          t.v[x][y][z][m] = v;
        }
      }
}

// (a|V|b) from [e|V|0] by HRR: (a, b+1_i) = (a+1_i, b) + AB_i (a, b).
double nuc_hrr(const NucTab& t, const double* AB, const int* a, const int* b) {
  int bi = -1;
  for (int d = 0; d < 3; ++d)
    if (b[d] > 0) {
      bi = d;
      break;
    }
  if (bi < 0) return t.v[a[0]][a[1]][a[2]][0];
  int a1[3] = {a[0], a[1], a[2]}, b1[3] = {b[0], b[1], b[2]};
  a1[bi] += 1;
  b1[bi] -= 1;
  return nuc_hrr(t, AB, a1, b1) + AB[bi] * nuc_hrr(t, AB, a, b1);
}

void to_pure2(int la, int lb, const double* cart, double* out) {
  double Ya[30], Yb[30];
  ylm(la, Ya);
  ylm(lb, Yb);
  const int ca = ncart(la), cb = ncart(lb), pa = 2 * la + 1, pb = 2 * lb + 1;
  for (int i = 0; i < pa; ++i)
    for (int j = 0; j < pb; ++j) {
      double v = 0;
      for (int p = 0; p < ca; ++p)
        for (int q = 0; q < cb; ++q) v += Ya[p * pa + i] * Yb[q * pb + j] * cart[p * cb + q];
      out[i * pb + j] = v;
    }
}

// Pure weights back to Cartesian: Wc = Ya W Yb^T.
void from_pure2(int la, int lb, const double* Wp, double* Wc) {
  double Ya[30], Yb[30];
  ylm(la, Ya);
  ylm(lb, Yb);
  const int ca = ncart(la), cb = ncart(lb), pa = 2 * la + 1, pb = 2 * lb + 1;
  for (int p = 0; p < ca; ++p)
    for (int q = 0; q < cb; ++q) {
      double v = 0;
      for (int i = 0; i < pa; ++i)
        for (int j = 0; j < pb; ++j) v += Ya[p * pa + i] * Yb[q * pb + j] * Wp[i * pb + j];
      Wc[p * cb + q] = v;
    }
}

}  // namespace

// Cartesian-block S, T, V for shells (s, t); optional derivative on centre A / B.
// mode 0: values; accumulates into S,T,V (n x n, final basis).
void hfgpu_onee_matrices(const OneEBasis& b, const double* Zc, const double* xyz, int natoms, double* S, double* T,
                         double* V) {
  const int ns = b.nshell, n = b.n;
  std::memset(S, 0, sizeof(double) * n * n);
  std::memset(T, 0, sizeof(double) * n * n);
  std::memset(V, 0, sizeof(double) * n * n);
#pragma omp parallel for schedule(dynamic) if (ns >= 24)
  for (int s = 0; s < ns; ++s)
    for (int t = s; t < ns; ++t) {
      const int la = b.L[s], lb = b.L[t], ca = ncart(la), cb = ncart(lb);
      int ea[10][3], eb[10][3];
      cart_comps(la, ea);
      cart_comps(lb, eb);
      const double* A = xyz + 3 * b.atom[s];
      const double* B = xyz + 3 * b.atom[t];
      const double AB[3] = {A[0] - B[0], A[1] - B[1], A[2] - B[2]};
      const double R2 = AB[0] * AB[0] + AB[1] * AB[1] + AB[2] * AB[2];
      double cs[36] = {0}, ct[36] = {0}, cv[36] = {0};
      for (int i = 0; i < b.nprim[s]; ++i)
        for (int j = 0; j < b.nprim[t]; ++j) {
          const double a1 = b.exps[b.off[s] + i], a2 = b.exps[b.off[t] + j];
          const double p = a1 + a2, mu = a1 * a2 / p;
          const double K = std::exp(-mu * R2) * b.coefs[b.off[s] + i] * b.coefs[b.off[t] + j];
          double P[3], PA[3], PB[3];
          for (int d = 0; d < 3; ++d) {
            P[d] = (a1 * A[d] + a2 * B[d]) / p;
            PA[d] = P[d] - A[d];
            PB[d] = P[d] - B[d];
          }
          double Sx[LM][LM], Sy[LM][LM], Sz[LM][LM];
          overlap1d(PA[0], PB[0], p, la, lb + 2, Sx);
          overlap1d(PA[1], PB[1], p, la, lb + 2, Sy);
          overlap1d(PA[2], PB[2], p, la, lb + 2, Sz);
          for (int x = 0; x < ca; ++x)
            for (int y = 0; y < cb; ++y) {
              double sv, tv;
              st_value(Sx, Sy, Sz, a2, ea[x], eb[y], sv, tv);
              cs[x * cb + y] += K * sv;
              ct[x * cb + y] += K * tv;
            }
          const int emax = la + lb;
          for (int c = 0; c < natoms; ++c) {
            const double* C = xyz + 3 * c;
            const double PC[3] = {P[0] - C[0], P[1] - C[1], P[2] - C[2]};
            double F[12];
            boys(emax, p * (PC[0] * PC[0] + PC[1] * PC[1] + PC[2] * PC[2]), F);
            NucTab tab;
            nuc_vrr(PA[0], PA[1], PA[2], PC[0], PC[1], PC[2], p, emax, F, -Zc[c] * 2.0 * kPi / p * K, tab);
            for (int x = 0; x < ca; ++x)
              for (int y = 0; y < cb; ++y) cv[x * cb + y] += nuc_hrr(tab, AB, ea[x], eb[y]);
          }
        }
      double ps[36], pt[36], pv[36];
      const double *os = cs, *ot = ct, *ov = cv;
      int na = ca, nb = cb;
      if (b.pure) {
        to_pure2(la, lb, cs, ps);
        to_pure2(la, lb, ct, pt);
        to_pure2(la, lb, cv, pv);
        os = ps;
        ot = pt;
        ov = pv;
        na = 2 * la + 1;
        nb = 2 * lb + 1;
      }
      for (int x = 0; x < na; ++x)
        for (int y = 0; y < nb; ++y) {
          const int i = b.first[s] + x, j = b.first[t] + y;
          S[i * n + j] = S[j * n + i] = os[x * nb + y];
          T[i * n + j] = T[j * n + i] = ot[x * nb + y];
          V[i * n + j] = V[j * n + i] = ov[x * nb + y];
        }
    }
}

// grad += cH sum_ij D_ij d(T+V)_ij/dX + cS sum_ij W_ij dS_ij/dX  (all atoms, x y z).
void hfgpu_onee_gradient(const OneEBasis& b, const double* Zc, const double* xyz, int natoms, const double* D,
                         const double* W, double cH, double cS, double* grad) {
  const int ns = b.nshell, n = b.n;
  std::vector<double> g(3 * natoms, 0.0);
#pragma omp parallel if (ns >= 24)
  {
    std::vector<double> gl(3 * natoms, 0.0);
#pragma omp for schedule(dynamic)
    for (int s = 0; s < ns; ++s)
      for (int t = 0; t < ns; ++t) {
        // ordered pairs: every (s, t) contributes its own block, no symmetry factor
        const int la = b.L[s], lb = b.L[t], ca = ncart(la), cb = ncart(lb);
        int ea[10][3], eb[10][3];
        cart_comps(la, ea);
        cart_comps(lb, eb);
        const int atA = b.atom[s], atB = b.atom[t];
        const double* A = xyz + 3 * atA;
        const double* B = xyz + 3 * atB;
        const double AB[3] = {A[0] - B[0], A[1] - B[1], A[2] - B[2]};
        const double R2 = AB[0] * AB[0] + AB[1] * AB[1] + AB[2] * AB[2];
        // Cartesian weight blocks for H (D) and S (W)
        const int na = b.pure ? 2 * la + 1 : ca, nb = b.pure ? 2 * lb + 1 : cb;
        double wd[36], ww[36], wdc[36], wwc[36];
        for (int x = 0; x < na; ++x)
          for (int y = 0; y < nb; ++y) {
            wd[x * nb + y] = cH * D[(b.first[s] + x) * n + b.first[t] + y];
            ww[x * nb + y] = cS * W[(b.first[s] + x) * n + b.first[t] + y];
          }
        if (b.pure) {
          from_pure2(la, lb, wd, wdc);
          from_pure2(la, lb, ww, wwc);
        } else {
          std::memcpy(wdc, wd, sizeof(double) * ca * cb);
          std::memcpy(wwc, ww, sizeof(double) * ca * cb);
        }
        double gA[3] = {0, 0, 0};
        std::vector<double> gC(3 * natoms, 0.0);
        double gAv[3] = {0, 0, 0}, gBv[3] = {0, 0, 0};
        for (int i = 0; i < b.nprim[s]; ++i)
          for (int j = 0; j < b.nprim[t]; ++j) {
            const double a1 = b.exps[b.off[s] + i], a2 = b.exps[b.off[t] + j];
            const double p = a1 + a2, mu = a1 * a2 / p;
            const double K = std::exp(-mu * R2) * b.coefs[b.off[s] + i] * b.coefs[b.off[t] + j];
            double P[3], PA[3], PB[3];
            for (int d = 0; d < 3; ++d) {
              P[d] = (a1 * A[d] + a2 * B[d]) / p;
              PA[d] = P[d] - A[d];
              PB[d] = P[d] - B[d];
            }
            double Sx[LM][LM], Sy[LM][LM], Sz[LM][LM];
            overlap1d(PA[0], PB[0], p, la + 1, lb + 2, Sx);
            overlap1d(PA[1], PB[1], p, la + 1, lb + 2, Sy);
            overlap1d(PA[2], PB[2], p, la + 1, lb + 2, Sz);
            // d/dA of S and T on the bra function (translational invariance gives d/dB = -d/dA)
            for (int x = 0; x < ca; ++x)
              for (int y = 0; y < cb; ++y) {
                const double wh = wdc[x * cb + y], wsv = wwc[x * cb + y];
                for (int d = 0; d < 3; ++d) {
                  int up[3] = {ea[x][0], ea[x][1], ea[x][2]};
                  up[d] += 1;
                  double su, tu;
                  st_value(Sx, Sy, Sz, a2, up, eb[y], su, tu);
                  double ds = 2.0 * a1 * su, dt = 2.0 * a1 * tu;
                  if (ea[x][d] > 0) {
                    int dn[3] = {ea[x][0], ea[x][1], ea[x][2]};
                    dn[d] -= 1;
                    double sd, td;
                    st_value(Sx, Sy, Sz, a2, dn, eb[y], sd, td);
                    ds -= ea[x][d] * sd;
                    dt -= ea[x][d] * td;
                  }
                  gA[d] += K * (wsv * ds + wh * dt);
                }
              }
            // nuclear attraction: d/dA and d/dB by the derivative rule; d/dC by invariance
            const int emax = la + lb + 2;
            int eaug[3];
            (void)eaug;
            for (int c = 0; c < natoms; ++c) {
              const double* C = xyz + 3 * c;
              const double PC[3] = {P[0] - C[0], P[1] - C[1], P[2] - C[2]};
              double F[12];
              boys(emax, p * (PC[0] * PC[0] + PC[1] * PC[1] + PC[2] * PC[2]), F);
              NucTab tab;
              nuc_vrr(PA[0], PA[1], PA[2], PC[0], PC[1], PC[2], p, emax, F, -Zc[c] * 2.0 * kPi / p * K, tab);
              double ga[3] = {0, 0, 0}, gb[3] = {0, 0, 0};
              for (int x = 0; x < ca; ++x)
                for (int y = 0; y < cb; ++y) {
                  const double wh = wdc[x * cb + y];
                  if (wh == 0.0) continue;
                  for (int d = 0; d < 3; ++d) {
                    int up[3] = {ea[x][0], ea[x][1], ea[x][2]};
                    up[d] += 1;
                    double va = 2.0 * a1 * nuc_hrr(tab, AB, up, eb[y]);
                    if (ea[x][d] > 0) {
                      int dn[3] = {ea[x][0], ea[x][1], ea[x][2]};
                      dn[d] -= 1;
                      va -= ea[x][d] * nuc_hrr(tab, AB, dn, eb[y]);
                    }
                    int ub[3] = {eb[y][0], eb[y][1], eb[y][2]};
                    ub[d] += 1;
                    double vb = 2.0 * a2 * nuc_hrr(tab, AB, ea[x], ub);
                    if (eb[y][d] > 0) {
                      int db[3] = {eb[y][0], eb[y][1], eb[y][2]};
                      db[d] -= 1;
                      vb -= eb[y][d] * nuc_hrr(tab, AB, ea[x], db);
                    }
                    ga[d] += wh * va;
                    gb[d] += wh * vb;
                  }
                }
              for (int d = 0; d < 3; ++d) {
                gAv[d] += ga[d];
                gBv[d] += gb[d];
                gC[3 * c + d] -= ga[d] + gb[d];
              }
            }
          }
        for (int d = 0; d < 3; ++d) {
          gl[3 * atA + d] += gA[d] + gAv[d];
          gl[3 * atB + d] += -gA[d] + gBv[d];
        }
        for (int x = 0; x < 3 * natoms; ++x) gl[x] += gC[x];
      }
#pragma omp critical
    for (int x = 0; x < 3 * natoms; ++x) g[x] += gl[x];
  }
  for (int x = 0; x < 3 * natoms; ++x) grad[x] += g[x];
}

// Cartesian -> pure coefficients of shell L (the table the device one-electron kernels use).
void hfgpu_onee_ylm(int L, double* out) { ylm(L, out); }
