/* CPU restatement of hfscf's two-electron algorithms: the test oracle.
 *
 * TEST INFRASTRUCTURE ONLY (see hfscf_oracle.h).  Plain C, written for clarity,
 * not speed; it is meant for molecules of a few dozen basis functions.
 *
 * Integral scheme, as the reference's Erios (src/integrals/hfscf_oseri.cpp:22-246):
 * Obara-Saika recurrences one Cartesian direction at a time.  The x table is
 * built once per primitive quartet carrying the auxiliary (Boys) index n; for each
 * Cartesian component the x values seed the y recurrence as functions of n, and
 * the y values seed the z recurrence (Helgaker, Jorgensen, Olsen, "Molecular
 * Electronic-Structure Theory", p.385).
 */
#include "hfscf_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define OR_LM 4            /* per-index angular momentum bound + 1 (f for derivatives of d) */
#define OR_NM 14           /* auxiliary index bound: 4 * 3 + 1 + 1 */
#define OR_NC 10           /* Cartesian components of an f shell */

static const double OR_PI = 3.14159265358979323846;

/* ---------------------------------------------------------------------------
 * Boys function F_m(T), restating extramath::F_nu (src/math/gamma.cpp:18-24):
 * F_m(x) = x^(-m-1/2) gamma(m+1/2, x) / 2 with x clamped to >= 1e-8 (:20-21),
 * the lower incomplete gamma from the series for x < a+1 and from the continued
 * fraction otherwise (gammp/gser/gcf, :33-135; Numerical Recipes 3rd ed. 6.2).
 * The reference's quadrature branch (a >= 100) is never reached for m <= 13.
 * ------------------------------------------------------------------------- */
double or_boys(int m, double T) {
  const double eps = 2.220446049250313e-16;
  const double fpmin = 2.2250738585072014e-308 / eps;
  const double a = m + 0.5;
  double x = fabs(T);
  if (x < 1e-8) x = 1e-8;
  if (x < a + 1.0) {
    /* gamma(a,x) = e^-x x^a sum_n x^n / (a (a+1) ... (a+n)) */
    double ap = a, del = 1.0 / a, sum = del;
    for (int it = 0; it < 100000; ++it) {
      ap += 1.0;
      del *= x / ap;
      sum += del;
      if (fabs(del) < fabs(sum) * eps) break;
    }
    return 0.5 * sum * exp(-x);
  }
  /* Gamma(a,x) = e^-x x^a h, modified Lentz continued fraction */
  double b = x + 1.0 - a, c = 1.0 / fpmin, d = 1.0 / b, h = d;
  for (int i = 1; i < 100000; ++i) {
    const double an = -i * (i - a);
    b += 2.0;
    d = an * d + b;
    if (fabs(d) < fpmin) d = fpmin;
    c = b + an / c;
    if (fabs(c) < fpmin) c = fpmin;
    d = 1.0 / d;
    const double del = d * c;
    h *= del;
    if (fabs(del - 1.0) <= eps) break;
  }
  return 0.5 * (tgamma(a) * pow(x, -a) - exp(-x) * h);
}

/* Contraction coefficients normalised so the x^L component is normalised,
 * restating BASIS::Shell::Shell (src/integrals/hfscf_shell.cpp:44-54). */
void or_shell_norm(int L, int nprim, const double* alpha, const double* coef, double* out) {
  const double m = L + 1.5, m2 = 0.5 * m;
  double sum = 0.0;
  for (int j = 0; j < nprim; ++j)
    for (int k = 0; k < nprim; ++k)
      sum += coef[j] * coef[k] * pow(alpha[j] * alpha[k], m2) / pow(alpha[j] + alpha[k], m);
  double dfac = 1.0;
  for (int n = 2 * L - 1; n > 1; n -= 2) dfac *= n;
  const double norm = 1.0 / sqrt(sum * pow(OR_PI, 1.5) * dfac / pow(2.0, L));
  for (int j = 0; j < nprim; ++j) out[j] = coef[j] * norm * pow(alpha[j], m2);
}

/* Cartesian component (lx, ly, lz) of index ci inside a shell of momentum L,
 * in the reference's order l = L-i, m = i-j, n = j (src/integrals/hfscf_shell.cpp:27-40). */
static void cart_comp(int L, int ci, int* lmn) {
  int c = 0;
  for (int i = 0; i <= L; ++i)
    for (int j = 0; j <= i; ++j, ++c)
      if (c == ci) {
        lmn[0] = L - i;
        lmn[1] = i - j;
        lmn[2] = j;
        return;
      }
}

static double binom(int n, int k) {
  if (k < 0 || k > n) return 0.0;
  double r = 1.0;
  for (int i = 1; i <= k; ++i) r = r * (n - k + i) / i;
  return r;
}

static double fact(int n) {
  double r = 1.0;
  for (int i = 2; i <= n; ++i) r *= i;
  return r;
}

/* Cartesian -> real solid harmonic matrix, ncart rows x (2L+1) columns m = -L..L,
 * restating hfscfmath::Ylm_transmat / calcYlm_coeff (src/math/solid_harmonics.cpp:16-108). */
void or_ylm(int L, double* out) {
  const int nc = (L + 1) * (L + 2) / 2, np = 2 * L + 1;
  memset(out, 0, sizeof(double) * nc * np);
  for (int mval = -L; mval <= L; ++mval) {
    const int m = abs(mval);
    double prefac = pow(2.0, -L);
    if (m != 0) prefac *= sqrt(fact(L - m) * 2.0 / fact(L + m));
    for (int k = 0; k <= (L - m) / 2; ++k) {
      double ffac = ((k % 2) ? -1.0 : 1.0) * binom(L, k) * binom(2 * (L - k), L);
      if (m != 0) ffac *= fact(L - 2 * k) / fact(L - 2 * k - m);
      ffac *= prefac;
      for (int a = 0; a <= k; ++a) {
        const double afac = binom(k, a) * ffac;
        for (int b = 0; b <= a; ++b) {
          const double fac = binom(a, b) * afac;
          const int zexp = 2 * (b - k) + L - m, yexp = 2 * (a - b);
          if (m == 0) {
            const int ii = yexp + zexp;
            out[(ii * (ii + 1) / 2 + zexp) * np + (L + mval)] += fac;
            continue;
          }
          for (int p = 0; p <= m; ++p) {
            /* cos((m-p) pi/2) for A_m (mval > 0), sin((m-p) pi/2) for B_m (mval < 0) */
            const int r = (m - p) % 4;
            const int f = mval > 0 ? (r == 0 ? 1 : (r == 2 ? -1 : 0)) : (r == 1 ? 1 : (r == 3 ? -1 : 0));
            if (f == 0) continue;
            const int ii = yexp + m - p + zexp;
            out[(ii * (ii + 1) / 2 + zexp) * np + (L + mval)] += f * binom(m, p) * fac;
          }
        }
      }
    }
  }
}

/* Packed 8-fold index, restating hfscfmath::index_ijkl (src/math/hfscf_math.hpp:90-101). */
long long or_index_ijkl(long long i, long long j, long long k, long long l) {
  const long long ij = i > j ? i * (i + 1) / 2 + j : j * (j + 1) / 2 + i;
  const long long kl = k > l ? k * (k + 1) / 2 + l : l * (l + 1) / 2 + k;
  return ij > kl ? ij * (ij + 1) / 2 + kl : kl * (kl + 1) / 2 + ij;
}

long long or_packed_len(long long n) { return n * (n + 1) * (n * n + n + 2) / 8; }

long long or_nbf(int nshell, const int* L, int pure) {
  long long n = 0;
  for (int s = 0; s < nshell; ++s) n += pure ? 2 * L[s] + 1 : (L[s] + 1) * (L[s] + 2) / 2;
  return n;
}

/* ---------------------------------------------------------------------------
 * 1-D Obara-Saika recurrence carrying the auxiliary index, restating
 * os_recursion::osrecur (src/integrals/hfscf_osrecur.hpp:17-81).  On entry
 * J(0,0,0,0,n) holds the seeds for n = 0..nmax; on exit J(l,k,j,i,n) is filled
 * for i<=l1, j<=l2, k<=l3, l<=l4, n <= nmax-i-j-k-l.
 * ------------------------------------------------------------------------- */
#define JI(l, k, j, i, n) (((((l) * OR_LM + (k)) * OR_LM + (j)) * OR_LM + (i)) * OR_NM + (n))

static void os1d(double PQ, double PA, double PB, double QC, double QD, double p2, double q2, double pr,
                 double qr, int l1, int l2, int l3, int l4, int nmax, double* J) {
  const double pq2 = p2 + q2;
  for (int i = 0; i < l1; ++i)
    for (int n = 0; n < nmax - i; ++n) {
      double v = PA * J[JI(0, 0, 0, i, n)] - pr * PQ * J[JI(0, 0, 0, i, n + 1)];
      if (i) v += (i / p2) * (J[JI(0, 0, 0, i - 1, n)] - pr * J[JI(0, 0, 0, i - 1, n + 1)]);
      J[JI(0, 0, 0, i + 1, n)] = v;
    }
  for (int j = 0; j < l2; ++j)
    for (int i = 0; i <= l1; ++i)
      for (int n = 0; n < nmax - i - j; ++n) {
        double v = PB * J[JI(0, 0, j, i, n)] - pr * PQ * J[JI(0, 0, j, i, n + 1)];
        if (i) v += (i / p2) * (J[JI(0, 0, j, i - 1, n)] - pr * J[JI(0, 0, j, i - 1, n + 1)]);
        if (j) v += (j / p2) * (J[JI(0, 0, j - 1, i, n)] - pr * J[JI(0, 0, j - 1, i, n + 1)]);
        J[JI(0, 0, j + 1, i, n)] = v;
      }
  for (int k = 0; k < l3; ++k)
    for (int j = 0; j <= l2; ++j)
      for (int i = 0; i <= l1; ++i)
        for (int n = 0; n < nmax - i - j - k; ++n) {
          double v = QC * J[JI(0, k, j, i, n)] + qr * PQ * J[JI(0, k, j, i, n + 1)];
          if (i) v += (i / pq2) * J[JI(0, k, j, i - 1, n + 1)];
          if (j) v += (j / pq2) * J[JI(0, k, j - 1, i, n + 1)];
          if (k) v += (k / q2) * (J[JI(0, k - 1, j, i, n)] - qr * J[JI(0, k - 1, j, i, n + 1)]);
          J[JI(0, k + 1, j, i, n)] = v;
        }
  for (int l = 0; l < l4; ++l)
    for (int k = 0; k <= l3; ++k)
      for (int j = 0; j <= l2; ++j)
        for (int i = 0; i <= l1; ++i)
          for (int n = 0; n < nmax - i - j - k - l; ++n) {
            double v = QD * J[JI(l, k, j, i, n)] + qr * PQ * J[JI(l, k, j, i, n + 1)];
            if (i) v += (i / pq2) * J[JI(l, k, j, i - 1, n + 1)];
            if (j) v += (j / pq2) * J[JI(l, k, j - 1, i, n + 1)];
            if (k) v += (k / q2) * (J[JI(l, k - 1, j, i, n)] - qr * J[JI(l, k - 1, j, i, n + 1)]);
            if (l) v += (l / q2) * (J[JI(l - 1, k, j, i, n)] - qr * J[JI(l - 1, k, j, i, n + 1)]);
            J[JI(l + 1, k, j, i, n)] = v;
          }
}

typedef struct {
  int nshell, pure;
  const int* L;
  const double* xyz;
  const int* nprim;
  const int* off;    /* first primitive of each shell */
  const double* alpha;
  double* c;         /* normalised coefficients */
  long long* first;  /* first function of each shell in the final basis */
} OrBasis;

static int or_basis_init(OrBasis* b, int nshell, const int* L, const double* xyz, const int* nprim,
                         const double* alpha, const double* coef, int pure) {
  int tot = 0;
  for (int s = 0; s < nshell; ++s) {
    if (L[s] < 0 || L[s] > 3 || nprim[s] < 1) return -1;
    tot += nprim[s];
  }
  int* off = (int*)malloc(sizeof(int) * (nshell + 1));
  double* c = (double*)malloc(sizeof(double) * tot);
  long long* first = (long long*)malloc(sizeof(long long) * (nshell + 1));
  if (!off || !c || !first) return -2;
  off[0] = 0;
  first[0] = 0;
  for (int s = 0; s < nshell; ++s) {
    off[s + 1] = off[s] + nprim[s];
    first[s + 1] = first[s] + (pure ? 2 * L[s] + 1 : (L[s] + 1) * (L[s] + 2) / 2);
    or_shell_norm(L[s], nprim[s], alpha + off[s], coef + off[s], c + off[s]);
  }
  b->nshell = nshell;
  b->pure = pure;
  b->L = L;
  b->xyz = xyz;
  b->nprim = nprim;
  b->off = off;
  b->alpha = alpha;
  b->c = c;
  b->first = first;
  return 0;
}

static void or_basis_free(OrBasis* b) {
  free((void*)b->off);
  free(b->c);
  free(b->first);
}

/* Contracted Cartesian block of shell quartet (s[0] s[1] | s[2] s[3]), laid out
 * [ca][cb][cc][cd].  With dcent >= 0 the block is the first derivative with respect
 * to centre dcent (0..3 = A..D) along direction ddir, using
 * d/dA_x g_a = 2 alpha g_{a+1x} - a_x g_{a-1x}, as the reference's deriv1 code does
 * (src/integrals/hfscf_oserideriv1.cpp:227-231).  Primitive data restate
 * BASIS::ShellPair::set_params (src/integrals/hfscf_shellpair.cpp:33-61); the
 * prefactor, primitive cut and Boys seeding restate hfscf_oseri.cpp:90-118. */
static void cart_block(const OrBasis* b, const int* s, int dcent, int ddir, double* out, double* Jx,
                       double* Jy, double* Jz) {
  const double cutoff = 1e-14, precut = cutoff / 10000.0;
  const double PI_25 = 2.0 * pow(OR_PI, 2.5);
  int Ls[4], nc[4];
  const double* R[4];
  for (int q = 0; q < 4; ++q) {
    Ls[q] = b->L[s[q]];
    nc[q] = (Ls[q] + 1) * (Ls[q] + 2) / 2;
    R[q] = b->xyz + 3 * s[q];
  }
  const int ntot = nc[0] * nc[1] * nc[2] * nc[3];
  memset(out, 0, sizeof(double) * ntot);
  int lt[4];
  for (int q = 0; q < 4; ++q) lt[q] = Ls[q] + (q == dcent ? 1 : 0);
  const int nmax = lt[0] + lt[1] + lt[2] + lt[3];
  double AB[3], CD[3], R2ab = 0, R2cd = 0;
  for (int d = 0; d < 3; ++d) {
    AB[d] = R[0][d] - R[1][d];
    CD[d] = R[2][d] - R[3][d];
    R2ab += AB[d] * AB[d];
    R2cd += CD[d] * CD[d];
  }
  int comp[4][OR_NC][3];
  for (int q = 0; q < 4; ++q)
    for (int ci = 0; ci < nc[q]; ++ci) cart_comp(Ls[q], ci, comp[q][ci]);

  for (int p1 = 0; p1 < b->nprim[s[0]]; ++p1)
    for (int p2 = 0; p2 < b->nprim[s[1]]; ++p2) {
      const double a1 = b->alpha[b->off[s[0]] + p1], a2 = b->alpha[b->off[s[1]] + p2];
      const double g = a1 + a2;
      const double Kab = exp(-a1 * a2 / g * R2ab) * b->c[b->off[s[0]] + p1] * b->c[b->off[s[1]] + p2];
      double P[3], PA[3], PB[3];
      for (int d = 0; d < 3; ++d) {
        P[d] = (a1 * R[0][d] + a2 * R[1][d]) / g;
        PA[d] = P[d] - R[0][d];
        PB[d] = P[d] - R[1][d];
      }
      for (int p3 = 0; p3 < b->nprim[s[2]]; ++p3)
        for (int p4 = 0; p4 < b->nprim[s[3]]; ++p4) {
          const double a3 = b->alpha[b->off[s[2]] + p3], a4 = b->alpha[b->off[s[3]] + p4];
          const double h = a3 + a4;
          const double Kcd = exp(-a3 * a4 / h * R2cd) * b->c[b->off[s[2]] + p3] * b->c[b->off[s[3]] + p4];
          double Q[3], QC[3], QD[3], PQ[3], rpq2 = 0;
          for (int d = 0; d < 3; ++d) {
            Q[d] = (a3 * R[2][d] + a4 * R[3][d]) / h;
            QC[d] = Q[d] - R[2][d];
            QD[d] = Q[d] - R[3][d];
            PQ[d] = P[d] - Q[d];
            rpq2 += PQ[d] * PQ[d];
          }
          const double eta = g * h / (g + h), pr = eta / g, qr = eta / h;
          const double pfac = Kab * Kcd * PI_25 / (g * h * sqrt(g + h));
          if (fabs(pfac) < precut) continue;
          const double T = eta * rpq2, eT = exp(-T);
          if (fabs(rpq2) > 1e-18) {
            Jx[JI(0, 0, 0, 0, nmax)] = or_boys(nmax, T);
            for (int n = nmax - 1; n >= 0; --n) Jx[JI(0, 0, 0, 0, n)] = (2.0 * T * Jx[JI(0, 0, 0, 0, n + 1)] + eT) / (2.0 * n + 1.0);
          } else {
            for (int n = nmax; n >= 0; --n) Jx[JI(0, 0, 0, 0, n)] = 1.0 / (2.0 * n + 1.0);
          }
          os1d(PQ[0], PA[0], PB[0], QC[0], QD[0], 2 * g, 2 * h, pr, qr, lt[0], lt[1], lt[2], lt[3], nmax, Jx);
          const double ex[4] = {2 * a1, 2 * a2, 2 * a3, 2 * a4};
          int idx = 0;
          for (int ia = 0; ia < nc[0]; ++ia)
            for (int ib = 0; ib < nc[1]; ++ib)
              for (int ic = 0; ic < nc[2]; ++ic)
                for (int id = 0; id < nc[3]; ++id, ++idx) {
                  const int* cs[4] = {comp[0][ia], comp[1][ib], comp[2][ic], comp[3][id]};
                  /* up to two terms: (coefficient, component shift) */
                  int nterm = 1;
                  double tc[2] = {1.0, 0.0};
                  int sh[2] = {0, 0};
                  if (dcent >= 0) {
                    tc[0] = ex[dcent];
                    sh[0] = +1;
                    nterm = 1;
                    if (cs[dcent][ddir] > 0) {
                      tc[1] = -(double)cs[dcent][ddir];
                      sh[1] = -1;
                      nterm = 2;
                    }
                  }
                  double acc = 0.0;
                  for (int t = 0; t < nterm; ++t) {
                    int e[4][3];
                    for (int q = 0; q < 4; ++q)
                      for (int d = 0; d < 3; ++d) e[q][d] = cs[q][d];
                    if (dcent >= 0) e[dcent][ddir] += sh[t];
                    const int nx = e[0][0] + e[1][0] + e[2][0] + e[3][0];
                    const int ny = e[0][1] + e[1][1] + e[2][1] + e[3][1];
                    const int nz = e[0][2] + e[1][2] + e[2][2] + e[3][2];
                    const int my = nmax - nx;
                    for (int n = 0; n <= my; ++n) Jy[JI(0, 0, 0, 0, n)] = Jx[JI(e[3][0], e[2][0], e[1][0], e[0][0], n)];
                    os1d(PQ[1], PA[1], PB[1], QC[1], QD[1], 2 * g, 2 * h, pr, qr, e[0][1], e[1][1], e[2][1], e[3][1], my, Jy);
                    const int mz = my - ny;
                    for (int n = 0; n <= mz; ++n) Jz[JI(0, 0, 0, 0, n)] = Jy[JI(e[3][1], e[2][1], e[1][1], e[0][1], n)];
                    os1d(PQ[2], PA[2], PB[2], QC[2], QD[2], 2 * g, 2 * h, pr, qr, e[0][2], e[1][2], e[2][2], e[3][2], mz, Jz);
                    (void)nz;
                    acc += tc[t] * Jz[JI(e[3][2], e[2][2], e[1][2], e[0][2], 0)];
                  }
                  out[idx] += pfac * acc;
                }
        }
    }
}

/* Cartesian -> pure on all four indices, restating TRANSFORM::transform
 * (src/integrals/hfscf_transform.cpp:80-154). */
static void to_pure(const int* Ls, const double* cart, double* pure) {
  double Y[4][OR_NC * 7];
  int nc[4], np[4];
  for (int q = 0; q < 4; ++q) {
    nc[q] = (Ls[q] + 1) * (Ls[q] + 2) / 2;
    np[q] = 2 * Ls[q] + 1;
    or_ylm(Ls[q], Y[q]);
  }
  const int n1 = np[0] * np[1] * np[2] * np[3];
  memset(pure, 0, sizeof(double) * n1);
  for (int i = 0; i < np[0]; ++i)
    for (int j = 0; j < np[1]; ++j)
      for (int k = 0; k < np[2]; ++k)
        for (int l = 0; l < np[3]; ++l) {
          double v = 0.0;
          for (int p = 0; p < nc[0]; ++p) {
            const double y0 = Y[0][p * np[0] + i];
            if (y0 == 0.0) continue;
            for (int q = 0; q < nc[1]; ++q) {
              const double y1 = y0 * Y[1][q * np[1] + j];
              if (y1 == 0.0) continue;
              for (int r = 0; r < nc[2]; ++r) {
                const double y2 = y1 * Y[2][r * np[2] + k];
                if (y2 == 0.0) continue;
                for (int s = 0; s < nc[3]; ++s)
                  v += y2 * Y[3][s * np[3] + l] * cart[((p * nc[1] + q) * nc[2] + r) * nc[3] + s];
              }
            }
          }
          pure[((i * np[1] + j) * np[2] + k) * np[3] + l] = v;
        }
}

static double* or_scratch(void) { return (double*)malloc(sizeof(double) * (3 * OR_LM * OR_LM * OR_LM * OR_LM * OR_NM + 2 * 10000)); }

/* Block in the final basis (pure or Cartesian), [a][b][c][d]. */
static void final_block(const OrBasis* b, const int* s, int dcent, int ddir, double* out, double* scr) {
  double* Jx = scr;
  double* Jy = Jx + OR_LM * OR_LM * OR_LM * OR_LM * OR_NM;
  double* Jz = Jy + OR_LM * OR_LM * OR_LM * OR_LM * OR_NM;
  double* cart = Jz + OR_LM * OR_LM * OR_LM * OR_LM * OR_NM;
  cart_block(b, s, dcent, ddir, cart, Jx, Jy, Jz);
  int Ls[4], n = 1;
  for (int q = 0; q < 4; ++q) {
    Ls[q] = b->L[s[q]];
    n *= (Ls[q] + 1) * (Ls[q] + 2) / 2;
  }
  if (b->pure)
    to_pure(Ls, cart, out);
  else
    memcpy(out, cart, sizeof(double) * n);
}

int or_shell_quartet(int nshell, const int* L, const double* xyz, const int* nprim, const double* alpha,
                     const double* coef, int pure, int si, int sj, int sk, int sl, double* block) {
  OrBasis b;
  if (or_basis_init(&b, nshell, L, xyz, nprim, alpha, coef, pure)) return -1;
  const int s[4] = {si, sj, sk, sl};
  double* scr = or_scratch();
  final_block(&b, s, -1, 0, block, scr);
  free(scr);
  or_basis_free(&b);
  return 0;
}

/* All unique shell quartets into the packed vector, restating
 * Mol::hf_solver::create_repulsion_matrix (src/scfsolver/hfscf_hf_hamiltonian.cpp:93-111)
 * and the packed scatter of Erios (src/integrals/hfscf_oseri.cpp:203-245). */
int or_eri_packed(int nshell, const int* L, const double* xyz, const int* nprim, const double* alpha,
                  const double* coef, int pure, double* eri) {
  OrBasis b;
  if (or_basis_init(&b, nshell, L, xyz, nprim, alpha, coef, pure)) return -1;
  const long long n = b.first[nshell];
  memset(eri, 0, sizeof(double) * or_packed_len(n));
#pragma omp parallel
  {
    double* scr = or_scratch();
    double* blk = (double*)malloc(sizeof(double) * 10000);
#pragma omp for schedule(dynamic)
    for (int i = 0; i < nshell; ++i)
      for (int j = i; j < nshell; ++j) {
        const long long ij = (long long)j * (j + 1) / 2 + i;
        for (int k = 0; k < nshell; ++k)
          for (int l = k; l < nshell; ++l) {
            const long long kl = (long long)l * (l + 1) / 2 + k;
            if (ij > kl) continue;
            const int s[4] = {i, j, k, l};
            final_block(&b, s, -1, 0, blk, scr);
            const long long f[4] = {b.first[i], b.first[j], b.first[k], b.first[l]};
            const long long m[4] = {b.first[i + 1] - f[0], b.first[j + 1] - f[1], b.first[k + 1] - f[2],
                                    b.first[l + 1] - f[3]};
            for (long long p = 0; p < m[0]; ++p)
              for (long long q = 0; q < m[1]; ++q)
                for (long long r = 0; r < m[2]; ++r)
                  for (long long t = 0; t < m[3]; ++t)
                    if (f[0] + p <= f[1] + q && f[2] + r <= f[3] + t)
                      eri[or_index_ijkl(f[0] + p, f[1] + q, f[2] + r, f[3] + t)] =
                          blk[((p * m[1] + q) * m[2] + r) * m[3] + t];
          }
      }
    free(scr);
    free(blk);
  }
  or_basis_free(&b);
  return 0;
}

/* F = H + sum_kl D_kl (2 (ij|kl) - (ik|jl)), restating Mol::hf_solver::update_fock_matrix
 * (src/scfsolver/hfscf_hf_solver.cpp:254-286); D carries no factor 2 (:221-231). */
int or_fock_rhf(long long n, const double* eri, const double* D, const double* H, double* F) {
#pragma omp parallel for schedule(dynamic)
  for (long long i = 0; i < n; ++i)
    for (long long j = i; j < n; ++j) {
      double f = H[i * n + j];
      for (long long k = 0; k < n; ++k)
        for (long long l = 0; l < n; ++l)
          f += D[k * n + l] * (2.0 * eri[or_index_ijkl(i, j, k, l)] - eri[or_index_ijkl(i, k, j, l)]);
      F[i * n + j] = F[j * n + i] = f;
    }
  return 0;
}

/* UHF Fock matrices, restating Mol::uhf_solver::update_fock_matrix
 * (src/scfsolver/hfscf_uhf_solver.cpp:155-191). */
int or_fock_uhf(long long n, const double* eri, const double* Da, const double* Db, const double* H,
                double* Fa, double* Fb) {
#pragma omp parallel for schedule(dynamic)
  for (long long i = 0; i < n; ++i)
    for (long long j = i; j < n; ++j) {
      double fa = H[i * n + j], fb = fa;
      for (long long k = 0; k < n; ++k)
        for (long long l = 0; l < n; ++l) {
          const double c = eri[or_index_ijkl(i, j, k, l)], x = eri[or_index_ijkl(i, k, j, l)];
          fa += Da[k * n + l] * (c - x) + Db[k * n + l] * c;
          fb += Db[k * n + l] * (c - x) + Da[k * n + l] * c;
        }
      Fa[i * n + j] = Fa[j * n + i] = fa;
      Fb[i * n + j] = Fb[j * n + i] = fb;
    }
  return 0;
}

/* J_ij = sum_kl D_kl (ij|kl), K_ij = sum_kl D_kl (ik|jl), the two halves of the
 * contraction in hfscf_hf_solver.cpp:266-273. */
int or_jk(long long n, const double* eri, const double* D, double* J, double* K) {
#pragma omp parallel for schedule(dynamic)
  for (long long i = 0; i < n; ++i)
    for (long long j = 0; j < n; ++j) {
      double jv = 0.0, kv = 0.0;
      for (long long k = 0; k < n; ++k)
        for (long long l = 0; l < n; ++l) {
          jv += D[k * n + l] * eri[or_index_ijkl(i, j, k, l)];
          kv += D[k * n + l] * eri[or_index_ijkl(i, k, j, l)];
        }
      J[i * n + j] = jv;
      K[i * n + j] = kv;
    }
  return 0;
}

/* Two-electron gradient at fixed density:
 *   dE/dX = sum_pqrs d(pq|rs)/dX [cJ DJ_pq DJ_rs - cK sum_m DK_m,pr DK_m,qs].
 * RHF (cJ = 2, one DK = D, cK = 1) is the contraction of
 * src/gradient/hfscf_grad_rhf.cpp:121-141 with dV/dX assembled as
 * src/gradient/hfscf_grad_ints.cpp:79-108 (centre D by translational invariance).
 * All ordered shell quartets are visited, so no degeneracy factors appear. */
int or_grad2e(int nshell, const int* L, const double* xyz, const int* nprim, const double* alpha,
              const double* coef, int pure, const int* shell_atom, int natoms, const double* DJ, double cJ,
              int nK, const double* DK, double cK, double* grad) {
  OrBasis b;
  if (or_basis_init(&b, nshell, L, xyz, nprim, alpha, coef, pure)) return -1;
  const long long n = b.first[nshell];
  memset(grad, 0, sizeof(double) * 3 * natoms);
#pragma omp parallel
  {
    double* scr = or_scratch();
    double* blk = (double*)malloc(sizeof(double) * 10000);
    double* W = (double*)malloc(sizeof(double) * 10000);
    double* g = (double*)calloc(3 * natoms, sizeof(double));
#pragma omp for schedule(dynamic)
    for (int i = 0; i < nshell; ++i)
      for (int j = 0; j < nshell; ++j)
        for (int k = 0; k < nshell; ++k)
          for (int l = 0; l < nshell; ++l) {
            const int s[4] = {i, j, k, l};
            const long long f[4] = {b.first[i], b.first[j], b.first[k], b.first[l]};
            const long long m[4] = {b.first[i + 1] - f[0], b.first[j + 1] - f[1], b.first[k + 1] - f[2],
                                    b.first[l + 1] - f[3]};
            for (long long p = 0; p < m[0]; ++p)
              for (long long q = 0; q < m[1]; ++q)
                for (long long r = 0; r < m[2]; ++r)
                  for (long long t = 0; t < m[3]; ++t) {
                    const long long P = f[0] + p, Q = f[1] + q, R = f[2] + r, S = f[3] + t;
                    double w = cJ * DJ[P * n + Q] * DJ[R * n + S];
                    for (int x = 0; x < nK; ++x) w -= cK * DK[x * n * n + P * n + R] * DK[x * n * n + Q * n + S];
                    W[((p * m[1] + q) * m[2] + r) * m[3] + t] = w;
                  }
            const long long nb = m[0] * m[1] * m[2] * m[3];
            for (int cen = 0; cen < 3; ++cen)
              for (int dir = 0; dir < 3; ++dir) {
                final_block(&b, s, cen, dir, blk, scr);
                double acc = 0.0;
                for (long long e = 0; e < nb; ++e) acc += W[e] * blk[e];
                g[3 * shell_atom[s[cen]] + dir] += acc;
                g[3 * shell_atom[l] + dir] -= acc;
              }
          }
#pragma omp critical
    for (int x = 0; x < 3 * natoms; ++x) grad[x] += g[x];
    free(scr);
    free(blk);
    free(W);
    free(g);
  }
  or_basis_free(&b);
  return 0;
}

/* J[D_m] and K[D_m] for nd densities from the packed 8-fold ERI vector, visiting each
 * unique integral once.  The same sums as the contraction of Mol::hf_solver::update_fock_matrix
 * (src/scfsolver/hfscf_hf_solver.cpp:261-278): J_ij = sum_kl D_kl (ij|kl), K_ij = sum_kl D_kl (ik|jl),
 * written as a scatter over the eight index images of (ij|kl) (i >= j, k >= l, ij >= kl) with
 * each image weighted by 1 / (number of coinciding images), so that an N = 250 basis takes
 * seconds instead of the N^4 gathers of the row-by-row form (or_jk, or_fock_rhf).
 * Densities need not be symmetric; J and K are n x n, row-major. */
int or_jk_packed(long long n, const double* eri, int nd, const double* D, double* J, double* K) {
  const long long nn = n * n;
  memset(J, 0, sizeof(double) * nn * nd);
  memset(K, 0, sizeof(double) * nn * nd);
#pragma omp parallel
  {
    double* Jt = (double*)calloc((size_t)(nn * nd), sizeof(double));
    double* Kt = (double*)calloc((size_t)(nn * nd), sizeof(double));
#pragma omp for schedule(dynamic, 1)
    for (long long i = n - 1; i >= 0; --i)
      for (long long j = 0; j <= i; ++j) {
        const long long ij = i * (i + 1) / 2 + j;
        for (long long k = 0; k <= i; ++k)
          for (long long l = 0; l <= k; ++l) {
            const long long kl = k * (k + 1) / 2 + l;
            if (kl > ij) break;
            const double v0 = eri[ij * (ij + 1) / 2 + kl];
            if (v0 == 0.0) continue;
            double w = v0;
            if (i == j) w *= 0.5;
            if (k == l) w *= 0.5;
            if (ij == kl) w *= 0.5;
            /* the eight images (p q | r s) of (i j | k l) */
            const long long im[8][4] = {{i, j, k, l}, {j, i, k, l}, {i, j, l, k}, {j, i, l, k},
                                        {k, l, i, j}, {l, k, i, j}, {k, l, j, i}, {l, k, j, i}};
            for (int m = 0; m < nd; ++m) {
              const double* Dm = D + m * nn;
              double* Jm = Jt + m * nn;
              double* Km = Kt + m * nn;
              for (int x = 0; x < 8; ++x) {
                const long long p = im[x][0], q = im[x][1], r = im[x][2], t = im[x][3];
                Jm[p * n + q] += w * Dm[r * n + t];
                Km[p * n + r] += w * Dm[q * n + t];
              }
            }
          }
      }
#pragma omp critical
    for (long long x = 0; x < nn * nd; ++x) {
      J[x] += Jt[x];
      K[x] += Kt[x];
    }
    free(Jt);
    free(Kt);
  }
  return 0;
}

/* Two-electron gradient from the reference's nine packed first-derivative tensors
 * (d/dXa, d/dXb, d/dXc, d/dYa, ..., d/dZc, each of the packed 8-fold length, from
 * Erios::compute_contracted_shell_quartet_deriv1).  Restates the dV/dX assembly of
 * Mol::scf_gradient::calc_coulomb_exchange_integrals (src/gradient/hfscf_grad_ints.cpp:79-108:
 * over canonical slots i >= j, k >= l, ij <= kl, the derivative belongs to the atom of function
 * i (A), j (B), k (C), and -(A + B + C) to the atom of l) and the contraction of
 * calc_scf_gradient_rhf (src/gradient/hfscf_grad_rhf.cpp:121-141), summed over all atoms at
 * once: every slot carries the sum, over its distinct index images (pq|rs), of
 * cJ DJ_pq DJ_rs - cK sum_m DK_m,pr DK_m,qs (RHF: cJ = 2, DK = {D}, cK = 1). */
int or_grad2e_from_deriv1(long long n, const double* deriv9, const int* bf_atom, int natoms, const double* DJ,
                          double cJ, int nK, const double* DK, double cK, double* grad) {
  const long long len = or_packed_len(n);
  const long long nn = n * n;
  memset(grad, 0, sizeof(double) * 3 * natoms);
#pragma omp parallel
  {
    double* g = (double*)calloc((size_t)(3 * natoms), sizeof(double));
#pragma omp for schedule(dynamic, 1)
    for (long long i = n - 1; i >= 0; --i)
      for (long long j = 0; j <= i; ++j) {
        const long long ij = i * (i + 1) / 2 + j;
        for (long long k = i; k < n; ++k)
          for (long long l = 0; l <= k; ++l) {
            const long long kl = k * (k + 1) / 2 + l;
            if (kl < ij) continue;
            const long long slot = kl * (kl + 1) / 2 + ij;
            double f = 1.0;
            if (i == j) f *= 0.5;
            if (k == l) f *= 0.5;
            if (ij == kl) f *= 0.5;
            const long long im[8][4] = {{i, j, k, l}, {j, i, k, l}, {i, j, l, k}, {j, i, l, k},
                                        {k, l, i, j}, {l, k, i, j}, {k, l, j, i}, {l, k, j, i}};
            double w = 0.0;
            for (int x = 0; x < 8; ++x) {
              const long long p = im[x][0], q = im[x][1], r = im[x][2], t = im[x][3];
              double v = cJ * DJ[p * n + q] * DJ[r * n + t];
              for (int m = 0; m < nK; ++m) v -= cK * DK[m * nn + p * n + r] * DK[m * nn + q * n + t];
              w += f * v;
            }
            if (w == 0.0) continue;
            for (int d = 0; d < 3; ++d) {
              const double A = deriv9[(3 * d + 0) * len + slot], B = deriv9[(3 * d + 1) * len + slot];
              const double C = deriv9[(3 * d + 2) * len + slot];
              g[3 * bf_atom[i] + d] += w * A;
              g[3 * bf_atom[j] + d] += w * B;
              g[3 * bf_atom[k] + d] += w * C;
              g[3 * bf_atom[l] + d] -= w * (A + B + C);
            }
          }
      }
#pragma omp critical
    for (int x = 0; x < 3 * natoms; ++x) grad[x] += g[x];
    free(g);
  }
  return 0;
}
