// One-electron integrals and their first derivatives on the device: overlap S, kinetic
// energy T and nuclear attraction V over the handle's shell pairs, and the one-electron
// part of the SCF gradient contracted with the densities on the fly.
//
// Reference routines restated: OSOVERLAP::OSOverlap::compute_contracted_shell
// (src/integrals/hfscf_osoverlap.cpp:10-61, S and T), OSNUCLEAR::OSNuclear::compute_contracted_shell
// (src/integrals/hfscf_osnuclear.cpp:17), and their _deriv1 forms
// (hfscf_osoverlapderiv1.cpp:8, hfscf_oskineticderiv1.cpp:8, hfscf_osnuclearderiv1.cpp:15)
// with the per-atom assembly of src/gradient/hfscf_grad_ints.cpp:14-77,153-199.
//
// Method.  S and T factor into one-dimensional Obara-Saika overlaps per direction,
//   s(i+1, j) = PA s(i, j) + (i s(i-1, j) + j s(i, j-1)) / 2p,   s(i, j+1) = PB s + (same),
// with the kinetic factor t(i, j) = -2 b^2 s(i, j+2) + b (2j+1) s(i, j) - j(j-1)/2 s(i, j-2).
// V uses the Obara-Saika recurrence on the bra with the auxiliary index,
//   Th(e+1_i)^m = PA_i Th(e)^m - PC_i Th(e)^(m+1) + e_i/2p (Th(e-1_i)^m - Th(e-1_i)^(m+1)),
//   Th(0)^m = F_m(p |PC|^2),
// and moves angular momentum to the ket with the binomial transfer
//   (a|b) = sum_k prod_i C(b_i, k_i) AB_i^(b_i - k_i) Th(a + k)     (AB = A - B).
// Derivatives: d/dA_i g_a = 2 alpha g_(a+1_i) - a_i g_(a-1_i) (the same rule as the two-electron
// gradient); for S and T the B derivative is minus the A derivative; for the nucleus C it is
// minus the sum of the A and B derivatives of that nucleus's term.
#pragma once
#include "hfgpu_common.cuh"

namespace onee {

__host__ __device__ constexpr int nc(int L) { return (L + 1) * (L + 2) / 2; }
__host__ __device__ constexpr int off(int L) { return L * (L + 1) * (L + 2) / 6; }

// exponents of component c of a shell of angular momentum L (the reference's order,
// l = L - i, m = i - j, n = j)
__device__ __forceinline__ void comp(int L, int c, int& x, int& y, int& z) {
  int i = 0;
  while ((i + 1) * (i + 2) / 2 <= c) ++i;
  const int j = c - i * (i + 1) / 2;
  x = L - i;
  y = i - j;
  z = j;
}
// index of (x, y, z) among all components of total degree <= x + y + z
__device__ __forceinline__ int gidx(int x, int y, int z) {
  const int L = x + y + z, i = L - x;
  return off(L) + i * (i + 1) / 2 + z;
}
__device__ __forceinline__ double binom(int n, int k) {
  double r = 1.0;
  for (int q = 1; q <= k; ++q) r = r * (n - k + q) / q;
  return r;
}

struct Atoms {
  const double* xyzZ;     // x, y, z, Z per atom (bohr)
  const int* mol_atom;    // atoms of molecule m: [mol_atom[m], mol_atom[m + 1])
  int slots;              // work items per shell pair: the largest molecule's atom count + 1
};

// Primitive-pair scalars.  Kp of PrimPair is K sqrt(2 pi^2.5) / p (scaled for the ERIs); the
// overlap prefactor K (pi/p)^1.5 and the nuclear prefactor 2 pi K / p follow from it.
__device__ __forceinline__ double ovl_pref(const PrimPair<double>& q) {
  return q.Kp * 0.941396263776714812 * rsqrt(q.p);  // pi^0.25 / sqrt(2)
}
__device__ __forceinline__ double nuc_pref(const PrimPair<double>& q) {
  return q.Kp * 1.062251932027196914;  // sqrt(2) pi^-0.25
}

// 1-D overlap table s[i][j], i <= IMAX, j <= JMAX, for one direction.
template <int IMAX, int JMAX>
__device__ __forceinline__ void ovl1d(double PA, double PB, double i2p, double (&s)[IMAX + 1][JMAX + 1]) {
  s[0][0] = 1.0;
#pragma unroll
  for (int i = 0; i <= IMAX; ++i) {
    if (i > 0) s[i][0] = PA * s[i - 1][0] + (i > 1 ? (i - 1) * i2p * s[i - 2][0] : 0.0);
#pragma unroll
    for (int j = 1; j <= JMAX; ++j)
      s[i][j] = PB * s[i][j - 1] + i2p * ((i > 0 ? i * s[i - 1][j - 1] : 0.0) + (j > 1 ? (j - 1) * s[i][j - 2] : 0.0));
  }
}

// Kinetic factor t(i, j) from the overlap table (needs s up to j + 2); b and b2 are the ket
// exponent and its square (means over the two orders for a folded self pair: t is linear in both).
template <int NI, int NJ>
__device__ __forceinline__ double kin1d(const double (&s)[NI][NJ], double b, double b2, int i, int j) {
  double t = -2.0 * b2 * s[i][j + 2] + b * (2 * j + 1) * s[i][j];
  if (j > 1) t -= 0.5 * j * (j - 1) * s[i][j - 2];
  return t;
}

// S and T Cartesian blocks (row a of shell LA, column b of shell LB) of one pair.
template <int LA, int LB>
__device__ void st_block(const PairInfo& P, const PrimPair<double>* __restrict__ pp, const double* __restrict__ eb,
                         double* S, double* T) {
  constexpr int NA = nc(LA), NB = nc(LB);
  for (int x = 0; x < NA * NB; ++x) S[x] = T[x] = 0.0;
  for (int k = 0; k < P.nprim; ++k) {
    const PrimPair<double> q = pp[k];
    const double b = eb[k], b2 = q.eb2, i2p = 0.5 * q.ip, pre = ovl_pref(q);
    double sx[LA + 1][LB + 3], sy[LA + 1][LB + 3], sz[LA + 1][LB + 3];
    ovl1d<LA, LB + 2>(q.PAx, q.PAx + P.ABx, i2p, sx);
    ovl1d<LA, LB + 2>(q.PAy, q.PAy + P.ABy, i2p, sy);
    ovl1d<LA, LB + 2>(q.PAz, q.PAz + P.ABz, i2p, sz);
    for (int ca = 0; ca < NA; ++ca) {
      int ax, ay, az;
      comp(LA, ca, ax, ay, az);
      for (int cb = 0; cb < NB; ++cb) {
        int bx, by, bz;
        comp(LB, cb, bx, by, bz);
        const double X = sx[ax][bx], Y = sy[ay][by], Z = sz[az][bz];
        S[ca * NB + cb] += pre * X * Y * Z;
        T[ca * NB + cb] += pre * (kin1d(sx, b, b2, ax, bx) * Y * Z + X * kin1d(sy, b, b2, ay, by) * Z +
                                  X * Y * kin1d(sz, b, b2, az, bz));
      }
    }
  }
}

// sum over the block of wS dS/dA + wT dT/dA (A = centre of the bra shell), per direction.
template <int LA, int LB>
__device__ void st_grad(const PairInfo& P, const PrimPair<double>* __restrict__ pp, const double* __restrict__ ea,
                        const double* __restrict__ eb, const double* wS, const double* wT, double* g) {
  constexpr int NA = nc(LA), NB = nc(LB);
  g[0] = g[1] = g[2] = 0.0;
  for (int k = 0; k < P.nprim; ++k) {
    const PrimPair<double> q = pp[k];
    const double a = ea[k], b = eb[k], b2 = q.eb2, i2p = 0.5 * q.ip, pre = ovl_pref(q);
    double s[3][LA + 2][LB + 3];
    ovl1d<LA + 1, LB + 2>(q.PAx, q.PAx + P.ABx, i2p, s[0]);
    ovl1d<LA + 1, LB + 2>(q.PAy, q.PAy + P.ABy, i2p, s[1]);
    ovl1d<LA + 1, LB + 2>(q.PAz, q.PAz + P.ABz, i2p, s[2]);
    for (int ca = 0; ca < NA; ++ca) {
      int ae[3];
      comp(LA, ca, ae[0], ae[1], ae[2]);
      for (int cb = 0; cb < NB; ++cb) {
        int be[3];
        comp(LB, cb, be[0], be[1], be[2]);
        const double ws = wS[ca * NB + cb], wt = wT[ca * NB + cb];
        if (ws == 0.0 && wt == 0.0) continue;
        double sv[3], tv[3], ds[3], dt[3];
        for (int d = 0; d < 3; ++d) {
          const int i = ae[d], j = be[d];
          sv[d] = s[d][i][j];
          tv[d] = kin1d(s[d], b, b2, i, j);
          ds[d] = 2.0 * a * s[d][i + 1][j] - (i > 0 ? i * s[d][i - 1][j] : 0.0);
          dt[d] = 2.0 * a * kin1d(s[d], b, b2, i + 1, j) - (i > 0 ? i * kin1d(s[d], b, b2, i - 1, j) : 0.0);
        }
        for (int d = 0; d < 3; ++d) {
          const int d1 = (d + 1) % 3, d2 = (d + 2) % 3;
          const double dS = ds[d] * sv[d1] * sv[d2];
          const double dT = dt[d] * sv[d1] * sv[d2] + ds[d] * (tv[d1] * sv[d2] + sv[d1] * tv[d2]);
          g[d] += pre * (ws * dS + wt * dT);
        }
      }
    }
  }
}

// Th(e)^(0) for |e| <= LT of one primitive pair and nucleus C, into th0[off(LT + 1)].
template <int LT>
__device__ __forceinline__ void nuc_theta(const PrimPair<double>& q, double Cx, double Cy, double Cz,
                                          const BoysTable<double>& boys, double* th0) {
  constexpr int NE = off(LT + 1);
  double th[NE][LT + 1];
  const double PCx = q.Px - Cx, PCy = q.Py - Cy, PCz = q.Pz - Cz;
  const double T = q.p * (PCx * PCx + PCy * PCy + PCz * PCz);
  double F[LT + 1];
  boys.template eval<LT>(T, 1.0, F);
  for (int m = 0; m <= LT; ++m) th[0][m] = F[m];
  const double i2p = 0.5 * q.ip;
  const double PA[3] = {q.PAx, q.PAy, q.PAz}, PC[3] = {PCx, PCy, PCz};
  for (int L = 1; L <= LT; ++L)
    for (int c = 0; c < nc(L); ++c) {
      int e[3];
      comp(L, c, e[0], e[1], e[2]);
      const int d = e[0] > 0 ? 0 : (e[1] > 0 ? 1 : 2);
      e[d] -= 1;  // e' = e - 1_d
      const int g = off(L) + c, g1 = gidx(e[0], e[1], e[2]);
      const int k = e[d];
      int g2 = 0;
      if (k > 0) {
        e[d] -= 1;
        g2 = gidx(e[0], e[1], e[2]);
      }
      for (int m = 0; m <= LT - L; ++m) {
        double v = PA[d] * th[g1][m] - PC[d] * th[g1][m + 1];
        if (k > 0) v += k * i2p * (th[g2][m] - th[g2][m + 1]);
        th[g][m] = v;
      }
    }
  for (int x = 0; x < NE; ++x) th0[x] = th[x][0];
}

// (a|b) from th0 by the binomial transfer, a and b given by exponents.
__device__ __forceinline__ double transfer(const double* th0, const int* a, const int* b, const double* AB) {
  double v = 0.0;
  for (int kx = 0; kx <= b[0]; ++kx) {
    const double fx = binom(b[0], kx) * pow(AB[0], b[0] - kx);
    for (int ky = 0; ky <= b[1]; ++ky) {
      const double fy = fx * binom(b[1], ky) * pow(AB[1], b[1] - ky);
      for (int kz = 0; kz <= b[2]; ++kz) {
        const double f = fy * binom(b[2], kz) * pow(AB[2], b[2] - kz);
        v += f * th0[gidx(a[0] + kx, a[1] + ky, a[2] + kz)];
      }
    }
  }
  return v;
}

// V block of one nucleus (charge Zc at C): V[a][b] += -Zc (a|1/r_C|b).
template <int LA, int LB>
__device__ void v_block(const PairInfo& P, const PrimPair<double>* __restrict__ pp, double Cx, double Cy, double Cz,
                        double Zc, const BoysTable<double>& boys, double* V) {
  constexpr int NA = nc(LA), NB = nc(LB), LT = LA + LB;
  const double AB[3] = {P.ABx, P.ABy, P.ABz};
  for (int x = 0; x < NA * NB; ++x) V[x] = 0.0;
  double th0[off(LT + 1)];
  for (int k = 0; k < P.nprim; ++k) {
    const PrimPair<double> q = pp[k];
    nuc_theta<LT>(q, Cx, Cy, Cz, boys, th0);
    const double pre = -Zc * nuc_pref(q);
    for (int ca = 0; ca < NA; ++ca) {
      int a[3];
      comp(LA, ca, a[0], a[1], a[2]);
      for (int cb = 0; cb < NB; ++cb) {
        int b[3];
        comp(LB, cb, b[0], b[1], b[2]);
        V[ca * NB + cb] += pre * transfer(th0, a, b, AB);
      }
    }
  }
}

// sum over the block of w dV_C/dA and w dV_C/dB for one nucleus, per direction.
template <int LA, int LB>
__device__ void v_grad(const PairInfo& P, const PrimPair<double>* __restrict__ pp, const double* __restrict__ ea,
                       const double* __restrict__ eb, double Cx, double Cy, double Cz, double Zc,
                       const BoysTable<double>& boys, const double* w, double* gA, double* gB) {
  constexpr int NA = nc(LA), NB = nc(LB), LT = LA + LB + 1;
  const double AB[3] = {P.ABx, P.ABy, P.ABz};
  for (int d = 0; d < 3; ++d) gA[d] = gB[d] = 0.0;
  double th0[off(LT + 1)];
  for (int k = 0; k < P.nprim; ++k) {
    const PrimPair<double> q = pp[k];
    nuc_theta<LT>(q, Cx, Cy, Cz, boys, th0);
    const double pre = -Zc * nuc_pref(q), al = 2.0 * ea[k], be = 2.0 * eb[k];
    for (int ca = 0; ca < NA; ++ca) {
      int a[3];
      comp(LA, ca, a[0], a[1], a[2]);
      for (int cb = 0; cb < NB; ++cb) {
        const double wab = w[ca * NB + cb];
        if (wab == 0.0) continue;
        int b[3];
        comp(LB, cb, b[0], b[1], b[2]);
        for (int d = 0; d < 3; ++d) {
          int a1[3] = {a[0], a[1], a[2]}, b1[3] = {b[0], b[1], b[2]};
          a1[d] += 1;
          double da = al * transfer(th0, a1, b, AB);
          if (a[d] > 0) {
            a1[d] -= 2;
            da -= a[d] * transfer(th0, a1, b, AB);
          }
          b1[d] += 1;
          double db = be * transfer(th0, a, b1, AB);
          if (b[d] > 0) {
            b1[d] -= 2;
            db -= b[d] * transfer(th0, a, b1, AB);
          }
          gA[d] += pre * wab * da;
          gB[d] += pre * wab * db;
        }
      }
    }
  }
}

struct Args {
  const PairInfo* pairs;
  const PrimPair<double>* prims;
  const double* alpha_a;  // exponent of the bra primitive of every primitive pair
  const double* alpha_b;
  int npairs;
  BoysTable<double> boys;
  Atoms atoms;
  const double* ylm;      // [3][6 * 5]: Cartesian -> pure of L = 0, 1, 2 (row-major ncart x npure)
  int pure;
  int n;                  // functions (single molecule)
  const long long* mol_off;  // batched handles: block offsets and sizes (else null)
  const int* mol_n;
};

__device__ __forceinline__ void block_of(const Args& a, int mol, long long& off_out, int& n_out) {
  if (a.mol_off) {
    off_out = a.mol_off[mol];
    n_out = a.mol_n[mol];
  } else {
    off_out = 0;
    n_out = a.n;
  }
}

// Cartesian block -> final basis block (pure: Y_a^T M Y_b).
template <int LA, int LB>
__device__ void to_final(const Args& a, const double* Mc, double* Mf, int& na, int& nb) {
  constexpr int NA = nc(LA), NB = nc(LB);
  if (!a.pure) {
    na = NA;
    nb = NB;
    for (int x = 0; x < NA * NB; ++x) Mf[x] = Mc[x];
    return;
  }
  constexpr int PA_ = 2 * LA + 1, PB_ = 2 * LB + 1;
  const double* Ya = a.ylm + LA * 30;
  const double* Yb = a.ylm + LB * 30;
  na = PA_;
  nb = PB_;
  for (int i = 0; i < PA_; ++i)
    for (int j = 0; j < PB_; ++j) {
      double v = 0.0;
      for (int ca = 0; ca < NA; ++ca) {
        const double ya = Ya[ca * PA_ + i];
        if (ya == 0.0) continue;
        for (int cb = 0; cb < NB; ++cb) v += ya * Mc[ca * NB + cb] * Yb[cb * PB_ + j];
      }
      Mf[i * PB_ + j] = v;
    }
}

// Final-basis weight block (the density entries of the pair) -> Cartesian weights (Y_a W Y_b^T).
template <int LA, int LB>
__device__ void weights(const Args& a, const double* M, long long off, int nm, int fa, int fb, double scale,
                        double* Wc) {
  constexpr int NA = nc(LA), NB = nc(LB);
  if (!a.pure) {
    for (int i = 0; i < NA; ++i)
      for (int j = 0; j < NB; ++j) Wc[i * NB + j] = scale * M[off + (long long)(fa + i) * nm + fb + j];
    return;
  }
  constexpr int PA_ = 2 * LA + 1, PB_ = 2 * LB + 1;
  const double* Ya = a.ylm + LA * 30;
  const double* Yb = a.ylm + LB * 30;
  for (int ca = 0; ca < NA; ++ca)
    for (int cb = 0; cb < NB; ++cb) {
      double v = 0.0;
      for (int i = 0; i < PA_; ++i) {
        const double ya = Ya[ca * PA_ + i];
        if (ya == 0.0) continue;
        for (int j = 0; j < PB_; ++j) v += ya * M[off + (long long)(fa + i) * nm + fb + j] * Yb[cb * PB_ + j];
      }
      Wc[ca * NB + cb] = scale * v;
    }
}

// Work item t: shell pair t / slots; slot t % slots is a nucleus of the pair's molecule, or
// (last slot) the overlap/kinetic item.  Returns false for slots past the molecule's atoms.
__device__ __forceinline__ bool item(const Args& a, long long t, int& pair, int& atom) {
  pair = (int)(t / a.atoms.slots);
  const int slot = (int)(t % a.atoms.slots);
  if (slot == a.atoms.slots - 1) {
    atom = -1;
    return true;
  }
  const int mol = a.pairs[pair].mol;
  const int a0 = a.atoms.mol_atom[mol], a1 = a.atoms.mol_atom[mol + 1];
  atom = a0 + slot;
  return atom < a1;
}

template <int LA, int LB>
__device__ void matrices_item(const Args& a, const PairInfo& P, int atom, double* S, double* T, double* V) {
  constexpr int NA = nc(LA), NB = nc(LB);
  double Mc[NA * NB], Mc2[NA * NB], Mf[NA * NB];
  long long off;
  int nm, na, nb;
  block_of(a, P.mol, off, nm);
  const bool diag = P.sa == P.sb;
  if (atom < 0) {
    st_block<LA, LB>(P, a.prims + P.prim_off, a.alpha_b + P.prim_off, Mc, Mc2);
    for (int which = 0; which < 2; ++which) {
      to_final<LA, LB>(a, which ? Mc2 : Mc, Mf, na, nb);
      double* out = which ? T : S;
      for (int i = 0; i < na; ++i)
        for (int j = 0; j < nb; ++j) {
          out[off + (long long)(P.fa + i) * nm + P.fb + j] = Mf[i * nb + j];
          if (!diag) out[off + (long long)(P.fb + j) * nm + P.fa + i] = Mf[i * nb + j];
        }
    }
    return;
  }
  const double* c = a.atoms.xyzZ + 4 * atom;
  v_block<LA, LB>(P, a.prims + P.prim_off, c[0], c[1], c[2], c[3], a.boys, Mc);
  to_final<LA, LB>(a, Mc, Mf, na, nb);
  for (int i = 0; i < na; ++i)
    for (int j = 0; j < nb; ++j) {
      atomicAdd(V + off + (long long)(P.fa + i) * nm + P.fb + j, Mf[i * nb + j]);
      if (!diag) atomicAdd(V + off + (long long)(P.fb + j) * nm + P.fa + i, Mf[i * nb + j]);
    }
}

template <int LA, int LB>
__device__ void grad_item(const Args& a, const PairInfo& P, int atom, const double* D, const double* W, double cH,
                          double cS, double* grad) {
  constexpr int NA = nc(LA), NB = nc(LB);
  double wD[NA * NB], wW[NA * NB];
  long long off;
  int nm;
  block_of(a, P.mol, off, nm);
  // the pair stands for the blocks (a, b) and (b, a) of the symmetric matrices
  const double sym = P.sa == P.sb ? 1.0 : 2.0;
  weights<LA, LB>(a, D, off, nm, P.fa, P.fb, sym * cH, wD);
  if (atom < 0) {
    if (P.atom_a == P.atom_b) return;  // A and B derivatives cancel on one atom
    weights<LA, LB>(a, W, off, nm, P.fa, P.fb, sym * cS, wW);
    double g[3];
    st_grad<LA, LB>(P, a.prims + P.prim_off, a.alpha_a + P.prim_off, a.alpha_b + P.prim_off, wW, wD, g);
    for (int d = 0; d < 3; ++d) {
      atomicAdd(grad + 3 * P.atom_a + d, g[d]);
      atomicAdd(grad + 3 * P.atom_b + d, -g[d]);
    }
    return;
  }
  const double* c = a.atoms.xyzZ + 4 * atom;
  double gA[3], gB[3];
  v_grad<LA, LB>(P, a.prims + P.prim_off, a.alpha_a + P.prim_off, a.alpha_b + P.prim_off, c[0], c[1], c[2], c[3],
                 a.boys, wD, gA, gB);
  for (int d = 0; d < 3; ++d) {
    atomicAdd(grad + 3 * P.atom_a + d, gA[d]);
    atomicAdd(grad + 3 * P.atom_b + d, gB[d]);
    atomicAdd(grad + 3 * atom + d, -(gA[d] + gB[d]));
  }
}

}  // namespace onee

__global__ void __launch_bounds__(128) onee_matrices_kernel(onee::Args a, long long nitems, double* S, double* T,
                                                            double* V) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nitems) return;
  int pair, atom;
  if (!onee::item(a, t, pair, atom)) return;
  const PairInfo P = a.pairs[pair];
  switch (P.cls) {
    case 0: onee::matrices_item<0, 0>(a, P, atom, S, T, V); break;
    case 1: onee::matrices_item<1, 0>(a, P, atom, S, T, V); break;
    case 2: onee::matrices_item<1, 1>(a, P, atom, S, T, V); break;
    case 3: onee::matrices_item<2, 0>(a, P, atom, S, T, V); break;
    case 4: onee::matrices_item<2, 1>(a, P, atom, S, T, V); break;
    default: onee::matrices_item<2, 2>(a, P, atom, S, T, V); break;
  }
}

__global__ void __launch_bounds__(128) onee_grad_kernel(onee::Args a, long long nitems, const double* D,
                                                        const double* W, double cH, double cS, double* grad) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nitems) return;
  int pair, atom;
  if (!onee::item(a, t, pair, atom)) return;
  const PairInfo P = a.pairs[pair];
  switch (P.cls) {
    case 0: onee::grad_item<0, 0>(a, P, atom, D, W, cH, cS, grad); break;
    case 1: onee::grad_item<1, 0>(a, P, atom, D, W, cH, cS, grad); break;
    case 2: onee::grad_item<1, 1>(a, P, atom, D, W, cH, cS, grad); break;
    case 3: onee::grad_item<2, 0>(a, P, atom, D, W, cH, cS, grad); break;
    case 4: onee::grad_item<2, 1>(a, P, atom, D, W, cH, cS, grad); break;
    default: onee::grad_item<2, 2>(a, P, atom, D, W, cH, cS, grad); break;
  }
}
