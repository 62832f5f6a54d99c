// C entry points around the reference's own integral code, compiled in place
// from the reference sources (see oracle/Makefile) into oracle/_ref/libhfref.so.
//
// TEST INFRASTRUCTURE ONLY.  Nothing in the product links or loads this
// library; tests and the CPU-baseline leg of bench.py use it as the checker.
//
// The shell-pair and shell-quartet loops below restate the reference's drivers:
//   - hfref_onee: Mol::hf_solver::create_one_electron_hamiltonian
//       (src/scfsolver/hfscf_hf_hamiltonian.cpp:14-37)
//   - hfref_onee_grad: the one-electron part of Mol::scf_gradient::calc_scf_gradient_rhf
//       (src/gradient/hfscf_grad_rhf.cpp:78-81,99-102,144-146,164) with
//       calc_overlap_centers / calc_kinetic_centers / calc_nuclear_potential_centers and
//       calc_overlap_kinetic_gradient / calc_potential_gradient
//       (src/gradient/hfscf_grad_ints.cpp:14-77,153-199)
//   - hfref_eri_packed: Mol::hf_solver::create_repulsion_matrix
//       (src/scfsolver/hfscf_hf_hamiltonian.cpp:67-112)
//   - hfref_deriv1: Mol::scf_gradient::calc_coulomb_exchange_integral_centers
//       (src/gradient/hfscf_grad_ints.cpp:110-151)
//   - hfref_hess2e: Mol::scf_hessian::calc_scf_hessian_tei
//       (src/hessian/hfscf_hessian_ints.cpp:20-303)
// Shell offsets follow BASIS::Basisset::get_shells (src/basis/hfscf_basis.cpp:244-274)
// and shell pairs are built for all ordered pairs as in
// MOLEC::Molecule::create_shell_pairs (src/molecule/hfscf_molecule.cpp:661-669).
#include <array>
#include <cstdint>
#include <memory>
#include <vector>

#include <omp.h>

#include "integrals/hfscf_oseri.hpp"
#include "integrals/hfscf_oskinetic.hpp"
#include "integrals/hfscf_osnuclear.hpp"
#include "integrals/hfscf_osoverlap.hpp"
#include "molecule/hfscf_atom.hpp"
#include "math/gamma.hpp"
#include "math/solid_harmonics.hpp"

namespace {

struct RefBasis {
  std::vector<BASIS::Shell> shells;
  std::vector<BASIS::ShellPair> pairs;
  Eigen::Index ncart = 0, npure = 0;
};

std::unique_ptr<RefBasis> make_basis(int nshell, const int* L, const double* xyz, const int* nprim,
                                     const double* alpha, const double* coef, int pure) {
  auto b = std::make_unique<RefBasis>();
  b->shells.reserve(static_cast<std::size_t>(nshell));
  Eigen::Index idx = 0, ids = 0, off = 0;
  for (int s = 0; s < nshell; ++s) {
    EigenVector<double> c(nprim[s]), a(nprim[s]);
    for (int k = 0; k < nprim[s]; ++k) {
      c(k) = coef[off + k];
      a(k) = alpha[off + k];
    }
    off += nprim[s];
    Vec3D r(xyz[3 * s], xyz[3 * s + 1], xyz[3 * s + 2]);
    b->shells.emplace_back(pure != 0, L[s], idx, ids, r, c, a);
    idx += (L[s] + 1) * (L[s] + 2) / 2;
    ids += 2 * L[s] + 1;
  }
  b->ncart = idx;
  b->npure = ids;
  b->pairs.reserve(static_cast<std::size_t>(nshell) * nshell);
  for (int i = 0; i < nshell; ++i)
    for (int j = 0; j < nshell; ++j) b->pairs.emplace_back(b->shells[i], b->shells[j]);
  return b;
}

}  // namespace

extern "C" {

// Normalised contraction coefficients, as BASIS::Shell's constructor makes them.
int hfref_shell_coefs(int L, int nprim, const double* alpha, const double* coef, double* c_out) {
  EigenVector<double> c(nprim), a(nprim);
  for (int k = 0; k < nprim; ++k) {
    c(k) = coef[k];
    a(k) = alpha[k];
  }
  Vec3D r(0.0, 0.0, 0.0);
  BASIS::Shell sh(false, L, 0, 0, r, c, a);
  for (int k = 0; k < nprim; ++k) c_out[k] = sh.c()(k);
  return 0;
}

// Cartesian -> pure matrix, (L+1)(L+2)/2 rows by 2L+1 columns, row-major.
int hfref_ylm(int L, double* out) {
  EigenMatrix<double> m = hfscfmath::Ylm_transmat(L);
  for (Eigen::Index i = 0; i < m.rows(); ++i)
    for (Eigen::Index j = 0; j < m.cols(); ++j) out[i * m.cols() + j] = m(i, j);
  return 0;
}

double hfref_boys(double m, double T) { return extramath::F_nu(m, T); }

// Number of basis functions for the given shells.
long long hfref_nbf(int nshell, const int* L, int pure) {
  long long n = 0;
  for (int s = 0; s < nshell; ++s) n += pure ? 2 * L[s] + 1 : (L[s] + 1) * (L[s] + 2) / 2;
  return n;
}

// Packed 8-fold ERI vector, length n(n+1)(n^2+n+2)/8, filled by the reference's
// Erios::compute_contracted_shell_quartet over all unique shell quartets.
int hfref_eri_packed(int nshell, const int* L, const double* xyz, const int* nprim, const double* alpha,
                     const double* coef, int pure, double cutoff, int do_screen, double* eri_out) {
  auto b = make_basis(nshell, L, xyz, nprim, alpha, coef, pure);
  const Eigen::Index n = pure ? b->npure : b->ncart;
  const Eigen::Index len = n * (n + 1) * (n * n + n + 2) / 8;
  EigenVector<double> eri(len);
  eri.setZero();
  ERIOS::Erios os(pure != 0, cutoff);
  if (do_screen) {
    os.init_screen(b->ncart);
    for (int i = 0; i < nshell; ++i)
      for (int j = i; j < nshell; ++j) os.compute_screen_matrix(b->pairs[i * nshell + j]);
  }
#pragma omp parallel for schedule(dynamic)
  for (int i = 0; i < nshell; ++i)
    for (int j = i; j < nshell; ++j) {
      const Eigen::Index ij = hfscfmath::index_ij(i, j);
      for (int k = 0; k < nshell; ++k)
        for (int l = k; l < nshell; ++l) {
          const Eigen::Index kl = hfscfmath::index_ij(k, l);
          if (ij > kl) continue;
          os.compute_contracted_shell_quartet(eri, b->pairs[i * nshell + j], b->pairs[k * nshell + l],
                                              do_screen != 0);
        }
    }
  for (Eigen::Index p = 0; p < len; ++p) eri_out[p] = eri(p);
  return 0;
}

// The reference's Schwarz diagonal (pq|pq) over Cartesian functions, as its screen matrix
// holds it.  Erios::init_screen and Erios::compute_screen_matrix over the shell pairs i <= j
// (as create_repulsion_matrix calls them, src/scfsolver/hfscf_hf_hamiltonian.cpp:77-89), then
// compute_contracted_shell_quartet(eri, s_ij, s_ij, do_screen = true) for every diagonal
// shell quartet: with screening on, a Cartesian basis stores screen(p, q) into the slot of
// (pq|pq) (src/integrals/hfscf_oseri.cpp:214-218), and the matrix itself is private.
// out: ncart x ncart, row-major; entries of shell pairs whose whole block the reference's
// block test skips (src/integrals/hfscf_oseri.cpp:36-46) are left at -1.
int hfref_screen_diagonal(int nshell, const int* L, const double* xyz, const int* nprim, const double* alpha,
                          const double* coef, double cutoff, double* out) {
  auto b = make_basis(nshell, L, xyz, nprim, alpha, coef, 0);
  const Eigen::Index n = b->ncart;
  const Eigen::Index len = n * (n + 1) * (n * n + n + 2) / 8;
  EigenVector<double> eri(len);
  for (Eigen::Index p = 0; p < len; ++p) eri(p) = -1.0;
  ERIOS::Erios os(false, cutoff);
  os.init_screen(n);
#pragma omp parallel for schedule(dynamic)
  for (int i = 0; i < nshell; ++i)
    for (int j = i; j < nshell; ++j) os.compute_screen_matrix(b->pairs[i * nshell + j]);
#pragma omp parallel for schedule(dynamic)
  for (int i = 0; i < nshell; ++i)
    for (int j = i; j < nshell; ++j)
      os.compute_contracted_shell_quartet(eri, b->pairs[i * nshell + j], b->pairs[i * nshell + j], true);
  for (Eigen::Index p = 0; p < n; ++p)
    for (Eigen::Index q = 0; q < n; ++q) out[p * n + q] = eri(hfscfmath::index_ijkl(p, q, p, q));
  return 0;
}

// Nine packed derivative-ERI tensors (d/dXa, d/dXb, d/dXc, d/dYa, ..., d/dZc), each
// of the packed 8-fold length, from Erios::compute_contracted_shell_quartet_deriv1.
// coords[3] selects the Cartesian directions, as the reference's out_of_plane mask.
int hfref_deriv1(int nshell, const int* L, const double* xyz, const int* nprim, const double* alpha,
                 const double* coef, int pure, double cutoff, const int* coords, double* out9) {
  auto b = make_basis(nshell, L, xyz, nprim, alpha, coef, pure);
  const Eigen::Index n = pure ? b->npure : b->ncart;
  const Eigen::Index len = n * (n + 1) * (n * n + n + 2) / 8;
  std::vector<bool> mask = {coords[0] != 0, coords[1] != 0, coords[2] != 0};
  std::vector<tensor4dmath::symm4dTensor<double>> t(9);
  for (int c = 0; c < 3; ++c)
    if (mask[c])
      for (int k = 0; k < 3; ++k) t[3 * c + k] = tensor4dmath::symm4dTensor<double>(n);
  ERIOS::Erios os(pure != 0, cutoff);
#pragma omp parallel for schedule(dynamic)
  for (int i = 0; i < nshell; ++i)
    for (int j = 0; j <= i; ++j) {
      const Eigen::Index ij = hfscfmath::index_ij(i, j);
      for (int k = 0; k < nshell; ++k)
        for (int l = 0; l <= k; ++l) {
          const Eigen::Index kl = hfscfmath::index_ij(k, l);
          if (ij > kl) continue;
          os.compute_contracted_shell_quartet_deriv1(t[0], t[1], t[2], t[3], t[4], t[5], t[6], t[7], t[8],
                                                     b->pairs[i * nshell + j], b->pairs[k * nshell + l], mask);
        }
    }
  for (int q = 0; q < 9; ++q) {
    if (!mask[q / 3]) {
      for (Eigen::Index p = 0; p < len; ++p) out9[q * len + p] = 0.0;
      continue;
    }
    for (Eigen::Index p = 0; p < len; ++p) out9[q * len + p] = t[q][p];
  }
  return 0;
}

// S, T, V (n x n each, row-major) from OSOverlap::compute_contracted_shell and
// OSNuclear::compute_contracted_shell over all shell pairs i <= j.  Atoms: natoms
// charges Z and positions atom_xyz (bohr); shell centres in xyz.
int hfref_onee(int nshell, const int* L, const double* xyz, const int* nprim, const double* alpha,
               const double* coef, int pure, int natoms, const int* Z, const double* atom_xyz, double* S_out,
               double* T_out, double* V_out) {
  auto b = make_basis(nshell, L, xyz, nprim, alpha, coef, pure);
  const Eigen::Index n = pure ? b->npure : b->ncart;
  std::vector<MOLEC::Atom> atoms;
  for (int a = 0; a < natoms; ++a) atoms.emplace_back(Z[a], Vec3D(atom_xyz[3 * a], atom_xyz[3 * a + 1], atom_xyz[3 * a + 2]));
  EigenMatrix<double> S = EigenMatrix<double>::Zero(n, n), T = S, V = S;
  OSOVERLAP::OSOverlap os(pure != 0);
  OSNUCLEAR::OSNuclear on(pure != 0);
  for (int i = 0; i < nshell; ++i)
    for (int j = i; j < nshell; ++j) {
      os.compute_contracted_shell(S, T, b->pairs[i * nshell + j]);
      on.compute_contracted_shell(V, b->pairs[i * nshell + j], atoms);
    }
  for (Eigen::Index i = 0; i < n; ++i)
    for (Eigen::Index j = 0; j < n; ++j) {
      S_out[i * n + j] = S(i, j);
      T_out[i * n + j] = T(i, j);
      V_out[i * n + j] = V(i, j);
    }
  return 0;
}

// One-electron gradient grad (natoms x 3) = cD sum D.(dT/dX + dV/dX) + cQ sum Q.dS/dX, from the
// reference's first-derivative shell routines and its per-atom assembly (cD = 2, cQ = -2 is
// the RHF gradient's one-electron part with Q = D F D).  shell_atom maps shells to atoms.
int hfref_onee_grad(int nshell, const int* L, const double* xyz, const int* nprim, const double* alpha,
                    const double* coef, int pure, int natoms, const int* Z, const double* atom_xyz,
                    const int* shell_atom, const double* D, const double* Q, double cD, double cQ, double* grad) {
  auto b = make_basis(nshell, L, xyz, nprim, alpha, coef, pure);
  const Eigen::Index n = pure ? b->npure : b->ncart;
  std::vector<MOLEC::Atom> atoms;
  for (int a = 0; a < natoms; ++a) atoms.emplace_back(Z[a], Vec3D(atom_xyz[3 * a], atom_xyz[3 * a + 1], atom_xyz[3 * a + 2]));
  tensor3d<double> dSdq(3, n, n), dTdq(3, n, n), dVdqa(3 * natoms, n, n), dVdqb(3 * natoms, n, n);
  OSOVERLAP::OSOverlap os(pure != 0);
  OSKINETIC::OSKinetic ok(pure != 0);
  OSNUCLEAR::OSNuclear on(pure != 0);
  const std::vector<bool> coords = {true, true, true};
  for (int i = 0; i < nshell; ++i)
    for (int j = i; j < nshell; ++j) {
      os.compute_contracted_shell_deriv1(dSdq, b->pairs[i * nshell + j]);
      ok.compute_contracted_shell_deriv1(dTdq, b->pairs[i * nshell + j]);
      on.compute_contracted_shell_deriv1(dVdqa, dVdqb, b->pairs[i * nshell + j], atoms, coords);
    }
  // function -> atom
  std::vector<int> fatom;
  for (int s = 0; s < nshell; ++s)
    for (int k = 0; k < (pure ? 2 * L[s] + 1 : (L[s] + 1) * (L[s] + 2) / 2); ++k) fatom.push_back(shell_atom[s]);
  for (int dir = 0; dir < 3; ++dir)
    for (int atom = 0; atom < natoms; ++atom) {
      double g = 0.0;
      for (Eigen::Index i = 0; i < n; ++i) {
        const bool mi = fatom[i] == atom;
        // overlap and kinetic: A-derivative with the B term by translational invariance
        for (Eigen::Index j = i + 1; j < n; ++j) {
          const bool mj = fatom[j] == atom;
          double ds = 0.0, dt = 0.0;
          if (mi) {
            ds = dSdq(dir, i, j);
            dt = dTdq(dir, i, j);
          }
          if (mj) {
            ds -= dSdq(dir, i, j);
            dt -= dTdq(dir, i, j);
          }
          g += 2.0 * (cQ * Q[i * n + j] * ds + cD * D[i * n + j] * dt);  // (i, j) and (j, i)
        }
        // nuclear attraction, upper triangle with the diagonal
        for (Eigen::Index j = i; j < n; ++j) {
          const bool mj = fatom[j] == atom;
          double dv = 0.0;
          for (int k = 0; k < natoms; ++k) {
            if (mi) dv -= dVdqa(natoms * dir + k, i, j);
            if (mj) dv -= dVdqb(natoms * dir + k, i, j);
            if (k == atom) dv += dVdqa(natoms * dir + atom, i, j) + dVdqb(natoms * dir + atom, i, j);
          }
          g += (j == i ? 1.0 : 2.0) * cD * D[i * n + j] * dv;
        }
      }
      grad[3 * atom + dir] = g;
    }
  return 0;
}

// Timing sample of the reference's ERI generation: runs
// Erios::compute_contracted_shell_quartet over every `stride`-th unique shell
// quartet of create_repulsion_matrix's loop (hfscf_hf_hamiltonian.cpp:95-111), with
// the reference's default eri_screen = true (screen matrix first, :77-89), on all
// OpenMP threads.  Returns the seconds of the sampled quartets (*sampled / *total give the
// scale factor); *fixed_s is the unscaled once-per-geometry part.
double hfref_time_eri_sample(int nshell, const int* L, const double* xyz, const int* nprim, const double* alpha,
                             const double* coef, int pure, double cutoff, long long stride, long long* sampled,
                             long long* total, double* fixed_s) {
  auto b = make_basis(nshell, L, xyz, nprim, alpha, coef, pure);
  const Eigen::Index n = pure ? b->npure : b->ncart;
  const Eigen::Index len = n * (n + 1) * (n * n + n + 2) / 8;
  EigenVector<double> eri(len);
  ERIOS::Erios os(pure != 0, cutoff);
  // Once-per-geometry work that does not scale with the sample: the first touch of the whole
  // packed ERI vector and the Schwarz screen matrix.  Timed apart and reported in *fixed_s.
  const double f0 = omp_get_wtime();
  eri.setZero();
  os.init_screen(b->ncart);
#pragma omp parallel for schedule(dynamic)
  for (int i = 0; i < nshell; ++i)
    for (int j = i; j < nshell; ++j) os.compute_screen_matrix(b->pairs[i * nshell + j]);
  *fixed_s = omp_get_wtime() - f0;
  std::vector<std::pair<int, int>> quartets;
  for (int i = 0; i < nshell; ++i)
    for (int j = i; j < nshell; ++j)
      for (int k = 0; k < nshell; ++k)
        for (int l = k; l < nshell; ++l)
          if (hfscfmath::index_ij(i, j) <= hfscfmath::index_ij(k, l)) quartets.emplace_back(i * nshell + j, k * nshell + l);
  std::vector<std::pair<int, int>> pick;
  for (size_t q = 0; q < quartets.size(); q += (size_t)stride) pick.push_back(quartets[q]);
  const double t0 = omp_get_wtime();
#pragma omp parallel for schedule(dynamic)
  for (long long q = 0; q < (long long)pick.size(); ++q)
    os.compute_contracted_shell_quartet(eri, b->pairs[pick[q].first], b->pairs[pick[q].second], true);
  const double t1 = omp_get_wtime();
  *sampled = (long long)pick.size();
  *total = (long long)quartets.size();
  return t1 - t0;
}

// Timing sample of the reference's per-iteration Fock contraction
// (Mol::hf_solver::update_fock_matrix, src/scfsolver/hfscf_hf_solver.cpp:258-279),
// restated: rows i in [0, rows) over a packed ERI vector of the full length.
// Returns seconds; the caller scales by the share of the N^3(N+1)/2 inner iterations.
double hfref_time_fock_sample(long long n, long long rows, double* checksum) {
  const long long len = n * (n + 1) * (n * n + n + 2) / 8;
  std::vector<double> eri((size_t)len, 1e-3), D((size_t)(n * n), 1e-2), F((size_t)(n * n), 0.0);
  // the sampled (i, j) elements are spread over all threads, as the reference's loop over every
  // row spreads them (a sample of a few rows parallelised by row would leave threads idle)
  std::vector<std::pair<long long, long long>> ij;
  for (long long i = 0; i < rows; ++i)
    for (long long j = i; j < n; ++j) ij.emplace_back(i, j);
  const double t0 = omp_get_wtime();
#pragma omp parallel for schedule(dynamic)
  for (long long x = 0; x < (long long)ij.size(); ++x) {
    const long long i = ij[(size_t)x].first, j = ij[(size_t)x].second;
    double f = 0.0;
    for (long long k = 0; k < n; ++k)
      for (long long l = 0; l < n; ++l)
        f += D[k * n + l] * (2.0 * eri[hfscfmath::index_ijkl(i, j, k, l)] - eri[hfscfmath::index_ijkl(i, k, j, l)]);
    F[i * n + j] = F[j * n + i] = f;
  }
  const double t1 = omp_get_wtime();
  double c = 0.0;
  for (double v : F) c += v;
  *checksum = c;
  return t1 - t0;
}

}  // extern "C"

extern "C" {

// Timing sample of the reference's RHF gradient two-electron part
// (Mol::scf_gradient::calc_scf_gradient_rhf, src/gradient/hfscf_grad_rhf.cpp:76-141):
//   *t_deriv_s   calc_coulomb_exchange_integral_centers (src/gradient/hfscf_grad_ints.cpp:110-151):
//                Erios::compute_contracted_shell_quartet_deriv1 over every `stride`-th unique shell
//                quartet of its loop, on all OpenMP threads, scaled to all quartets (the nine packed
//                tensors are allocated and first touched outside the timed part, which is added in
//                full to *t_fixed_s);
//   *t_assemble_s  one call of calc_coulomb_exchange_integrals (:79-108) for atom 0, x, over all
//                canonical slots (the reference makes 3 natoms of them);
//   *t_contract_s  the dG/dX contraction of one (atom, direction) (hfscf_grad_rhf.cpp:121-134) over
//                the rows i < rows, scaled to all N(N+1)/2 elements (3 natoms of them).
// Returns 0.  Only the timings are of interest; the sums are kept in *checksum.
int hfref_time_grad_sample(int nshell, const int* L, const double* xyz, const int* nprim, const double* alpha,
                           const double* coef, int pure, double cutoff, long long stride, long long rows,
                           double* t_deriv_s, double* t_fixed_s, double* t_assemble_s, double* t_contract_s,
                           double* checksum) {
  auto b = make_basis(nshell, L, xyz, nprim, alpha, coef, pure);
  const Eigen::Index n = pure ? b->npure : b->ncart;
  const double f0 = omp_get_wtime();
  std::vector<bool> mask = {true, true, true};
  std::vector<tensor4dmath::symm4dTensor<double>> t(9);
  for (int q = 0; q < 9; ++q) t[q] = tensor4dmath::symm4dTensor<double>(n);
  *t_fixed_s = omp_get_wtime() - f0;
  std::vector<std::pair<int, int>> quartets;
  for (int i = 0; i < nshell; ++i)
    for (int j = 0; j <= i; ++j)
      for (int k = 0; k < nshell; ++k)
        for (int l = 0; l <= k; ++l)
          if (hfscfmath::index_ij(i, j) <= hfscfmath::index_ij(k, l)) quartets.emplace_back(i * nshell + j, k * nshell + l);
  std::vector<std::pair<int, int>> pick;
  for (size_t q = 0; q < quartets.size(); q += (size_t)stride) pick.push_back(quartets[q]);
  ERIOS::Erios os(pure != 0, cutoff);
  const double t0 = omp_get_wtime();
#pragma omp parallel for schedule(dynamic)
  for (long long q = 0; q < (long long)pick.size(); ++q)
    os.compute_contracted_shell_quartet_deriv1(t[0], t[1], t[2], t[3], t[4], t[5], t[6], t[7], t[8],
                                               b->pairs[pick[q].first], b->pairs[pick[q].second], mask);
  *t_deriv_s = (omp_get_wtime() - t0) * (double)quartets.size() / (double)std::max<size_t>(pick.size(), 1);
  // function -> atom of shell, for the mask of atom 0
  std::vector<char> m0((size_t)n, 0);
  {
    Eigen::Index f = 0;
    for (int s = 0; s < nshell; ++s) {
      const int nf = pure ? 2 * L[s] + 1 : (L[s] + 1) * (L[s] + 2) / 2;
      const bool on0 = xyz[3 * s] == xyz[0] && xyz[3 * s + 1] == xyz[1] && xyz[3 * s + 2] == xyz[2];
      for (int k = 0; k < nf; ++k) m0[(size_t)(f + k)] = on0;
      f += nf;
    }
  }
  tensor4dmath::symm4dTensor<double> dV(n);
  const double t1 = omp_get_wtime();
#pragma omp parallel for schedule(dynamic)
  for (Eigen::Index i = 0; i < n; ++i)
    for (Eigen::Index j = 0; j <= i; ++j) {
      const Eigen::Index ij = hfscfmath::index_ij(i, j);
      for (Eigen::Index k = 0; k < n; ++k)
        for (Eigen::Index l = 0; l <= k; ++l) {
          const Eigen::Index kl = hfscfmath::index_ij(k, l);
          if (ij <= kl) {
            if (m0[(size_t)i]) dV(i, j, k, l) += t[0](i, j, k, l);
            if (m0[(size_t)j]) dV(i, j, k, l) += t[1](i, j, k, l);
            if (m0[(size_t)k]) dV(i, j, k, l) += t[2](i, j, k, l);
            if (m0[(size_t)l]) dV(i, j, k, l) += -t[0](i, j, k, l) - t[1](i, j, k, l) - t[2](i, j, k, l);
          }
        }
    }
  *t_assemble_s = omp_get_wtime() - t1;
  std::vector<double> D((size_t)(n * n), 1e-2);
  std::vector<std::pair<Eigen::Index, Eigen::Index>> ij;
  for (Eigen::Index i = 0; i < std::min<Eigen::Index>(rows, n); ++i)
    for (Eigen::Index j = i; j < n; ++j) ij.emplace_back(i, j);
  double c = 0.0;
  const double t2 = omp_get_wtime();
#pragma omp parallel for schedule(dynamic) reduction(+ : c)
  for (long long x = 0; x < (long long)ij.size(); ++x) {
    const Eigen::Index i = ij[(size_t)x].first, j = ij[(size_t)x].second;
    double gc = 0.0, ge = 0.0;
    for (Eigen::Index k = 0; k < n; ++k)
      for (Eigen::Index l = 0; l < n; ++l) {
        gc += D[(size_t)(k * n + l)] * (2.0 * dV(i, j, k, l));
        ge -= D[(size_t)(k * n + l)] * dV(i, k, j, l);
      }
    c += gc + ge;
  }
  const double frac = (double)ij.size() / (0.5 * (double)n * (double)(n + 1));
  *t_contract_s = (omp_get_wtime() - t2) / frac;
  *checksum = c;
  return 0;
}

// Two-electron part of the RHF Hessian at a fixed density D (n x n, row-major, without the
// factor 2 of the closed-shell density): hessC = sum D_ij D_kl 2 d2(ij|kl)/dX dY and
// hessEx = -sum D_ij D_kl d2(ik|jl)/dX dY, both 3 natoms x 3 natoms, row-major, from the
// reference's second-derivative shell routines Erios::compute_contracted_shell_quartet_deriv2_qq
// and _pq.  The loops, the translational-invariance relations and the per-atom masks restate
// Mol::scf_hessian::calc_scf_hessian_tei (src/hessian/hfscf_hessian_ints.cpp:20-303); the
// reference skips the off-diagonal direction pairs of a planar or linear molecule (zero by
// symmetry in its aligned frame, :145-166), here every direction pair is computed.
// shell_atom maps shells to atoms.
int hfref_hess2e(int nshell, const int* L, const double* xyz, const int* nprim, const double* alpha,
                 const double* coef, int pure, double cutoff, const int* shell_atom, int natoms, const double* Dm,
                 double* hessC, double* hessEx) {
  using tensor4dmath::symm4dTensor;
  using tensor4dmath::tensor4d;
  auto b = make_basis(nshell, L, xyz, nprim, alpha, coef, pure);
  const Eigen::Index n = pure ? b->npure : b->ncart;
  const int na3 = 3 * natoms;
  // mask[atom][function]: the function sits on the atom
  std::vector<std::vector<bool>> mask((size_t)natoms, std::vector<bool>((size_t)n, false));
  {
    Eigen::Index f = 0;
    for (int s = 0; s < nshell; ++s) {
      const int nf = pure ? 2 * L[s] + 1 : (L[s] + 1) * (L[s] + 2) / 2;
      for (int k = 0; k < nf; ++k) mask[(size_t)shell_atom[s]][(size_t)(f + k)] = true;
      f += nf;
    }
  }
  auto D = [&](Eigen::Index k, Eigen::Index l) { return Dm[k * n + l]; };
  for (int q = 0; q < na3 * na3; ++q) hessC[q] = hessEx[q] = 0.0;
  ERIOS::Erios os(pure != 0, cutoff);
  // XX, YY, ZZ
  for (int cart2 = 0; cart2 < 3; ++cart2) {
    symm4dTensor<double> AA(n), AB(n), AC(n), BD(n), CC(n), CD(n);
#pragma omp parallel for schedule(dynamic)
    for (int i = 0; i < nshell; ++i)
      for (int j = 0; j <= i; ++j)
        for (int k = 0; k < nshell; ++k)
          for (int l = 0; l <= k; ++l)
            os.compute_contracted_shell_quartet_deriv2_qq(AA, AB, AC, BD, CC, CD, b->pairs[i * nshell + j],
                                                          b->pairs[k * nshell + l], cart2);
    for (int atom = 0; atom < natoms; ++atom) {
      const std::vector<bool>& m1 = mask[(size_t)atom];
      for (int atom2 = 0; atom2 <= atom; ++atom2) {
        const std::vector<bool>& m2 = mask[(size_t)atom2];
        symm4dTensor<double> t(n);
#pragma omp parallel for schedule(dynamic)
        for (Eigen::Index i = 0; i < n; ++i)
          for (Eigen::Index j = 0; j <= i; ++j) {
            const Eigen::Index ij = hfscfmath::index_ij(i, j);
            for (Eigen::Index k = 0; k < n; ++k)
              for (Eigen::Index l = 0; l <= k; ++l) {
                if (ij > hfscfmath::index_ij(k, l)) continue;
                const double ad = -(AA(i, j, k, l) + AB(i, j, k, l) + AC(i, j, k, l));
                const double dd = -(ad + BD(i, j, k, l) + CD(i, j, k, l));
                const double bb = AA(i, j, k, l) + 2 * AC(i, j, k, l) + 2 * ad + CC(i, j, k, l) +
                                  2 * CD(i, j, k, l) + dd;
                const double bc = -(AC(i, j, k, l) + CC(i, j, k, l) + CD(i, j, k, l));
                double v = 0.0;
                if (atom == atom2) {
                  if (m1[i]) v += AA(i, j, k, l);
                  if (m1[j]) v += bb;
                  if (m1[k]) v += CC(i, j, k, l);
                  if (m1[l]) v += dd;
                  if (m1[i] && m1[j]) v += 2 * AB(i, j, k, l);
                  if (m1[i] && m1[k]) v += 2 * AC(i, j, k, l);
                  if (m1[i] && m1[l]) v += 2 * ad;
                  if (m1[j] && m1[k]) v += 2 * bc;
                  if (m1[j] && m1[l]) v += 2 * BD(i, j, k, l);
                  if (m1[k] && m1[l]) v += 2 * CD(i, j, k, l);
                } else {
                  if ((m1[i] && m2[j]) || (m1[j] && m2[i])) v += AB(i, j, k, l);
                  if ((m1[i] && m2[k]) || (m1[k] && m2[i])) v += AC(i, j, k, l);
                  if ((m1[i] && m2[l]) || (m1[l] && m2[i])) v += ad;
                  if ((m1[j] && m2[k]) || (m1[k] && m2[j])) v += bc;
                  if ((m1[j] && m2[l]) || (m1[l] && m2[j])) v += BD(i, j, k, l);
                  if ((m1[k] && m2[l]) || (m1[l] && m2[k])) v += CD(i, j, k, l);
                }
                t(i, j, k, l) = v;
              }
          }
        double hc = 0.0, he = 0.0;
#pragma omp parallel for schedule(dynamic) reduction(+ : hc, he)
        for (Eigen::Index i = 0; i < n; ++i)
          for (Eigen::Index j = i; j < n; ++j) {
            double gc = 0.0, ge = 0.0;
            for (Eigen::Index k = 0; k < n; ++k)
              for (Eigen::Index l = 0; l < n; ++l) {
                gc += D(k, l) * (2.0 * t(i, j, k, l));
                ge -= D(k, l) * t(i, k, j, l);
              }
            const double w = i == j ? 1.0 : 2.0;  // dG(j, i) = dG(i, j)
            hc += w * D(i, j) * gc;
            he += w * D(i, j) * ge;
          }
        const int r = 3 * atom + cart2, c = 3 * atom2 + cart2;
        hessC[r * na3 + c] = hessC[c * na3 + r] = hc;
        hessEx[r * na3 + c] = hessEx[c * na3 + r] = he;
      }
    }
  }
  // XY, XZ, YZ
  for (int cart2 = 3; cart2 <= 5; ++cart2) {
    tensor4d<double> AA(n), AB(n), AC(n);
    AA.setZero();
    AB.setZero();
    AC.setZero();
#pragma omp parallel for schedule(dynamic)
    for (int i = 0; i < nshell; ++i)
      for (int j = 0; j < nshell; ++j)
        for (int k = 0; k < nshell; ++k)
          for (int l = 0; l < nshell; ++l)
            os.compute_contracted_shell_quartet_deriv2_pq(AA, AB, AC, b->pairs[i * nshell + j],
                                                          b->pairs[k * nshell + l], cart2,
                                                          l <= k ? ERIOS::Permute::ALL : ERIOS::Permute::ACONLY);
    for (int atom = 0; atom < natoms; ++atom) {
      const std::vector<bool>& m1 = mask[(size_t)atom];
      for (int atom2 = 0; atom2 < natoms; ++atom2) {
        const std::vector<bool>& m2 = mask[(size_t)atom2];
        tensor4d<double> t(n);
#pragma omp parallel for schedule(dynamic)
        for (Eigen::Index i = 0; i < n; ++i)
          for (Eigen::Index j = 0; j < n; ++j)
            for (Eigen::Index k = 0; k < n; ++k)
              for (Eigen::Index l = 0; l < n; ++l) {
                const double ad = -(AA(i, j, k, l) + AB(i, j, k, l) + AC(i, j, k, l));
                const double ad1 = -(AA(i, j, k, l) + AB(j, i, k, l) + AC(k, l, i, j));
                const double dd = -(ad + AC(j, i, l, k) + AB(k, l, i, j));
                const double bb = AA(i, j, k, l) + AC(i, j, k, l) + ad + AC(k, l, i, j) + AA(k, l, i, j) +
                                  AB(k, l, i, j) + ad1 + AB(l, k, i, j) + dd;
                const double bc = -(AC(i, j, k, l) + AA(k, l, i, j) + AB(l, k, i, j));
                const double bc1 = -(AC(k, l, i, j) + AA(k, l, i, j) + AB(k, l, i, j));
                const double bd1 = -(ad1 + AB(l, k, i, j) + dd);
                double v = 0.0;
                if (atom == atom2) {
                  if (m1[i]) v += AA(i, j, k, l);
                  if (m1[j]) v += bb;
                  if (m1[k]) v += AA(k, l, i, j);
                  if (m1[l]) v += dd;
                  if (m1[i] && m1[j]) v += 2 * AB(i, j, k, l);
                  if (m1[i] && m1[k]) v += 2 * AC(i, j, k, l);
                  if (m1[i] && m1[l]) v += 2 * ad;
                  if (m1[j] && m1[k]) v += 2 * bc;
                  if (m1[j] && m1[l]) v += 2 * AC(j, i, l, k);
                  if (m1[k] && m1[l]) v += 2 * AB(k, l, i, j);
                } else {
                  if (m1[i] && m2[j]) v += AB(i, j, k, l);
                  if (m1[j] && m2[i]) v += AB(j, i, k, l);
                  if (m1[i] && m2[k]) v += AC(i, j, k, l);
                  if (m1[k] && m2[i]) v += AC(k, l, i, j);
                  if (m1[i] && m2[l]) v += ad;
                  if (m1[l] && m2[i]) v += ad1;
                  if (m1[j] && m2[k]) v += bc;
                  if (m1[k] && m2[j]) v += bc1;
                  if (m1[j] && m2[l]) v += AC(j, i, l, k);
                  if (m1[l] && m2[j]) v += bd1;
                  if (m1[k] && m2[l]) v += AB(k, l, i, j);
                  if (m1[l] && m2[k]) v += AB(l, k, i, j);
                }
                t(i, j, k, l) = v;
              }
        double hc = 0.0, he = 0.0;
#pragma omp parallel for schedule(dynamic) reduction(+ : hc, he)
        for (Eigen::Index i = 0; i < n; ++i)
          for (Eigen::Index j = 0; j < n; ++j) {
            double gc = 0.0, ge = 0.0;
            for (Eigen::Index k = 0; k < n; ++k)
              for (Eigen::Index l = 0; l < n; ++l) {
                gc += D(k, l) * (2.0 * t(i, j, k, l));
                ge -= D(k, l) * t(i, k, j, l);
              }
            hc += D(i, j) * gc;
            he += D(i, j) * ge;
          }
        const int d1 = cart2 == 5 ? 1 : 0, d2 = cart2 == 3 ? 1 : 2;
        const int r = 3 * atom + d1, c = 3 * atom2 + d2;
        hessC[r * na3 + c] = hessC[c * na3 + r] = hc;
        hessEx[r * na3 + c] = hessEx[c * na3 + r] = he;
      }
    }
  }
  return 0;
}

}  // extern "C"

extern "C" {

// Timing sample of the reference's Hessian two-electron part (calc_scf_hessian_tei,
// src/hessian/hfscf_hessian_ints.cpp:20-303) on all OpenMP threads: the second-derivative
// shell routines of one direction pair of each kind (xx via deriv2_qq, xy via deriv2_pq) over
// every `stride`-th shell quartet of its loop, scaled to the whole loop (*t_qq_ints, *t_pq_ints,
// per direction pair), and the per-atom-pair assembly + contraction of one atom pair of each
// kind (*t_pair_qq, *t_pair_pq).  The whole term costs 3 (t_qq_ints + t_pq_ints) +
// 3 natoms (natoms + 1) / 2 t_pair_qq + 3 natoms^2 t_pair_pq.
int hfref_time_hess_sample(int nshell, const int* L, const double* xyz, const int* nprim, const double* alpha,
                           const double* coef, int pure, double cutoff, const int* shell_atom, int natoms,
                           int stride, double* t_qq_ints, double* t_pq_ints, double* t_pair_qq,
                           double* t_pair_pq) {
  using tensor4dmath::symm4dTensor;
  using tensor4dmath::tensor4d;
  auto b = make_basis(nshell, L, xyz, nprim, alpha, coef, pure);
  const Eigen::Index n = pure ? b->npure : b->ncart;
  std::vector<std::vector<bool>> mask((size_t)natoms, std::vector<bool>((size_t)n, false));
  {
    Eigen::Index f = 0;
    for (int s = 0; s < nshell; ++s) {
      const int nf = pure ? 2 * L[s] + 1 : (L[s] + 1) * (L[s] + 2) / 2;
      for (int k = 0; k < nf; ++k) mask[(size_t)shell_atom[s]][(size_t)(f + k)] = true;
      f += nf;
    }
  }
  std::vector<double> D((size_t)(n * n), 1e-2);
  ERIOS::Erios os(pure != 0, cutoff);
  const int a1 = natoms > 1 ? 1 : 0, a0 = 0;
  {
    std::vector<std::array<int, 4>> qs;
    for (int i = 0; i < nshell; ++i)
      for (int j = 0; j <= i; ++j)
        for (int k = 0; k < nshell; ++k)
          for (int l = 0; l <= k; ++l) qs.push_back({i, j, k, l});
    std::vector<std::array<int, 4>> pick;
    for (size_t q = 0; q < qs.size(); q += (size_t)stride) pick.push_back(qs[q]);
    symm4dTensor<double> AA(n), AB(n), AC(n), BD(n), CC(n), CD(n);
    double t0 = omp_get_wtime();
#pragma omp parallel for schedule(dynamic)
    for (long long q = 0; q < (long long)pick.size(); ++q) {
      const auto& s = pick[(size_t)q];
      os.compute_contracted_shell_quartet_deriv2_qq(AA, AB, AC, BD, CC, CD, b->pairs[s[0] * nshell + s[1]],
                                                    b->pairs[s[2] * nshell + s[3]], 0);
    }
    *t_qq_ints = (omp_get_wtime() - t0) * (double)qs.size() / (double)std::max<size_t>(pick.size(), 1);
    // one atom pair: the mask assembly into a packed tensor and the Coulomb/exchange contraction
    const std::vector<bool>& m1 = mask[(size_t)a1];
    const std::vector<bool>& m2 = mask[(size_t)a0];
    t0 = omp_get_wtime();
    symm4dTensor<double> t(n);
#pragma omp parallel for schedule(dynamic)
    for (Eigen::Index i = 0; i < n; ++i)
      for (Eigen::Index j = 0; j <= i; ++j) {
        const Eigen::Index ij = hfscfmath::index_ij(i, j);
        for (Eigen::Index k = 0; k < n; ++k)
          for (Eigen::Index l = 0; l <= k; ++l) {
            if (ij > hfscfmath::index_ij(k, l)) continue;
            const double ad = -(AA(i, j, k, l) + AB(i, j, k, l) + AC(i, j, k, l));
            const double dd = -(ad + BD(i, j, k, l) + CD(i, j, k, l));
            const double bc = -(AC(i, j, k, l) + CC(i, j, k, l) + CD(i, j, k, l));
            double v = 0.0;
            if ((m1[i] && m2[j]) || (m1[j] && m2[i])) v += AB(i, j, k, l);
            if ((m1[i] && m2[k]) || (m1[k] && m2[i])) v += AC(i, j, k, l);
            if ((m1[i] && m2[l]) || (m1[l] && m2[i])) v += ad;
            if ((m1[j] && m2[k]) || (m1[k] && m2[j])) v += bc;
            if ((m1[j] && m2[l]) || (m1[l] && m2[j])) v += BD(i, j, k, l);
            if ((m1[k] && m2[l]) || (m1[l] && m2[k])) v += CD(i, j, k, l) + 0.0 * dd;
            t(i, j, k, l) = v;
          }
      }
    double hc = 0.0;
#pragma omp parallel for schedule(dynamic) reduction(+ : hc)
    for (Eigen::Index i = 0; i < n; ++i)
      for (Eigen::Index j = i; j < n; ++j) {
        double gc = 0.0, ge = 0.0;
        for (Eigen::Index k = 0; k < n; ++k)
          for (Eigen::Index l = 0; l < n; ++l) {
            gc += D[(size_t)(k * n + l)] * (2.0 * t(i, j, k, l));
            ge -= D[(size_t)(k * n + l)] * t(i, k, j, l);
          }
        hc += D[(size_t)(i * n + j)] * (gc + ge);
      }
    *t_pair_qq = omp_get_wtime() - t0 + 0.0 * hc;
  }
  {
    std::vector<std::array<int, 4>> qs;
    for (int i = 0; i < nshell; ++i)
      for (int j = 0; j < nshell; ++j)
        for (int k = 0; k < nshell; ++k)
          for (int l = 0; l < nshell; ++l) qs.push_back({i, j, k, l});
    std::vector<std::array<int, 4>> pick;
    for (size_t q = 0; q < qs.size(); q += (size_t)stride) pick.push_back(qs[q]);
    tensor4d<double> AA(n), AB(n), AC(n);
    AA.setZero();
    AB.setZero();
    AC.setZero();
    double t0 = omp_get_wtime();
#pragma omp parallel for schedule(dynamic)
    for (long long q = 0; q < (long long)pick.size(); ++q) {
      const auto& s = pick[(size_t)q];
      os.compute_contracted_shell_quartet_deriv2_pq(AA, AB, AC, b->pairs[s[0] * nshell + s[1]],
                                                    b->pairs[s[2] * nshell + s[3]], 3,
                                                    s[3] <= s[2] ? ERIOS::Permute::ALL : ERIOS::Permute::ACONLY);
    }
    *t_pq_ints = (omp_get_wtime() - t0) * (double)qs.size() / (double)std::max<size_t>(pick.size(), 1);
    const std::vector<bool>& m1 = mask[(size_t)a1];
    const std::vector<bool>& m2 = mask[(size_t)a0];
    t0 = omp_get_wtime();
    tensor4d<double> t(n);
#pragma omp parallel for schedule(dynamic)
    for (Eigen::Index i = 0; i < n; ++i)
      for (Eigen::Index j = 0; j < n; ++j)
        for (Eigen::Index k = 0; k < n; ++k)
          for (Eigen::Index l = 0; l < n; ++l) {
            const double ad = -(AA(i, j, k, l) + AB(i, j, k, l) + AC(i, j, k, l));
            const double ad1 = -(AA(i, j, k, l) + AB(j, i, k, l) + AC(k, l, i, j));
            const double dd = -(ad + AC(j, i, l, k) + AB(k, l, i, j));
            const double bc = -(AC(i, j, k, l) + AA(k, l, i, j) + AB(l, k, i, j));
            const double bc1 = -(AC(k, l, i, j) + AA(k, l, i, j) + AB(k, l, i, j));
            const double bd1 = -(ad1 + AB(l, k, i, j) + dd);
            double v = 0.0;
            if (m1[i] && m2[j]) v += AB(i, j, k, l);
            if (m1[j] && m2[i]) v += AB(j, i, k, l);
            if (m1[i] && m2[k]) v += AC(i, j, k, l);
            if (m1[k] && m2[i]) v += AC(k, l, i, j);
            if (m1[i] && m2[l]) v += ad;
            if (m1[l] && m2[i]) v += ad1;
            if (m1[j] && m2[k]) v += bc;
            if (m1[k] && m2[j]) v += bc1;
            if (m1[j] && m2[l]) v += AC(j, i, l, k);
            if (m1[l] && m2[j]) v += bd1;
            if (m1[k] && m2[l]) v += AB(k, l, i, j);
            if (m1[l] && m2[k]) v += AB(l, k, i, j);
            t(i, j, k, l) = v;
          }
    double hc = 0.0;
#pragma omp parallel for schedule(dynamic) reduction(+ : hc)
    for (Eigen::Index i = 0; i < n; ++i)
      for (Eigen::Index j = 0; j < n; ++j) {
        double gc = 0.0, ge = 0.0;
        for (Eigen::Index k = 0; k < n; ++k)
          for (Eigen::Index l = 0; l < n; ++l) {
            gc += D[(size_t)(k * n + l)] * (2.0 * t(i, j, k, l));
            ge -= D[(size_t)(k * n + l)] * t(i, k, j, l);
          }
        hc += D[(size_t)(i * n + j)] * (gc + ge);
      }
    *t_pair_pq = omp_get_wtime() - t0 + 0.0 * hc;
  }
  return 0;
}

}  // extern "C"
