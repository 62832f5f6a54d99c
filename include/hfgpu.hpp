// hfgpu: C++ classes over the C ABI of hfgpu.h, shaped like the reference's integral
// engine and Fock hooks, so that hfscf's own call sites keep their method names and
// argument order.  Header-only; link libhfgpu.so.
//
//   hfgpu::Engine     one handle: a basis (flat arrays as hfgpu_basis takes them) on one GPU,
//                     with the current geometry; replaces constructing the shell pairs
//                     (MOLEC::Molecule::create_shell_pairs, src/molecule/hfscf_molecule.cpp:661-669).
//   hfgpu::GpuErios   ERIOS::Erios (src/integrals/hfscf_oseri.hpp:27-123): packed ERIs of one
//                     shell quartet at a time and the Schwarz screen matrix.  The GPU computes
//                     every unique integral in one launch sequence on the first request after a
//                     geometry change (hfgpu_eri_packed) and each call copies its quartet's
//                     slots out of that vector; create_repulsion_matrix's loop over all quartets
//                     (src/scfsolver/hfscf_hf_hamiltonian.cpp:95-111) therefore costs one GPU
//                     pass.  The first-derivative method of the reference has no counterpart:
//                     the gradient is contracted on the GPU without storing derivative
//                     integrals (GpuGradient).
//   hfgpu::GpuJK      the Fock hooks Mol::hf_solver::update_fock_matrix
//                     (src/scfsolver/hfscf_hf_solver.cpp:254-286, declared hfscf_hf_solver.hpp:105-107)
//                     and Mol::uhf_solver::update_fock_matrix (src/scfsolver/hfscf_uhf_solver.cpp:155-191),
//                     taking the solver's row-major matrices.
//   hfgpu::GpuGradient  the two-electron term of Mol::scf_gradient::calc_scf_gradient_rhf
//                     (src/gradient/hfscf_grad_rhf.cpp:76-141) and its UHF form.
//
// Shell pairs are named by their two shell indices (ShellPairRef), in the basis order of the
// handle.  Errors throw hfgpu::Error carrying the status code and hfgpu_last_error's message.
#ifndef HFGPU_HPP
#define HFGPU_HPP

#include <cmath>
#include <stdexcept>
#include <string>
#include <vector>

#include "hfgpu.h"

namespace hfgpu {

class Error : public std::runtime_error {
 public:
  Error(int code, const std::string& msg) : std::runtime_error(msg), code_(code) {}
  int code() const { return code_; }

 private:
  int code_;
};

inline void check(int rc, const hfgpu_handle* h, const char* what) {
  if (rc != HFGPU_OK)
    throw Error(rc, std::string(what) + ": status " + std::to_string(rc) + (h ? std::string(": ") + hfgpu_last_error(h) : ""));
}

// The two shells (i, j) of a shell pair, as BASIS::ShellPair joins them (i <= j in the loops of
// create_repulsion_matrix; any order is accepted).
struct ShellPairRef {
  int i, j;
};

// Index of (ij|kl) in the packed 8-fold vector, hfscfmath::index_ijkl (src/math/hfscf_math.hpp:90-101).
inline long long index_ijkl(long long i, long long j, long long k, long long l) {
  const long long ij = i > j ? i * (i + 1) / 2 + j : j * (j + 1) / 2 + i;
  const long long kl = k > l ? k * (k + 1) / 2 + l : l * (l + 1) / 2 + k;
  return ij > kl ? ij * (ij + 1) / 2 + kl : kl * (kl + 1) / 2 + ij;
}

inline long long packed_length(long long n) { return n * (n + 1) * (n * n + n + 2) / 8; }

class Engine {
 public:
  // basis: flat arrays (unnormalised .gbs coefficients); xyz_bohr: natoms x 3.
  Engine(const hfgpu_basis& basis, const double* xyz_bohr, const hfgpu_opts* opts = nullptr)
      : L_(basis.L, basis.L + basis.nshell), pure_(basis.pure != 0), natoms_(basis.natoms) {
    hfgpu_opts o;
    if (opts) {
      o = *opts;
    } else {
      hfgpu_default_opts(&o);
    }
    check(hfgpu_create(&basis, &o, &h_), nullptr, "hfgpu_create");
    first_.resize(L_.size() + 1, 0);
    for (size_t s = 0; s < L_.size(); ++s) first_[s + 1] = first_[s] + nfunc(L_[s]);
    set_geometry(xyz_bohr);
  }
  ~Engine() { hfgpu_destroy(h_); }
  Engine(const Engine&) = delete;
  Engine& operator=(const Engine&) = delete;

  void set_geometry(const double* xyz_bohr) {
    check(hfgpu_set_geometry(h_, xyz_bohr, natoms_), h_, "hfgpu_set_geometry");
    packed_.clear();  // every cached integral belongs to the old geometry
  }
  hfgpu_handle* handle() const { return h_; }
  int nbf() const { return first_.back(); }
  int natoms() const { return natoms_; }
  bool pure() const { return pure_; }
  int nshell() const { return (int)L_.size(); }
  int shell_L(int s) const { return L_[(size_t)s]; }
  int first_function(int s) const { return first_[(size_t)s]; }
  int nfunc(int L) const { return pure_ ? 2 * L + 1 : (L + 1) * (L + 2) / 2; }

  // Every unique ERI of the current geometry, computed on the GPU on first use.
  const std::vector<double>& packed_eris() {
    if (packed_.empty()) {
      packed_.resize((size_t)packed_length(nbf()));
      check(hfgpu_eri_packed(h_, packed_.data(), (long long)packed_.size()), h_, "hfgpu_eri_packed");
    }
    return packed_;
  }

 private:
  hfgpu_handle* h_ = nullptr;
  std::vector<int> L_, first_;
  bool pure_;
  int natoms_;
  std::vector<double> packed_;
};

class GpuErios {
 public:
  // Erios(bool is_pure, double cut_off = 1e-14): screen_tol = 100 * cut_off (hfscf_oseri.hpp:31-32).
  GpuErios(Engine& engine, bool is_pure, double cut_off = 1e-14)
      : eng_(engine), cutoff_(cut_off), screen_tol_(100.0 * cut_off) {
    if (is_pure != engine.pure()) throw Error(HFGPU_ERR_INVALID, "GpuErios: is_pure differs from the engine's basis");
  }
  GpuErios(const GpuErios&) = delete;
  GpuErios& operator=(const GpuErios&) = delete;

  // compute_contracted_shell_quartet(eri, s12, s34, do_screen) (hfscf_oseri.cpp:22-246): assigns
  // the packed slots (pq|rs) of the quartet, p in shell s12.i, q in s12.j, r in s34.i, s in
  // s34.j, with p <= q and r <= s, as the reference does.  do_screen leaves the slots whose
  // Schwarz bound sqrt((pq|pq)(rs|rs)) is below screen_tol untouched (init_screen and
  // compute_screen_matrix must have filled the screen matrix, as in the reference).
  void compute_contracted_shell_quartet(double* eri, long long eri_len, ShellPairRef s12, ShellPairRef s34,
                                        bool do_screen = false) const {
    const long long n = eng_.nbf();
    if (eri_len != packed_length(n)) throw Error(HFGPU_ERR_INVALID, "compute_contracted_shell_quartet: eri length");
    if (do_screen && (long long)screen_.size() != n * n)
      throw Error(HFGPU_ERR_STATE, "compute_contracted_shell_quartet: screening without init_screen");
    const std::vector<double>& all = eng_.packed_eris();
    const int sh[4] = {s12.i, s12.j, s34.i, s34.j};
    int f0[4], f1[4];
    for (int x = 0; x < 4; ++x) {
      if (sh[x] < 0 || sh[x] >= eng_.nshell()) throw Error(HFGPU_ERR_INVALID, "shell index out of range");
      f0[x] = eng_.first_function(sh[x]);
      f1[x] = f0[x] + eng_.nfunc(eng_.shell_L(sh[x]));
    }
    for (int p = f0[0]; p < f1[0]; ++p)
      for (int q = f0[1]; q < f1[1]; ++q) {
        if (p > q) continue;
        for (int r = f0[2]; r < f1[2]; ++r)
          for (int s = f0[3]; s < f1[3]; ++s) {
            if (r > s) continue;
            if (do_screen && std::sqrt(std::fabs(screen_[(size_t)(p * n + q)] * screen_[(size_t)(r * n + s)])) < screen_tol_)
              continue;
            const long long x = index_ijkl(p, q, r, s);
            eri[x] = all[(size_t)x];
          }
      }
  }

  // init_screen(num_orbitals) / compute_screen_matrix(s12) (hfscf_oseri_screen.cpp:17-181):
  // screen(p, q) = (pq|pq) for the functions of the pair.  The reference's matrix spans
  // Cartesian functions; this one spans the engine's basis functions (pure or Cartesian).
  void init_screen(long long num_orbitals) {
    if (num_orbitals != eng_.nbf()) throw Error(HFGPU_ERR_INVALID, "init_screen: basis size");
    screen_.assign((size_t)(num_orbitals * num_orbitals), 0.0);
  }
  void compute_screen_matrix(ShellPairRef s12) {
    const long long n = eng_.nbf();
    if ((long long)screen_.size() != n * n) throw Error(HFGPU_ERR_STATE, "compute_screen_matrix before init_screen");
    const std::vector<double>& all = eng_.packed_eris();
    const int a0 = eng_.first_function(s12.i), a1 = a0 + eng_.nfunc(eng_.shell_L(s12.i));
    const int b0 = eng_.first_function(s12.j), b1 = b0 + eng_.nfunc(eng_.shell_L(s12.j));
    for (int p = a0; p < a1; ++p)
      for (int q = b0; q < b1; ++q) {
        const double v = all[(size_t)index_ijkl(p, q, p, q)];
        screen_[(size_t)(p * n + q)] = screen_[(size_t)(q * n + p)] = v;
      }
  }
  const std::vector<double>& screen() const { return screen_; }
  double cutoff() const { return cutoff_; }
  double screen_tol() const { return screen_tol_; }

 private:
  Engine& eng_;
  double cutoff_, screen_tol_;
  std::vector<double> screen_;
};

class GpuJK {
 public:
  explicit GpuJK(Engine& engine, hfgpu_precision precision = HFGPU_FP64) : eng_(engine), precision_(precision) {}

  // RHF: f_mat = hcore_mat + 2 J[d_mat] - K[d_mat] (hfscf_hf_solver.cpp:261-278), row-major N x N.
  void update_fock_matrix(const double* d_mat, const double* hcore_mat, double* f_mat) const {
    check(hfgpu_fock_rhf(eng_.handle(), d_mat, hcore_mat, f_mat, precision_), eng_.handle(), "hfgpu_fock_rhf");
  }
  // UHF: f_mat = H + J[Da + Db] - K[Da], f_mat_b = H + J[Da + Db] - K[Db] (hfscf_uhf_solver.cpp:160-180).
  void update_fock_matrix(const double* d_mat, const double* d_mat_b, const double* hcore_mat, double* f_mat,
                          double* f_mat_b) const {
    check(hfgpu_fock_uhf(eng_.handle(), d_mat, d_mat_b, hcore_mat, f_mat, f_mat_b, precision_), eng_.handle(),
          "hfgpu_fock_uhf");
  }
  // The direct-SCF hook (hfscf_hf_solver.cpp:288-291, disabled in the reference): the same build.
  void update_fock_matrix_scf_direct(const double* d_mat, const double* hcore_mat, double* f_mat) const {
    update_fock_matrix(d_mat, hcore_mat, f_mat);
  }
  // Incremental build F += 2 J[dD] - K[dD].
  void update_fock_matrix_delta(const double* delta_d_mat, double* f_mat) const {
    check(hfgpu_fock_delta(eng_.handle(), delta_d_mat, f_mat, precision_), eng_.handle(), "hfgpu_fock_delta");
  }

 private:
  Engine& eng_;
  hfgpu_precision precision_;
};

class GpuGradient {
 public:
  explicit GpuGradient(Engine& engine, hfgpu_precision precision = HFGPU_FP64) : eng_(engine), precision_(precision) {}
  // grad (natoms x 3, row-major) += the two-electron RHF gradient at d_mat: the contraction of
  // hfscf_grad_rhf.cpp:121-141 over the derivative integrals, computed without storing them.
  void calc_two_electron_gradient_rhf(const double* d_mat, double* grad) const {
    check(hfgpu_grad2e_backward(eng_.handle(), d_mat, 1.0, grad, precision_), eng_.handle(), "hfgpu_grad2e_backward");
  }
  // UHF form (hfscf_grad_uhf.cpp:124-150).
  void calc_two_electron_gradient_uhf(const double* d_mat, const double* d_mat_b, double* grad) const {
    check(hfgpu_grad2e_uhf_backward(eng_.handle(), d_mat, d_mat_b, 1.0, grad, precision_), eng_.handle(),
          "hfgpu_grad2e_uhf_backward");
  }

 private:
  Engine& eng_;
  hfgpu_precision precision_;
};

// The two-electron part of the analytic Hessian, in place of Mol::scf_hessian::calc_scf_hessian_tei
// (src/hessian/hfscf_hessian_ints.cpp:20-303): hess (3 natoms x 3 natoms, row-major) += the
// reference's m_hessianC + m_hessianEx at d_mat, from second-derivative integrals that are never stored.
class GpuHessian {
 public:
  explicit GpuHessian(Engine& engine) : eng_(engine) {}
  void calc_scf_hessian_tei(const double* d_mat, double* hess) const {
    check(hfgpu_hess2e(eng_.handle(), d_mat, 1.0, hess), eng_.handle(), "hfgpu_hess2e");
  }
  void calc_scf_hessian_tei_uhf(const double* d_mat_a, const double* d_mat_b, double* hess) const {
    check(hfgpu_hess2e_uhf(eng_.handle(), d_mat_a, d_mat_b, 1.0, hess), eng_.handle(), "hfgpu_hess2e_uhf");
  }

 private:
  Engine& eng_;
};

}  // namespace hfgpu

#endif
