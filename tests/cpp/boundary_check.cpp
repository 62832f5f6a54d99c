// A C++ caller of the engine through include/hfgpu.hpp, built with g++ by tests/test_cpp_boundary.py:
// the loops the reference runs over its integral engine and Fock hook, written against the
// GPU classes.
//
// Usage: boundary_check INPUT OUTPUT
//   INPUT (whitespace-separated numbers): nshell natoms pure; L[nshell]; atom[nshell];
//     nprim[nshell]; exps[sum nprim]; coefs[sum nprim]; xyz[natoms*3] (bohr); D[n*n]; H[n*n]
//   OUTPUT (raw float64): the packed ERI vector filled quartet by quartet as
//     create_repulsion_matrix fills it (src/scfsolver/hfscf_hf_hamiltonian.cpp:77-111, screening
//     on), F = H + 2J[D] - K[D], the two-electron gradient (natoms x 3) and the two-electron
//     Hessian (3 natoms x 3 natoms)
#include <cstdio>
#include <fstream>
#include <iostream>
#include <vector>

#include "hfgpu.hpp"

int main(int argc, char** argv) {
  if (argc != 3) {
    std::cerr << "usage: boundary_check INPUT OUTPUT\n";
    return 2;
  }
  std::ifstream in(argv[1]);
  int nshell = 0, natoms = 0, pure = 0;
  in >> nshell >> natoms >> pure;
  std::vector<int> L(nshell), atom(nshell), nprim(nshell);
  for (int& v : L) in >> v;
  for (int& v : atom) in >> v;
  int np = 0;
  for (int& v : nprim) {
    in >> v;
    np += v;
  }
  std::vector<double> exps(np), coefs(np), xyz(3 * natoms);
  for (double& v : exps) in >> v;
  for (double& v : coefs) in >> v;
  for (double& v : xyz) in >> v;
  const hfgpu_basis b{nshell, natoms, pure, L.data(), atom.data(), nprim.data(), exps.data(), coefs.data()};
  try {
    hfgpu::Engine eng(b, xyz.data());
    const int n = eng.nbf();
    std::vector<double> D((size_t)n * n), H((size_t)n * n), F((size_t)n * n), grad(3 * (size_t)natoms, 0.0);
    for (double& v : D) in >> v;
    for (double& v : H) in >> v;
    if (!in) {
      std::cerr << "short input\n";
      return 2;
    }
    // the reference's ERI generation loop with screening on (hfscf_hf_hamiltonian.cpp:77-111)
    hfgpu::GpuErios os(eng, pure != 0);
    os.init_screen(n);
    for (int i = 0; i < nshell; ++i)
      for (int j = i; j < nshell; ++j) os.compute_screen_matrix({i, j});
    std::vector<double> eri((size_t)hfgpu::packed_length(n), 0.0);
    for (int i = 0; i < nshell; ++i)
      for (int j = i; j < nshell; ++j)
        for (int k = 0; k < nshell; ++k)
          for (int l = k; l < nshell; ++l) {
            const long long ij = (long long)j * (j + 1) / 2 + i, kl = (long long)l * (l + 1) / 2 + k;
            if (ij > kl) continue;
            os.compute_contracted_shell_quartet(eri.data(), (long long)eri.size(), {i, j}, {k, l}, true);
          }
    hfgpu::GpuJK jk(eng);
    jk.update_fock_matrix(D.data(), H.data(), F.data());
    hfgpu::GpuGradient gr(eng);
    gr.calc_two_electron_gradient_rhf(D.data(), grad.data());
    std::vector<double> hess(9 * (size_t)natoms * natoms, 0.0);
    hfgpu::GpuHessian(eng).calc_scf_hessian_tei(D.data(), hess.data());
    FILE* out = std::fopen(argv[2], "wb");
    if (!out) return 2;
    std::fwrite(eri.data(), sizeof(double), eri.size(), out);
    std::fwrite(F.data(), sizeof(double), F.size(), out);
    std::fwrite(grad.data(), sizeof(double), grad.size(), out);
    std::fwrite(hess.data(), sizeof(double), hess.size(), out);
    std::fclose(out);
  } catch (const hfgpu::Error& e) {
    std::cerr << "hfgpu error " << e.code() << ": " << e.what() << "\n";
    return 1;
  }
  return 0;
}
