// One-electron integrals on the host (see hfgpu_onee.cpp).
#pragma once

struct OneEBasis {
  int nshell, n, pure;
  const int* L;
  const int* atom;
  const int* nprim;
  const int* off;    // first primitive of each shell
  const int* first;  // first function of each shell (final basis)
  const double* exps;
  const double* coefs;  // normalised
};

void hfgpu_onee_matrices(const OneEBasis& b, const double* Zc, const double* xyz, int natoms, double* S, double* T,
                         double* V);
void hfgpu_onee_gradient(const OneEBasis& b, const double* Zc, const double* xyz, int natoms, const double* D,
                         const double* W, double cH, double cS, double* grad);
// Cartesian -> pure coefficients, (L+1)(L+2)/2 x (2L+1) row-major (the reference's Ylm_transmat).
void hfgpu_onee_ylm(int L, double* out);
