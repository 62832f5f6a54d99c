// Batched SCF density by trace-correcting purification (TC2; Niklasson, Phys. Rev. B 66,
// 155115 (2002)): one thread block per molecule, the molecule's whole matrix and its square in
// shared memory, so a step needs no other block and a molecule stops at its own converged step.
// Replaces the batched Jacobi diagonalisation of the SCF iterations (the projector onto the nocc
// lowest eigenvectors is C_occ C_occ^T of Mol::hf_solver::calc_density_matrix,
// src/scfsolver/hfscf_hf_solver.cpp:206-231); the same steps as the single-molecule purification.
#pragma once
#include <cuda_runtime.h>

constexpr int kBatchPurifyThreads = 512;
constexpr int kBatchPurifyMaxN = 116;  // 2 (n rounded up to 4)^2 doubles of shared memory <= 227 KB

__host__ __device__ inline int batch_purify_stride(int n) { return (n + 3) & ~3; }

inline size_t batch_purify_smem_bytes(int nmax) {
  const size_t s = (size_t)batch_purify_stride(nmax);
  return 2 * s * s * sizeof(double);
}

// Fo: nmol x nmax x nmax (padded; molecule b uses its leading n_b x n_b block).  P: the same
// layout, zero outside each block.  err[b] = tr P - tr P^2 at the step that converged, or 1.
// The square C = A A takes 4 x 4 output tiles of the upper triangle per thread; A is symmetric,
// so A_ik = A_ki and both operands of a tile are rows of A (two 32-byte loads per k).
__global__ void __launch_bounds__(kBatchPurifyThreads) batch_purify_kernel(
    const double* __restrict__ Fo, int nmax, const int* __restrict__ mol_n, const int* __restrict__ nocc,
    int max_steps, double tol, double* __restrict__ P, double* __restrict__ err) {
  extern __shared__ __align__(16) double bp_sm[];
  __shared__ double red[2][kBatchPurifyThreads];
  const int b = blockIdx.x;
  const int n = mol_n[b], no = nocc[b];
  const int s = batch_purify_stride(n);
  double* A = bp_sm;
  double* C = bp_sm + (size_t)s * s;
  const double* F = Fo + (size_t)b * nmax * nmax;
  double* Pb = P + (size_t)b * nmax * nmax;
  const int tid = threadIdx.x;
  // Gershgorin bounds of the molecule's block
  double lo = 1e300, hi = -1e300;
  for (int i = tid; i < n; i += blockDim.x) {
    double r = 0.0;
    for (int j = 0; j < n; ++j)
      if (j != i) r += fabs(F[(size_t)i * nmax + j]);
    lo = fmin(lo, F[(size_t)i * nmax + i] - r);
    hi = fmax(hi, F[(size_t)i * nmax + i] + r);
  }
  red[0][tid] = lo;
  red[1][tid] = hi;
  __syncthreads();
  for (int off = blockDim.x / 2; off > 0; off >>= 1) {
    if (tid < off) {
      red[0][tid] = fmin(red[0][tid], red[0][tid + off]);
      red[1][tid] = fmax(red[1][tid], red[1][tid + off]);
    }
    __syncthreads();
  }
  const double emin = red[0][0], emax = red[1][0];
  __syncthreads();
  for (int e = tid; e < s * s; e += blockDim.x) {
    const int i = e / s, j = e % s;
    A[e] = (i < n && j < n) ? ((i == j ? emax : 0.0) - F[(size_t)i * nmax + j]) / (emax - emin) : 0.0;
  }
  __syncthreads();
  const int nt = s / 4;
  const int ntiles = nt * (nt + 1) / 2;
  double e_out = 1.0;
  for (int k = 0; k < max_steps; ++k) {
    // C = A A on the upper-triangle tiles, mirrored into the lower triangle
    for (int t = tid; t < ntiles; t += blockDim.x) {
      int ti = 0, rem = t;
      while (rem >= nt - ti) {
        rem -= nt - ti;
        ++ti;
      }
      const int tj = ti + rem;
      const int i0 = 4 * ti, j0 = 4 * tj;
      double c[4][4];
#pragma unroll
      for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int q = 0; q < 4; ++q) c[p][q] = 0.0;
      for (int kk = 0; kk < s; ++kk) {
        const double2 a01 = *reinterpret_cast<const double2*>(A + (size_t)kk * s + i0);
        const double2 a23 = *reinterpret_cast<const double2*>(A + (size_t)kk * s + i0 + 2);
        const double2 b01 = *reinterpret_cast<const double2*>(A + (size_t)kk * s + j0);
        const double2 b23 = *reinterpret_cast<const double2*>(A + (size_t)kk * s + j0 + 2);
        const double av[4] = {a01.x, a01.y, a23.x, a23.y}, bv[4] = {b01.x, b01.y, b23.x, b23.y};
#pragma unroll
        for (int p = 0; p < 4; ++p)
#pragma unroll
          for (int q = 0; q < 4; ++q) c[p][q] = fma(av[p], bv[q], c[p][q]);
      }
#pragma unroll
      for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          C[(size_t)(i0 + p) * s + j0 + q] = c[p][q];
          C[(size_t)(j0 + q) * s + i0 + p] = c[p][q];
        }
    }
    __syncthreads();
    double ta = 0.0, tc = 0.0;
    for (int i = tid; i < n; i += blockDim.x) {
      ta += A[(size_t)i * s + i];
      tc += C[(size_t)i * s + i];
    }
    red[0][tid] = ta;
    red[1][tid] = tc;
    __syncthreads();
    for (int off = blockDim.x / 2; off > 0; off >>= 1) {
      if (tid < off) {
        red[0][tid] += red[0][tid + off];
        red[1][tid] += red[1][tid + off];
      }
      __syncthreads();
    }
    const double tr = red[0][0], tr2 = red[1][0];
    __syncthreads();
    if (tr - tr2 < tol) {  // block-uniform: every thread read the same sums
      e_out = tr - tr2;
      break;
    }
    const bool up = tr > (double)no;
    for (int e = tid; e < s * s; e += blockDim.x) A[e] = up ? C[e] : 2.0 * A[e] - C[e];
    __syncthreads();
  }
  for (int e = tid; e < nmax * nmax; e += blockDim.x) {
    const int i = e / nmax, j = e % nmax;
    Pb[e] = (i < n && j < n) ? A[(size_t)i * s + j] : 0.0;
  }
  if (tid == 0) err[b] = e_out;
}
