// Batched symmetric eigensolver for the SCF of many small molecules: one thread block per
// molecule, cyclic Jacobi with the round-robin (tournament) ordering, matrix and
// eigenvectors in shared memory.
//
// Each round applies n/2 disjoint plane rotations at once: the rotation of pair (p, q) is
// taken from a_pp, a_qq, a_pq (Golub & Van Loan, Matrix Computations, sym.schur2:
// tau = (a_qq - a_pp) / 2 a_pq, t = sign(tau) / (|tau| + sqrt(1 + tau^2)), c = 1/sqrt(1 + t^2),
// s = t c), then rows p, q of A are rotated for every pair, then columns p, q of A and of V.
// n - 1 rounds (n even; a dummy index pads odd n) make one sweep over every pair; sweeps
// repeat until the off-diagonal part is below 1e-14 of the diagonal (relative, squared
// norms) or `max_sweeps` have run.  Eigenvalues are returned ascending with their
// eigenvectors (columns); entries of the padded matrices outside a molecule's n_m x n_m
// block pass through (identity eigenvectors, their diagonal as eigenvalues).
//
// The reference diagonalises one molecule at a time with Eigen's SelfAdjointEigenSolver
// (src/scfsolver/hfscf_hf_solver.cpp:206-242); this kernel has no counterpart there.
#pragma once
#include <cuda_runtime.h>

constexpr int kJacobiThreads = 512;
constexpr int kJacobiMaxN = 118;  // two (n+1) x n FP64 arrays in 227 KB of shared memory

__host__ __device__ inline size_t jacobi_smem_bytes(int n) {
  const int ld = n + 1;
  return sizeof(double) * ((size_t)2 * ld * n + 2 * (n / 2 + 1) + kJacobiThreads / 32 * 2) +
         sizeof(int) * 2 * (n / 2 + 1);
}

__global__ void __launch_bounds__(kJacobiThreads) batch_jacobi_kernel(const double* __restrict__ A, int nmax,
                                                                     const int* __restrict__ mol_n, double* W,
                                                                     double* V, int max_sweeps, int* sweeps_out) {
  extern __shared__ __align__(16) double jsm[];
  const int mol = blockIdx.x;
  const int n = mol_n[mol];
  const int ld = n + 1;  // odd pitch: rows and columns both spread over the banks
  const int npair = (n + 1) / 2;
  double* a = jsm;
  double* v = a + (size_t)ld * n;
  double* cs = v + (size_t)ld * n;        // c, s per pair
  double* red = cs + 2 * (n / 2 + 1);     // block reduction scratch
  int* pq = reinterpret_cast<int*>(red + kJacobiThreads / 32 * 2);
  const int tid = threadIdx.x, nt = blockDim.x;
  const double* Am = A + (size_t)mol * nmax * nmax;
  for (int x = tid; x < n * n; x += nt) {
    const int i = x / n, j = x % n;
    a[i * ld + j] = Am[(size_t)i * nmax + j];
    v[i * ld + j] = i == j ? 1.0 : 0.0;
  }
  __syncthreads();
  const int N = n + (n & 1);  // tournament size; index n is the dummy when n is odd
  int sweep = 0;
  for (; sweep < max_sweeps; ++sweep) {
    // convergence: off-diagonal and diagonal squared norms
    double off = 0.0, dia = 0.0;
    for (int x = tid; x < n * n; x += nt) {
      const int i = x / n, j = x % n;
      const double e = a[i * ld + j];
      if (i == j) dia += e * e; else off += e * e;
    }
    for (int o = 16; o > 0; o >>= 1) {
      off += __shfl_xor_sync(0xffffffffu, off, o);
      dia += __shfl_xor_sync(0xffffffffu, dia, o);
    }
    if ((tid & 31) == 0) {
      red[2 * (tid >> 5)] = off;
      red[2 * (tid >> 5) + 1] = dia;
    }
    __syncthreads();
    off = dia = 0.0;
    for (int w = 0; w < nt / 32; ++w) {
      off += red[2 * w];
      dia += red[2 * w + 1];
    }
    __syncthreads();  // red is rewritten next sweep
    if (!(off > 1e-28 * dia)) break;  // also stops on 0/0 (n = 1) and NaN
    for (int r = 0; r < N - 1; ++r) {
      // pairs of this round: position 0 is fixed, the others rotate
      for (int k = tid; k < npair; k += nt) {
        const int i0 = k, i1 = N - 1 - k;
        const int p0 = i0 == 0 ? 0 : 1 + (i0 - 1 + r) % (N - 1);
        const int q0 = i1 == 0 ? 0 : 1 + (i1 - 1 + r) % (N - 1);
        const int p = min(p0, q0), q = max(p0, q0);
        double c = 1.0, s = 0.0;
        if (q < n) {
          const double apq = a[p * ld + q];
          if (apq != 0.0) {
            const double tau = (a[q * ld + q] - a[p * ld + p]) / (2.0 * apq);
            const double t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
            c = rsqrt(1.0 + t * t);
            s = t * c;
          }
        }
        pq[2 * k] = p;
        pq[2 * k + 1] = q < n ? q : -1;
        cs[2 * k] = c;
        cs[2 * k + 1] = s;
      }
      __syncthreads();
      // rows p, q of A
      for (int x = tid; x < npair * n; x += nt) {
        const int k = x / n, j = x % n;
        const int q = pq[2 * k + 1];
        if (q < 0) continue;
        const int p = pq[2 * k];
        const double c = cs[2 * k], s = cs[2 * k + 1];
        const double ap = a[p * ld + j], aq = a[q * ld + j];
        a[p * ld + j] = c * ap - s * aq;
        a[q * ld + j] = s * ap + c * aq;
      }
      __syncthreads();
      // columns p, q of A and V
      for (int x = tid; x < npair * n; x += nt) {
        const int k = x / n, i = x % n;
        const int q = pq[2 * k + 1];
        if (q < 0) continue;
        const int p = pq[2 * k];
        const double c = cs[2 * k], s = cs[2 * k + 1];
        const double ap = a[i * ld + p], aq = a[i * ld + q];
        a[i * ld + p] = c * ap - s * aq;
        a[i * ld + q] = s * ap + c * aq;
        const double vp = v[i * ld + p], vq = v[i * ld + q];
        v[i * ld + p] = c * vp - s * vq;
        v[i * ld + q] = s * vp + c * vq;
      }
      __syncthreads();
      for (int k = tid; k < npair; k += nt) {  // the rotated pair is now decoupled
        const int q = pq[2 * k + 1];
        if (q < 0) continue;
        const int p = pq[2 * k];
        a[p * ld + q] = 0.0;
        a[q * ld + p] = 0.0;
      }
      __syncthreads();
    }
  }
  if (tid == 0 && sweeps_out) sweeps_out[mol] = sweep;
  // ascending order: rank of eigenvalue i (ties by index)
  double* Wm = W + (size_t)mol * nmax;
  double* Vm = V + (size_t)mol * nmax * nmax;
  for (int i = tid; i < n; i += nt) {
    const double wi = a[i * ld + i];
    int rank = 0;
    for (int j = 0; j < n; ++j) {
      const double wj = a[j * ld + j];
      rank += (wj < wi || (wj == wi && j < i)) ? 1 : 0;
    }
    Wm[rank] = wi;
    for (int row = 0; row < n; ++row) Vm[(size_t)row * nmax + rank] = v[row * ld + i];
    for (int row = n; row < nmax; ++row) Vm[(size_t)row * nmax + rank] = 0.0;
  }
  // padding: identity eigenvectors, diagonal eigenvalues
  for (int x = tid; x < (nmax - n) * nmax; x += nt) {
    const int col = n + x / nmax, row = x % nmax;
    Vm[(size_t)row * nmax + col] = row == col ? 1.0 : 0.0;
    if (row == col) Wm[col] = Am[(size_t)col * nmax + col];
  }
}
