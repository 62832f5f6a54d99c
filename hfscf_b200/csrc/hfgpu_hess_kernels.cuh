// Adjoint second derivatives of the two-electron energy at a fixed density: the two-electron
// part of the analytic Hessian, sum_abcd W_abcd d2(ab|cd)/dX dY, with the same weight block
// W as the adjoint gradient (RHF: W = 8 s [2 D_ab D_cd - (D_ac D_bd + D_ad D_bc)/2]).
//
// Replaces the reference's second-derivative ERI tensors and their contraction:
// Erios::compute_contracted_shell_quartet_deriv2_qq / _pq (src/integrals/hfscf_oserideriv2qq.cpp:28-853,
// hfscf_oserideriv2pq.cpp:23-891) and Mol::scf_hessian::calc_scf_hessian_tei
// (src/hessian/hfscf_hessian_ints.cpp:20-303), which store six packed derivative tensors per
// direction pair and then contract them once per atom pair.  Here nothing is stored: per unique
// shell quartet the class's generated op tables run the VRR two orders higher, the HRR of ten
// exponent-weighted sets and the contraction of every shifted integral with W, and the quartet's
// 12 x 12 block (centres A, B, C, D by x, y, z; D from translational invariance) is added into
// the 3 natoms x 3 natoms Hessian.  Four forms: hess_kernel, one thread per quartet on
// thread-interleaved global scratch (gen_eri.py gen_hess_table); hess_block_kernel with one
// block of 128 threads or one warp per quartet over levelised tables in shared memory
// (gen_hess_block); hess_line_kernel, one thread per quartet on straight-line register code
// (gen_hess_line, the classes whose terms fit at most 24 passes of 64 accumulators).
#pragma once
#include "hfgpu_kernels.cuh"

// Hessian output of a launch: 3 natoms x 3 natoms, row-major.  smem > 0: the block sums its
// contributions in shared memory (9 natoms^2 doubles) and adds them once at its end.
struct HessOut {
  double* __restrict__ hess;
  int natoms;
  int smem;
};

// Executor of a table-mode Hessian class.  Weight sets, in the generator's order:
// 1, 2a_a, 2a_b, 2a_c, (2a_a)^2, (2a_b)^2, (2a_c)^2, 2a_a 2a_b, 2a_a 2a_c, 2a_b 2a_c.
// h45: the 45 upper-triangle entries of the 9 x 9 block over (A, B, C) x (x, y, z).
template <typename Tab>
__device__ void hess_table(const PrimPair<double>* __restrict__ bp, const double* __restrict__ ea,
                           const double* __restrict__ eb, int nbp, const PrimPair<double>* __restrict__ kp,
                           const double* __restrict__ ec, int nkp, double ABx, double ABy, double ABz, double CDx,
                           double CDy, double CDz, const BoysTable<double>& boys, Strided<double> W,
                           Strided<double> vs, Strided<double> hs, Strided<double> h45) {
  using R = double;
  vs[0] = R(0);
  hs[0] = R(0);
  for (int x = 1; x <= Tab::NACC; ++x) hs[x] = R(0);
  const int4* vo = Tab::vrr();  // packed rows: gen_eri.py pack_grad_vrr / pack_hess_hrr
  const int2* ho = Tab::hrr();
  for (int ib = 0; ib < nbp; ++ib) {
    const R p = bp[ib].p, ip = bp[ib].ip, Px = bp[ib].Px, Py = bp[ib].Py, Pz = bp[ib].Pz;
    const R PAx = bp[ib].PAx, PAy = bp[ib].PAy, PAz = bp[ib].PAz, Kab = bp[ib].Kp;
    const R wa = R(2) * ea[ib], wb = R(2) * eb[ib];
    for (int ik = 0; ik < nkp; ++ik) {
      const R q = kp[ik].p, iq = kp[ik].ip, Qx = kp[ik].Px, Qy = kp[ik].Py, Qz = kp[ik].Pz;
      const R QCx = kp[ik].PAx, QCy = kp[ik].PAy, QCz = kp[ik].PAz, Kcd = kp[ik].Kp;
      const R wc = R(2) * ec[ik];
      const R pq = p + q;
      const R rsq = rsqrt_t(pq);
      const R ipq = rsq * rsq;
      const R rho = p * q * ipq;
      const R rp = q * ipq, rq = p * ipq;
      const R inv2p = R(0.5) * ip, inv2q = R(0.5) * iq, inv2pq = R(0.5) * ipq;
      const R PQx = Px - Qx, PQy = Py - Qy, PQz = Pz - Qz;
      const R T = rho * (PQx * PQx + PQy * PQy + PQz * PQz);
      const R pre = Kab * Kcd * rsq;
      R F[Tab::L + 1];
      boys.template eval<Tab::L>(T, pre, F);
#pragma unroll
      for (int m = 0; m <= Tab::L; ++m) vs[1 + m] = F[m];
      for (int o = 0; o < Tab::NVOPS; ++o) {
        const int4 op = __ldg(vo + o);
        const int kind = op.w & 15, dir = (op.w >> 4) & 15, dst = op.x & 0xffff;
        const int sa = (unsigned)op.x >> 16, sb = op.y & 0xffff, sc = (unsigned)op.y >> 16, sd = op.z & 0xffff;
        if (kind == 2) {
          R w;
          switch (dir) {
            case 0: w = R(1); break;
            case 1: w = wa; break;
            case 2: w = wb; break;
            case 3: w = wc; break;
            case 4: w = wa * wa; break;
            case 5: w = wb * wb; break;
            case 6: w = wc * wc; break;
            case 7: w = wa * wb; break;
            case 8: w = wa * wc; break;
            default: w = wb * wc; break;
          }
          hs[1 + dst] += w * vs[sa];
          continue;
        }
        const R PQd = dir == 0 ? PQx : (dir == 1 ? PQy : PQz);
        const int k1 = (op.w >> 8) & 255;
        if (kind == 0) {
          const R PA = dir == 0 ? PAx : (dir == 1 ? PAy : PAz);
          vs[dst] = PA * vs[sa] - rp * PQd * vs[sb] + small_int<R>(k1) * inv2p * (vs[sc] - rp * vs[sd]);
        } else {
          const R QC = dir == 0 ? QCx : (dir == 1 ? QCy : QCz);
          const int sg = (unsigned)op.z >> 16, k2 = (unsigned)op.w >> 16;
          vs[dst] = QC * vs[sa] + rq * PQd * vs[sb] + small_int<R>(k1) * inv2q * (vs[sc] - rq * vs[sd]) +
                    small_int<R>(k2) * inv2pq * vs[sg];
        }
      }
    }
  }
  for (int x = 0; x < 45; ++x) h45[x] = R(0);
  for (int o = 0; o < Tab::NHOPS; ++o) {
    const int2 op = __ldg(ho + o);
    const int kind = (op.y >> 16) & 15;
    const int sx = (unsigned)op.x >> 16;
    if (kind == 2) {
      const int wi = op.x & 0xffff, k = (op.y & 0xffff) - 128, hi = (op.y >> 20) & 63;
      h45[hi] += R(k) * W[wi] * hs[sx];
    } else {
      const int dst = op.x & 0xffff, sy = op.y & 0xffff, dir = (op.y >> 20) & 15;
      const R d = kind == 0 ? (dir == 0 ? ABx : (dir == 1 ? ABy : ABz)) : (dir == 0 ? CDx : (dir == 1 ? CDy : CDz));
      hs[dst] = hs[sx] + d * hs[sy];
    }
  }
}

// Position of coordinate pair (r, s), r <= s, of the 9 x 9 block in the 45-entry upper triangle.
__device__ __forceinline__ int hess_tri(int r, int s) { return r * 9 - r * (r - 1) / 2 + (s - r); }

// Adds the quartet's 12 x 12 block over centres A, B, C, D (atoms at[0..3]) into the
// 3 natoms x 3 natoms Hessian hout: the A, B, C part from the 45 entries h45, a D row or column
// as minus the sum of the A, B, C ones (translational invariance).
template <typename H>
__device__ __forceinline__ void hess_add_block(const H& h45, const int (&at)[4], double* hout, int n3) {
  // unrolled, so that a register array h45 is read at constant indexes
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      double hx[4][4];
#pragma unroll
      for (int X = 0; X < 3; ++X)
#pragma unroll
        for (int Y = 0; Y < 3; ++Y) {
          const int r = 3 * X + i, c = 3 * Y + j;
          hx[X][Y] = r <= c ? h45[hess_tri(r, c)] : h45[hess_tri(c, r)];
        }
#pragma unroll
      for (int X = 0; X < 3; ++X) hx[X][3] = -(hx[X][0] + hx[X][1] + hx[X][2]);
#pragma unroll
      for (int Y = 0; Y < 4; ++Y) hx[3][Y] = -(hx[0][Y] + hx[1][Y] + hx[2][Y]);
#pragma unroll
      for (int X = 0; X < 4; ++X)
#pragma unroll
        for (int Y = 0; Y < 4; ++Y)
          if (hx[X][Y] != 0.0) atomicAdd(hout + (size_t)(3 * at[X] + i) * n3 + 3 * at[Y] + j, hx[X][Y]);
    }
}

template <int LA, int LB, int LC, int LD, bool PURE, typename Tab>
__device__ __forceinline__ void hess_quartet(const GradArgs<double>& a, const HessOut& o, int tid, const int2 pq,
                                             double* hout, int n3) {
  using Dm = BlockDims<LA, LB, LC, LD, PURE>;
  const PairInfo P = a.pairs[pq.x];
  const PairInfo Q = a.pairs[pq.y];
  double s = 8.0;
  if (P.sa == P.sb) s *= 0.5;
  if (Q.sa == Q.sb) s *= 0.5;
  if (pq.x == pq.y) s *= 0.5;
  // scratch per thread: [VRR slots | HRR slots | 45 outputs | W cart | 2 transform buffers]
  double* base = a.scratch + tid;
  const int st = a.scratch_threads;
  Strided<double> vs{base, st};
  Strided<double> hs{base + (size_t)Tab::NVSLOT * st, st};
  Strided<double> h45{base + (size_t)(Tab::NVSLOT + Tab::NHSLOT) * st, st};
  Strided<double> Wc{base + (size_t)(Tab::NVSLOT + Tab::NHSLOT + 45) * st, st};
  Strided<double> t0{base + (size_t)(Tab::NVSLOT + Tab::NHSLOT + 45 + Dm::NCART) * st, st};
  Strided<double> t1{base + (size_t)(Tab::NVSLOT + Tab::NHSLOT + 45 + 2 * Dm::NCART) * st, st};
  if constexpr (PURE) {
    grad_weights<Dm::NA, Dm::NB, Dm::NC, Dm::ND>(a.DJ, a.cJ, a.nK, a.DK, a.cK, a.n, P.fa, P.fb, Q.fa, Q.fb, s, t0);
    // pure -> Cartesian weights, one index at a time: t0 -> t1 -> t0 -> t1 -> Wc
    const int Ls[4] = {LA, LB, LC, LD};
    int dims[4] = {Dm::NA, Dm::NB, Dm::NC, Dm::ND};
    Strided<double> src = t0, dst = t1;
    for (int stp = 0; stp < 4; ++stp) {
      const int nc = ncart_of(Ls[stp]), np = npure_of(Ls[stp]);
      int nd[4] = {dims[0], dims[1], dims[2], dims[3]};
      nd[stp] = nc;
      Strided<double> out = (stp == 3) ? Wc : dst;
      const int tot = nd[0] * nd[1] * nd[2] * nd[3];
      for (int e = 0; e < tot; ++e) {
        int id[4];
        int r = e;
        for (int qq = 3; qq >= 0; --qq) {
          id[qq] = r % nd[qq];
          r /= nd[qq];
        }
        double v = 0.0;
        for (int c = 0; c < np; ++c) {
          const double y = c_ylm[Ls[stp]][id[stp] * np + c];
          if (y == 0.0) continue;
          int jd[4] = {id[0], id[1], id[2], id[3]};
          jd[stp] = c;
          v += y * src[((jd[0] * dims[1] + jd[1]) * dims[2] + jd[2]) * dims[3] + jd[3]];
        }
        out[e] = v;
      }
      for (int qq = 0; qq < 4; ++qq) dims[qq] = nd[qq];
      Strided<double> tmp = src;
      src = dst;
      dst = tmp;
    }
  } else {
    grad_weights<Dm::NA, Dm::NB, Dm::NC, Dm::ND>(a.DJ, a.cJ, a.nK, a.DK, a.cK, a.n, P.fa, P.fb, Q.fa, Q.fb, s, Wc);
  }
  hess_table<Tab>(a.prims + P.prim_off, a.alpha_a + P.prim_off, a.alpha_b + P.prim_off, P.nprim,
                  a.prims + Q.prim_off, a.alpha_a + Q.prim_off, Q.nprim, P.ABx, P.ABy, P.ABz, Q.ABx, Q.ABy, Q.ABz,
                  a.boys, Wc, vs, hs, h45);
  const int at[4] = {P.atom_a, P.atom_b, Q.atom_a, Q.atom_b};
  hess_add_block(h45, at, hout, n3);
}

template <int LA, int LB, int LC, int LD, typename Tab>
__global__ void __launch_bounds__(128) hess_kernel(GradArgs<double> a, HessOut o, int pure,
                                                   const int2* __restrict__ quartets, int nq) {
  extern __shared__ double hess_sh[];
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int nthr = gridDim.x * blockDim.x;
  const int n3 = 3 * o.natoms;
  double* hout = o.hess;
  if (o.smem) {
    for (int i = threadIdx.x; i < n3 * n3; i += blockDim.x) hess_sh[i] = 0.0;
    __syncthreads();
    hout = hess_sh;
  }
  const int np = a.nparts > 1 ? a.nparts : 1, p0 = np > 1 ? a.part : 0;
  for (int t = tid; t < nq; t += nthr) {
    const int2 pq = quartets[(size_t)t * np + p0];
    if (pure)
      hess_quartet<LA, LB, LC, LD, true, Tab>(a, o, tid, pq, hout, n3);
    else
      hess_quartet<LA, LB, LC, LD, false, Tab>(a, o, tid, pq, hout, n3);
  }
  if (o.smem) {
    __syncthreads();
    for (int i = threadIdx.x; i < n3 * n3; i += blockDim.x)
      if (hess_sh[i] != 0.0) atomicAdd(o.hess + i, hess_sh[i]);
  }
}

// ---------------------------------------------------------------------------
// Straight-line form: one thread per quartet, the class's generated code (gen_eri.py
// gen_hess_line) with every value in registers, in passes of at most 64 accumulators.  Each pass
// adds its terms into the thread's 45 entries of the 9 x 9 block, kept in shared memory (45 x 128
// doubles per block, behind the block's Hessian when that is in shared memory too) so that they
// hold no registers through the primitive loops; the 12 x 12 block goes into the output once per
// quartet.  For the many-quartet classes, whose table forms spend their time on level barriers
// or on global scratch round trips rather than on the few dozen ops of a level.
// ---------------------------------------------------------------------------
constexpr int kHessLineThreads = 128;
constexpr int kHessLineH45Bytes = 45 * kHessLineThreads * (int)sizeof(double);

// grad_weights with every loop over the block unrolled, so that W stays in registers
template <int NA, int NB, int NC, int ND>
__device__ __forceinline__ void hess_line_weights(const double* __restrict__ DJ, double cJ, int nK,
                                                  const double* __restrict__ DK, double cK, int n, int fa, int fb,
                                                  int fc, int fd, double s8, double* W) {
#pragma unroll
  for (int i = 0; i < NA; ++i)
#pragma unroll
    for (int j = 0; j < NB; ++j) {
      const double dab = DJ ? __ldg(DJ + (size_t)(fa + i) * n + fb + j) : 0.0;
#pragma unroll
      for (int k = 0; k < NC; ++k)
#pragma unroll
        for (int l = 0; l < ND; ++l) {
          double w = DJ ? cJ * dab * __ldg(DJ + (size_t)(fc + k) * n + fd + l) : 0.0;
          for (int m = 0; m < nK; ++m) {
            const double* D = DK + (size_t)m * n * n;
            w -= 0.5 * cK *
                 (__ldg(D + (size_t)(fa + i) * n + fc + k) * __ldg(D + (size_t)(fb + j) * n + fd + l) +
                  __ldg(D + (size_t)(fa + i) * n + fd + l) * __ldg(D + (size_t)(fb + j) * n + fc + k));
          }
          W[((i * NB + j) * NC + k) * ND + l] = s8 * w;
        }
    }
}

template <int LA, int LB, int LC, int LD, bool PURE, typename Line>
__device__ __forceinline__ void hess_line_quartet(const GradArgs<double>& a, const int2 pq, Strided<double> h45,
                                                  double* hout, int n3) {
  using Dm = BlockDims<LA, LB, LC, LD, PURE>;
  const PairInfo P = a.pairs[pq.x];
  const PairInfo Q = a.pairs[pq.y];
  double s = 8.0;
  if (P.sa == P.sb) s *= 0.5;
  if (Q.sa == Q.sb) s *= 0.5;
  if (pq.x == pq.y) s *= 0.5;
  // the weight block, Cartesian, fetched by each pass after its primitive loops
  auto weights = [&](double* Wc) {
    if constexpr (PURE) {
      double Wp[Dm::NOUT];
      hess_line_weights<Dm::NA, Dm::NB, Dm::NC, Dm::ND>(a.DJ, a.cJ, a.nK, a.DK, a.cK, a.n, P.fa, P.fb, Q.fa, Q.fb, s,
                                                        Wp);
      ClassCode<LA, LB, LC, LD>::template from_pure<double>(Wp, Wc);
    } else {
      hess_line_weights<Dm::NA, Dm::NB, Dm::NC, Dm::ND>(a.DJ, a.cJ, a.nK, a.DK, a.cK, a.n, P.fa, P.fb, Q.fa, Q.fb, s,
                                                        Wc);
    }
  };
#pragma unroll
  for (int x = 0; x < 45; ++x) h45[x] = 0.0;
  Line::template run<double>(a.prims + P.prim_off, a.alpha_a + P.prim_off, a.alpha_b + P.prim_off, P.nprim,
                             a.prims + Q.prim_off, a.alpha_a + Q.prim_off, Q.nprim, P.ABx, P.ABy, P.ABz, Q.ABx,
                             Q.ABy, Q.ABz, a.boys, weights, h45);
  const int at[4] = {P.atom_a, P.atom_b, Q.atom_a, Q.atom_b};
  hess_add_block(h45, at, hout, n3);
}

// dynamic shared memory: [the block's Hessian, 9 natoms^2 doubles, when o.smem | h45 slices]
template <int LA, int LB, int LC, int LD, typename Line>
__global__ void __launch_bounds__(kHessLineThreads) hess_line_kernel(GradArgs<double> a, HessOut o, int pure,
                                                                     const int2* __restrict__ quartets, int nq) {
  extern __shared__ double hess_sh[];
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int nthr = gridDim.x * blockDim.x;
  const int n3 = 3 * o.natoms;
  double* hout = o.hess;
  double* h45_base = hess_sh;
  if (o.smem) {
    for (int i = threadIdx.x; i < n3 * n3; i += blockDim.x) hess_sh[i] = 0.0;
    __syncthreads();
    hout = hess_sh;
    h45_base = hess_sh + n3 * n3;
  }
  const Strided<double> h45{h45_base + threadIdx.x, kHessLineThreads};
  const int np = a.nparts > 1 ? a.nparts : 1, p0 = np > 1 ? a.part : 0;
  for (int t = tid; t < nq; t += nthr) {
    const int2 pq = quartets[(size_t)t * np + p0];
    if (pure)
      hess_line_quartet<LA, LB, LC, LD, true, Line>(a, pq, h45, hout, n3);
    else
      hess_line_quartet<LA, LB, LC, LD, false, Line>(a, pq, h45, hout, n3);
  }
  if (o.smem) {
    __syncthreads();
    for (int i = threadIdx.x; i < n3 * n3; i += blockDim.x)
      if (hess_sh[i] != 0.0) atomicAdd(o.hess + i, hess_sh[i]);
  }
}

// ---------------------------------------------------------------------------
// Block form: one block of NT threads per quartet over levelised tables (gen_eri.py
// gen_hess_block).  The ops of one level read only values of earlier levels, so the threads run
// a level's ops in parallel and synchronise between levels.  The VRR slots, the weights and the
// 45 outputs live in shared memory; the HRR slots (accumulators first) too when the whole table
// fits (HS_GLOBAL false), else in a per-block region of global scratch (the two largest classes).
// Each HRR level ends with its contraction rows sorted by output entry; a thread takes a
// contiguous chunk of them and adds one register sum per run of equal entries.
// ---------------------------------------------------------------------------
template <typename Tab>
__host__ __device__ constexpr int hess_block_shared_doubles(bool hs_global) {
  return Tab::NVSLOT + 1 + (hs_global ? 0 : Tab::NHSLOT + 1) + 3 * Tab::NCART + 45;
}

// NT = 128: one block per quartet; NT = 32: one warp per quartet, four quartets per 128-thread
// block, each warp with its own shared-memory region (the small classes, whose levels hold a
// few dozen ops), synchronised with __syncwarp.
template <int LA, int LB, int LC, int LD, typename Tab, bool HS_GLOBAL, int NT = 128>
__global__ void __launch_bounds__(128) hess_block_kernel(GradArgs<double> a, HessOut o, int pure,
                                                         const int2* __restrict__ quartets, int nq) {
  static_assert(NT == 128 || (NT == 32 && !HS_GLOBAL), "threads per quartet");
  using R = double;
  extern __shared__ __align__(16) unsigned char hbsm[];
  constexpr int GROUPS = 128 / NT;  // quartets per block
  const int tid = threadIdx.x % NT, grp = threadIdx.x / NT;
  R* vs = reinterpret_cast<R*>(hbsm) + (size_t)grp * hess_block_shared_doubles<Tab>(HS_GLOBAL);
  R* hs;
  R* W;
  if constexpr (HS_GLOBAL) {
    hs = a.scratch + (size_t)blockIdx.x * (Tab::NHSLOT + 1);
    W = vs + Tab::NVSLOT + 1;
  } else {
    hs = vs + Tab::NVSLOT + 1;
    W = hs + Tab::NHSLOT + 1;
  }
  R* t0 = W + Tab::NCART;
  R* t1 = t0 + Tab::NCART;
  R* h45 = t1 + Tab::NCART;
  const int n3 = 3 * o.natoms;
  const int np = a.nparts > 1 ? a.nparts : 1, p0 = np > 1 ? a.part : 0;
  for (int qb = blockIdx.x * GROUPS; qb < nq; qb += gridDim.x * GROUPS) {
    const int qi = qb + grp;
    if (qi >= nq) break;  // only a warp of an NT = 32 block gets here: its barriers are its own
    const int2 pq = quartets[(size_t)qi * np + p0];
    const PairInfo P = a.pairs[pq.x];
    const PairInfo Q = a.pairs[pq.y];
    double s8 = 8.0;
    if (P.sa == P.sb) s8 *= 0.5;
    if (Q.sa == Q.sb) s8 *= 0.5;
    if (pq.x == pq.y) s8 *= 0.5;
    // weight block in the final basis (t0 when pure), then back to Cartesian one index at a time
    const int Ls[4] = {LA, LB, LC, LD};
    int dims[4];
    for (int q = 0; q < 4; ++q) dims[q] = pure ? npure_of(Ls[q]) : ncart_of(Ls[q]);
    {
      const int tot = dims[0] * dims[1] * dims[2] * dims[3];
      R* dstw = pure ? t0 : W;
      for (int e = tid; e < tot; e += NT) {
        const int l = e % dims[3], k = (e / dims[3]) % dims[2], j = (e / (dims[3] * dims[2])) % dims[1];
        const int i = e / (dims[3] * dims[2] * dims[1]);
        const int ia = P.fa + i, jb = P.fb + j, kc = Q.fa + k, ld = Q.fb + l;
        const int n = a.n;
        double w = a.DJ ? a.cJ * __ldg(a.DJ + (size_t)ia * n + jb) * __ldg(a.DJ + (size_t)kc * n + ld) : 0.0;
        for (int m = 0; m < a.nK; ++m) {
          const double* D = a.DK + (size_t)m * n * n;
          w -= 0.5 * a.cK *
               (__ldg(D + (size_t)ia * n + kc) * __ldg(D + (size_t)jb * n + ld) +
                __ldg(D + (size_t)ia * n + ld) * __ldg(D + (size_t)jb * n + kc));
        }
        dstw[e] = s8 * w;
      }
      group_sync<NT>();
    }
    if (pure) {
      R* bufs[2] = {t1, t0};
      const R* in = t0;
      for (int st = 0; st < 4; ++st) {
        const int nc = ncart_of(Ls[st]), npu = npure_of(Ls[st]);
        int nd[4] = {dims[0], dims[1], dims[2], dims[3]};
        nd[st] = nc;
        R* out = st == 3 ? W : bufs[st & 1];
        const int tot = nd[0] * nd[1] * nd[2] * nd[3];
        for (int e = tid; e < tot; e += NT) {
          int id[4];
          int r = e;
          for (int q = 3; q >= 0; --q) {
            id[q] = r % nd[q];
            r /= nd[q];
          }
          R v = R(0);
          for (int c = 0; c < npu; ++c) {
            const double y = c_ylm[Ls[st]][id[st] * npu + c];
            if (y == 0.0) continue;
            int jd[4] = {id[0], id[1], id[2], id[3]};
            jd[st] = c;
            v += y * in[((jd[0] * dims[1] + jd[1]) * dims[2] + jd[2]) * dims[3] + jd[3]];
          }
          out[e] = v;
        }
        group_sync<NT>();
        for (int q = 0; q < 4; ++q) dims[q] = nd[q];
        in = out;
      }
    }
    for (int t = tid; t < Tab::NACC; t += NT) hs[t] = R(0);
    for (int t = tid; t < 45; t += NT) h45[t] = R(0);
    if (tid == 0) vs[Tab::NVSLOT] = R(0);
    group_sync<NT>();
    const PrimPair<R>* bp = a.prims + P.prim_off;
    const PrimPair<R>* kp = a.prims + Q.prim_off;
    const R* eA = a.alpha_a + P.prim_off;
    const R* eB = a.alpha_b + P.prim_off;
    const R* eC = a.alpha_a + Q.prim_off;
    const int4* vo = Tab::vrr();
    const int* vl = Tab::vlev();
    const int2* acc = Tab::acc();
    for (int ib = 0; ib < P.nprim; ++ib) {
      const R p = bp[ib].p, ip = bp[ib].ip, Px = bp[ib].Px, Py = bp[ib].Py, Pz = bp[ib].Pz;
      const R PAx = bp[ib].PAx, PAy = bp[ib].PAy, PAz = bp[ib].PAz, Kab = bp[ib].Kp;
      const R wa = R(2) * eA[ib], wb = R(2) * eB[ib];
      for (int ik = 0; ik < Q.nprim; ++ik) {
        const R q = kp[ik].p, iq = kp[ik].ip, Qx = kp[ik].Px, Qy = kp[ik].Py, Qz = kp[ik].Pz;
        const R QCx = kp[ik].PAx, QCy = kp[ik].PAy, QCz = kp[ik].PAz, Kcd = kp[ik].Kp;
        const R wc = R(2) * eC[ik];
        const R pqs = p + q;
        const R rs = rsqrt_t(pqs);
        const R ipq = rs * rs;
        const R rho = p * q * ipq;
        const R rp = q * ipq, rq = p * ipq;
        const R inv2p = R(0.5) * ip, inv2q = R(0.5) * iq, inv2pq = R(0.5) * ipq;
        const R PQx = Px - Qx, PQy = Py - Qy, PQz = Pz - Qz;
        const R T = rho * (PQx * PQx + PQy * PQy + PQz * PQz);
        if (tid <= Tab::L) {
          R F[Tab::L + 1];
          a.boys.template eval<Tab::L>(T, Kab * Kcd * rs, F);
#pragma unroll
          for (int m = 0; m <= Tab::L; ++m)
            if (tid == m) vs[m] = F[m];
        }
        group_sync<NT>();
        for (int l = 0; l < Tab::NVLEV; ++l) {
          const int e = __ldg(vl + l + 1);
          for (int oi = __ldg(vl + l) + tid; oi < e; oi += NT) {
            const int4 op = __ldg(vo + oi);
            const int dst = op.x & 0xffff, sa = (unsigned)op.x >> 16, sb = op.y & 0xffff, sc = (unsigned)op.y >> 16;
            const int sd = op.z & 0xffff, kd = op.w & 255, k12 = (unsigned)op.w >> 8;
            const int dir = kd >> 2;
            const R PQd = dir == 0 ? PQx : (dir == 1 ? PQy : PQz);
            const R k1 = small_int<R>(k12 & 255);
            R v;
            if ((kd & 1) == 0) {
              const R PA = dir == 0 ? PAx : (dir == 1 ? PAy : PAz);
              v = PA * vs[sa] - rp * PQd * vs[sb] + k1 * inv2p * (vs[sc] - rp * vs[sd]);
            } else {
              const R QC = dir == 0 ? QCx : (dir == 1 ? QCy : QCz);
              const int sg = (unsigned)op.z >> 16;
              v = QC * vs[sa] + rq * PQd * vs[sb] + k1 * inv2q * (vs[sc] - rq * vs[sd]) +
                  small_int<R>(k12 >> 8) * inv2pq * vs[sg];
            }
            vs[dst] = v;
          }
          group_sync<NT>();
        }
        for (int t = tid; t < Tab::NACC; t += NT) {
          const int2 ac = __ldg(acc + t);
          R w;
          switch (ac.y) {
            case 0: w = R(1); break;
            case 1: w = wa; break;
            case 2: w = wb; break;
            case 3: w = wc; break;
            case 4: w = wa * wa; break;
            case 5: w = wb * wb; break;
            case 6: w = wc * wc; break;
            case 7: w = wa * wb; break;
            case 8: w = wa * wc; break;
            default: w = wb * wc; break;
          }
          hs[t] += w * vs[ac.x];
        }
        group_sync<NT>();
      }
    }
    // HRR levels; each ends with its contraction rows (sorted by output entry), taken by the
    // threads in contiguous chunks
    const int4* ho = Tab::hrr();
    const int2* hl = Tab::hlev();
    const R ABx = P.ABx, ABy = P.ABy, ABz = P.ABz, CDx = Q.ABx, CDy = Q.ABy, CDz = Q.ABz;
    for (int l = 0; l < Tab::NHLEV; ++l) {
      const int2 lv = __ldg(hl + l);
      const int end = __ldg(hl + l + 1).x;
      for (int oi = lv.x + tid; oi < lv.y; oi += NT) {
        const int4 op = __ldg(ho + oi);
        const int dir = (op.w >> 2) & 3;
        const R d = (op.w & 1) ? (dir == 0 ? CDx : (dir == 1 ? CDy : CDz)) : (dir == 0 ? ABx : (dir == 1 ? ABy : ABz));
        hs[op.x] = hs[op.y] + d * hs[op.z];
      }
      const int nc = end - lv.y;
      if (nc > 0) {
        const int chunk = (nc + NT - 1) / NT;
        const int c0 = lv.y + tid * chunk, c1 = min(c0 + chunk, end);
        int cur = -1;
        R sum = R(0);
        for (int oi = c0; oi < c1; ++oi) {
          const int4 op = __ldg(ho + oi);
          const int hi = (op.w >> 4) & 63, k = ((op.w >> 10) & 255) - 128;
          if (hi != cur) {
            if (cur >= 0) atomicAdd(h45 + cur, sum);
            cur = hi;
            sum = R(0);
          }
          sum += R(k) * W[op.x] * hs[op.y];
        }
        if (cur >= 0) atomicAdd(h45 + cur, sum);
      }
      group_sync<NT>();
    }
    // the 12 x 12 block over centres A, B, C, D into the Hessian (D by translational invariance)
    if (tid < 9) {
      const int i = tid / 3, j = tid % 3;
      const int at[4] = {P.atom_a, P.atom_b, Q.atom_a, Q.atom_b};
      double hx[4][4];
      for (int X = 0; X < 3; ++X)
        for (int Y = 0; Y < 3; ++Y) {
          const int r = 3 * X + i, c = 3 * Y + j;
          hx[X][Y] = r <= c ? h45[hess_tri(r, c)] : h45[hess_tri(c, r)];
        }
      for (int X = 0; X < 3; ++X) hx[X][3] = -(hx[X][0] + hx[X][1] + hx[X][2]);
      for (int Y = 0; Y < 4; ++Y) hx[3][Y] = -(hx[0][Y] + hx[1][Y] + hx[2][Y]);
      for (int X = 0; X < 4; ++X)
        for (int Y = 0; Y < 4; ++Y)
          if (hx[X][Y] != 0.0) atomicAdd(o.hess + (size_t)(3 * at[X] + i) * n3 + 3 * at[Y] + j, hx[X][Y]);
    }
    group_sync<NT>();
  }
}
