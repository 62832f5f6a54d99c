// Two-electron kernels, templated on the shell-quartet class.
//
// One thread owns one unique shell quartet (ab|cd) (a b and c d canonical pairs,
// pair(ab) <= pair(cd) in the sorted pair order) and
//   * computes its contracted block with the class's generated VRR/HRR code,
//   * transforms it to spherical functions when the basis is pure,
//   * digests it straight into J and K (FP64 atomics into half-matrices that are
//     symmetrised afterwards), or contracts it with density weights for the
//     adjoint gradient.
// Quartets are listed per class (one launch per class), grouped by primitive
// counts so that a warp's threads run loops of equal length.
#pragma once
#include "hfgpu_common.cuh"
#include "generated/common.cuh"

// Arguments shared by every J/K launch.
template <typename R>
struct JKArgs {
  const PairInfo* __restrict__ pairs;
  const PrimPair<R>* __restrict__ prims;
  BoysTable<R> boys;
  int n;                             // basis functions
  int nshell;
  const double* __restrict__ DJ;     // density for J (n x n) or nullptr
  int nK;                            // densities for K
  const double* __restrict__ DK;     // nK x n x n
  double* __restrict__ Jh;           // n x n half accumulator (symmetrised later)
  double* __restrict__ Kh;           // nK x n x n
  const float* __restrict__ dmax;    // nshell x nshell max |D| over all densities, or nullptr
  double dtol;                       // density-weighted screening threshold
  const long long* __restrict__ mol_off;  // batched handle: start of each molecule's n_m x n_m block, else nullptr
  const int* __restrict__ mol_n;          // batched handle: n_m
  unsigned long long* __restrict__ counters;  // per class: computed, skipped by density, primitive quartets
};

template <typename R>
struct GradArgs {
  const PairInfo* __restrict__ pairs;
  const PrimPair<R>* __restrict__ prims;
  const R* __restrict__ alpha_a;     // per primitive pair: exponent of shell a
  const R* __restrict__ alpha_b;     // per primitive pair: exponent of shell b
  BoysTable<R> boys;
  int n;
  const double* __restrict__ DJ;
  double cJ;
  int nK;
  const double* __restrict__ DK;
  double cK;
  double* __restrict__ grad;         // natoms x 3
  const long long* __restrict__ mol_off;  // batched handle (see JKArgs)
  const int* __restrict__ mol_n;
  R* __restrict__ scratch;           // thread-interleaved scratch (table-mode classes)
  int scratch_threads;               // threads sharing the scratch (stride)
  int smem_atoms;                    // grad_kernel: > 0 = accumulate 3 x smem_atoms entries per block in
                                     // shared memory, then one atomic per entry (0: atomics into grad)
  int warp_split;                    // grad_warp_kernel: 1 = four launches, one accumulator set each
  int warp_threads;                  // grad_warp_kernel: threads per quartet (32, 128 or 256; 0 = 32)
  int part, nparts;                  // partitioned gradients: the launch's quartet t is list entry
                                     // t * nparts + part (nparts <= 1: t); nq counts this part's
};

template <int NA, int NB, int NC, int ND>
__device__ __forceinline__ void load_block(const double* __restrict__ D, int n, int f0, int f1, int n0, int n1,
                                           double* out) {
#pragma unroll
  for (int i = 0; i < n0; ++i)
#pragma unroll
    for (int j = 0; j < n1; ++j) out[i * n1 + j] = __ldg(D + (size_t)(f0 + i) * n + f1 + j);
}

// J/K digestion of one block V[a][b][c][d] (final basis), scaled by the quartet's
// degeneracy s: Jh_ab += 2s sum_cd D_cd V, Jh_cd += 2s sum_ab D_ab V,
// Kh_ac += s sum_bd D_bd V, Kh_ad += s D_bc V, Kh_bc += s D_ad V, Kh_bd += s D_ac V.
// coop: all 32 lanes of the warp call this with valid quartets of the same bra pair.
template <int NA, int NB, int NC, int ND>
__device__ __forceinline__ void digest_jk(const double* V, int fa, int fb, int fc, int fd, double s,
                                          const double* __restrict__ DJ,
                                          int nK, const double* __restrict__ DK, double* Jh, double* Kh, int n,
                                          bool coop = false) {
  constexpr int NV = NA * NB * NC * ND;
  constexpr bool SMALL = NV <= 81;
  if (DJ != nullptr) {
    double dcd[NC * ND], dab[NA * NB];
    load_block<NA, NB, NC, ND>(DJ, n, fc, fd, NC, ND, dcd);
    load_block<NA, NB, NC, ND>(DJ, n, fa, fb, NA, NB, dab);
    double jcd[NC * ND];
#pragma unroll
    for (int x = 0; x < NC * ND; ++x) jcd[x] = 0.0;
#pragma unroll(SMALL ? NA * NB : 1)
    for (int ab = 0; ab < NA * NB; ++ab) {
      double jab = 0.0;
      const double dv = dab[ab];
#pragma unroll
      for (int cd = 0; cd < NC * ND; ++cd) {
        const double v = V[ab * NC * ND + cd];
        jab += dcd[cd] * v;
        jcd[cd] += dv * v;
      }
      if (coop) {
        // the whole warp shares this bra pair: one atomic per J_ab element
        double v = 2.0 * s * jab;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
        if ((threadIdx.x & 31) == 0) atomicAdd(Jh + (size_t)(fa + ab / NB) * n + fb + ab % NB, v);
      } else {
        atomicAdd(Jh + (size_t)(fa + ab / NB) * n + fb + ab % NB, 2.0 * s * jab);
      }
    }
#pragma unroll
    for (int cd = 0; cd < NC * ND; ++cd) atomicAdd(Jh + (size_t)(fc + cd / ND) * n + fd + cd % ND, 2.0 * s * jcd[cd]);
  }
  for (int m = 0; m < nK; ++m) {
    const double* D = DK + (size_t)m * n * n;
    double* K = Kh + (size_t)m * n * n;
    double dbd[NB * ND], dbc[NB * NC], dad[NA * ND], dac[NA * NC];
    load_block<NA, NB, NC, ND>(D, n, fb, fd, NB, ND, dbd);
    load_block<NA, NB, NC, ND>(D, n, fb, fc, NB, NC, dbc);
    load_block<NA, NB, NC, ND>(D, n, fa, fd, NA, ND, dad);
    load_block<NA, NB, NC, ND>(D, n, fa, fc, NA, NC, dac);
    double kbc[NB * NC], kbd[NB * ND];
#pragma unroll
    for (int x = 0; x < NB * NC; ++x) kbc[x] = 0.0;
#pragma unroll
    for (int x = 0; x < NB * ND; ++x) kbd[x] = 0.0;
#pragma unroll(SMALL ? NA : 1)
    for (int i = 0; i < NA; ++i) {
      double kac[NC], kad[ND];
#pragma unroll
      for (int x = 0; x < NC; ++x) kac[x] = 0.0;
#pragma unroll
      for (int x = 0; x < ND; ++x) kad[x] = 0.0;
#pragma unroll
      for (int j = 0; j < NB; ++j)
#pragma unroll
        for (int k = 0; k < NC; ++k)
#pragma unroll
          for (int l = 0; l < ND; ++l) {
            const double v = V[((i * NB + j) * NC + k) * ND + l];
            kac[k] += dbd[j * ND + l] * v;
            kad[l] += dbc[j * NC + k] * v;
            kbc[j * NC + k] += dad[i * ND + l] * v;
            kbd[j * ND + l] += dac[i * NC + k] * v;
          }
#pragma unroll
      for (int k = 0; k < NC; ++k) atomicAdd(K + (size_t)(fa + i) * n + fc + k, s * kac[k]);
#pragma unroll
      for (int l = 0; l < ND; ++l) atomicAdd(K + (size_t)(fa + i) * n + fd + l, s * kad[l]);
    }
#pragma unroll
    for (int x = 0; x < NB * NC; ++x) atomicAdd(K + (size_t)(fb + x / NC) * n + fc + x % NC, s * kbc[x]);
#pragma unroll
    for (int x = 0; x < NB * ND; ++x) atomicAdd(K + (size_t)(fb + x / ND) * n + fd + x % ND, s * kbd[x]);
  }
}

template <int LA, int LB, int LC, int LD, bool PURE>
struct BlockDims {
  static constexpr int CA = ncart_of(LA), CB = ncart_of(LB), CC = ncart_of(LC), CD = ncart_of(LD);
  static constexpr int NA = PURE ? npure_of(LA) : CA, NB = PURE ? npure_of(LB) : CB;
  static constexpr int NC = PURE ? npure_of(LC) : CC, ND = PURE ? npure_of(LD) : CD;
  static constexpr int NCART = CA * CB * CC * CD;
  static constexpr int NOUT = NA * NB * NC * ND;
};

// Contracted block of quartet (P|Q) in the final basis, as doubles.
template <int LA, int LB, int LC, int LD, typename R, bool PURE>
__device__ __forceinline__ void finish_block(const R* cart, double* V) {
  using Dm = BlockDims<LA, LB, LC, LD, PURE>;
  if constexpr (PURE) {
    R pure[Dm::NOUT];
    ClassCode<LA, LB, LC, LD>::template to_pure<R>(cart, pure);
#pragma unroll
    for (int x = 0; x < Dm::NOUT; ++x) V[x] = double(pure[x]);
  } else {
#pragma unroll
    for (int x = 0; x < Dm::NOUT; ++x) V[x] = double(cart[x]);
  }
}

template <int LA, int LB, int LC, int LD, typename R>
__device__ __forceinline__ void cart_block(const PairInfo& P, const PairInfo& Q, const PrimPair<R>* prims,
                                           const BoysTable<R>& boys, R* cart) {
  ClassCode<LA, LB, LC, LD>::template eri<R>(prims + P.prim_off, P.nprim, prims + Q.prim_off, Q.nprim,
                                              R(P.ABx), R(P.ABy), R(P.ABz), R(Q.ABx), R(Q.ABy), R(Q.ABz), boys, cart);
}

__device__ __forceinline__ long long packed_index(long long i, long long j, long long k, long long l) {
  const long long ij = i > j ? i * (i + 1) / 2 + j : j * (j + 1) / 2 + i;
  const long long kl = k > l ? k * (k + 1) / 2 + l : l * (l + 1) / 2 + k;
  return ij > kl ? ij * (ij + 1) / 2 + kl : kl * (kl + 1) / 2 + ij;
}

enum : int { QMODE_JK = 0, QMODE_PACKED = 1, QMODE_SCHWARZ = 2 };

// Matrix block of the quartet's molecule: offset into D/J/K storage and its leading dimension.
__device__ __forceinline__ void mol_block(const long long* mol_off, const int* mol_n, int mol, int n, long long& blk,
                                          int& nm) {
  if (mol_off != nullptr) {
    blk = mol_off[mol];
    nm = mol_n[mol];
  } else {
    blk = 0;
    nm = n;
  }
}

__device__ __forceinline__ const double* off_ptr(const double* p, long long b) { return p ? p + b : p; }
__device__ __forceinline__ double* off_ptr(double* p, long long b) { return p ? p + b : p; }

// What one thread does with its block, by mode:
//   JK      digest into J/K;
//   PACKED  write the unique ERIs into the reference's packed 8-fold vector
//           (hfscfmath::index_ijkl, src/math/hfscf_math.hpp:90-101);
//   SCHWARZ (P|P) only: store sqrt(max |(ab|ab)|) into the pair.
template <int LA, int LB, int LC, int LD, bool PURE>
__device__ __forceinline__ void use_block(const double* V, int mode, const int2 pq, const PairInfo& P,
                                          const PairInfo& Q, double s, const double* __restrict__ DJ, int nK,
                                          const double* __restrict__ DK, double* Jh, double* Kh, int n, double* eri,
                                          PairInfo* pairs_rw, bool coop = false) {
  using Dm = BlockDims<LA, LB, LC, LD, PURE>;
  if (mode == QMODE_JK) {
    digest_jk<Dm::NA, Dm::NB, Dm::NC, Dm::ND>(V, P.fa, P.fb, Q.fa, Q.fb, s, DJ, nK, DK, Jh, Kh, n, coop);
  } else if (mode == QMODE_PACKED) {
    for (int i = 0; i < Dm::NA; ++i)
      for (int j = 0; j < Dm::NB; ++j)
        for (int k = 0; k < Dm::NC; ++k)
          for (int l = 0; l < Dm::ND; ++l)
            eri[packed_index(P.fa + i, P.fb + j, Q.fa + k, Q.fb + l)] = V[((i * Dm::NB + j) * Dm::NC + k) * Dm::ND + l];
  } else {
    double m = 0.0;
    for (int i = 0; i < Dm::NA; ++i)
      for (int j = 0; j < Dm::NB; ++j) m = fmax(m, fabs(V[((i * Dm::NB + j) * Dm::NC + i) * Dm::ND + j]));
    pairs_rw[pq.x].schwarz = sqrt(m);
  }
}

template <typename R>
struct QuartetArgs {
  JKArgs<R> jk;
  int mode;
  int pure;
  double* eri;          // PACKED output
  PairInfo* pairs_rw;   // SCHWARZ output
  int warp_max;         // large classes: warp per quartet up to this many quartets
  int warp_threads;     // threads per quartet of that form: 32 (four quartets per block) or 128
  int block;            // threads per block of the thread-per-quartet form (32, 64 or 128; 0 = 64)
  int group;            // lanes per quartet of the primitive-split form (4, 8, 16 or 32; 0 = 32)
  int capped;           // 1: the register-capped variant of the thread form (classes that have one)
  // Density-screened builds: a launch covers up to four consecutive list segments; segment k
  // starts at seg_off[k] (relative to the launch's list pointer) and only its first dyn_nq[k]
  // quartets (written on the device by an earlier kernel of the same build) are processed.
  // dyn_nq == nullptr: all nq quartets.
  const int* dyn_nq;
  int nseg;
  int seg_off[4];
  int staged;           // 1: the persistent form with the Boys table staged in shared memory (low L)
  const R* boys_planes; // the Boys table in plane layout, one block of boys_plane_bytes<R>() per order
  int* status;          // device status word (HFGPU_DEV_STAGE_TIMEOUT when a staging wait ran out)
  int stage_test;       // 1: arm the staging barrier without a copy, so that its wait runs out (test only)
  const int* abort_flag;  // device word the host sets to stop persistent launches early (nullptr: none)
  // Partitioned builds (one molecule's quartets split over nparts devices or passes): the
  // launch processes every nparts-th quartet of its range, starting at number `part`, and its
  // nq is the per-part upper bound.  nparts <= 1: all quartets.  full_nq: the range's quartets
  // when dyn_nq == nullptr.
  int part;
  int nparts;
  int full_nq;
};

// Quartets this launch processes: nq, or the sum of the device-side segment counts of a
// density-screened build; of a partitioned build, this part's share of them.
template <typename R>
__device__ __forceinline__ int launch_count(const QuartetArgs<R>& qa, int nq) {
  const int np = qa.nparts > 1 ? qa.nparts : 1;
  int tot;
  if (qa.dyn_nq == nullptr) {
    if (np == 1) return nq;
    tot = qa.full_nq;
  } else {
    tot = 0;
    for (int k = 0; k < qa.nseg; ++k) tot += __ldg(qa.dyn_nq + k);
  }
  if (np > 1) tot = tot > qa.part ? (tot - qa.part + np - 1) / np : 0;
  return min(nq, tot);
}

// List position of the launch's t-th processed quartet (t < launch_count): t itself, or, in a
// density-screened build, the t-th quartet of the segments' kept prefixes in segment order
// (in a partitioned build, the (t nparts + part)-th).
template <typename R>
__device__ __forceinline__ int quartet_slot(const QuartetArgs<R>& qa, int t) {
  if (qa.nparts > 1) t = t * qa.nparts + qa.part;
  if (qa.dyn_nq == nullptr) return t;
  for (int k = 0; k < qa.nseg - 1; ++k) {
    const int c = __ldg(qa.dyn_nq + k);
    if (t < c) return qa.seg_off[k] + t;
    t -= c;
  }
  return qa.seg_off[qa.nseg - 1] + t;
}

// One thread per quartet: quartet t of the launch's list (t >= nq: an idle lane that still
// takes part in the warp's shuffles).  Called by all 32 lanes of a warp with consecutive t.
template <int LA, int LB, int LC, int LD, typename R, typename BT>
__device__ __forceinline__ void quartet_thread(const QuartetArgs<R>& qa, const BT& boys,
                                               const int2* __restrict__ quartets, int nq, int t) {
  const JKArgs<R>& a = qa.jk;
  // every lane stays to the end (lanes without work carry valid = false), so
  // that the digestion can use whole-warp shuffles
  const bool in_range = t < nq;
  const int2 pq = in_range ? quartets[quartet_slot(qa, t)] : make_int2(0, 0);
  const PairInfo P = a.pairs[pq.x];
  const PairInfo Q = a.pairs[pq.y];
  bool skip = !in_range;
  if (in_range && qa.mode == QMODE_JK && a.dmax != nullptr) {
    // density-weighted Schwarz bound: Q_ab Q_cd max(4|D_ab|, 4|D_cd|, |D_ac|, |D_ad|, |D_bc|, |D_bd|)
    const float* dm = a.dmax;
    const int ns = a.nshell;
    float m = 4.f * fmaxf(dm[P.sa * ns + P.sb], dm[Q.sa * ns + Q.sb]);
    m = fmaxf(m, fmaxf(fmaxf(dm[P.sa * ns + Q.sa], dm[P.sa * ns + Q.sb]), fmaxf(dm[P.sb * ns + Q.sa], dm[P.sb * ns + Q.sb])));
    skip = P.schwarz * Q.schwarz * double(m) < a.dtol;
  }
  const bool valid = !skip;
  if (a.counters != nullptr) {
    // per-class work counters, one atomic per warp: [0] quartets computed,
    // [1] quartets skipped by the density bound, [2] primitive quartets computed
    const unsigned nvalid = __popc(__ballot_sync(0xffffffffu, valid));
    const unsigned nin = __popc(__ballot_sync(0xffffffffu, in_range));
    const unsigned prims = __reduce_add_sync(0xffffffffu, valid ? unsigned(P.nprim * Q.nprim) : 0u);
    if ((threadIdx.x & 31) == 0) {
      atomicAdd(a.counters + 0, (unsigned long long)nvalid);
      atomicAdd(a.counters + 1, (unsigned long long)(nin - nvalid));
      atomicAdd(a.counters + 2, (unsigned long long)prims);
    }
  }
  if (!__any_sync(0xffffffffu, valid)) return;  // whole warp leaves together
  // J_ab contributions can be summed across the warp when every lane works on the same bra pair.
  // The shuffle is taken by all 32 lanes before any predicate (a shuffle skipped by some
  // lanes, e.g. through && short-circuiting, would leave the others waiting).
  const int px0 = __shfl_sync(0xffffffffu, pq.x, 0);
  const bool same_bra = valid && pq.x == px0;
  const bool coop = __all_sync(0xffffffffu, same_bra) && qa.mode == QMODE_JK;
  using Dc = BlockDims<LA, LB, LC, LD, false>;
  R cart[Dc::NCART];
  if (valid)
    ClassCode<LA, LB, LC, LD>::template eri<R>(a.prims + P.prim_off, P.nprim, a.prims + Q.prim_off, Q.nprim,
                                                R(P.ABx), R(P.ABy), R(P.ABz), R(Q.ABx), R(Q.ABy), R(Q.ABz), boys,
                                                cart);
  double s = 1.0;
  if (P.sa == P.sb) s *= 0.5;
  if (Q.sa == Q.sb) s *= 0.5;
  if (pq.x == pq.y) s *= 0.5;
  long long blk;
  int nm;
  mol_block(a.mol_off, a.mol_n, P.mol, a.n, blk, nm);
  if (qa.pure) {
    using Dp = BlockDims<LA, LB, LC, LD, true>;
    double V[Dp::NOUT];
    if (valid) finish_block<LA, LB, LC, LD, R, true>(cart, V);
    if (valid || coop)
      use_block<LA, LB, LC, LD, true>(V, qa.mode, pq, P, Q, s, off_ptr(a.DJ, blk), a.nK, off_ptr(a.DK, blk),
                                      off_ptr(a.Jh, blk), off_ptr(a.Kh, blk), nm, qa.eri, qa.pairs_rw, coop);
  } else {
    double V[Dc::NOUT];
    if (valid) finish_block<LA, LB, LC, LD, R, false>(cart, V);
    if (valid || coop)
      use_block<LA, LB, LC, LD, false>(V, qa.mode, pq, P, Q, s, off_ptr(a.DJ, blk), a.nK, off_ptr(a.DK, blk),
                                       off_ptr(a.Jh, blk), off_ptr(a.Kh, blk), nm, qa.eri, qa.pairs_rw, coop);
  }
}

// MINB > 1: the register-capped variant (at least MINB blocks of 128 threads per SM) of the
// small classes, for more warps in flight.
template <int LA, int LB, int LC, int LD, typename R, int MINB = 1>
__global__ void __launch_bounds__(128, MINB) quartet_kernel(QuartetArgs<R> qa, const int2* __restrict__ quartets,
                                                            int nq) {
  nq = launch_count(qa, nq);
  quartet_thread<LA, LB, LC, LD, R>(qa, qa.jk.boys, quartets, nq, blockIdx.x * blockDim.x + threadIdx.x);
}

// The thread-per-quartet form as a persistent kernel with the class's Boys table in shared
// memory, for the low-L classes whose time goes to the lanes' scattered Boys-row loads: every
// block stages the table of the class's single order L = la+lb+lc+ld with one bulk copy
// (stage_to_shared), then its warps take 32 quartets at a time, grid-stride.  Launched with
// about as many blocks as the GPU holds at once, so the copy is made once per resident block.
template <int LA, int LB, int LC, int LD, typename R>
__global__ void __launch_bounds__(128) quartet_staged_kernel(QuartetArgs<R> qa, const int2* __restrict__ quartets,
                                                             int nq) {
  constexpr int L = LA + LB + LC + LD;
  extern __shared__ __align__(16) unsigned char staged_smem[];
  __shared__ unsigned long long stage_bar;
  R* tab = reinterpret_cast<R*>(staged_smem);
  const unsigned char* src = reinterpret_cast<const unsigned char*>(qa.boys_planes) + (size_t)L * boys_plane_bytes<R>();
  if (!stage_to_shared(tab, src, boys_plane_bytes<R>(), &stage_bar, qa.status, qa.stage_test == 0)) return;
  const BoysShared<R, L> boys{tab};
  nq = launch_count(qa, nq);
  const int warps = gridDim.x * (blockDim.x >> 5);
  for (int w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); w * 32 < nq; w += warps) {
    // a host request to stop (hfgpu_request_abort) ends the launch between two warp chunks
    if (qa.abort_flag != nullptr && *reinterpret_cast<const volatile int*>(qa.abort_flag) != 0) {
      if ((threadIdx.x & 31) == 0 && qa.status != nullptr) atomicExch(qa.status, HFGPU_DEV_ABORTED);
      break;
    }
    quartet_thread<LA, LB, LC, LD, R>(qa, boys, quartets, nq, w * 32 + (threadIdx.x & 31));
  }
}

// G lanes per quartet (G = 4, 8, 16 or 32) for small classes and quartets with many
// primitive quartets: the lanes of a group split the primitive quartets (consecutive ket
// primitives, one bra primitive per run: coalesced and broadcast loads), the
// accumulators are reduced with shuffles inside the group, and the group's first lane
// transforms and digests the block.  Every lane stays to the end: the shuffles take the
// whole warp.
template <int LA, int LB, int LC, int LD, typename R, int G>
__global__ void __launch_bounds__(128) quartet_primwarp_kernel(QuartetArgs<R> qa, const int2* __restrict__ quartets,
                                                               int nq) {
  static_assert(G == 4 || G == 8 || G == 16 || G == 32, "group size");
  const JKArgs<R>& a = qa.jk;
  nq = launch_count(qa, nq);
  const int sub = threadIdx.x & (G - 1);
  const int qi = (blockIdx.x * blockDim.x + threadIdx.x) / G;
  const bool in_range = qi < nq;
  if (!__any_sync(0xffffffffu, in_range)) return;  // whole warp leaves together
  const int2 pq = in_range ? quartets[quartet_slot(qa, qi)] : make_int2(0, 0);
  const PairInfo P = a.pairs[pq.x];
  const PairInfo Q = a.pairs[pq.y];
  bool skip = !in_range;
  if (in_range && qa.mode == QMODE_JK && a.dmax != nullptr) {
    const float* dm = a.dmax;
    const int ns = a.nshell;
    float m = 4.f * fmaxf(dm[P.sa * ns + P.sb], dm[Q.sa * ns + Q.sb]);
    m = fmaxf(m, fmaxf(fmaxf(dm[P.sa * ns + Q.sa], dm[P.sa * ns + Q.sb]), fmaxf(dm[P.sb * ns + Q.sa], dm[P.sb * ns + Q.sb])));
    skip = P.schwarz * Q.schwarz * double(m) < a.dtol;
  }
  if (a.counters != nullptr) {
    // per-class work counters, one atomic per warp (see quartet_kernel)
    const bool lead = sub == 0;
    const unsigned nvalid = __popc(__ballot_sync(0xffffffffu, lead && !skip));
    const unsigned nin = __popc(__ballot_sync(0xffffffffu, lead && in_range));
    const unsigned prims = __reduce_add_sync(0xffffffffu, (lead && !skip) ? unsigned(P.nprim * Q.nprim) : 0u);
    if ((threadIdx.x & 31) == 0) {
      atomicAdd(a.counters + 0, (unsigned long long)nvalid);
      atomicAdd(a.counters + 1, (unsigned long long)(nin - nvalid));
      atomicAdd(a.counters + 2, (unsigned long long)prims);
    }
  }
  using Dc = BlockDims<LA, LB, LC, LD, false>;
  R cart[Dc::NCART];
  // skipped and out-of-range groups run an empty primitive loop but still take the shuffles
  ClassCode<LA, LB, LC, LD>::template eri_pw<R, G>(a.prims + P.prim_off, skip ? 0 : P.nprim,
                                                    a.prims + Q.prim_off, Q.nprim, R(P.ABx), R(P.ABy), R(P.ABz),
                                                    R(Q.ABx), R(Q.ABy), R(Q.ABz), a.boys, cart, sub);
  if (skip || sub != 0) return;
  double s = 1.0;
  if (P.sa == P.sb) s *= 0.5;
  if (Q.sa == Q.sb) s *= 0.5;
  if (pq.x == pq.y) s *= 0.5;
  long long blk;
  int nm;
  mol_block(a.mol_off, a.mol_n, P.mol, a.n, blk, nm);
  if (qa.pure) {
    using Dp = BlockDims<LA, LB, LC, LD, true>;
    double V[Dp::NOUT];
    finish_block<LA, LB, LC, LD, R, true>(cart, V);
    use_block<LA, LB, LC, LD, true>(V, qa.mode, pq, P, Q, s, off_ptr(a.DJ, blk), a.nK, off_ptr(a.DK, blk),
                                    off_ptr(a.Jh, blk), off_ptr(a.Kh, blk), nm, qa.eri, qa.pairs_rw);
  } else {
    double V[Dc::NOUT];
    finish_block<LA, LB, LC, LD, R, false>(cart, V);
    use_block<LA, LB, LC, LD, false>(V, qa.mode, pq, P, Q, s, off_ptr(a.DJ, blk), a.nK, off_ptr(a.DK, blk),
                                     off_ptr(a.Jh, blk), off_ptr(a.Kh, blk), nm, qa.eri, qa.pairs_rw);
  }
}

// ---------------------------------------------------------------------------
// Adjoint gradient.
// ---------------------------------------------------------------------------
template <typename R>
struct Strided {
  R* base;
  int stride;
  __device__ __forceinline__ R& operator[](int i) const { return base[(size_t)i * stride]; }
};


// Executor of a table-mode gradient class (ops generated by gen_eri.py).
template <typename R, typename Tab>
__device__ void grad_table(const PrimPair<R>* __restrict__ bp, const R* __restrict__ ea, const R* __restrict__ eb,
                           int nbp, const PrimPair<R>* __restrict__ kp, const R* __restrict__ ec, int nkp, R ABx,
                           R ABy, R ABz, R CDx, R CDy, R CDz, const BoysTable<R>& boys, Strided<R> W, Strided<R> vs,
                           Strided<R> hs, R* g) {
  vs[0] = R(0);
  hs[0] = R(0);
  for (int x = 1; x <= Tab::NACC; ++x) hs[x] = R(0);
  const int4* vo = Tab::vrr();  // packed rows, see gen_eri.py pack_grad_vrr / pack_grad_hrr
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
          const R w = dir == 0 ? R(1) : (dir == 1 ? wa : (dir == 2 ? wb : wc));
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
#pragma unroll
  for (int x = 0; x < 9; ++x) g[x] = R(0);
  for (int o = 0; o < Tab::NHOPS; ++o) {
    const int2 op = __ldg(ho + o);
    const int dst = op.x & 0xffff, sx = (unsigned)op.x >> 16, sy = op.y & 0xffff;
    const int kind = (op.y >> 16) & 15, dir = (op.y >> 20) & 15;
    if (kind == 2) {
      const int k = (op.y >> 24) & 127;
      const R v = W[dst] * (hs[sx] - small_int<R>(k) * hs[sy]);
#pragma unroll
      for (int x = 0; x < 9; ++x)
        if (x == dir) g[x] += v;
    } else {
      const R d = kind == 0 ? (dir == 0 ? ABx : (dir == 1 ? ABy : ABz)) : (dir == 0 ? CDx : (dir == 1 ? CDy : CDz));
      hs[dst] = hs[sx] + d * hs[sy];
    }
  }
}

// Weight block of a unique quartet in the final basis:
// W_abcd = 8 s [cJ DJ_ab DJ_cd - (cK/2) sum_m (DK_ac DK_bd + DK_ad DK_bc)],
// the average of cJ DJ_pq DJ_rs - cK DK_pr DK_qs over the quartet's 8 index images.
template <int NA, int NB, int NC, int ND, typename Out>
__device__ __forceinline__ void grad_weights(const double* __restrict__ DJ, double cJ,
                                             int nK, const double* __restrict__ DK, double cK, int n, int fa, int fb,
                                             int fc, int fd, double s8, Out W) {
  for (int i = 0; i < NA; ++i)
    for (int j = 0; j < NB; ++j) {
      const double dab = DJ ? __ldg(DJ + (size_t)(fa + i) * n + fb + j) : 0.0;
      for (int k = 0; k < NC; ++k)
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

// PASS < 0: the whole gradient of the quartet; PASS = 0..3: the part that accumulator set
// U, A, B or C carries (classes generated with kGradPasses = 4 run one launch per pass); for
// kGradPasses = 2, PASS = 0, 1: the part that sets U and A, or B and C, carry.
template <int LA, int LB, int LC, int LD, typename R, bool PURE, int PASS = -1>
__device__ __forceinline__ void grad_quartet(const GradArgs<R>& a, int tid, const int2 pq, double* gout) {
  using Dm = BlockDims<LA, LB, LC, LD, PURE>;
  using CC = ClassCode<LA, LB, LC, LD>;
  {
    const PairInfo P = a.pairs[pq.x];
    const PairInfo Q = a.pairs[pq.y];
    double s = 8.0;
    if (P.sa == P.sb) s *= 0.5;
    if (Q.sa == Q.sb) s *= 0.5;
    if (pq.x == pq.y) s *= 0.5;
    long long gblk;
    int gnm;
    mol_block(a.mol_off, a.mol_n, P.mol, a.n, gblk, gnm);
    R g[9];
    if constexpr (CC::kGradTable) {
      using Tab = typename CC::GradTab;
      // scratch layout per thread: [VRR slots | HRR slots | W cart | 2 transform buffers]
      R* base = a.scratch + tid;
      Strided<R> vs{base, a.scratch_threads};
      Strided<R> hs{base + (size_t)Tab::NVSLOT * a.scratch_threads, a.scratch_threads};
      Strided<R> Wc{base + (size_t)(Tab::NVSLOT + Tab::NHSLOT) * a.scratch_threads, a.scratch_threads};
      Strided<R> t0{base + (size_t)(Tab::NVSLOT + Tab::NHSLOT + Dm::NCART) * a.scratch_threads, a.scratch_threads};
      Strided<R> t1{base + (size_t)(Tab::NVSLOT + Tab::NHSLOT + 2 * Dm::NCART) * a.scratch_threads, a.scratch_threads};
      if constexpr (PURE) {
        grad_weights<Dm::NA, Dm::NB, Dm::NC, Dm::ND>(off_ptr(a.DJ, gblk), a.cJ, a.nK, off_ptr(a.DK, gblk), a.cK, gnm, P.fa, P.fb,
                                                     Q.fa, Q.fb, s, t0);
        // pure -> Cartesian weights, one index at a time: t0 -> t1 -> t0 -> t1 -> Wc
        const int Ls[4] = {LA, LB, LC, LD};
        int dims[4] = {Dm::NA, Dm::NB, Dm::NC, Dm::ND};
        Strided<R> src = t0, dst = t1;
        for (int st = 0; st < 4; ++st) {
          const int nc = ncart_of(Ls[st]), np = npure_of(Ls[st]);
          int nd[4] = {dims[0], dims[1], dims[2], dims[3]};
          nd[st] = nc;
          Strided<R> out = (st == 3) ? Wc : dst;
          const int tot = nd[0] * nd[1] * nd[2] * nd[3];
          for (int e = 0; e < tot; ++e) {
            int id[4];
            int r = e;
            for (int q = 3; q >= 0; --q) {
              id[q] = r % nd[q];
              r /= nd[q];
            }
            R v = R(0);
            for (int c = 0; c < np; ++c) {
              const double y = c_ylm[Ls[st]][id[st] * np + c];
              if (y == 0.0) continue;
              int jd[4] = {id[0], id[1], id[2], id[3]};
              jd[st] = c;
              v += R(y) * src[((jd[0] * dims[1] + jd[1]) * dims[2] + jd[2]) * dims[3] + jd[3]];
            }
            out[e] = v;
          }
          for (int q = 0; q < 4; ++q) dims[q] = nd[q];
          Strided<R> tmp = src;
          src = dst;
          dst = tmp;
        }
      } else {
        grad_weights<Dm::NA, Dm::NB, Dm::NC, Dm::ND>(off_ptr(a.DJ, gblk), a.cJ, a.nK, off_ptr(a.DK, gblk), a.cK, gnm, P.fa, P.fb,
                                                     Q.fa, Q.fb, s, Wc);
      }
      grad_table<R, Tab>(a.prims + P.prim_off, a.alpha_a + P.prim_off, a.alpha_b + P.prim_off, P.nprim,
                         a.prims + Q.prim_off, a.alpha_a + Q.prim_off, Q.nprim, R(P.ABx), R(P.ABy), R(P.ABz),
                         R(Q.ABx), R(Q.ABy), R(Q.ABz), a.boys, Wc, vs, hs, g);
    } else {
      R Wc[Dm::NCART];
      if constexpr (PURE) {
        R Wp[Dm::NOUT];
        grad_weights<Dm::NA, Dm::NB, Dm::NC, Dm::ND>(off_ptr(a.DJ, gblk), a.cJ, a.nK, off_ptr(a.DK, gblk), a.cK, gnm, P.fa, P.fb,
                                                     Q.fa, Q.fb, s, Wp);
        CC::template from_pure<R>(Wp, Wc);
      } else {
        grad_weights<Dm::NA, Dm::NB, Dm::NC, Dm::ND>(off_ptr(a.DJ, gblk), a.cJ, a.nK, off_ptr(a.DK, gblk), a.cK, gnm, P.fa, P.fb,
                                                     Q.fa, Q.fb, s, Wc);
      }
      if constexpr (PASS >= 0) {
        CC::template grad_pass<R, PASS>(a.prims + P.prim_off, a.alpha_a + P.prim_off, a.alpha_b + P.prim_off,
                                        P.nprim, a.prims + Q.prim_off, a.alpha_a + Q.prim_off, Q.nprim, R(P.ABx),
                                        R(P.ABy), R(P.ABz), R(Q.ABx), R(Q.ABy), R(Q.ABz), a.boys, Wc, g, g + 3,
                                        g + 6);
      } else {
        CC::template grad<R>(a.prims + P.prim_off, a.alpha_a + P.prim_off, a.alpha_b + P.prim_off, P.nprim,
                             a.prims + Q.prim_off, a.alpha_a + Q.prim_off, Q.nprim, R(P.ABx), R(P.ABy), R(P.ABz),
                             R(Q.ABx), R(Q.ABy), R(Q.ABz), a.boys, Wc, g, g + 3, g + 6);
      }
    }
    const int at[3] = {P.atom_a, P.atom_b, Q.atom_a};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double gA = double(g[d]), gB = double(g[3 + d]), gC = double(g[6 + d]);
      atomicAdd(gout + 3 * at[0] + d, gA);
      atomicAdd(gout + 3 * at[1] + d, gB);
      atomicAdd(gout + 3 * at[2] + d, gC);
      atomicAdd(gout + 3 * Q.atom_b + d, -(gA + gB + gC));
    }
  }
}

// Every quartet adds 12 values into the natoms x 3 gradient.  Straight into global memory
// those are millions of atomics on a few dozen addresses, serialised in L2; with
// a.smem_atoms > 0 each block sums into shared memory first and adds its 3 natoms totals
// once at the end.
template <int LA, int LB, int LC, int LD, typename R, int PASS = -1>
__global__ void __launch_bounds__(128) grad_kernel(GradArgs<R> a, int pure, const int2* __restrict__ quartets, int nq) {
  extern __shared__ double grad_sh[];
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int nthr = gridDim.x * blockDim.x;
  const int nsh = 3 * a.smem_atoms;
  double* gout = a.grad;
  if (nsh > 0) {
    for (int i = threadIdx.x; i < nsh; i += blockDim.x) grad_sh[i] = 0.0;
    __syncthreads();
    gout = grad_sh;
  }
  const int np = a.nparts > 1 ? a.nparts : 1, p0 = np > 1 ? a.part : 0;
  for (int t = tid; t < nq; t += nthr) {
    const int2 pq = quartets[(size_t)t * np + p0];
    if (pure)
      grad_quartet<LA, LB, LC, LD, R, true, PASS>(a, tid, pq, gout);
    else
      grad_quartet<LA, LB, LC, LD, R, false, PASS>(a, tid, pq, gout);
  }
  if (nsh > 0) {
    __syncthreads();
    for (int i = threadIdx.x; i < nsh; i += blockDim.x)
      if (grad_sh[i] != 0.0) atomicAdd(a.grad + i, grad_sh[i]);
  }
}


// ---------------------------------------------------------------------------
// Warp-per-quartet kernel for the large classes (generated levelised tables).
// ---------------------------------------------------------------------------
// Synchronisation of the threads that share one quartet: a warp, or a whole block.
template <int NT>
__device__ __forceinline__ void group_sync() {
  if constexpr (NT == 32)
    __syncwarp();
  else
    __syncthreads();
}

template <typename R, int NT = 32>
__device__ __forceinline__ void warp_to_pure(const R* src, R* dst0, R* dst1, const int* Ls, int lane, const R** out) {
  // one index at a time, ping-pong between dst0 and dst1
  int dims[4] = {ncart_of(Ls[0]), ncart_of(Ls[1]), ncart_of(Ls[2]), ncart_of(Ls[3])};
  const R* in = src;
  R* bufs[2] = {dst0, dst1};
  for (int st = 0; st < 4; ++st) {
    const int nc = ncart_of(Ls[st]), np = npure_of(Ls[st]);
    int nd[4] = {dims[0], dims[1], dims[2], dims[3]};
    nd[st] = np;
    R* o = bufs[st & 1];
    const int tot = nd[0] * nd[1] * nd[2] * nd[3];
    for (int e = lane; e < tot; e += NT) {
      int id[4];
      int r = e;
      for (int q = 3; q >= 0; --q) {
        id[q] = r % nd[q];
        r /= nd[q];
      }
      R v = R(0);
      for (int c = 0; c < nc; ++c) {
        const double y = c_ylm[Ls[st]][c * np + id[st]];
        if (y == 0.0) continue;
        int jd[4] = {id[0], id[1], id[2], id[3]};
        jd[st] = c;
        v += R(y) * in[((jd[0] * dims[1] + jd[1]) * dims[2] + jd[2]) * dims[3] + jd[3]];
      }
      o[e] = v;
    }
    group_sync<NT>();
    for (int q = 0; q < 4; ++q) dims[q] = nd[q];
    in = o;
  }
  *out = in;
}

template <typename R, int NT = 32>
__device__ __forceinline__ void warp_digest(const R* V, int NA, int NB, int NC, int ND, int fa, int fb, int fc, int fd,
                                            double s, const double* __restrict__ DJ, int nK,
                                            const double* __restrict__ DK, double* Jh, double* Kh, int n, int lane) {
  const int NCD = NC * ND;
  if (DJ != nullptr) {
    for (int x = lane; x < NA * NB; x += NT) {
      double acc = 0.0;
      for (int c = 0; c < NC; ++c)
        for (int d = 0; d < ND; ++d) acc += __ldg(DJ + (size_t)(fc + c) * n + fd + d) * double(V[x * NCD + c * ND + d]);
      atomicAdd(Jh + (size_t)(fa + x / NB) * n + fb + x % NB, 2.0 * s * acc);
    }
    for (int y = lane; y < NCD; y += NT) {
      double acc = 0.0;
      for (int a = 0; a < NA; ++a)
        for (int b = 0; b < NB; ++b) acc += __ldg(DJ + (size_t)(fa + a) * n + fb + b) * double(V[(a * NB + b) * NCD + y]);
      atomicAdd(Jh + (size_t)(fc + y / ND) * n + fd + y % ND, 2.0 * s * acc);
    }
  }
  for (int m = 0; m < nK; ++m) {
    const double* D = DK + (size_t)m * n * n;
    double* K = Kh + (size_t)m * n * n;
    for (int x = lane; x < NA * NC; x += NT) {  // K_ac += D_bd V
      const int a = x / NC, c = x % NC;
      double acc = 0.0;
      for (int b = 0; b < NB; ++b)
        for (int d = 0; d < ND; ++d) acc += __ldg(D + (size_t)(fb + b) * n + fd + d) * double(V[((a * NB + b) * NC + c) * ND + d]);
      atomicAdd(K + (size_t)(fa + a) * n + fc + c, s * acc);
    }
    for (int x = lane; x < NA * ND; x += NT) {  // K_ad += D_bc V
      const int a = x / ND, d = x % ND;
      double acc = 0.0;
      for (int b = 0; b < NB; ++b)
        for (int c = 0; c < NC; ++c) acc += __ldg(D + (size_t)(fb + b) * n + fc + c) * double(V[((a * NB + b) * NC + c) * ND + d]);
      atomicAdd(K + (size_t)(fa + a) * n + fd + d, s * acc);
    }
    for (int x = lane; x < NB * NC; x += NT) {  // K_bc += D_ad V
      const int b = x / NC, c = x % NC;
      double acc = 0.0;
      for (int a = 0; a < NA; ++a)
        for (int d = 0; d < ND; ++d) acc += __ldg(D + (size_t)(fa + a) * n + fd + d) * double(V[((a * NB + b) * NC + c) * ND + d]);
      atomicAdd(K + (size_t)(fb + b) * n + fc + c, s * acc);
    }
    for (int x = lane; x < NB * ND; x += NT) {  // K_bd += D_ac V
      const int b = x / ND, d = x % ND;
      double acc = 0.0;
      for (int a = 0; a < NA; ++a)
        for (int c = 0; c < NC; ++c) acc += __ldg(D + (size_t)(fa + a) * n + fc + c) * double(V[((a * NB + b) * NC + c) * ND + d]);
      atomicAdd(K + (size_t)(fb + b) * n + fd + d, s * acc);
    }
  }
}

template <typename Tab, typename R>
constexpr int warp_slots() {
  return Tab::NVSLOT + 1 + Tab::NHSLOT + 1 + 2 * Tab::NCART;
}

// One warp per unique quartet (NT = 32, four quartets per 128-thread block) or one block of
// NT = 128 threads per quartet: the levelised VRR and HRR run lane-parallel out of shared
// memory; transform and digestion are lane-parallel over the quartet's threads.
template <int LA, int LB, int LC, int LD, typename R, typename Tab, int NT = 32>
__global__ void __launch_bounds__(128) quartet_warp_kernel(QuartetArgs<R> qa, const int2* __restrict__ quartets,
                                                           int nq) {
  static_assert(NT == 32 || NT == 128, "threads per quartet");
  extern __shared__ __align__(16) unsigned char wsmem[];
  __shared__ double wred[4];
  constexpr int PER = warp_slots<Tab, R>();
  const int lane = NT == 32 ? (threadIdx.x & 31) : threadIdx.x, w = NT == 32 ? (threadIdx.x >> 5) : 0;
  const int qi = NT == 32 ? blockIdx.x * (blockDim.x >> 5) + w : blockIdx.x;
  if (qi >= launch_count(qa, nq)) return;  // the quartet's whole warp or block
  R* vs = reinterpret_cast<R*>(wsmem) + (size_t)w * PER;
  R* hs = vs + Tab::NVSLOT + 1;
  R* A = hs + Tab::NHSLOT + 1;
  R* Bb = A + Tab::NCART;
  const JKArgs<R>& a = qa.jk;
  const int2 pq = quartets[quartet_slot(qa, qi)];
  const PairInfo P = a.pairs[pq.x];
  const PairInfo Q = a.pairs[pq.y];
  bool skip = false;
  if (qa.mode == QMODE_JK && a.dmax != nullptr) {
    const float* dm = a.dmax;
    const int ns = a.nshell;
    float m = 4.f * fmaxf(dm[P.sa * ns + P.sb], dm[Q.sa * ns + Q.sb]);
    m = fmaxf(m, fmaxf(fmaxf(dm[P.sa * ns + Q.sa], dm[P.sa * ns + Q.sb]), fmaxf(dm[P.sb * ns + Q.sa], dm[P.sb * ns + Q.sb])));
    skip = P.schwarz * Q.schwarz * double(m) < a.dtol;
  }
  if (a.counters != nullptr && lane == 0) {
    atomicAdd(a.counters + (skip ? 1 : 0), 1ull);
    if (!skip) atomicAdd(a.counters + 2, (unsigned long long)(P.nprim * Q.nprim));
  }
  if (skip) return;
  if (lane == 0) {
    vs[Tab::NVSLOT] = R(0);
    hs[Tab::NHSLOT] = R(0);
  }
  for (int t = lane; t < Tab::NACC; t += NT) hs[t] = R(0);
  group_sync<NT>();
  const PrimPair<R>* bp = a.prims + P.prim_off;
  const PrimPair<R>* kp = a.prims + Q.prim_off;
  const int4* vo = Tab::vrr();  // packed rows, see gen_eri.py pack_warp_vrr / pack_warp_hrr
  const int* vl = Tab::vlev();
  const int* accs = Tab::acc();
  for (int ib = 0; ib < P.nprim; ++ib) {
    const R p = bp[ib].p, ip = bp[ib].ip, Px = bp[ib].Px, Py = bp[ib].Py, Pz = bp[ib].Pz;
    const R PAx = bp[ib].PAx, PAy = bp[ib].PAy, PAz = bp[ib].PAz, Kab = bp[ib].Kp;
    for (int ik = 0; ik < Q.nprim; ++ik) {
      const R q = kp[ik].p, iq = kp[ik].ip, Qx = kp[ik].Px, Qy = kp[ik].Py, Qz = kp[ik].Pz;
      const R QCx = kp[ik].PAx, QCy = kp[ik].PAy, QCz = kp[ik].PAz, Kcd = kp[ik].Kp;
      const R pqs = p + q;
      const R rs = rsqrt_t(pqs);
      const R ipq = rs * rs;
      const R rho = p * q * ipq;
      const R rp = q * ipq, rq = p * ipq;
      const R inv2p = R(0.5) * ip, inv2q = R(0.5) * iq, inv2pq = R(0.5) * ipq;
      const R PQx = Px - Qx, PQy = Py - Qy, PQz = Pz - Qz;
      const R T = rho * (PQx * PQx + PQy * PQy + PQz * PQz);
      R F[Tab::L + 1];
      a.boys.template eval<Tab::L>(T, Kab * Kcd * rs, F);
#pragma unroll
      for (int m = 0; m <= Tab::L; ++m)
        if (lane == m) vs[m] = F[m];
      group_sync<NT>();
      for (int l = 0; l < Tab::NVLEV; ++l) {
        const int e = __ldg(vl + l + 1);
        // two op rows in flight per lane: the rows of one level are independent
        auto body = [&](const int4 op) {
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
            v = QC * vs[sa] + rq * PQd * vs[sb] + k1 * inv2q * (vs[sc] - rq * vs[sd]) + small_int<R>(k12 >> 8) * inv2pq * vs[sg];
          }
          vs[dst] = v;
        };
        for (int o = __ldg(vl + l) + lane; o < e; o += 2 * NT) {
          const int4 opa = __ldg(vo + o);
          const bool two = o + NT < e;
          const int4 opb = two ? __ldg(vo + o + NT) : opa;
          body(opa);
          if (two) body(opb);
        }
        group_sync<NT>();
      }
      for (int t = lane; t < Tab::NACC; t += NT) hs[t] += vs[__ldg(accs + t)];
      group_sync<NT>();
    }
  }
  const int2* ho = Tab::hrr();
  const int* hl = Tab::hlev();
  const R ABx = R(P.ABx), ABy = R(P.ABy), ABz = R(P.ABz), CDx = R(Q.ABx), CDy = R(Q.ABy), CDz = R(Q.ABz);
  for (int l = 0; l < Tab::NHLEV; ++l) {
    const int e = __ldg(hl + l + 1);
    // two op rows in flight per lane: the rows of one level are independent
    auto body = [&](const int2 op) {
      const int kd = (unsigned)op.y >> 16, dir = kd >> 2;
      const R d = (kd & 1) ? (dir == 0 ? CDx : (dir == 1 ? CDy : CDz)) : (dir == 0 ? ABx : (dir == 1 ? ABy : ABz));
      hs[op.x & 0xffff] = hs[(unsigned)op.x >> 16] + d * hs[op.y & 0xffff];
    };
    for (int o = __ldg(hl + l) + lane; o < e; o += 2 * NT) {
      const int2 opa = __ldg(ho + o);
      const bool two = o + NT < e;
      const int2 opb = two ? __ldg(ho + o + NT) : opa;
      body(opa);
      if (two) body(opb);
    }
    group_sync<NT>();
  }
  const int* outs = Tab::out();
  for (int o = lane; o < Tab::NCART; o += NT) A[o] = hs[__ldg(outs + o)];
  group_sync<NT>();
  const R* V = A;
  int NA = ncart_of(LA), NB = ncart_of(LB), NC = ncart_of(LC), ND = ncart_of(LD);
  if (qa.pure) {
    const int Ls[4] = {LA, LB, LC, LD};
    warp_to_pure<R, NT>(A, Bb, A, Ls, lane, &V);
    NA = npure_of(LA);
    NB = npure_of(LB);
    NC = npure_of(LC);
    ND = npure_of(LD);
  }
  double s = 1.0;
  if (P.sa == P.sb) s *= 0.5;
  if (Q.sa == Q.sb) s *= 0.5;
  if (pq.x == pq.y) s *= 0.5;
  if (qa.mode == QMODE_JK) {
    long long blk;
    int nm;
    mol_block(a.mol_off, a.mol_n, P.mol, a.n, blk, nm);
    warp_digest<R, NT>(V, NA, NB, NC, ND, P.fa, P.fb, Q.fa, Q.fb, s, off_ptr(a.DJ, blk), a.nK, off_ptr(a.DK, blk),
                   off_ptr(a.Jh, blk), off_ptr(a.Kh, blk), nm, lane);
  } else if (qa.mode == QMODE_PACKED) {
    for (int e = lane; e < NA * NB * NC * ND; e += NT) {
      const int l = e % ND, k = (e / ND) % NC, j = (e / (ND * NC)) % NB, i = e / (ND * NC * NB);
      qa.eri[packed_index(P.fa + i, P.fb + j, Q.fa + k, Q.fb + l)] = double(V[e]);
    }
  } else {
    double m = 0.0;
    for (int x = lane; x < NA * NB; x += NT) {
      const int i = x / NB, j = x % NB;
      m = fmax(m, fabs(double(V[((i * NB + j) * NC + i) * ND + j])));
    }
    for (int off = 16; off > 0; off >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, off));
    if constexpr (NT > 32) {  // the block's warps through shared memory
      if ((lane & 31) == 0) wred[lane >> 5] = m;
      __syncthreads();
      if (lane == 0)
        for (int k = 1; k < NT / 32; ++k) m = fmax(m, wred[k]);
    }
    if (lane == 0) qa.pairs_rw[pq.x].schwarz = sqrt(m);
  }
}

// ---------------------------------------------------------------------------
// Warp-per-quartet adjoint gradient for the large classes: the weight block, the VRR one
// order higher with its four weighted accumulations, and the HRR of the four sets with
// the contractions against W all run lane-parallel out of shared memory, level by level
// (generated tables, gen_eri.py gen_grad_warp).  One block per quartet, of one warp or four.
// ---------------------------------------------------------------------------
// t0 holds a pure weight block or an intermediate of its transform (NCART values), and at the end
// the per-warp gradient sums of a multi-warp block (9 per warp, up to 8 warps): at least 72.
template <typename Tab, typename R>
__host__ __device__ constexpr int grad_warp_t0() {
  return Tab::NCART > 72 ? Tab::NCART : 72;
}

template <typename Tab, typename R>
__host__ __device__ constexpr int grad_warp_slots() {
  return Tab::NVSLOT + 1 + Tab::NHSLOT + 1 + 2 * Tab::NCART + grad_warp_t0<Tab, R>();
}

// NT = 32: one warp per quartet; NT = 128 or 256: one block of four or eight warps per quartet
// (the same shared-memory tables, each level's rows spread over more threads, so that a
// quartet finishes sooner and more warps per SM hide the shared-memory latency).
template <int LA, int LB, int LC, int LD, typename R, typename Tab, int NT = 32>
__global__ void __launch_bounds__(NT) grad_warp_kernel(GradArgs<R> a, int pure, const int2* __restrict__ quartets,
                                                       int nq) {
  static_assert(NT == 32 || NT == 128 || NT == 256, "threads per quartet");
  extern __shared__ __align__(16) unsigned char gwsm[];
  const int lane = threadIdx.x;  // 0 .. NT-1
  const int qi = blockIdx.x;
  if (qi >= nq) return;
  R* vs = reinterpret_cast<R*>(gwsm);
  R* hs = vs + Tab::NVSLOT + 1;
  R* W = hs + Tab::NHSLOT + 1;
  R* t0 = W + Tab::NCART;
  R* t1 = t0 + grad_warp_t0<Tab, R>();
  const int2 pq = quartets[(size_t)qi * (a.nparts > 1 ? a.nparts : 1) + (a.nparts > 1 ? a.part : 0)];
  const PairInfo P = a.pairs[pq.x];
  const PairInfo Q = a.pairs[pq.y];
  double s8 = 8.0;
  if (P.sa == P.sb) s8 *= 0.5;
  if (Q.sa == Q.sb) s8 *= 0.5;
  if (pq.x == pq.y) s8 *= 0.5;
  long long blk;
  int nm;
  mol_block(a.mol_off, a.mol_n, P.mol, a.n, blk, nm);
  const double* DJ = off_ptr(a.DJ, blk);
  const double* DK = off_ptr(a.DK, blk);
  // weight block W_abcd = s8 [cJ DJ_ab DJ_cd - cK/2 sum_m (DK_ac DK_bd + DK_ad DK_bc)] in the final
  // basis (t0), then (pure) back to Cartesian one index at a time
  const int Ls[4] = {LA, LB, LC, LD};
  int dims[4];
  for (int q = 0; q < 4; ++q) dims[q] = pure ? npure_of(Ls[q]) : ncart_of(Ls[q]);
  {
    const int tot = dims[0] * dims[1] * dims[2] * dims[3];
    R* dstw = pure ? t0 : W;
    for (int e = lane; e < tot; e += NT) {
      const int l = e % dims[3], k = (e / dims[3]) % dims[2], j = (e / (dims[3] * dims[2])) % dims[1];
      const int i = e / (dims[3] * dims[2] * dims[1]);
      const int ia = P.fa + i, jb = P.fb + j, kc = Q.fa + k, ld = Q.fb + l;
      double w = DJ ? a.cJ * __ldg(DJ + (size_t)ia * nm + jb) * __ldg(DJ + (size_t)kc * nm + ld) : 0.0;
      for (int m = 0; m < a.nK; ++m) {
        const double* D = DK + (size_t)m * nm * nm;
        w -= 0.5 * a.cK *
             (__ldg(D + (size_t)ia * nm + kc) * __ldg(D + (size_t)jb * nm + ld) +
              __ldg(D + (size_t)ia * nm + ld) * __ldg(D + (size_t)jb * nm + kc));
      }
      dstw[e] = R(s8 * w);
    }
    group_sync<NT>();
  }
  if (pure) {
    R* bufs[2] = {t1, t0};
    const R* in = t0;
    for (int st = 0; st < 4; ++st) {
      const int nc = ncart_of(Ls[st]), np = npure_of(Ls[st]);
      int nd[4] = {dims[0], dims[1], dims[2], dims[3]};
      nd[st] = nc;
      R* o = st == 3 ? W : bufs[st & 1];
      const int tot = nd[0] * nd[1] * nd[2] * nd[3];
      for (int e = lane; e < tot; e += NT) {
        int id[4];
        int r = e;
        for (int q = 3; q >= 0; --q) {
          id[q] = r % nd[q];
          r /= nd[q];
        }
        R v = R(0);
        for (int c = 0; c < np; ++c) {
          const double y = c_ylm[Ls[st]][id[st] * np + c];
          if (y == 0.0) continue;
          int jd[4] = {id[0], id[1], id[2], id[3]};
          jd[st] = c;
          v += R(y) * in[((jd[0] * dims[1] + jd[1]) * dims[2] + jd[2]) * dims[3] + jd[3]];
        }
        o[e] = v;
      }
      group_sync<NT>();
      for (int q = 0; q < 4; ++q) dims[q] = nd[q];
      in = o;
    }
  }
  for (int t = lane; t < Tab::NACC; t += NT) hs[t] = R(0);
  if (lane == 0) {
    vs[Tab::NVSLOT] = R(0);
    hs[Tab::NHSLOT] = R(0);
  }
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
      R F[Tab::L + 1];
      a.boys.template eval<Tab::L>(T, Kab * Kcd * rs, F);
#pragma unroll
      for (int m = 0; m <= Tab::L; ++m)
        if (lane == m) vs[m] = F[m];
      group_sync<NT>();
      for (int l = 0; l < Tab::NVLEV; ++l) {
        const int e = __ldg(vl + l + 1);
        // two op rows in flight per lane: the rows of one level are independent
        auto body = [&](const int4 op) {
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
        };
        for (int o = __ldg(vl + l) + lane; o < e; o += 2 * NT) {
          const int4 opa = __ldg(vo + o);
          const bool two = o + NT < e;
          const int4 opb = two ? __ldg(vo + o + NT) : opa;
          body(opa);
          if (two) body(opb);
        }
        group_sync<NT>();
      }
      for (int t = lane; t < Tab::NACC; t += NT) {
        const int2 ac = __ldg(acc + t);
        const R w = ac.y == 0 ? R(1) : (ac.y == 1 ? wa : (ac.y == 2 ? wb : wc));
        hs[t] += w * vs[ac.x];
      }
      group_sync<NT>();
    }
  }
  // HRR of the four sets and the contractions with W, per lane into nine partial sums
  R g[9];
#pragma unroll
  for (int x = 0; x < 9; ++x) g[x] = R(0);
  const int2* ho = Tab::hrr();
  const int* hl = Tab::hlev();
  const R ABx = R(P.ABx), ABy = R(P.ABy), ABz = R(P.ABz), CDx = R(Q.ABx), CDy = R(Q.ABy), CDz = R(Q.ABz);
  for (int l = 0; l < Tab::NHLEV; ++l) {
    const int e = __ldg(hl + l + 1);
    // two op rows in flight per lane: the rows of one level are independent
    auto body = [&](const int2 op) {
      const int kd = (unsigned)op.y >> 16;
      const int x = (unsigned)op.x >> 16, y = op.y & 0xffff;
      if ((kd & 3) == 2) {
        const int gi = (kd >> 2) & 15;
        const R v = W[op.x & 0xffff] * (hs[x] - small_int<R>(kd >> 6) * hs[y]);
#pragma unroll
        for (int c = 0; c < 9; ++c)
          if (c == gi) g[c] += v;
      } else {
        const int dir = kd >> 2;
        const R d = (kd & 1) ? (dir == 0 ? CDx : (dir == 1 ? CDy : CDz)) : (dir == 0 ? ABx : (dir == 1 ? ABy : ABz));
        hs[op.x & 0xffff] = hs[x] + d * hs[y];
      }
    };
    for (int o = __ldg(hl + l) + lane; o < e; o += 2 * NT) {
      const int2 opa = __ldg(ho + o);
      const bool two = o + NT < e;
      const int2 opb = two ? __ldg(ho + o + NT) : opa;
      body(opa);
      if (two) body(opb);
    }
    group_sync<NT>();
  }
#pragma unroll
  for (int c = 0; c < 9; ++c)
    for (int off = 16; off > 0; off >>= 1) g[c] += __shfl_xor_sync(0xffffffffu, g[c], off);
  if constexpr (NT > 32) {
    // warp sums across the block through t0 (free after the weights; the last level synced)
    if ((lane & 31) == 0)
#pragma unroll
      for (int c = 0; c < 9; ++c) t0[(lane >> 5) * 9 + c] = g[c];
    __syncthreads();
    if (lane == 0)
      for (int w = 1; w < NT / 32; ++w)
#pragma unroll
        for (int c = 0; c < 9; ++c) g[c] += t0[w * 9 + c];
  }
  if (lane == 0) {
    const int at[3] = {P.atom_a, P.atom_b, Q.atom_a};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double gA = double(g[d]), gB = double(g[3 + d]), gC = double(g[6 + d]);
      atomicAdd(a.grad + 3 * at[0] + d, gA);
      atomicAdd(a.grad + 3 * at[1] + d, gB);
      atomicAdd(a.grad + 3 * at[2] + d, gC);
      atomicAdd(a.grad + 3 * Q.atom_b + d, -(gA + gB + gC));
    }
  }
}
