// Host side of the hfgpu engine: basis set-up, primitive-pair data, Schwarz
// factors, screened quartet lists, and the C ABI of include/hfgpu.h.
#include <algorithm>
#include <cooperative_groups.h>
#include <atomic>
#include <chrono>
#include <thread>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/hfgpu.h"
#include "hfgpu_kernels.cuh"
#include "hfgpu_launch.h"
#include "hfgpu_hess_kernels.cuh"
#include "hfgpu_hess_launch.h"
#include "hfgpu_onee.h"
#include "hfgpu_onee_kernels.cuh"
#include "hfgpu_batch_eigh.cuh"
#include "hfgpu_batch_purify.cuh"

namespace {

constexpr int kPairClasses = 6;
constexpr double kPi = 3.14159265358979323846;
// A primitive quartet contributes at most |Kp_ab Kp_cd| / sqrt(p + q) (times F_m <= 1 and
// the recurrence factors) to any integral; primitive pairs whose bound against the
// largest pair of the molecule is below kPrimQuartetCut are dropped.
constexpr double kPrimQuartetCut = 1e-16;

int pair_class(int la, int lb) { return la * (la + 1) / 2 + lb; }  // la >= lb: ss ps pp ds dp dd
int quartet_class(int cp, int cq) { return cp * (cp + 1) / 2 + cq; }  // cp >= cq

// Boys table rows (layout in hfgpu_common.cuh): F_m(k h), m < BOYS_NM, from the series
// e^-T sum_i (2T)^i / (2m+1)(2m+3)...(2m+2i+1) in long double, divided by j! for the j-th
// Taylor term, and e^-T_k.  `terms` = 7 (FP64 rows) or 4 (FP32 rows).
template <typename R>
std::vector<R> boys_table(int terms) {
  std::vector<long double> F((size_t)BOYS_NGRID * BOYS_NM), ek(BOYS_NGRID);
  for (int k = 0; k < BOYS_NGRID; ++k) {
    const long double T = (long double)k * (long double)BOYS_H;
    for (int m = 0; m < BOYS_NM; ++m) {
      long double term = 1.0L / (2 * m + 1), sum = term;
      for (int i = 0; i < 2000; ++i) {
        term *= 2.0L * T / (long double)(2 * m + 2 * i + 3);
        sum += term;
        if (term < sum * 1e-21L) break;
      }
      F[(size_t)k * BOYS_NM + m] = expl(-T) * sum;
    }
    ek[k] = expl(-T);
  }
  std::vector<R> t((size_t)(BOYS_MMAX + 1) * BOYS_NGRID * BOYS_ROW, R(0));
  for (int M = 0; M <= BOYS_MMAX; ++M)
    for (int k = 0; k < BOYS_NGRID; ++k) {
      R* row = &t[((size_t)M * BOYS_NGRID + k) * BOYS_ROW];
      long double fact = 1.0L;
      for (int j = 0; j < terms; ++j) {
        if (j > 0) fact *= j;
        row[j] = (R)(F[(size_t)k * BOYS_NM + M + j] / fact);
      }
      row[terms] = (R)ek[k];
    }
  return t;
}

// The same table in the plane layout of BoysShared (hfgpu_common.cuh): per order, FP64 planes
// j = 0..3 of (row[2j], row[2j+1]) over the grid points; FP32 one plane of row[0..3].
template <typename R>
std::vector<R> boys_planes(const std::vector<R>& rows) {
  const int per = boys_plane_bytes<R>() / (int)sizeof(R);  // values per order
  std::vector<R> t((size_t)(BOYS_MMAX + 1) * per, R(0));
  for (int M = 0; M <= BOYS_MMAX; ++M)
    for (int k = 0; k < BOYS_NGRID; ++k) {
      const R* row = &rows[((size_t)M * BOYS_NGRID + k) * BOYS_ROW];
      R* o = &t[(size_t)M * per];
      if (sizeof(R) == 8) {
        for (int j = 0; j < BOYS_PLANES_D; ++j) {
          o[((size_t)j * BOYS_NGRID + k) * 2 + 0] = row[2 * j];
          o[((size_t)j * BOYS_NGRID + k) * 2 + 1] = row[2 * j + 1];
        }
      } else {
        for (int j = 0; j < 4; ++j) o[(size_t)k * 4 + j] = row[j];
      }
    }
  return t;
}

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  cudaError_t ensure(size_t b) {
    if (b <= bytes) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
    cudaError_t e = cudaMalloc(&p, b);
    if (e == cudaSuccess) bytes = b;
    return e;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  template <typename T>
  T* as() const {
    return static_cast<T*>(p);
  }
};

}  // namespace

struct hfgpu_handle {
  // basis
  int nshell = 0, natoms = 0, pure = 0, n = 0;
  std::vector<int> L, shell_atom, nprim, prim_off, first;
  std::vector<double> exps, coefs;  // normalised coefficients
  std::vector<double> xyz;
  bool have_geometry = false;
  hfgpu_opts opts{};
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  std::string err;

  // batched handles: several molecules; shells of molecule m are [mol_shell[m], mol_shell[m+1]),
  // its matrices the n_m x n_m block at mol_off[m] of the block storage (mat_total doubles)
  int nmol = 1;
  bool batched = false;
  std::vector<int> mol_shell, mol_n, mol_atom;
  std::vector<long long> mol_off;
  long long mat_total = 0;
  DevBuf d_mol;

  // pair data (host mirror) and class ranges; cm_begin[c * (nmol+1) + m]: first pair of class c, molecule m
  std::vector<PairInfo> pairs;
  int class_begin[kPairClasses + 1] = {0};
  std::vector<int> cm_begin;
  int nprimpairs = 0;

  // quartet lists per class: [beg, mid) high bound (FP64 always), [mid, end) low bound;
  // inside each part the quartets with many primitive quartets come first:
  // [beg, hik1) and [mid, hik2) run the warp-over-primitives kernel where the class has one
  std::vector<long long> q_beg, q_mid, q_end, q_hik1, q_hik2;
  std::vector<long long> q_prims;  // per class: primitive quartets of the Schwarz-screened quartets
  int part = 0, nparts = 1;        // partition of every quartet list (hfgpu_set_partition)
  // classes of a J/K build / a gradient on the auxiliary streams concurrently (0) or one after
  // another on one of them (1); chosen by the autotuners on whole builds
  int jk_serial = 0, grad_serial = 0;
  // inside each of the four segments quartets are ordered by Schwarz-bound decade
  // (largest first; inside a decade by primitive-quartet count, then bra-major):
  // bucket_end[(c * 4 + seg) * kBuckets + e] is the
  // end of decade e (bound in [10^-e, 10^(1-e)), e = 0 collects bounds >= 1)
  std::vector<long long> bucket_end;
  DevBuf d_gmax;
  // per geometry, for density-screened builds without a host round trip: d_launch holds per
  // (class, list segment) the segment's [lo, hi) and its decade ends (2 + kBuckets longs),
  // d_dyn the counts a build's launches process, d_first the first function of every shell
  DevBuf d_launch, d_dyn, d_first;
  // the Boys table in the plane layout of the staged kernels, and the device status word
  DevBuf d_boys_pd, d_boys_pf, d_status, d_abort;
  DevBuf d_purify;  // workspace of hfgpu_purify_device
  cudaStream_t ctl_stream = nullptr;  // non-blocking stream of hfgpu_request_abort
  int status_host = 0;  // the status word as the last host-pointer entry point read it
  long long nquartets = 0;

  DevBuf d_pairs, d_prim_d, d_prim_f, d_alpha_d, d_alpha_f, d_boys_d, d_boys_f, d_quart;
  DevBuf d_onee;  // one-electron kernels: atoms (x, y, z, Z), molecule atom ranges, Cartesian -> pure tables
  DevBuf d_mats, d_half, d_dmax, d_counters, d_grad, d_scratch, d_eri, d_eriq;
  long long last_launched = 0, last_skipped = 0;
  int last_kernels = 0;                 // kernel launches of the last J/K build
  double setup_ms[4] = {0, 0, 0, 0};    // last set_geometry: pairs, Schwarz, quartet lists (host), list upload
  // class kernels run concurrently on auxiliary streams (fork/join with events)
  static constexpr int kAux = 6;
  cudaStream_t aux[kAux] = {};
  cudaEvent_t fork_ev = nullptr, join_ev[kAux] = {};
  bool timing = false;                  // record CUDA events around every class launch
  cudaEvent_t ev[2 * 21 + 2] = {};
  bool ev_used[21] = {};
  // per-class launch schedule (hfgpu_autotune / hfgpu_set_schedule): threads per block of
  // the thread-per-quartet form, warp-over-primitives form for the many-primitive parts,
  // warp-per-quartet form (-1 = follow opts.warp_max_quartets)
  int sched_block[21], sched_primwarp[21], sched_warp[21], sched_cap[21];
  unsigned class_mask = ~0u;            // classes a J/K build launches (autotuning runs one at a time)
  // gradient form per class (hfgpu_autotune_grad): 1 warp per quartet, 0 one thread per
  // quartet, 3/4 (5/6) block of four (eight) warps per quartet (whole / split), -1 the default
  // (grad_form_of)
  int grad_form[21];
  unsigned grad_class_mask = ~0u;       // classes a gradient launches (autotuning runs one at a time)
  // Hessian form (hfgpu_set_hess_form): -1 by class, 0 one thread per quartet, 1 one block per
  // quartet, 2 one warp per quartet (where the class's tables fit), 3 one thread per quartet on
  // straight-line code (where the class has it)
  int hess_form = -1;
  int purify_blocks = -1;               // co-resident blocks of the cooperative purification (0: not available)
  int purify_coop = 1;                  // hfgpu_set_purify_mode: 1 one cooperative launch, 0 two launches per step
  int hess_cls_form[21];                // per class (hfgpu_autotune_hess): 0 thread, 1 block, 2 warp, 3 line,
                                        // -1 hess_form
  unsigned hess_class_mask = ~0u;       // classes a Hessian launches (autotuning runs one at a time)

  hfgpu_handle() : q_beg(21), q_mid(21), q_end(21), q_hik1(21), q_hik2(21), q_prims(21) {
    for (int c = 0; c < 21; ++c) {
      sched_block[c] = 64;
      sched_primwarp[c] = 0;
      sched_warp[c] = c < hfgpu::kNumClasses && hfgpu::kClassLaunchers[c]->warp_default ? -1 : 0;
      sched_cap[c] = 0;
      grad_form[c] = -1;
      hess_cls_form[c] = -1;
    }
  }
};

namespace {

int fail(hfgpu_handle* h, int code, const std::string& msg) {
  if (h) h->err = msg;
  return code;
}

// warp_max of QuartetArgs for class c under the handle's schedule
int class_warp_max(const hfgpu_handle* h, int c) {
  const int w = h->sched_warp[c];
  return w < 0 ? h->opts.warp_max_quartets : (w ? INT_MAX : -1);
}

// threads per quartet of that form: schedule entry 2 = one block of 128 threads per quartet
int class_warp_threads(const hfgpu_handle* h, int c) { return h->sched_warp[c] == 2 ? 128 : 32; }

int cuda_fail(hfgpu_handle* h, cudaError_t e, const char* where) {
  return fail(h, e == cudaErrorMemoryAllocation ? HFGPU_ERR_NOMEM : HFGPU_ERR_CUDA,
              std::string(where) + ": " + cudaGetErrorString(e));
}

#define HF_CUDA(h, call)                                    \
  do {                                                      \
    cudaError_t e_ = (call);                                \
    if (e_ != cudaSuccess) return cuda_fail(h, e_, #call);  \
  } while (0)

#define HF_CHECK_LAUNCH(h, what)                              \
  do {                                                        \
    cudaError_t e_ = cudaGetLastError();                      \
    if (e_ != cudaSuccess) return cuda_fail(h, e_, what);     \
  } while (0)

// Normalisation of BASIS::Shell::Shell (src/integrals/hfscf_shell.cpp:44-54).
void normalise(int L, int np, const double* a, const double* c, double* out) {
  const double m = L + 1.5, m2 = 0.5 * m;
  double sum = 0.0;
  for (int j = 0; j < np; ++j)
    for (int k = 0; k < np; ++k) sum += c[j] * c[k] * std::pow(a[j] * a[k], m2) / std::pow(a[j] + a[k], m);
  double dfac = 1.0;
  for (int x = 2 * L - 1; x > 1; x -= 2) dfac *= x;
  const double norm = 1.0 / std::sqrt(sum * std::pow(kPi, 1.5) * dfac / std::pow(2.0, L));
  for (int j = 0; j < np; ++j) out[j] = c[j] * norm * std::pow(a[j], m2);
}

// Makes the handle's device current for the duration of one entry point and restores the
// caller's current device when the entry point returns (on every path).
struct DeviceGuard {
  int prev = -1;
  int rc = HFGPU_OK;
  explicit DeviceGuard(hfgpu_handle* h) {
    if (cudaGetDevice(&prev) != cudaSuccess) {
      (void)cudaGetLastError();
      prev = -1;
    }
    if (prev != h->device) {
      const cudaError_t e = cudaSetDevice(h->device);
      if (e != cudaSuccess) rc = cuda_fail(h, e, "cudaSetDevice");
    }
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
  DeviceGuard(const DeviceGuard&) = delete;
  DeviceGuard& operator=(const DeviceGuard&) = delete;
};

// Runs f(0) ... f(ntask - 1) on up to max_threads threads (the caller's thread among them).
template <typename F>
void run_parallel(int ntask, int max_threads, F&& f) {
  std::atomic<int> next{0};
  auto work = [&]() {
    for (int i = next++; i < ntask; i = next++) f(i);
  };
  const int nthr = std::max(1, std::min(ntask, max_threads));
  std::vector<std::thread> pool;
  for (int t = 1; t < nthr; ++t) pool.emplace_back(work);
  work();
  for (auto& t : pool) t.join();
}

// Primitive pairs of every canonical shell pair; pairs sorted by class, then by
// primitive count (descending) so that quartet lists group equal loop lengths.
int build_pairs(hfgpu_handle* h) {
  struct Tmp {
    int sa, sb, cls, np, mol;
  };
  std::vector<Tmp> tmp;
  for (int m = 0; m < h->nmol; ++m)
    for (int i = h->mol_shell[m]; i < h->mol_shell[m + 1]; ++i)
      for (int j = i; j < h->mol_shell[m + 1]; ++j) {
        int sa = i, sb = j;
        if (h->L[sa] < h->L[sb]) std::swap(sa, sb);
        tmp.push_back({sa, sb, pair_class(h->L[sa], h->L[sb]), h->nprim[sa] * h->nprim[sb], m});
      }
  std::stable_sort(tmp.begin(), tmp.end(), [](const Tmp& x, const Tmp& y) {
    if (x.cls != y.cls) return x.cls < y.cls;
    if (x.mol != y.mol) return x.mol < y.mol;
    return x.np > y.np;
  });
  const int nm1 = h->nmol + 1;
  h->cm_begin.assign((size_t)kPairClasses * nm1, 0);
  for (int c = 0; c < kPairClasses; ++c)
    for (int m = 0; m <= h->nmol; ++m) {
      // first pair at or after (class c, molecule m) in the (class, molecule) order
      const auto it = std::lower_bound(tmp.begin(), tmp.end(), std::make_pair(c, m), [](const Tmp& x, const std::pair<int, int>& k) {
        return x.cls < k.first || (x.cls == k.first && x.mol < k.second);
      });
      h->cm_begin[(size_t)c * nm1 + m] = (int)(it - tmp.begin());
    }
  // The primitive pairs are made on all host threads, in chunks of consecutive pairs: (1) the
  // largest |Kp| and smallest p over all primitive pairs, for the primitive-pair cut, (2) the
  // kept primitive pairs of every pair, (3) after a prefix sum, every pair's records at its offset.
  // Same arithmetic and order as one pass over the pairs.
  const int npairs = (int)tmp.size();
  const int threads = npairs < 4096 ? 1 : (int)std::max(1u, std::thread::hardware_concurrency());
  const int nchunk = std::max(1, std::min(npairs, 8 * threads));
  auto chunk_range = [&](int ci, int& x0, int& x1) {
    x0 = (int)((long long)npairs * ci / nchunk);
    x1 = (int)((long long)npairs * (ci + 1) / nchunk);
  };
  // K of primitive pair (i, j) of pair t (self pairs: (i, j) and (j, i) stored once, K doubled)
  auto prim_k = [&](const Tmp& t, double R2, int i, int j, double& p) {
    const double a1 = h->exps[h->prim_off[t.sa] + i], a2 = h->exps[h->prim_off[t.sb] + j];
    p = a1 + a2;
    return std::exp(-a1 * a2 / p * R2) * h->coefs[h->prim_off[t.sa] + i] * h->coefs[h->prim_off[t.sb] + j] *
           ((t.sa == t.sb && j > i) ? 2.0 : 1.0);
  };
  auto pair_r2 = [&](const Tmp& t) {
    const double* A = &h->xyz[3 * h->shell_atom[t.sa]];
    const double* B = &h->xyz[3 * h->shell_atom[t.sb]];
    return (A[0] - B[0]) * (A[0] - B[0]) + (A[1] - B[1]) * (A[1] - B[1]) + (A[2] - B[2]) * (A[2] - B[2]);
  };
  std::vector<double> ck_max(nchunk, 0.0), cp_min(nchunk, 1e300);
  run_parallel(nchunk, threads, [&](int ci) {
    int x0, x1;
    chunk_range(ci, x0, x1);
    double km = 0.0, pm = 1e300;
    for (int x = x0; x < x1; ++x) {
      const Tmp& t = tmp[x];
      const double R2 = pair_r2(t);
      for (int i = 0; i < h->nprim[t.sa]; ++i)
        for (int j = 0; j < h->nprim[t.sb]; ++j) {
          const double a1 = h->exps[h->prim_off[t.sa] + i], a2 = h->exps[h->prim_off[t.sb] + j];
          const double p = a1 + a2;
          const double fold = (t.sa == t.sb && i != j) ? 2.0 : 1.0;  // see the folding below
          const double kp = fold * std::fabs(std::exp(-a1 * a2 / p * R2) * h->coefs[h->prim_off[t.sa] + i] *
                                             h->coefs[h->prim_off[t.sb] + j]) * std::sqrt(PI_2_5) / p;
          km = std::max(km, kp);
          pm = std::min(pm, p);
        }
    }
    ck_max[ci] = km;
    cp_min[ci] = pm;
  });
  double kp_max = 0.0, p_min = 1e300;
  for (int ci = 0; ci < nchunk; ++ci) {
    kp_max = std::max(kp_max, ck_max[ci]);
    p_min = std::min(p_min, cp_min[ci]);
  }
  const double kp_cut = kPrimQuartetCut * std::sqrt(2.0 * p_min) / std::max(kp_max, 1e-300);
  // (2) kept primitive pairs per pair
  std::vector<int> kept(npairs + 1, 0);
  run_parallel(nchunk, threads, [&](int ci) {
    int x0, x1;
    chunk_range(ci, x0, x1);
    for (int x = x0; x < x1; ++x) {
      const Tmp& t = tmp[x];
      const double R2 = pair_r2(t);
      const bool self = t.sa == t.sb;
      int k = 0;
      for (int i = 0; i < h->nprim[t.sa]; ++i)
        for (int j = self ? i : 0; j < h->nprim[t.sb]; ++j) {
          double p;
          const double K = prim_k(t, R2, i, j, p);
          if (!(std::fabs(K) * std::sqrt(PI_2_5) / p < kp_cut)) ++k;
        }
      kept[x + 1] = k;
    }
  });
  for (int x = 0; x < npairs; ++x) kept[x + 1] += kept[x];
  h->pairs.assign(tmp.size(), PairInfo{});
  std::vector<PrimPair<double>> pd((size_t)kept[npairs]);
  std::vector<double> aa((size_t)kept[npairs]), ab((size_t)kept[npairs]);
  for (int c = 0; c <= kPairClasses; ++c) h->class_begin[c] = (int)tmp.size();
  for (size_t x = 0; x < tmp.size(); ++x) h->class_begin[tmp[x].cls] = std::min(h->class_begin[tmp[x].cls], (int)x);
  // (3) the records
  run_parallel(nchunk, threads, [&](int ci) {
    int x0, x1;
    chunk_range(ci, x0, x1);
    for (int x = x0; x < x1; ++x) {
      const Tmp& t = tmp[x];
      PairInfo& P = h->pairs[x];
      P.sa = t.sa;
      P.sb = t.sb;
      P.fa = h->first[t.sa];
      P.fb = h->first[t.sb];
      P.cls = t.cls;
      P.mol = t.mol;
      P.atom_a = h->shell_atom[t.sa];
      P.atom_b = h->shell_atom[t.sb];
      const double* A = &h->xyz[3 * P.atom_a];
      const double* B = &h->xyz[3 * P.atom_b];
      P.ABx = A[0] - B[0];
      P.ABy = A[1] - B[1];
      P.ABz = A[2] - B[2];
      const double R2 = P.ABx * P.ABx + P.ABy * P.ABy + P.ABz * P.ABz;
      P.prim_off = kept[x];
      // A pair of a shell with itself has A = B, so primitive pairs (i, j) and (j, i) have the
      // same p, P, PA and K: they are stored once, j >= i, with K doubled for j > i.  For the
      // gradient both exponent weights become (a_i + a_j)/2: the A and B derivatives then
      // have the right sum, which is all that reaches the atom the two centres share.
      const bool self = t.sa == t.sb;
      int o = kept[x];
      for (int i = 0; i < h->nprim[t.sa]; ++i)
        for (int j = self ? i : 0; j < h->nprim[t.sb]; ++j) {
          double a1 = h->exps[h->prim_off[t.sa] + i], a2 = h->exps[h->prim_off[t.sb] + j];
          double p;
          const double K = prim_k(t, R2, i, j, p);
          double eb2 = a2 * a2;  // the kinetic integral is quadratic in the ket exponent
          if (self && j > i) {
            eb2 = 0.5 * (a1 * a1 + a2 * a2);
            a1 = a2 = 0.5 * p;
          }
          if (std::fabs(K) * std::sqrt(PI_2_5) / p < kp_cut) continue;
          PrimPair<double>& q = pd[(size_t)o];
          q.p = p;
          q.ip = 1.0 / p;
          q.eb2 = eb2;
          q.Px = (a1 * A[0] + a2 * B[0]) / p;
          q.Py = (a1 * A[1] + a2 * B[1]) / p;
          q.Pz = (a1 * A[2] + a2 * B[2]) / p;
          q.PAx = q.Px - A[0];
          q.PAy = q.Py - A[1];
          q.PAz = q.Pz - A[2];
          q.Kp = K * std::sqrt(PI_2_5) / p;
          aa[(size_t)o] = a1;
          ab[(size_t)o] = a2;
          ++o;
        }
      P.nprim = o - kept[x];
      P.schwarz = 0.0;
    }
  });
  for (int c = kPairClasses - 1; c >= 0; --c)
    if (h->class_begin[c] > h->class_begin[c + 1]) h->class_begin[c] = h->class_begin[c + 1];
  h->nprimpairs = (int)pd.size();
  const size_t np = std::max<size_t>(pd.size(), 1);
  std::vector<PrimPair<float>> pf(np);
  std::vector<float> aaf(np), abf(np);
  for (size_t i = 0; i < pd.size(); ++i) {
    pf[i] = {(float)pd[i].p, (float)pd[i].ip, (float)pd[i].Px, (float)pd[i].Py, (float)pd[i].Pz,
             (float)pd[i].PAx, (float)pd[i].PAy, (float)pd[i].PAz, (float)pd[i].Kp, (float)pd[i].eb2};
    aaf[i] = (float)aa[i];
    abf[i] = (float)ab[i];
  }
  HF_CUDA(h, h->d_pairs.ensure(sizeof(PairInfo) * std::max<size_t>(h->pairs.size(), 1)));
  HF_CUDA(h, h->d_prim_d.ensure(sizeof(PrimPair<double>) * np));
  HF_CUDA(h, h->d_prim_f.ensure(sizeof(PrimPair<float>) * np));
  HF_CUDA(h, h->d_alpha_d.ensure(sizeof(double) * 2 * np));
  HF_CUDA(h, h->d_alpha_f.ensure(sizeof(float) * 2 * np));
  cudaStream_t s = h->stream;
  HF_CUDA(h, cudaMemcpyAsync(h->d_pairs.p, h->pairs.data(), sizeof(PairInfo) * h->pairs.size(), cudaMemcpyHostToDevice, s));
  if (!pd.empty()) {
    HF_CUDA(h, cudaMemcpyAsync(h->d_prim_d.p, pd.data(), sizeof(PrimPair<double>) * pd.size(), cudaMemcpyHostToDevice, s));
    HF_CUDA(h, cudaMemcpyAsync(h->d_prim_f.p, pf.data(), sizeof(PrimPair<float>) * pd.size(), cudaMemcpyHostToDevice, s));
    HF_CUDA(h, cudaMemcpyAsync(h->d_alpha_d.p, aa.data(), sizeof(double) * pd.size(), cudaMemcpyHostToDevice, s));
    HF_CUDA(h, cudaMemcpyAsync(h->d_alpha_d.as<double>() + np, ab.data(), sizeof(double) * pd.size(), cudaMemcpyHostToDevice, s));
    HF_CUDA(h, cudaMemcpyAsync(h->d_alpha_f.p, aaf.data(), sizeof(float) * pd.size(), cudaMemcpyHostToDevice, s));
    HF_CUDA(h, cudaMemcpyAsync(h->d_alpha_f.as<float>() + np, abf.data(), sizeof(float) * pd.size(), cudaMemcpyHostToDevice, s));
  }
  HF_CUDA(h, cudaStreamSynchronize(s));
  return HFGPU_OK;
}

JKArgs<double> jk_args_d(hfgpu_handle* h) {
  JKArgs<double> a{};
  a.pairs = h->d_pairs.as<PairInfo>();
  a.prims = h->d_prim_d.as<PrimPair<double>>();
  a.boys.tab = h->d_boys_d.as<double>();
  a.n = h->n;
  a.nshell = h->nshell;
  return a;
}

JKArgs<float> jk_args_f(hfgpu_handle* h) {
  JKArgs<float> a{};
  a.pairs = h->d_pairs.as<PairInfo>();
  a.prims = h->d_prim_f.as<PrimPair<float>>();
  a.boys.tab = h->d_boys_f.as<float>();
  a.n = h->n;
  a.nshell = h->nshell;
  return a;
}

// Schwarz factors: (P|P) for every pair, class by class.
int compute_schwarz(hfgpu_handle* h) {
  const int npairs = (int)h->pairs.size();
  std::vector<int2> diag(std::max(npairs, 1));
  for (int x = 0; x < npairs; ++x) diag[x] = make_int2(x, x);
  HF_CUDA(h, h->d_quart.ensure(sizeof(int2) * diag.size()));
  HF_CUDA(h, cudaMemcpyAsync(h->d_quart.p, diag.data(), sizeof(int2) * npairs, cudaMemcpyHostToDevice, h->stream));
  QuartetArgs<double> qa{};
  qa.jk = jk_args_d(h);
  qa.mode = QMODE_SCHWARZ;
  qa.pure = h->pure;
  qa.pairs_rw = h->d_pairs.as<PairInfo>();
  for (int c = 0; c < kPairClasses; ++c) {
    const int b = h->class_begin[c], e = h->class_begin[c + 1];
    if (e <= b) continue;
    qa.warp_max = class_warp_max(h, quartet_class(c, c));
    qa.warp_threads = class_warp_threads(h, quartet_class(c, c));
    qa.block = h->sched_block[quartet_class(c, c)];
    qa.capped = h->sched_cap[quartet_class(c, c)];
    const hfgpu::ClassLaunchers* L = hfgpu::kClassLaunchers[quartet_class(c, c)];
    L->quartet_d(qa, h->d_quart.as<int2>() + b, e - b, h->stream);
    HF_CHECK_LAUNCH(h, "schwarz kernel");
  }
  HF_CUDA(h, cudaMemcpyAsync(h->pairs.data(), h->d_pairs.p, sizeof(PairInfo) * npairs, cudaMemcpyDeviceToHost, h->stream));
  HF_CUDA(h, cudaStreamSynchronize(h->stream));
  for (const PairInfo& P : h->pairs)
    if (!std::isfinite(P.schwarz)) return fail(h, HFGPU_ERR_NONFINITE, "non-finite Schwarz factor");
  return HFGPU_OK;
}

constexpr int kPrimWarpMinPrims = 16;  // primitive quartets per quartet for the primitive-split kernel
constexpr int kBuckets = 18;           // Schwarz-bound decades of the quartet lists

// Decade of a Schwarz bound: 0 for b >= 1, else the e >= 1 with b in [10^-e, 10^(1-e)) (the last
// decade also takes everything smaller), by comparisons with the same powers of ten that bound the
// decades on the device (kDecadeUpper), which is all the density-screened launches rely on.
int bound_decade(double b) {
  static const double lo[kBuckets] = {1.0,  1e-1,  1e-2,  1e-3,  1e-4,  1e-5,  1e-6,  1e-7,  1e-8,
                                      1e-9, 1e-10, 1e-11, 1e-12, 1e-13, 1e-14, 1e-15, 1e-16, 1e-17};
  if (b >= 1.0) return 0;
  int e = 1;
  while (e < kBuckets - 1 && b < lo[e]) ++e;
  return e;
}

// Screened unique quartets (P <= Q within a class; bra class >= ket class), per class.
// Quartet list of one class (pair classes cp >= cq), in four segments (Schwarz bound at or
// above the mixed-precision bound / below, each split into quartets with at least
// kPrimWarpMinPrims primitive quartets / fewer), each ordered by one stable counting sort
// on (bound decade, then the primitive shape: ket primitive pairs, then bra primitive pairs,
// largest first): the decades make the prefix launches of density-screened builds possible,
// the shapes let the 32 lanes of a warp run the same trip counts of both primitive loops (a
// sort on the product alone mixes 3 x 1 with 1 x 3).
//
// Built in two parallel phases on all host threads.  Phase 1 filters the candidates of
// chunks of about kListChunkWork candidate quartets (consecutive bra pairs of one class) and
// keeps each chunk's survivors in bra-pair order with their sort keys; phase 2 sorts every
// (class, segment) with one counting sort over its chunks in order and writes it into place.
// The lists are the same as those of one serial pass per class in bra-pair order.
constexpr long long kListChunkWork = 1 << 20;
constexpr int kProdSpan = 1 << 16;  // primitive shapes above this share the last sort slot

struct ListChunk {
  int cls = 0;                  // index into the class table (cp, cq)
  int P0 = 0, P1 = 0;           // bra pairs [P0, P1)
  std::vector<int2> q[4];       // survivors per segment, in list order
  std::vector<int> key[4];      // bound decade * kProdSpan + primitive shape
  int maxprod[4] = {0, 0, 0, 0};
  long long prims = 0;          // primitive quartets of the survivors
};

int build_quartets(hfgpu_handle* h) {
  using clk = std::chrono::steady_clock;
  const auto t0 = clk::now();
  std::vector<std::pair<int, int>> cls;
  for (int cp = 0; cp < kPairClasses; ++cp)
    for (int cq = 0; cq <= cp; ++cq) cls.emplace_back(cp, cq);
  const int ncls = (int)cls.size();
  const int nm1 = h->nmol + 1;
  // ket pair range [k0, ke) of bra pair P in class (cp, cq)
  auto ket_range = [&](int cp, int cq, int P, int& k0, int& ke) {
    const int mol = h->pairs[P].mol;
    const int kb = h->cm_begin[(size_t)cq * nm1 + mol];
    ke = h->cm_begin[(size_t)cq * nm1 + mol + 1];
    k0 = (cp == cq) ? P : kb;
  };
  // chunks of consecutive bra pairs, about kListChunkWork candidates each
  std::vector<ListChunk> chunks;
  std::vector<int> cls_chunk0(ncls + 1, 0);
  long long all_work = 0;  // candidate quartets of every class
  for (int i = 0; i < ncls; ++i) {
    const int cp = cls[i].first, cq = cls[i].second;
    cls_chunk0[i] = (int)chunks.size();
    const int pb = h->class_begin[cp], pe = h->class_begin[cp + 1];
    long long work = 0;
    int start = pb;
    for (int P = pb; P < pe; ++P) {
      int k0, ke;
      ket_range(cp, cq, P, k0, ke);
      work += std::max(0, ke - k0);
      all_work += std::max(0, ke - k0);
      if (work >= kListChunkWork || P + 1 == pe) {
        ListChunk c;
        c.cls = i;
        c.P0 = start;
        c.P1 = P + 1;
        chunks.push_back(std::move(c));
        start = P + 1;
        work = 0;
      }
    }
  }
  cls_chunk0[ncls] = (int)chunks.size();
  // small lists (fewer than two chunks' worth of candidates) are built on the calling thread
  const int threads = all_work < 2 * kListChunkWork ? 1 : (int)std::max(1u, std::thread::hardware_concurrency());
  // phase 1: filter
  const double tol = h->opts.schwarz_tol, mix = h->opts.mixed_fp32_bound;
  // primitive shape of a quartet: ket primitive pairs * shape_mul + bra primitive pairs
  int shape_mul = 1;
  for (int P = 0; P < (int)h->pairs.size(); ++P) shape_mul = std::max(shape_mul, h->pairs[P].nprim + 1);
  // the pairs' Schwarz factors and primitive counts as plain arrays (the inner loop reads them
  // for every candidate ket; PairInfo is 72 bytes)
  std::vector<double> pq_s(h->pairs.size());
  std::vector<int> pq_n(h->pairs.size());
  for (size_t P = 0; P < h->pairs.size(); ++P) {
    pq_s[P] = h->pairs[P].schwarz;
    pq_n[P] = h->pairs[P].nprim;
  }
  run_parallel((int)chunks.size(), threads, [&](int ci) {
    ListChunk& c = chunks[ci];
    const int cp = cls[c.cls].first, cq = cls[c.cls].second;
    for (int P = c.P0; P < c.P1; ++P) {
      const double qp = h->pairs[P].schwarz;
      const int np = h->pairs[P].nprim;
      int k0, ke;
      ket_range(cp, cq, P, k0, ke);
      for (int Q = k0; Q < ke; ++Q) {
        const double b = qp * pq_s[Q];
        if (b < tol) continue;
        const int nq = pq_n[Q];
        c.prims += (long long)np * nq;
        const int prod = np * nq;
        const int shape = (int)std::min<long long>((long long)nq * shape_mul + np, kProdSpan - 1);
        const int sg = (b >= mix ? 0 : 2) + (prod >= kPrimWarpMinPrims ? 0 : 1);
        c.q[sg].push_back(make_int2(P, Q));
        c.key[sg].push_back(bound_decade(b) * kProdSpan + shape);
        c.maxprod[sg] = std::max(c.maxprod[sg], shape);
      }
    }
  });
  // offsets: classes in class order, segments in order inside a class
  std::vector<long long> seg_base((size_t)ncls * 5, 0);
  long long total = 0;
  for (int i = 0; i < ncls; ++i) {
    for (int sg = 0; sg < 4; ++sg) {
      seg_base[(size_t)i * 5 + sg] = total;
      for (int ci = cls_chunk0[i]; ci < cls_chunk0[i + 1]; ++ci) total += (long long)chunks[ci].q[sg].size();
    }
    seg_base[(size_t)i * 5 + 4] = total;
  }
  // left uninitialised: every slot is written by the scatter below (a zero-filled vector of the
  // octane-to-batch sizes, 10^7-10^8 quartets, cost 0.15 s of single-threaded page touching)
  std::unique_ptr<int2[]> all(new int2[(size_t)std::max<long long>(total, 1)]);
  h->bucket_end.assign((size_t)hfgpu::kNumClasses * 4 * kBuckets, 0);
  // phase 2: one stable counting sort per (class, segment) on (decade, count descending),
  // itself parallel over the class's chunks: (a) per-chunk key histograms, (b) per (class,
  // segment) the histograms become each chunk's first slot per key (keys in order, chunks in
  // order inside a key), (c) every chunk scatters its quartets.
  std::vector<int> seg_span((size_t)ncls * 4, 1);
  for (int i = 0; i < ncls; ++i)
    for (int sg = 0; sg < 4; ++sg) {
      int maxprod = 0;
      for (int ci = cls_chunk0[i]; ci < cls_chunk0[i + 1]; ++ci) maxprod = std::max(maxprod, chunks[ci].maxprod[sg]);
      seg_span[(size_t)i * 4 + sg] = maxprod + 1;
    }
  auto key_of = [&](int raw, int span) { return (raw / kProdSpan) * span + (span - 1 - raw % kProdSpan); };
  std::vector<std::vector<long long>> slot(chunks.size() * 4);  // per (chunk, segment): next slot per key
  run_parallel((int)chunks.size() * 4, threads, [&](int task) {
    const int ci = task / 4, sg = task % 4;
    const ListChunk& c = chunks[ci];
    if (c.key[sg].empty()) return;
    const int span = seg_span[(size_t)c.cls * 4 + sg];
    std::vector<long long>& hst = slot[task];
    hst.assign((size_t)kBuckets * span, 0);
    for (const int raw : c.key[sg]) ++hst[(size_t)key_of(raw, span)];
  });
  run_parallel(ncls * 4, threads, [&](int task) {
    const int i = task / 4, sg = task % 4;
    const int qc = quartet_class(cls[i].first, cls[i].second);
    const int span = seg_span[(size_t)task];
    const int nk = kBuckets * span;
    long long next = seg_base[(size_t)i * 5 + sg];
    for (int k = 0; k < nk; ++k) {
      if (k % span == 0) {
        const int e = k / span;  // decade e starts here; decade e-1 ends here
        if (e > 0) h->bucket_end[((size_t)qc * 4 + sg) * kBuckets + e - 1] = next;
      }
      for (int ci = cls_chunk0[i]; ci < cls_chunk0[i + 1]; ++ci) {
        std::vector<long long>& hst = slot[(size_t)ci * 4 + sg];
        if (hst.empty()) continue;
        const long long n = hst[(size_t)k];
        hst[(size_t)k] = next;
        next += n;
      }
    }
    h->bucket_end[((size_t)qc * 4 + sg) * kBuckets + kBuckets - 1] = next;
  });
  run_parallel((int)chunks.size() * 4, threads, [&](int task) {
    const int ci = task / 4, sg = task % 4;
    const ListChunk& c = chunks[ci];
    if (c.key[sg].empty()) return;
    const int span = seg_span[(size_t)c.cls * 4 + sg];
    std::vector<long long>& nxt = slot[task];
    for (size_t x = 0; x < c.q[sg].size(); ++x) all[(size_t)nxt[(size_t)key_of(c.key[sg][x], span)]++] = c.q[sg][x];
  });
  for (int i = 0; i < ncls; ++i) {
    const int qc = quartet_class(cls[i].first, cls[i].second);
    h->q_beg[qc] = seg_base[(size_t)i * 5 + 0];
    h->q_hik1[qc] = seg_base[(size_t)i * 5 + 1];
    h->q_mid[qc] = seg_base[(size_t)i * 5 + 2];
    h->q_hik2[qc] = seg_base[(size_t)i * 5 + 3];
    h->q_end[qc] = seg_base[(size_t)i * 5 + 4];
    h->q_prims[qc] = 0;
    for (int ci = cls_chunk0[i]; ci < cls_chunk0[i + 1]; ++ci) h->q_prims[qc] += chunks[ci].prims;
  }
  h->nquartets = total;
  const auto t1 = clk::now();
  HF_CUDA(h, h->d_quart.ensure(sizeof(int2) * (size_t)std::max<long long>(total, 1)));
  if (total > 0)
    HF_CUDA(h, cudaMemcpyAsync(h->d_quart.p, all.get(), sizeof(int2) * (size_t)total, cudaMemcpyHostToDevice,
                               h->stream));
  {
    // launch table of the density-screened builds (see launch_counts_kernel)
    const int nslot = hfgpu::kNumClasses * 4;
    std::vector<long long> lt((size_t)nslot * (2 + kBuckets), 0);
    for (int c = 0; c < hfgpu::kNumClasses; ++c) {
      const long long pstart[5] = {h->q_beg[c], h->q_hik1[c], h->q_mid[c], h->q_hik2[c], h->q_end[c]};
      for (int part = 0; part < 4; ++part) {
        long long* row = lt.data() + (size_t)(c * 4 + part) * (2 + kBuckets);
        row[0] = pstart[part];
        row[1] = pstart[part + 1];
        for (int e = 0; e < kBuckets; ++e) row[2 + e] = h->bucket_end[((size_t)c * 4 + part) * kBuckets + e];
      }
    }
    HF_CUDA(h, h->d_launch.ensure(sizeof(long long) * lt.size()));
    HF_CUDA(h, h->d_dyn.ensure(sizeof(int) * nslot));
    HF_CUDA(h, h->d_first.ensure(sizeof(int) * h->first.size()));
    HF_CUDA(h, cudaMemcpyAsync(h->d_launch.p, lt.data(), sizeof(long long) * lt.size(), cudaMemcpyHostToDevice,
                               h->stream));
    if (!h->first.empty())
      HF_CUDA(h, cudaMemcpyAsync(h->d_first.p, h->first.data(), sizeof(int) * h->first.size(),
                                 cudaMemcpyHostToDevice, h->stream));
  }
  HF_CUDA(h, cudaStreamSynchronize(h->stream));
  h->setup_ms[2] = std::chrono::duration<double, std::milli>(t1 - t0).count();
  h->setup_ms[3] = std::chrono::duration<double, std::milli>(clk::now() - t1).count();
  return HFGPU_OK;
}

__global__ void dmax_kernel(const int* __restrict__ first, int nshell, int n, const double* __restrict__ DJ, int nK,
                            const double* __restrict__ DK, float* __restrict__ out) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= nshell * nshell) return;
  const int s = idx / nshell, t = idx % nshell;
  double m = 0.0;
  for (int i = first[s]; i < first[s + 1]; ++i)
    for (int j = first[t]; j < first[t + 1]; ++j) {
      if (DJ) m = fmax(m, fabs(DJ[(size_t)i * n + j]));
      for (int k = 0; k < nK; ++k) m = fmax(m, fabs(DK[(size_t)k * n * n + (size_t)i * n + j]));
    }
  out[idx] = (float)m;
}

// J = Jh + Jh^T, K = Kh + Kh^T (in place into J/K outputs).
// Largest entry of the shell-pair density maxima (non-negative floats compare as ints).
__global__ void gmax_kernel(const float* __restrict__ dmax, int n, unsigned int* out) {
  unsigned int m = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    m = max(m, __float_as_uint(dmax[i]));
  for (int off = 16; off > 0; off >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, off));
  if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

// Per launch of a density-screened build: how many quartets of its list segment can pass the
// per-quartet test.  A segment is ordered by Schwarz-bound decade, largest first; decade e holds
// bounds below kDecadeUpper[e], so with 4 max|D| = dm4 only the decades with
// kDecadeUpper[e] * dm4 >= dtol can hold a surviving quartet.  table: per slot (class * 4 +
// segment) lo, hi and the end of every decade; dyn[slot] = quartets from lo to the end of the
// last such decade.  Runs on the device, so the build needs no host round trip.
__constant__ double kDecadeUpper[18] = {1e300, 1.0,   1e-1,  1e-2,  1e-3,  1e-4,  1e-5,  1e-6,  1e-7,
                                        1e-8,  1e-9,  1e-10, 1e-11, 1e-12, 1e-13, 1e-14, 1e-15, 1e-16};
__global__ void launch_counts_kernel(const unsigned int* __restrict__ gmax_bits, double dtol,
                                     const long long* __restrict__ table, int nslot, int nbuckets,
                                     int* __restrict__ dyn) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nslot) return;
  const double dm4 = 4.0 * (double)__uint_as_float(*gmax_bits);
  int keep = 0;
  for (int e = 0; e < nbuckets; ++e)
    if (kDecadeUpper[e] * dm4 >= dtol) keep = e + 1;
  const long long* row = table + (size_t)s * (2 + nbuckets);
  const long long lo = row[0], hi = row[1];
  const long long end = keep > 0 ? min(hi, row[2 + keep - 1]) : lo;
  dyn[s] = (int)max(0LL, end - lo);
}

// J = Jh + Jh^T inside every molecule's block of a batched handle.
__global__ void batch_symmetrise_kernel(const double* __restrict__ h, double* __restrict__ out, long long tot,
                                        const long long* __restrict__ mol_off, const int* __restrict__ mol_n,
                                        int nmol) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= tot) return;
  int lo = 0, hi = nmol - 1;  // last molecule whose block starts at or before e
  while (lo < hi) {
    const int mid = (lo + hi + 1) / 2;
    if (mol_off[mid] <= e) lo = mid; else hi = mid - 1;
  }
  const long long b = mol_off[lo];
  const int nm = mol_n[lo];
  const long long r = e - b;
  const long long i = r / nm, j = r % nm;
  out[e] = h[e] + h[b + j * nm + i];
}

__global__ void symmetrise_kernel(const double* __restrict__ h, double* __restrict__ out, int n, int nmat) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  const int tot = n * n;
  if (idx >= tot * nmat) return;
  const int m = idx / tot, e = idx % tot;
  const int i = e / n, j = e % n;
  out[idx] = h[(size_t)m * tot + i * n + j] + h[(size_t)m * tot + j * n + i];
}

// F = H + 2J - K (F may alias J).
__global__ void fock_combine_kernel(double* F, const double* __restrict__ H, const double* J,
                                    const double* __restrict__ K, int tot) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < tot) F[i] = H[i] + 2.0 * J[i] - K[i];
}

// F_0 .. F_M at count points T through the engine's own Boys evaluation (BoysTable::eval, the
// routine every quartet kernel calls), F[i * (M + 1) + m], for the direct Boys tests.
template <typename R, int M>
__global__ void boys_eval_kernel(BoysTable<R> bt, const double* __restrict__ T, long long count,
                                 double* __restrict__ F) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  R f[M + 1];
  bt.template eval<M>(R(T[i]), R(1), f);
#pragma unroll
  for (int m = 0; m <= M; ++m) F[i * (M + 1) + m] = double(f[m]);
}

template <typename R, int M>
void launch_boys_eval(const R* tab, const double* T, long long count, double* F, cudaStream_t st) {
  BoysTable<R> bt{tab};
  boys_eval_kernel<R, M><<<(unsigned)((count + 127) / 128), 128, 0, st>>>(bt, T, count, F);
}

template <typename R>
void boys_eval_dispatch(int m, const R* tab, const double* T, long long count, double* F, cudaStream_t st) {
  switch (m) {
    case 0: launch_boys_eval<R, 0>(tab, T, count, F, st); break;
    case 1: launch_boys_eval<R, 1>(tab, T, count, F, st); break;
    case 2: launch_boys_eval<R, 2>(tab, T, count, F, st); break;
    case 3: launch_boys_eval<R, 3>(tab, T, count, F, st); break;
    case 4: launch_boys_eval<R, 4>(tab, T, count, F, st); break;
    case 5: launch_boys_eval<R, 5>(tab, T, count, F, st); break;
    case 6: launch_boys_eval<R, 6>(tab, T, count, F, st); break;
    case 7: launch_boys_eval<R, 7>(tab, T, count, F, st); break;
    case 8: launch_boys_eval<R, 8>(tab, T, count, F, st); break;
    case 9: launch_boys_eval<R, 9>(tab, T, count, F, st); break;
    default: launch_boys_eval<R, 10>(tab, T, count, F, st); break;
  }
}

// ---------------------------------------------------------------------------
// Density by trace-correcting purification (TC2; Niklasson, Phys. Rev. B 66, 155115 (2002)) of
// an orthonormal-basis Fock matrix, for the SCF loop: the projector onto the nocc lowest
// eigenvectors without a diagonalisation.  Workspace (doubles): A, C (n x n each), then per
// step k: tr A_k, tr A_k^2, and a frozen flag f_k (as a double), then emin, emax.
//   purify_bounds_kernel   Gershgorin bounds of Fo (one block), zeroes the per-step slots;
//   purify_init_kernel     A_0 = (emax I - Fo) / (emax - emin);
//   purify_square_kernel   C = A_k A_k (16 x 16 output tiles, shared-memory k tiles), and the
//                          traces of A_k and C from the diagonal tiles; skipped once frozen;
//   purify_update_kernel   frozen_{k+1} = frozen_k or tr A_k - tr A_k^2 < tol;
//                          A_{k+1} = A_k if frozen, C if tr A_k > nocc, else 2 A_k - C.
// Every step reads the slots of its own index only, so no kernel reads what it writes.
// ---------------------------------------------------------------------------
constexpr int kPurifyTile = 16;

__global__ void purify_bounds_kernel(const double* __restrict__ F, int n, double* __restrict__ slots, int nslot,
                                     double* __restrict__ bounds) {
  __shared__ double smin[1024], smax[1024];
  double lo = 1e300, hi = -1e300;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    double r = 0.0;
    for (int j = 0; j < n; ++j)
      if (j != i) r += fabs(F[(size_t)i * n + j]);
    lo = fmin(lo, F[(size_t)i * n + i] - r);
    hi = fmax(hi, F[(size_t)i * n + i] + r);
  }
  smin[threadIdx.x] = lo;
  smax[threadIdx.x] = hi;
  for (int i = threadIdx.x; i < nslot; i += blockDim.x) slots[i] = 0.0;
  __syncthreads();
  for (int off = blockDim.x / 2; off > 0; off >>= 1) {
    if ((int)threadIdx.x < off) {
      smin[threadIdx.x] = fmin(smin[threadIdx.x], smin[threadIdx.x + off]);
      smax[threadIdx.x] = fmax(smax[threadIdx.x], smax[threadIdx.x + off]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    bounds[0] = smin[0];
    bounds[1] = smax[0];
  }
}

__global__ void purify_init_kernel(const double* __restrict__ F, int n, const double* __restrict__ bounds,
                                   double* __restrict__ A) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (long long)n * n) return;
  const int i = (int)(e / n), j = (int)(e % n);
  const double emin = bounds[0], emax = bounds[1];
  A[e] = ((i == j ? emax : 0.0) - F[e]) / (emax - emin);
}

__global__ void __launch_bounds__(kPurifyTile * kPurifyTile) purify_square_kernel(const double* __restrict__ A, int n,
                                                                                   double* __restrict__ C,
                                                                                   double* __restrict__ step) {
  if (step[2] != 0.0) return;  // frozen: nothing to compute
  __shared__ double ta[kPurifyTile][kPurifyTile + 1], tb[kPurifyTile][kPurifyTile + 1];
  const int tx = threadIdx.x % kPurifyTile, ty = threadIdx.x / kPurifyTile;
  const int row = blockIdx.y * kPurifyTile + ty, col = blockIdx.x * kPurifyTile + tx;
  double acc = 0.0;
  for (int k0 = 0; k0 < n; k0 += kPurifyTile) {
    ta[ty][tx] = (row < n && k0 + tx < n) ? A[(size_t)row * n + k0 + tx] : 0.0;
    tb[ty][tx] = (k0 + ty < n && col < n) ? A[(size_t)(k0 + ty) * n + col] : 0.0;
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kPurifyTile; ++k) acc = fma(ta[ty][k], tb[k][tx], acc);
    __syncthreads();
  }
  if (row < n && col < n) {
    C[(size_t)row * n + col] = acc;
    if (row == col) {
      atomicAdd(step + 0, A[(size_t)row * n + col]);
      atomicAdd(step + 1, acc);
    }
  }
}

__global__ void purify_update_kernel(double* __restrict__ A, const double* __restrict__ C, int n, int nocc,
                                     double tol, const double* __restrict__ step, double* __restrict__ next,
                                     double* __restrict__ err) {
  const bool frozen = step[2] != 0.0 || (step[0] - step[1]) < tol;
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e == 0) {
    next[2] = frozen ? 1.0 : 0.0;
    // error report: tr A - tr A^2 (= sum lambda (1 - lambda)) of the step that froze, else 1
    if (err != nullptr) *err = frozen ? (step[2] != 0.0 ? *err : step[0] - step[1]) : 1.0;
  }
  if (frozen || e >= (long long)n * n) return;
  A[e] = step[0] > (double)nocc ? C[e] : 2.0 * A[e] - C[e];
}

// The same purification as one cooperative launch: every block owns 16 x 16 output tiles
// (grid-stride), computes the Gershgorin bounds itself, and the blocks meet at a grid-wide
// barrier twice per step (after the squares and traces, after the update of their own tiles);
// once a step freezes, every block leaves the loop at the same step, so the frozen steps cost
// nothing.  Same arithmetic, step for step, as the kernels above.
__global__ void __launch_bounds__(kPurifyTile * kPurifyTile) purify_coop_kernel(
    const double* __restrict__ F, int n, int nocc, int max_steps, double tol, double* __restrict__ A,
    double* __restrict__ C, double* __restrict__ slots, double* __restrict__ err) {
  namespace cg = cooperative_groups;
  cg::grid_group grid = cg::this_grid();
  __shared__ double ta[kPurifyTile][kPurifyTile + 1], tb[kPurifyTile][kPurifyTile + 1];
  __shared__ double red[2][kPurifyTile * kPurifyTile];
  const int tx = threadIdx.x % kPurifyTile, ty = threadIdx.x / kPurifyTile;
  const int nt = (n + kPurifyTile - 1) / kPurifyTile;
  const int ntiles = nt * nt;
  // Gershgorin bounds of F, by every block for itself
  double lo = 1e300, hi = -1e300;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    double r = 0.0;
    for (int j = 0; j < n; ++j)
      if (j != i) r += fabs(F[(size_t)i * n + j]);
    lo = fmin(lo, F[(size_t)i * n + i] - r);
    hi = fmax(hi, F[(size_t)i * n + i] + r);
  }
  red[0][threadIdx.x] = lo;
  red[1][threadIdx.x] = hi;
  __syncthreads();
  for (int off = blockDim.x / 2; off > 0; off >>= 1) {
    if ((int)threadIdx.x < off) {
      red[0][threadIdx.x] = fmin(red[0][threadIdx.x], red[0][threadIdx.x + off]);
      red[1][threadIdx.x] = fmax(red[1][threadIdx.x], red[1][threadIdx.x + off]);
    }
    __syncthreads();
  }
  const double emin = red[0][0], emax = red[1][0];
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int row = (t / nt) * kPurifyTile + ty, col = (t % nt) * kPurifyTile + tx;
    if (row < n && col < n) A[(size_t)row * n + col] = ((row == col ? emax : 0.0) - F[(size_t)row * n + col]) / (emax - emin);
  }
  if (blockIdx.x == 0)
    for (int i = threadIdx.x; i < 3 * (max_steps + 1); i += blockDim.x) slots[i] = 0.0;
  grid.sync();
  for (int k = 0; k < max_steps; ++k) {
    double* step = slots + 3 * k;
    // the step's flags and traces are read from L2 (__ldcg), never from a block's L1, so that every
    // block takes the same decision after the barrier
    if (__ldcg(step + 2) != 0.0) break;  // frozen at an earlier step
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
      const int row = (t / nt) * kPurifyTile + ty, col = (t % nt) * kPurifyTile + tx;
      double acc = 0.0;
      for (int k0 = 0; k0 < n; k0 += kPurifyTile) {
        ta[ty][tx] = (row < n && k0 + tx < n) ? A[(size_t)row * n + k0 + tx] : 0.0;
        tb[ty][tx] = (k0 + ty < n && col < n) ? A[(size_t)(k0 + ty) * n + col] : 0.0;
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < kPurifyTile; ++kk) acc = fma(ta[ty][kk], tb[kk][tx], acc);
        __syncthreads();
      }
      if (row < n && col < n) {
        C[(size_t)row * n + col] = acc;
        if (row == col) {
          atomicAdd(step + 0, A[(size_t)row * n + col]);
          atomicAdd(step + 1, acc);
        }
      }
    }
    grid.sync();
    const double tr = __ldcg(step + 0), tr2 = __ldcg(step + 1);
    const bool frozen = (tr - tr2) < tol;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      step[5] = frozen ? 1.0 : 0.0;  // the next step's flag
      *err = frozen ? tr - tr2 : 1.0;
    }
    if (!frozen) {
      const bool up = tr > (double)nocc;
      for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int row = (t / nt) * kPurifyTile + ty, col = (t % nt) * kPurifyTile + tx;
        if (row < n && col < n) {
          const size_t e = (size_t)row * n + col;
          A[e] = up ? C[e] : 2.0 * A[e] - C[e];
        }
      }
    }
    grid.sync();
  }
}

// FP64 FMA throughput probe: 8 independent FMA chains per thread.
__global__ void fp64_peak_kernel(double* out, int iters, double a, double b) {
  double x[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) x[k] = threadIdx.x * 1e-3 + k;
  for (int i = 0; i < iters; ++i)
#pragma unroll
    for (int k = 0; k < 8; ++k) x[k] = fma(x[k], a, b);
  double s = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) s += x[k];
  if (s == 12345.678) out[0] = s;  // keeps the loop alive, never true in practice
}

}  // namespace

static int ensure_aux(hfgpu_handle* h) {
  if (h->aux[0]) return HFGPU_OK;
  for (int i = 0; i < hfgpu_handle::kAux; ++i) {
    HF_CUDA(h, cudaStreamCreateWithFlags(&h->aux[i], cudaStreamNonBlocking));
    HF_CUDA(h, cudaEventCreateWithFlags(&h->join_ev[i], cudaEventDisableTiming));
  }
  HF_CUDA(h, cudaEventCreateWithFlags(&h->fork_ev, cudaEventDisableTiming));
  return HFGPU_OK;
}

// Fork: every auxiliary stream waits for the work already queued on the handle's stream.
static int fork_streams(hfgpu_handle* h) {
  int rc = ensure_aux(h);
  if (rc) return rc;
  HF_CUDA(h, cudaEventRecord(h->fork_ev, h->stream));
  for (int i = 0; i < hfgpu_handle::kAux; ++i) HF_CUDA(h, cudaStreamWaitEvent(h->aux[i], h->fork_ev, 0));
  return HFGPU_OK;
}

// Join: the handle's stream waits for all auxiliary streams.
static int join_streams(hfgpu_handle* h) {
  for (int i = 0; i < hfgpu_handle::kAux; ++i) {
    HF_CUDA(h, cudaEventRecord(h->join_ev[i], h->aux[i]));
    HF_CUDA(h, cudaStreamWaitEvent(h->stream, h->join_ev[i], 0));
  }
  return HFGPU_OK;
}

// Largest classes first, each of the first kAux on its own stream, the rest
// round-robin: the few-quartet, long-latency d classes then overlap the
// many-quartet s/p classes instead of running alone on a handful of SMs.
static void class_schedule(int* order, int* stream_of) {
  for (int i = 0; i < hfgpu::kNumClasses; ++i) {
    order[i] = hfgpu::kNumClasses - 1 - i;
    stream_of[i] = i % hfgpu_handle::kAux;
  }
}

static int read_counters(hfgpu_handle* h, long long* computed, long long* skipped) {
  std::vector<unsigned long long> c(3 * hfgpu::kNumClasses);
  HF_CUDA(h, cudaMemcpy(c.data(), h->d_counters.p, sizeof(unsigned long long) * c.size(), cudaMemcpyDeviceToHost));
  long long a = 0, b = 0;
  for (int k = 0; k < hfgpu::kNumClasses; ++k) {
    a += (long long)c[3 * k];
    b += (long long)c[3 * k + 1];
  }
  if (computed) *computed = a;
  if (skipped) *skipped = b;
  return HFGPU_OK;
}

// Host-pointer entry points read the device status word back with their results (in stream
// order) and clear it; a staging wait that ran out fails the call.
static int enqueue_status_read(hfgpu_handle* h) {
  HF_CUDA(h, cudaMemcpyAsync(&h->status_host, h->d_status.p, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  HF_CUDA(h, cudaMemsetAsync(h->d_status.p, 0, sizeof(int), h->stream));
  return HFGPU_OK;
}
static int status_after_sync(hfgpu_handle* h) {
  const int st = h->status_host;
  h->status_host = 0;
  if (st == HFGPU_DEV_STAGE_TIMEOUT)
    return fail(h, HFGPU_ERR_CUDA, "a shared-memory staging wait ran out (bounded wait); the build is incomplete");
  if (st == HFGPU_DEV_ABORTED) return fail(h, HFGPU_ERR_STATE, "the build was stopped by hfgpu_request_abort");
  return st == 0 ? HFGPU_OK : fail(h, HFGPU_ERR_CUDA, "device status " + std::to_string(st));
}

// Device J/K: all pointers on the device.  Jout/Kout may be null to skip.
static int jk_device_impl(hfgpu_handle* h, const double* DJ, int nK, const double* DK, double* Jout, double* Kout,
                          int precision, bool delta = false) {
  if (!h->have_geometry) return fail(h, HFGPU_ERR_STATE, "no geometry set");
  if (nK < 0 || nK > 8) return fail(h, HFGPU_ERR_INVALID, "nK out of range");
  const int n = h->n, ns = h->nshell;
  const size_t nn = (size_t)h->mat_total;  // n*n, or the block storage of a batched handle
  if (h->batched && nK > 1) return fail(h, HFGPU_ERR_UNSUPPORTED, "batched handles build RHF J/K (one density)");
  HF_CUDA(h, h->d_half.ensure(sizeof(double) * nn * (1 + std::max(nK, 1))));
  HF_CUDA(h, h->d_counters.ensure(sizeof(unsigned long long) * 3 * hfgpu::kNumClasses));
  double* Jh = h->d_half.as<double>();
  double* Kh = Jh + nn;
  HF_CUDA(h, cudaMemsetAsync(Jh, 0, sizeof(double) * nn * (1 + nK), h->stream));
  HF_CUDA(h, cudaMemsetAsync(h->d_counters.p, 0, sizeof(unsigned long long) * 3 * hfgpu::kNumClasses, h->stream));
  int kernels = 0;
  // mixed-precision Delta-D builds screen at their own (looser) threshold; full builds never do
  const double dtol = delta && precision == HFGPU_MIXED ? h->opts.mixed_density_tol : h->opts.density_tol;
  const float* dmax = nullptr;
  if (dtol > 0.0 && !h->batched) {
    HF_CUDA(h, h->d_dmax.ensure(sizeof(float) * ns * ns));
    dmax_kernel<<<(ns * ns + 127) / 128, 128, 0, h->stream>>>(h->d_first.as<int>(), ns, n, DJ, nK, DK,
                                                              h->d_dmax.as<float>());
    HF_CHECK_LAUNCH(h, "dmax kernel");
    ++kernels;
    dmax = h->d_dmax.as<float>();
  }
  // Quartets whose Schwarz bound times 4 max|D| is below the threshold cannot survive the
  // per-quartet density test: with the lists ordered by bound decade, only a prefix of every
  // segment can.  The prefix lengths are computed on the device (launch_counts_kernel) and read
  // by the class kernels, so a density-screened build never waits for the host.
  const int nslot = hfgpu::kNumClasses * 4;
  if (dmax != nullptr) {
    static_assert(kBuckets == 18, "launch_counts_kernel's decade table");
    HF_CUDA(h, h->d_gmax.ensure(sizeof(unsigned int)));
    HF_CUDA(h, cudaMemsetAsync(h->d_gmax.p, 0, sizeof(unsigned int), h->stream));
    gmax_kernel<<<std::min((ns * ns + 255) / 256, 1024), 256, 0, h->stream>>>(h->d_dmax.as<float>(), ns * ns,
                                                                            h->d_gmax.as<unsigned int>());
    launch_counts_kernel<<<1, 128, 0, h->stream>>>(h->d_gmax.as<unsigned int>(), dtol, h->d_launch.as<long long>(),
                                                   nslot, kBuckets, h->d_dyn.as<int>());
    HF_CHECK_LAUNCH(h, "launch counts");
    kernels += 2;
  }
  QuartetArgs<double> qd{};
  qd.jk = jk_args_d(h);
  QuartetArgs<float> qf{};
  qf.jk = jk_args_f(h);
  for (JKArgs<double>* a : {&qd.jk}) {
    a->DJ = DJ; a->nK = nK; a->DK = DK; a->Jh = Jh; a->Kh = Kh; a->dmax = dmax; a->dtol = dtol;
    a->counters = h->d_counters.as<unsigned long long>();
  }
  qf.jk.DJ = DJ; qf.jk.nK = nK; qf.jk.DK = DK; qf.jk.Jh = Jh; qf.jk.Kh = Kh; qf.jk.dmax = dmax;
  qf.jk.dtol = dtol; qf.jk.counters = h->d_counters.as<unsigned long long>();
  if (h->batched) {
    const long long* mo = h->d_mol.as<long long>();
    const int* mn = reinterpret_cast<const int*>(mo + h->nmol);
    qd.jk.mol_off = qf.jk.mol_off = mo;
    qd.jk.mol_n = qf.jk.mol_n = mn;
  }
  qd.mode = qf.mode = QMODE_JK;
  qd.pure = qf.pure = h->pure;
  qd.boys_planes = h->d_boys_pd.as<double>();
  qf.boys_planes = h->d_boys_pf.as<float>();
  qd.status = qf.status = h->d_status.as<int>();
  qd.stage_test = qf.stage_test = h->opts.reserved[0] == 1 ? 1 : 0;
  qd.abort_flag = qf.abort_flag = h->d_abort.as<int>();
  qd.part = qf.part = h->part;
  qd.nparts = qf.nparts = h->nparts;
  const int2* q = h->d_quart.as<int2>();
  long long launched = 0;
  // largest classes first so that they overlap the tail of the smaller ones
  unsigned long long* cnt = h->d_counters.as<unsigned long long>();
  int rc0 = fork_streams(h);
  if (rc0) return rc0;
  int order[32], sidx[32];
  class_schedule(order, sidx);
  for (int i = 0; i < hfgpu::kNumClasses; ++i) {
    const int c = order[i];
    cudaStream_t st = h->aux[h->jk_serial ? 0 : sidx[i]];
    const hfgpu::ClassLaunchers* L = hfgpu::kClassLaunchers[c];
    const long long b = h->q_beg[c], m = h->q_mid[c], e = h->q_end[c];
    qd.jk.counters = cnt + 3 * c;
    qf.jk.counters = cnt + 3 * c;
    qd.block = qf.block = h->sched_block[c];
    qd.capped = qf.capped = h->sched_cap[c];
    qd.group = qf.group = h->sched_primwarp[c] == 1 ? 32 : h->sched_primwarp[c];
    qd.warp_max = qf.warp_max = class_warp_max(h, c);
    qd.warp_threads = qf.warp_threads = class_warp_threads(h, c);
    qd.staged = qf.staged = (h->sched_cap[c] == 2 && L->has_staged) ? 1 : 0;
    h->ev_used[c] = false;
    if (e <= b || !((h->class_mask >> c) & 1u)) continue;
    if (h->timing) HF_CUDA(h, cudaEventRecord(h->ev[2 * c], st));
    // Four parts in list order: [beg,hik1) many-primitive / [hik1,mid) few-primitive (high
    // bound, FP64), [mid,hik2) / [hik2,end) (low bound, FP32 in mixed mode).  Adjacent parts
    // that run the same kernel are launched together.  In a density-screened build each part
    // keeps the device-computed prefix of its bound decades: the launch gets the parts' offsets
    // and their slots of the device counts (consecutive, one per part).
    const long long pstart[5] = {b, h->q_hik1[c], m, h->q_hik2[c], e};
    struct Range { long long lo, hi; bool fp32, many; int part0, nseg; long long off[4]; };
    Range rg[4];
    int nr = 0;
    for (int part = 0; part < 4; ++part) {
      const long long lo = pstart[part], hi = pstart[part + 1];
      const bool fp32 = precision == HFGPU_MIXED && part >= 2;
      const bool many = (part % 2) == 0 && L->has_primwarp && h->sched_primwarp[c];
      if (nr > 0 && rg[nr - 1].hi == lo && rg[nr - 1].fp32 == fp32 && rg[nr - 1].many == many) {
        Range& r = rg[nr - 1];  // contiguous and the same kernel: extend
        r.off[r.nseg++] = lo - r.lo;
        r.hi = hi;
      } else {
        Range& r = rg[nr++];
        r = Range{lo, hi, fp32, many, part, 1, {0, 0, 0, 0}};
      }
    }
    for (int r = 0; r < nr; ++r) {
      const int nq_all = (int)(rg[r].hi - rg[r].lo);
      // the grid covers every quartet of the parts (this partition's share of them)
      const int nq_max = (int)((nq_all + h->nparts - 1) / h->nparts);
      if (nq_max <= 0 || (h->nparts > 1 && nq_all <= h->part)) continue;
      const int2* qs = q + rg[r].lo;
      const int* dyn = dmax != nullptr ? h->d_dyn.as<int>() + c * 4 + rg[r].part0 : nullptr;
      if (rg[r].fp32) {
        qf.dyn_nq = dyn;
        qf.nseg = rg[r].nseg;
        qf.full_nq = nq_all;
        for (int k = 0; k < 4; ++k) qf.seg_off[k] = (int)rg[r].off[k];
        if (!(rg[r].many && L->primwarp_f(qf, qs, nq_max, st))) L->quartet_f(qf, qs, nq_max, st);
      } else {
        qd.dyn_nq = dyn;
        qd.nseg = rg[r].nseg;
        qd.full_nq = nq_all;
        for (int k = 0; k < 4; ++k) qd.seg_off[k] = (int)rg[r].off[k];
        if (!(rg[r].many && L->primwarp_d(qd, qs, nq_max, st))) L->quartet_d(qd, qs, nq_max, st);
      }
      ++kernels;
    }
    HF_CHECK_LAUNCH(h, "quartet kernel");
    if (h->timing) {
      HF_CUDA(h, cudaEventRecord(h->ev[2 * c + 1], st));
      h->ev_used[c] = true;
    }
    launched += e - b;
  }
  if ((rc0 = join_streams(h))) return rc0;
  h->last_launched = launched;
  const int tot = (int)nn;
  h->last_kernels = kernels + ((Jout && DJ) ? 1 : 0) + ((Kout && nK > 0) ? 1 : 0);
  if (h->batched) {
    const long long* mo = h->d_mol.as<long long>();
    const int* mn = reinterpret_cast<const int*>(mo + h->nmol);
    const int nb = (int)((nn + 255) / 256);
    if (Jout && DJ) batch_symmetrise_kernel<<<nb, 256, 0, h->stream>>>(Jh, Jout, (long long)nn, mo, mn, h->nmol);
    if (Kout && nK > 0) batch_symmetrise_kernel<<<nb, 256, 0, h->stream>>>(Kh, Kout, (long long)nn, mo, mn, h->nmol);
    HF_CHECK_LAUNCH(h, "symmetrise blocks");
  } else {
    if (Jout && DJ) {
      symmetrise_kernel<<<(tot + 255) / 256, 256, 0, h->stream>>>(Jh, Jout, n, 1);
      HF_CHECK_LAUNCH(h, "symmetrise J");
    }
    if (Kout && nK > 0) {
      symmetrise_kernel<<<(tot * nK + 255) / 256, 256, 0, h->stream>>>(Kh, Kout, n, nK);
      HF_CHECK_LAUNCH(h, "symmetrise K");
    }
  }
  return HFGPU_OK;
}

// Gradient accumulation of grad_kernel: per block in shared memory when the natoms x 3
// totals fit in kGradSmemBytes, and then no more than kGradMaxBlocks blocks for the
// straight-line classes (their grid-stride loop takes the rest), so that the flush at the
// end of each block stays a small number of atomics.
constexpr int kGradSmemBytes = 24 * 1024;
constexpr int kGradMaxBlocks = 2048;
// blocks of a straight-line gradient launch: opts.reserved[1] when set (> 0), else kGradMaxBlocks
static int grad_max_blocks(const hfgpu_handle* h) {
  return h->opts.reserved[1] > 0 ? h->opts.reserved[1] : kGradMaxBlocks;
}
int grad_smem_atoms(const hfgpu_handle* h) {
  return (size_t)h->natoms * 3 * sizeof(double) <= (size_t)kGradSmemBytes ? h->natoms : 0;
}

// Gradient forms of the op-table classes: 0 one thread per quartet (global scratch), 1 one warp
// per quartet, 2 one warp per quartet in four one-set launches, 3 one block of 128 threads per
// quartet, 4 the same in four one-set launches, 5 and 6 the same with 256 threads.
constexpr int kGradForms = 7;
static int grad_form_threads(int form) { return form >= 5 ? 256 : (form >= 3 ? 128 : 32); }
static bool grad_form_split(int form) { return form == 2 || form == 4 || form == 6; }

// Form of a gradient launch of class c: the one hfgpu_autotune_grad or hfgpu_set_grad_forms
// chose, else the block form (3), which was the fastest single form on every workload measured
// (octane, anthracene, the water octamer), when the class has shared-memory tables that fit one
// block; opts.grad_warp_max_waves <= 0 asks for the thread form instead.
static int grad_form_of(const hfgpu_handle* h, int c, bool fp32) {
  const hfgpu::ClassLaunchers* L = hfgpu::kClassLaunchers[c];
  if (!L->has_grad_warp) return 0;
  const int bytes = L->grad_warp_bytes(fp32 ? 1 : 0);
  if (bytes <= 0 || bytes > 232448) return 0;
  if (h->grad_form[c] >= 0) return h->grad_form[c];
  return h->opts.grad_warp_max_waves > 0 ? 3 : 0;
}

static bool grad_use_warp(const hfgpu_handle* h, int c, bool fp32) { return grad_form_of(h, c, fp32) >= 1; }

// Quartets of a list range of n that this handle's partition processes (every nparts-th,
// starting at number part).
static long long part_share(const hfgpu_handle* h, long long n) {
  if (h->nparts <= 1) return n;
  return n > h->part ? (n - h->part + h->nparts - 1) / h->nparts : 0;
}

static int grad_device_impl(hfgpu_handle* h, const double* DJ, double cJ, int nK, const double* DK, double cK,
                            double* grad, int precision) {
  if (!h->have_geometry) return fail(h, HFGPU_ERR_STATE, "no geometry set");
  GradArgs<double> gd{};
  gd.pairs = h->d_pairs.as<PairInfo>();
  gd.prims = h->d_prim_d.as<PrimPair<double>>();
  const size_t np = std::max<size_t>(h->nprimpairs, 1);
  gd.alpha_a = h->d_alpha_d.as<double>();
  gd.alpha_b = h->d_alpha_d.as<double>() + np;
  gd.boys.tab = h->d_boys_d.as<double>();
  gd.n = h->n;
  gd.DJ = DJ; gd.cJ = cJ; gd.nK = nK; gd.DK = DK; gd.cK = cK; gd.grad = grad;
  if (h->batched) {
    if (nK > 1) return fail(h, HFGPU_ERR_UNSUPPORTED, "batched handles take one density");
    gd.mol_off = h->d_mol.as<long long>();
    gd.mol_n = reinterpret_cast<const int*>(gd.mol_off + h->nmol);
  }
  GradArgs<float> gf{};
  gf.pairs = gd.pairs;
  gf.prims = h->d_prim_f.as<PrimPair<float>>();
  gf.alpha_a = h->d_alpha_f.as<float>();
  gf.alpha_b = h->d_alpha_f.as<float>() + np;
  gf.boys.tab = h->d_boys_f.as<float>();
  gf.n = h->n;
  gf.DJ = DJ; gf.cJ = cJ; gf.nK = nK; gf.DK = DK; gf.cK = cK; gf.grad = grad;
  gf.mol_off = gd.mol_off;
  gf.mol_n = gd.mol_n;
  gd.smem_atoms = gf.smem_atoms = grad_smem_atoms(h);
  gd.part = gf.part = h->part;
  gd.nparts = gf.nparts = h->nparts;
  const int2* q = h->d_quart.as<int2>();
  const size_t budget = (size_t)1 << 30;  // scratch bytes per table-mode class and precision
  // threads of a table-mode launch: as many as the budget allows (at least 4736),
  // at most one per quartet, a whole number of 128-thread blocks
  auto table_threads = [&](int slots, long long nq) -> long long {
    long long thr = std::max<long long>((long long)(budget / ((size_t)slots * sizeof(double))), 4736);
    thr = std::min<long long>(thr, ((nq + 127) / 128) * 128);
    return ((thr + 127) / 128) * 128;
  };
  // Every table-mode class gets its own slice of the scratch buffer, so the classes run
  // concurrently on the auxiliary streams like the straight-line ones.
  // In mixed mode the FP32 part of a class gets a second slice and its own stream, so the two
  // parts of a class run concurrently too.
  size_t slice_off[32] = {0}, slice_off_f[32] = {0};
  size_t need_total = 0;
  for (int c = 0; c < hfgpu::kNumClasses; ++c) {
    const int slots = hfgpu::kClassLaunchers[c]->grad_scratch_slots(h->pure);
    const long long nq = h->q_end[c] - h->q_beg[c];
    slice_off[c] = slice_off_f[c] = need_total;
    if (slots <= 0 || nq <= 0) continue;
    if (grad_use_warp(h, c, false) && grad_use_warp(h, c, true)) continue;  // warp/block form: no scratch
    const size_t one = (size_t)slots * sizeof(double) * (size_t)table_threads(slots, nq);
    need_total += (one + 255) / 256 * 256;
    if (precision == HFGPU_MIXED) {
      slice_off_f[c] = need_total;
      need_total += (one + 255) / 256 * 256;
    }
  }
  if (need_total) HF_CUDA(h, h->d_scratch.ensure(need_total));
  int rc = fork_streams(h);
  if (rc) return rc;
  int rr = 1;
  for (int c = hfgpu::kNumClasses - 1; c >= 0; --c) {
    const hfgpu::ClassLaunchers* L = hfgpu::kClassLaunchers[c];
    const long long b = h->q_beg[c], m = h->q_mid[c], e = h->q_end[c];
    if (e <= b || !((h->grad_class_mask >> c) & 1u)) continue;
    const int slots = L->grad_scratch_slots(h->pure);
    cudaStream_t st_d = h->aux[h->grad_serial ? 0 : rr++ % hfgpu_handle::kAux];
    cudaStream_t st_f = precision == HFGPU_MIXED ? h->aux[h->grad_serial ? 0 : rr++ % hfgpu_handle::kAux] : st_d;
    auto run = [&](bool fp32, long long lo, long long hi) -> int {
      const int nq = (int)part_share(h, hi - lo);
      if (nq <= 0) return HFGPU_OK;
      const int form = grad_form_of(h, c, fp32);
      gd.warp_split = gf.warp_split = grad_form_split(form) ? 1 : 0;
      gd.warp_threads = gf.warp_threads = grad_form_threads(form);
      if (form >= 1) {
        const bool done = fp32 ? L->grad_warp_f(gf, h->pure, q + lo, nq, fp32 ? st_f : st_d)
                               : L->grad_warp_d(gd, h->pure, q + lo, nq, st_d);
        if (done) {
          HF_CHECK_LAUNCH(h, "grad warp kernel");
          return HFGPU_OK;
        }
      }
      const size_t off = fp32 ? slice_off_f[c] : slice_off[c];
      unsigned char* slice = h->d_scratch.as<unsigned char>() + off;
      cudaStream_t st = fp32 ? st_f : st_d;
      int grid = (nq + 127) / 128;
      if (slots == 0 && gd.smem_atoms > 0) grid = std::min(grid, grad_max_blocks(h));
      if (slots > 0) {
        const size_t rb = fp32 ? sizeof(float) : sizeof(double);
        grid = (int)(table_threads(slots, nq) / 128);
        if (off + (size_t)slots * rb * (size_t)grid * 128 > h->d_scratch.bytes)
          return fail(h, HFGPU_ERR_NOMEM, "gradient scratch too small");
      }
      if (fp32) {
        gf.scratch = reinterpret_cast<float*>(slice);
        gf.scratch_threads = grid * 128;
        L->grad_f(gf, h->pure, q + lo, nq, grid, st);
      } else {
        gd.scratch = reinterpret_cast<double*>(slice);
        gd.scratch_threads = grid * 128;
        L->grad_d(gd, h->pure, q + lo, nq, grid, st);
      }
      HF_CHECK_LAUNCH(h, "grad kernel");
      return HFGPU_OK;
    };
    if (precision == HFGPU_MIXED) {
      if ((rc = run(false, b, m))) return rc;
      if ((rc = run(true, m, e))) return rc;
    } else if ((rc = run(false, b, e))) {
      return rc;
    }
  }
  return join_streams(h);
}

// Gradient with caller-provided scratch of fixed capacity, on the handle's stream
// only.  Allocates nothing: table-mode classes get as many threads as the scratch
// holds (whole 128-thread blocks); a class that cannot fit one block is rejected.
int hfgpu_grad_fixed_scratch(hfgpu_handle* h, const double* DJ, double cJ, int nK, const double* DK, double cK,
                             double* grad, int precision, void* scratch, size_t scratch_bytes) {
  if (!h || !grad || !scratch) return HFGPU_ERR_INVALID;
  if (!h->have_geometry) return fail(h, HFGPU_ERR_STATE, "no geometry set");
  DeviceGuard dev_guard(h);
  int rc = dev_guard.rc;
  if (rc) return rc;
  GradArgs<double> gd{};
  gd.pairs = h->d_pairs.as<PairInfo>();
  gd.prims = h->d_prim_d.as<PrimPair<double>>();
  const size_t np = std::max<size_t>(h->nprimpairs, 1);
  gd.alpha_a = h->d_alpha_d.as<double>();
  gd.alpha_b = h->d_alpha_d.as<double>() + np;
  gd.boys.tab = h->d_boys_d.as<double>();
  gd.n = h->n;
  gd.DJ = DJ; gd.cJ = cJ; gd.nK = nK; gd.DK = DK; gd.cK = cK; gd.grad = grad;
  gd.scratch = static_cast<double*>(scratch);
  if (h->batched) {
    if (nK > 1) return fail(h, HFGPU_ERR_UNSUPPORTED, "batched handles take one density");
    gd.mol_off = h->d_mol.as<long long>();
    gd.mol_n = reinterpret_cast<const int*>(gd.mol_off + h->nmol);
  }
  GradArgs<float> gf{};
  gf.pairs = gd.pairs;
  gf.prims = h->d_prim_f.as<PrimPair<float>>();
  gf.alpha_a = h->d_alpha_f.as<float>();
  gf.alpha_b = h->d_alpha_f.as<float>() + np;
  gf.boys.tab = h->d_boys_f.as<float>();
  gf.n = h->n;
  gf.DJ = DJ; gf.cJ = cJ; gf.nK = nK; gf.DK = DK; gf.cK = cK; gf.grad = grad;
  gf.scratch = static_cast<float*>(scratch);
  gf.mol_off = gd.mol_off;
  gf.mol_n = gd.mol_n;
  gd.smem_atoms = gf.smem_atoms = grad_smem_atoms(h);
  gd.part = gf.part = h->part;
  gd.nparts = gf.nparts = h->nparts;
  const int2* q = h->d_quart.as<int2>();
  // quartet range of part 0 / 1 of class c (FP64 and, in mixed mode, the FP32 low-bound part)
  auto part_range = [&](int c, int part, long long& lo, long long& hi) {
    const long long b = h->q_beg[c], m = h->q_mid[c], e = h->q_end[c];
    lo = (precision == HFGPU_MIXED) ? (part == 0 ? b : m) : (part == 0 ? b : e);
    hi = (precision == HFGPU_MIXED) ? (part == 0 ? m : e) : e;
  };
  // First pass: every table-mode launch must fit one 128-thread block into the scratch.
  // Checked before anything is enqueued, so that a rejected call leaves grad untouched.
  for (int c = hfgpu::kNumClasses - 1; c >= 0; --c) {
    const int slots = hfgpu::kClassLaunchers[c]->grad_scratch_slots(h->pure);
    if (slots <= 0) continue;
    for (int part = 0; part < 2; ++part) {
      long long lo, hi;
      part_range(c, part, lo, hi);
      if (hi <= lo) continue;
      const bool fp32 = precision == HFGPU_MIXED && part == 1;
      const size_t per_thread = (size_t)slots * (fp32 ? sizeof(float) : sizeof(double));
      if (scratch_bytes / per_thread < 128)
        return fail(h, HFGPU_ERR_INVALID,
                    "gradient class needs " + std::to_string(per_thread * 128) +
                        " bytes of scratch for one 128-thread block, more than the fixed scratch of " +
                        std::to_string(scratch_bytes) + " bytes");
    }
  }
  for (int c = hfgpu::kNumClasses - 1; c >= 0; --c) {
    const hfgpu::ClassLaunchers* L = hfgpu::kClassLaunchers[c];
    if (h->q_end[c] <= h->q_beg[c]) continue;
    const int slots = L->grad_scratch_slots(h->pure);
    for (int part = 0; part < 2; ++part) {
      const bool fp32 = precision == HFGPU_MIXED && part == 1;
      long long lo, hi;
      part_range(c, part, lo, hi);
      const int nq = (int)part_share(h, hi - lo);
      if (nq <= 0) continue;
      int grid = (nq + 127) / 128;
      if (slots == 0 && gd.smem_atoms > 0) grid = std::min(grid, grad_max_blocks(h));
      if (slots > 0) {
        const size_t per_thread = (size_t)slots * (fp32 ? sizeof(float) : sizeof(double));
        const long long fit = (long long)(scratch_bytes / per_thread) / 128 * 128;  // >= 128 (first pass)
        grid = (int)(std::min<long long>(fit, (long long)grid * 128) / 128);
      }
      if (fp32) {
        gf.scratch_threads = grid * 128;
        L->grad_f(gf, h->pure, q + lo, nq, grid, h->stream);
      } else {
        gd.scratch_threads = grid * 128;
        L->grad_d(gd, h->pure, q + lo, nq, grid, h->stream);
      }
      HF_CHECK_LAUNCH(h, "grad kernel (fixed scratch)");
    }
  }
  return HFGPU_OK;
}

int hfgpu_device_of(const hfgpu_handle* h) { return h ? h->device : -1; }

// Records a CUDA failure on the handle (status and hfgpu_last_error message) and clears the
// runtime's sticky last error, so that a later launch check on any handle does not report it.
int hfgpu_cuda_error(hfgpu_handle* h, int cuda_code, const char* where) {
  (void)cudaGetLastError();
  return cuda_fail(h, static_cast<cudaError_t>(cuda_code), where);
}

extern "C" {

int hfgpu_default_opts(hfgpu_opts* o) {
  if (!o) return HFGPU_ERR_INVALID;
  std::memset(o, 0, sizeof(*o));
  o->schwarz_tol = 1e-12;
  o->density_tol = 1e-12;
  o->mixed_fp32_bound = 1e-4;
  o->mixed_density_tol = 1e-12;
  o->device = 0;
  o->warp_max_quartets = 1 << 30;
  o->grad_warp_max_waves = 48;
  return HFGPU_OK;
}

const char* hfgpu_last_error(const hfgpu_handle* h) { return h ? h->err.c_str() : "null handle"; }

int hfgpu_nbf(const hfgpu_handle* h, int* nbf) {
  if (!h || !nbf) return HFGPU_ERR_INVALID;
  *nbf = h->n;
  return HFGPU_OK;
}

int hfgpu_create(const hfgpu_basis* b, const hfgpu_opts* opts, hfgpu_handle** out) {
  if (!b || !out || b->nshell <= 0 || b->natoms <= 0 || !b->L || !b->shell_atom || !b->nprim || !b->exps || !b->coefs)
    return HFGPU_ERR_INVALID;
  *out = nullptr;
  hfgpu_handle* h = new (std::nothrow) hfgpu_handle();
  if (!h) return HFGPU_ERR_NOMEM;
  if (opts)
    h->opts = *opts;
  else
    hfgpu_default_opts(&h->opts);
  h->device = h->opts.device;
  h->nshell = b->nshell;
  h->natoms = b->natoms;
  h->pure = b->pure ? 1 : 0;
  h->L.assign(b->L, b->L + b->nshell);
  h->shell_atom.assign(b->shell_atom, b->shell_atom + b->nshell);
  h->nprim.assign(b->nprim, b->nprim + b->nshell);
  h->prim_off.resize(b->nshell + 1);
  h->first.resize(b->nshell + 1);
  h->prim_off[0] = 0;
  h->first[0] = 0;
  for (int s = 0; s < b->nshell; ++s) {
    if (h->L[s] < 0 || h->L[s] > 2 || h->nprim[s] < 1 || h->shell_atom[s] < 0 || h->shell_atom[s] >= b->natoms) {
      delete h;
      return HFGPU_ERR_INVALID;
    }
    h->prim_off[s + 1] = h->prim_off[s] + h->nprim[s];
    h->first[s + 1] = h->first[s] + (h->pure ? 2 * h->L[s] + 1 : (h->L[s] + 1) * (h->L[s] + 2) / 2);
  }
  const int nprim_tot = h->prim_off[b->nshell];
  h->exps.assign(b->exps, b->exps + nprim_tot);
  h->coefs.resize(nprim_tot);
  for (int p = 0; p < nprim_tot; ++p)
    if (!std::isfinite(b->exps[p]) || !(b->exps[p] > 0.0) || !std::isfinite(b->coefs[p])) {
      delete h;
      return HFGPU_ERR_INVALID;
    }
  for (int s = 0; s < b->nshell; ++s)
    normalise(h->L[s], h->nprim[s], &b->exps[h->prim_off[s]], &b->coefs[h->prim_off[s]], &h->coefs[h->prim_off[s]]);
  h->n = h->first[b->nshell];
  h->nmol = 1;
  h->mol_shell = {0, b->nshell};
  h->mol_n = {h->n};
  h->mol_off = {0};
  h->mol_atom = {0, b->natoms};
  h->mat_total = (long long)h->n * h->n;
  DeviceGuard dev_guard(h);
  int rc = dev_guard.rc;
  if (rc) {
    delete h;
    return rc;
  }
  if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete h;
    return HFGPU_ERR_CUDA;
  }
  h->own_stream = true;
  // the tables are constants: computed once per process (the long-double series take milliseconds),
  // uploaded per handle
  static const std::vector<double> bt = boys_table<double>(7);
  static const std::vector<float> btf = boys_table<float>(4);
  static const std::vector<double> bpd = boys_planes(bt);
  static const std::vector<float> bpf = boys_planes(btf);
  if (h->d_boys_d.ensure(sizeof(double) * bt.size()) || h->d_boys_f.ensure(sizeof(float) * btf.size()) ||
      h->d_boys_pd.ensure(sizeof(double) * bpd.size()) || h->d_boys_pf.ensure(sizeof(float) * bpf.size()) ||
      h->d_status.ensure(sizeof(int)) || h->d_abort.ensure(sizeof(int)) ||
      cudaMemset(h->d_abort.p, 0, sizeof(int)) ||
      cudaMemcpy(h->d_boys_d.p, bt.data(), sizeof(double) * bt.size(), cudaMemcpyHostToDevice) ||
      cudaMemcpy(h->d_boys_f.p, btf.data(), sizeof(float) * btf.size(), cudaMemcpyHostToDevice) ||
      cudaMemcpy(h->d_boys_pd.p, bpd.data(), sizeof(double) * bpd.size(), cudaMemcpyHostToDevice) ||
      cudaMemcpy(h->d_boys_pf.p, bpf.data(), sizeof(float) * bpf.size(), cudaMemcpyHostToDevice) ||
      cudaMemset(h->d_status.p, 0, sizeof(int))) {
    hfgpu_destroy(h);
    return HFGPU_ERR_CUDA;
  }
  *out = h;
  return HFGPU_OK;
}

int hfgpu_destroy(hfgpu_handle* h) {
  if (!h) return HFGPU_OK;
  {
    DeviceGuard dev_guard(h);
    if (h->stream) cudaStreamSynchronize(h->stream);
  for (DevBuf* d : {&h->d_onee, &h->d_pairs, &h->d_prim_d, &h->d_prim_f, &h->d_alpha_d, &h->d_alpha_f, &h->d_boys_d, &h->d_boys_f,
                    &h->d_quart, &h->d_mats, &h->d_half, &h->d_dmax, &h->d_counters, &h->d_grad, &h->d_scratch,
                    &h->d_eri, &h->d_eriq, &h->d_launch, &h->d_dyn, &h->d_first, &h->d_boys_pd,
                    &h->d_boys_pf, &h->d_status, &h->d_abort, &h->d_purify})
    d->release();
  h->d_mol.release();
  if (h->ev[0])
    for (auto& e : h->ev) cudaEventDestroy(e);
  for (int i = 0; i < hfgpu_handle::kAux; ++i) {
    if (h->aux[i]) cudaStreamDestroy(h->aux[i]);
    if (h->join_ev[i]) cudaEventDestroy(h->join_ev[i]);
  }
  if (h->fork_ev) cudaEventDestroy(h->fork_ev);
  if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
  if (h->ctl_stream) cudaStreamDestroy(h->ctl_stream);
  }  // the caller's current device is restored here, before the handle goes
  delete h;
  return HFGPU_OK;
}

int hfgpu_set_stream(hfgpu_handle* h, void* stream) {
  if (!h) return HFGPU_ERR_INVALID;
  if (h->own_stream && h->stream) {
    cudaStreamSynchronize(h->stream);
    cudaStreamDestroy(h->stream);
  }
  h->own_stream = false;
  h->stream = static_cast<cudaStream_t>(stream);
  if (!stream) {
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) return HFGPU_ERR_CUDA;
    h->own_stream = true;
  }
  return HFGPU_OK;
}

int hfgpu_set_geometry(hfgpu_handle* h, const double* xyz, int natoms) {
  if (!h || !xyz || natoms != h->natoms) return fail(h, HFGPU_ERR_INVALID, "bad geometry arguments");
  for (int i = 0; i < 3 * natoms; ++i)
    if (!std::isfinite(xyz[i])) return fail(h, HFGPU_ERR_INVALID, "non-finite coordinate");
  DeviceGuard dev_guard(h);
  int rc = dev_guard.rc;
  if (rc) return rc;
  h->xyz.assign(xyz, xyz + 3 * natoms);
  h->have_geometry = false;
  using clk = std::chrono::steady_clock;
  const auto t0 = clk::now();
  if ((rc = build_pairs(h))) return rc;
  const auto t1 = clk::now();
  if ((rc = compute_schwarz(h))) return rc;
  const auto t2 = clk::now();
  if ((rc = build_quartets(h))) return rc;  // sets setup_ms[2] and [3]
  h->setup_ms[0] = std::chrono::duration<double, std::milli>(t1 - t0).count();
  h->setup_ms[1] = std::chrono::duration<double, std::milli>(t2 - t1).count();
  h->have_geometry = true;
  return HFGPU_OK;
}

int hfgpu_schwarz(hfgpu_handle* h, double* Q) {
  if (!h || !Q) return HFGPU_ERR_INVALID;
  if (!h->have_geometry) return fail(h, HFGPU_ERR_STATE, "no geometry set");
  const int ns = h->nshell;
  for (const PairInfo& P : h->pairs) {
    Q[P.sa * ns + P.sb] = P.schwarz;
    Q[P.sb * ns + P.sa] = P.schwarz;
  }
  return HFGPU_OK;
}

int hfgpu_eri_packed(hfgpu_handle* h, double* eri_out, long long eri_len) {
  if (!h || !eri_out) return HFGPU_ERR_INVALID;
  if (!h->have_geometry) return fail(h, HFGPU_ERR_STATE, "no geometry set");
  const long long n = h->n, len = n * (n + 1) * (n * n + n + 2) / 8;
  if (eri_len != len) return fail(h, HFGPU_ERR_INVALID, "eri_len must be n(n+1)(n^2+n+2)/8");
  DeviceGuard dev_guard(h);
  int rc = dev_guard.rc;
  if (rc) return rc;
  HF_CUDA(h, h->d_eri.ensure(sizeof(double) * len));
  HF_CUDA(h, cudaMemsetAsync(h->d_eri.p, 0, sizeof(double) * len, h->stream));
  QuartetArgs<double> qa{};
  qa.jk = jk_args_d(h);
  qa.mode = QMODE_PACKED;
  qa.pure = h->pure;
  qa.eri = h->d_eri.as<double>();
  for (int cp = 0; cp < kPairClasses; ++cp)
    for (int cq = 0; cq <= cp; ++cq) {
      std::vector<int2> list;
      for (int P = h->class_begin[cp]; P < h->class_begin[cp + 1]; ++P)
        for (int Q = (cp == cq) ? P : h->class_begin[cq]; Q < h->class_begin[cq + 1]; ++Q)
          list.push_back(make_int2(P, Q));
      if (list.empty()) continue;
      HF_CUDA(h, h->d_eriq.ensure(sizeof(int2) * list.size()));
      HF_CUDA(h, cudaMemcpyAsync(h->d_eriq.p, list.data(), sizeof(int2) * list.size(), cudaMemcpyHostToDevice, h->stream));
      qa.warp_max = class_warp_max(h, quartet_class(cp, cq));
      qa.warp_threads = class_warp_threads(h, quartet_class(cp, cq));
      qa.block = h->sched_block[quartet_class(cp, cq)];
      qa.capped = h->sched_cap[quartet_class(cp, cq)];
      hfgpu::kClassLaunchers[quartet_class(cp, cq)]->quartet_d(qa, h->d_eriq.as<int2>(), (int)list.size(), h->stream);
      HF_CHECK_LAUNCH(h, "packed eri kernel");
      HF_CUDA(h, cudaStreamSynchronize(h->stream));
    }
  HF_CUDA(h, cudaMemcpyAsync(eri_out, h->d_eri.p, sizeof(double) * len, cudaMemcpyDeviceToHost, h->stream));
  HF_CUDA(h, cudaStreamSynchronize(h->stream));
  return HFGPU_OK;
}

int hfgpu_jk_device(hfgpu_handle* h, const double* DJ, int nK, const double* DK, double* J, double* K, int precision) {
  if (!h) return HFGPU_ERR_INVALID;
  DeviceGuard dev_guard(h);
  int rc = dev_guard.rc;
  if (rc) return rc;
  return jk_device_impl(h, DJ, nK, DK, J, K, precision);
}

int hfgpu_jk(hfgpu_handle* h, const double* DJ, int nK, const double* DK, double* J, double* K, int precision) {
  if (!h || (nK > 0 && (!DK || !K)) || (DJ && !J)) return HFGPU_ERR_INVALID;
  DeviceGuard dev_guard(h);
  int rc = dev_guard.rc;
  if (rc) return rc;
  const size_t nn = (size_t)h->n * h->n;
  // device layout: [DJ | DK (nK) | J | K (nK)]
  HF_CUDA(h, h->d_mats.ensure(sizeof(double) * nn * (2 + 2 * nK)));
  double* dDJ = h->d_mats.as<double>();
  double* dDK = dDJ + nn;
  double* dJ = dDK + nn * nK;
  double* dK = dJ + nn;
  if (DJ) HF_CUDA(h, cudaMemcpyAsync(dDJ, DJ, sizeof(double) * nn, cudaMemcpyHostToDevice, h->stream));
  if (nK) HF_CUDA(h, cudaMemcpyAsync(dDK, DK, sizeof(double) * nn * nK, cudaMemcpyHostToDevice, h->stream));
  if ((rc = jk_device_impl(h, DJ ? dDJ : nullptr, nK, dDK, dJ, dK, precision))) return rc;
  if (DJ) HF_CUDA(h, cudaMemcpyAsync(J, dJ, sizeof(double) * nn, cudaMemcpyDeviceToHost, h->stream));
  if (nK) HF_CUDA(h, cudaMemcpyAsync(K, dK, sizeof(double) * nn * nK, cudaMemcpyDeviceToHost, h->stream));
  if ((rc = enqueue_status_read(h))) return rc;
  HF_CUDA(h, cudaStreamSynchronize(h->stream));
  if ((rc = status_after_sync(h))) return rc;
  long long sk = 0;
  if ((rc = read_counters(h, nullptr, &sk))) return rc;
  h->last_skipped = sk;
  return HFGPU_OK;
}

int hfgpu_last_counts(const hfgpu_handle* h, long long* launched, long long* skipped) {
  if (!h) return HFGPU_ERR_INVALID;
  if (launched) *launched = h->last_launched;
  if (skipped) *skipped = h->last_skipped;
  return HFGPU_OK;
}

int hfgpu_fock_rhf(hfgpu_handle* h, const double* D, const double* H, double* F, int precision) {
  if (!h || !D || !H || !F) return HFGPU_ERR_INVALID;
  if (h->nparts > 1) return fail(h, HFGPU_ERR_STATE, "a partitioned handle builds partial J/K only: the Fock entry points add H and are refused");
  DeviceGuard dev_guard(h);
  int rc = dev_guard.rc;
  if (rc) return rc;
  const size_t nn = (size_t)h->n * h->n;
  // device layout: [D | H | J | K]; only D and H go up, only F comes back
  HF_CUDA(h, h->d_mats.ensure(sizeof(double) * nn * 4));
  double* dD = h->d_mats.as<double>();
  double* dH = dD + nn;
  double* dJ = dH + nn;
  double* dK = dJ + nn;
  HF_CUDA(h, cudaMemcpyAsync(dD, D, sizeof(double) * nn, cudaMemcpyHostToDevice, h->stream));
  HF_CUDA(h, cudaMemcpyAsync(dH, H, sizeof(double) * nn, cudaMemcpyHostToDevice, h->stream));
  if ((rc = jk_device_impl(h, dD, 1, dD, dJ, dK, precision))) return rc;
  fock_combine_kernel<<<(int)((nn + 255) / 256), 256, 0, h->stream>>>(dJ, dH, dJ, dK, (int)nn);
  HF_CHECK_LAUNCH(h, "fock combine");
  ++h->last_kernels;
  HF_CUDA(h, cudaMemcpyAsync(F, dJ, sizeof(double) * nn, cudaMemcpyDeviceToHost, h->stream));
  if ((rc = enqueue_status_read(h))) return rc;
  HF_CUDA(h, cudaStreamSynchronize(h->stream));
  return status_after_sync(h);
}

int hfgpu_fock_uhf(hfgpu_handle* h, const double* Da, const double* Db, const double* H, double* Fa, double* Fb,
                   int precision) {
  if (!h || !Da || !Db || !H || !Fa || !Fb) return HFGPU_ERR_INVALID;
  if (h->nparts > 1) return fail(h, HFGPU_ERR_STATE, "a partitioned handle builds partial J/K only: the Fock entry points add H and are refused");
  const size_t nn = (size_t)h->n * h->n;
  std::vector<double> Dt(nn), DK(2 * nn), J(nn), K(2 * nn);
  for (size_t i = 0; i < nn; ++i) {
    Dt[i] = Da[i] + Db[i];
    DK[i] = Da[i];
    DK[nn + i] = Db[i];
  }
  int rc = hfgpu_jk(h, Dt.data(), 2, DK.data(), J.data(), K.data(), precision);
  if (rc) return rc;
  for (size_t i = 0; i < nn; ++i) {
    Fa[i] = H[i] + J[i] - K[i];
    Fb[i] = H[i] + J[i] - K[nn + i];
  }
  return HFGPU_OK;
}

int hfgpu_fock_delta(hfgpu_handle* h, const double* dD, double* F, int precision) {
  if (!h || !dD || !F) return HFGPU_ERR_INVALID;
  if (h->nparts > 1) return fail(h, HFGPU_ERR_STATE, "a partitioned handle builds partial J/K only: the Fock entry points add H and are refused");
  DeviceGuard dev_guard(h);
  int rc = dev_guard.rc;
  if (rc) return rc;
  const size_t nn = (size_t)h->n * h->n;
  // same device layout as hfgpu_fock_rhf, with F_in in place of H
  HF_CUDA(h, h->d_mats.ensure(sizeof(double) * nn * 4));
  double* ddD = h->d_mats.as<double>();
  double* dF = ddD + nn;
  double* dJ = dF + nn;
  double* dK = dJ + nn;
  HF_CUDA(h, cudaMemcpyAsync(ddD, dD, sizeof(double) * nn, cudaMemcpyHostToDevice, h->stream));
  HF_CUDA(h, cudaMemcpyAsync(dF, F, sizeof(double) * nn, cudaMemcpyHostToDevice, h->stream));
  if ((rc = jk_device_impl(h, ddD, 1, ddD, dJ, dK, precision, true))) return rc;
  fock_combine_kernel<<<(int)((nn + 255) / 256), 256, 0, h->stream>>>(dJ, dF, dJ, dK, (int)nn);
  HF_CHECK_LAUNCH(h, "fock combine");
  ++h->last_kernels;
  HF_CUDA(h, cudaMemcpyAsync(F, dJ, sizeof(double) * nn, cudaMemcpyDeviceToHost, h->stream));
  if ((rc = enqueue_status_read(h))) return rc;
  HF_CUDA(h, cudaStreamSynchronize(h->stream));
  return status_after_sync(h);
}

int hfgpu_energy_forward(hfgpu_handle* h, const double* D, double* E2, int precision) {
  if (!h || !D || !E2) return HFGPU_ERR_INVALID;
  const size_t nn = (size_t)h->n * h->n;
  std::vector<double> J(nn), K(nn);
  int rc = hfgpu_jk(h, D, 1, D, J.data(), K.data(), precision);
  if (rc) return rc;
  double e = 0.0;
  for (size_t i = 0; i < nn; ++i) e += D[i] * (2.0 * J[i] - K[i]);
  *E2 = e;
  return std::isfinite(e) ? HFGPU_OK : fail(h, HFGPU_ERR_NONFINITE, "non-finite energy");
}

int hfgpu_grad2e_device(hfgpu_handle* h, const double* DJ, double cJ, int nK, const double* DK, double cK,
                        double* grad, int precision) {
  if (!h || !grad) return HFGPU_ERR_INVALID;
  DeviceGuard dev_guard(h);
  int rc = dev_guard.rc;
  if (rc) return rc;
  return grad_device_impl(h, DJ, cJ, nK, DK, cK, grad, precision);
}

static int grad_host(hfgpu_handle* h, const double* DJ, double cJ, int nK, const double* const* DKs, double cK,
                     double scale, double* dE_dR, int precision) {
  DeviceGuard dev_guard(h);
  int rc = dev_guard.rc;
  if (rc) return rc;
  const size_t nn = (size_t)h->n * h->n;
  HF_CUDA(h, h->d_mats.ensure(sizeof(double) * nn * (1 + nK)));
  HF_CUDA(h, h->d_grad.ensure(sizeof(double) * 3 * h->natoms));
  double* dDJ = h->d_mats.as<double>();
  double* dDK = dDJ + nn;
  HF_CUDA(h, cudaMemcpyAsync(dDJ, DJ, sizeof(double) * nn, cudaMemcpyHostToDevice, h->stream));
  for (int m = 0; m < nK; ++m)
    HF_CUDA(h, cudaMemcpyAsync(dDK + m * nn, DKs[m], sizeof(double) * nn, cudaMemcpyHostToDevice, h->stream));
  HF_CUDA(h, cudaMemsetAsync(h->d_grad.p, 0, sizeof(double) * 3 * h->natoms, h->stream));
  if ((rc = grad_device_impl(h, dDJ, cJ, nK, dDK, cK, h->d_grad.as<double>(), precision))) return rc;
  std::vector<double> g(3 * h->natoms);
  HF_CUDA(h, cudaMemcpyAsync(g.data(), h->d_grad.p, sizeof(double) * g.size(), cudaMemcpyDeviceToHost, h->stream));
  HF_CUDA(h, cudaStreamSynchronize(h->stream));
  for (size_t i = 0; i < g.size(); ++i) {
    if (!std::isfinite(g[i])) return fail(h, HFGPU_ERR_NONFINITE, "non-finite gradient");
    dE_dR[i] += scale * g[i];
  }
  return HFGPU_OK;
}

int hfgpu_grad2e_backward(hfgpu_handle* h, const double* D, double scale, double* dE_dR, int precision) {
  if (!h || !D || !dE_dR) return HFGPU_ERR_INVALID;
  if (!h->have_geometry) return fail(h, HFGPU_ERR_STATE, "no geometry set");
  const double* dk[1] = {D};
  return grad_host(h, D, 2.0, 1, dk, 1.0, scale, dE_dR, precision);
}

int hfgpu_grad2e_uhf_backward(hfgpu_handle* h, const double* Da, const double* Db, double scale, double* dE_dR,
                              int precision) {
  if (!h || !Da || !Db || !dE_dR) return HFGPU_ERR_INVALID;
  if (!h->have_geometry) return fail(h, HFGPU_ERR_STATE, "no geometry set");
  const size_t nn = (size_t)h->n * h->n;
  std::vector<double> Dt(nn);
  for (size_t i = 0; i < nn; ++i) Dt[i] = Da[i] + Db[i];
  const double* dk[2] = {Da, Db};
  return grad_host(h, Dt.data(), 0.5, 2, dk, 0.5, scale, dE_dR, precision);
}

// ---- Two-electron part of the Hessian at a fixed density (adjoint second derivatives) ----
// The classes run on the auxiliary streams (fork/join with the handle's stream, as the J/K
// classes do), so the few-quartet, long-table d classes overlap the many-quartet s/p classes.
// Every auxiliary stream owns one slice of the scratch buffer, which its classes use one after
// another; a class gets as many threads (whole 128-thread blocks) as kHessScratchBudget holds
// (enough to fill the GPU for the largest tables), at most one per quartet, and loops over the rest.
constexpr size_t kHessScratchBudget = (size_t)2 << 30;
constexpr size_t kHessSmemBytes = 96 * 1024;  // per-block Hessian in shared memory up to 36 atoms
constexpr int kHessBlockMinSlots = 1000;       // thread-form tables from this size run in the block form,
constexpr long long kHessBlockMaxQuartets = 4096;  // and so do classes with at most this many quartets
constexpr long long kHessLineGrid = 4 * 148;     // straight-line form: at most four blocks per SM, grid-stride
constexpr long long kHessBlockGrid = 296;      // blocks of a block-form launch with global HRR slots

static int hess_device_impl(hfgpu_handle* h, const double* DJ, double cJ, int nK, const double* DK, double cK,
                            double* hess) {
  if (!h->have_geometry) return fail(h, HFGPU_ERR_STATE, "no geometry set");
  if (h->batched) return fail(h, HFGPU_ERR_UNSUPPORTED, "the Hessian takes a single-molecule handle");
  if (hfgpu::kNumHessClasses != hfgpu::kNumClasses) return fail(h, HFGPU_ERR_STATE, "Hessian class table");
  GradArgs<double> gd{};
  gd.pairs = h->d_pairs.as<PairInfo>();
  gd.prims = h->d_prim_d.as<PrimPair<double>>();
  const size_t np = std::max<size_t>(h->nprimpairs, 1);
  gd.alpha_a = h->d_alpha_d.as<double>();
  gd.alpha_b = h->d_alpha_d.as<double>() + np;
  gd.boys.tab = h->d_boys_d.as<double>();
  gd.n = h->n;
  gd.DJ = DJ; gd.cJ = cJ; gd.nK = nK; gd.DK = DK; gd.cK = cK; gd.grad = nullptr;
  gd.part = h->part;
  gd.nparts = h->nparts;
  const size_t n3 = 3 * (size_t)h->natoms;
  const size_t smem = sizeof(double) * n3 * n3;
  HessOut o{hess, h->natoms, smem <= kHessSmemBytes ? 1 : 0};
  const int2* q = h->d_quart.as<int2>();
  auto threads_of = [&](int slots, long long nq) -> long long {
    long long thr = (long long)(kHessScratchBudget / ((size_t)slots * sizeof(double)));
    thr = std::min<long long>(thr, ((nq + 127) / 128) * 128);
    return std::max<long long>(128, thr / 128 * 128);
  };
  // form per class: 0 one thread per quartet on global scratch, 1 one block of 128 threads per
  // quartet over levelised tables, 2 one warp per quartet over the same tables, 3 one thread per
  // quartet on straight-line register code (the classes that have it; a class without it takes
  // the default).  Default: the straight-line form where the class has one; else the block form
  // for the classes whose tables are large or whose quartets are too few to fill the GPU (one
  // thread would run a long chain of dependent table ops on global scratch), the warp form for
  // the small many-quartet classes (their levels hold a few dozen ops).
  auto form_of = [&](int c) -> int {
    const bool line = hfgpu::kHessLaunchers[c]->has_line;
    int f = h->hess_cls_form[c] >= 0 ? h->hess_cls_form[c] : h->hess_form;
    if (f == 3 && !line) f = -1;
    if (f >= 0) return f;
    if (line) return 3;
    const bool big = hfgpu::kHessLaunchers[c]->scratch_slots(h->pure) >= kHessBlockMinSlots ||
                     part_share(h, h->q_end[c] - h->q_beg[c]) <= kHessBlockMaxQuartets;
    return big ? 1 : 2;
  };
  auto use_block = [&](int c) -> bool { return form_of(c) == 1 || form_of(c) == 2; };
  // block-form grid: one block per quartet, or kHessBlockGrid blocks when the HRR slots live in
  // global scratch (one region per block)
  auto block_grid = [&](int c, long long nq) -> long long {
    return hfgpu::kHessLaunchers[c]->block_global_slots() > 0 ? std::min<long long>(nq, kHessBlockGrid) : nq;
  };
  // classes largest first, round-robin over the auxiliary streams; each stream's slice is the
  // largest need of its classes
  constexpr int kS = hfgpu_handle::kAux;
  int stream_of[32];
  size_t slice[kS] = {0}, off[kS] = {0}, need = 0;
  int rr = 0;
  for (int c = hfgpu::kNumClasses - 1; c >= 0; --c) {
    const hfgpu::HessLaunchers* L = hfgpu::kHessLaunchers[c];
    const hfgpu::ClassLaunchers* C = hfgpu::kClassLaunchers[c];
    if (L->la != C->la || L->lb != C->lb || L->lc != C->lc || L->ld != C->ld)
      return fail(h, HFGPU_ERR_STATE, "Hessian class order");
    stream_of[c] = -1;
    const long long nq = part_share(h, h->q_end[c] - h->q_beg[c]);
    if (nq <= 0 || !((h->hess_class_mask >> c) & 1u)) continue;
    stream_of[c] = rr++ % kS;
    size_t bytes;
    if (form_of(c) == 3) {
      bytes = 0;
    } else if (use_block(c)) {
      bytes = sizeof(double) * (size_t)L->block_global_slots() * (size_t)block_grid(c, nq);
    } else {
      const int slots = L->scratch_slots(h->pure);
      bytes = (size_t)slots * sizeof(double) * (size_t)threads_of(slots, nq);
    }
    slice[stream_of[c]] = std::max(slice[stream_of[c]], (bytes + 255) / 256 * 256);
  }
  for (int st = 0; st < kS; ++st) {
    off[st] = need;
    need += slice[st];
  }
  if (need) HF_CUDA(h, h->d_scratch.ensure(need));
  int rc = fork_streams(h);
  if (rc) return rc;
  for (int c = hfgpu::kNumClasses - 1; c >= 0; --c) {
    if (stream_of[c] < 0) continue;
    const hfgpu::HessLaunchers* L = hfgpu::kHessLaunchers[c];
    const long long nq = part_share(h, h->q_end[c] - h->q_beg[c]);
    if (form_of(c) == 3) {
      const long long grid = std::min<long long>((nq + 127) / 128, kHessLineGrid);
      if (!L->launch_line(gd, o, h->pure, q + h->q_beg[c], (int)nq, (int)grid, o.smem ? (int)smem : 0,
                          h->aux[stream_of[c]]))
        return fail(h, HFGPU_ERR_STATE, "class without a Hessian straight-line form");
      HF_CHECK_LAUNCH(h, "hess line kernel");
      continue;
    }
    if (use_block(c)) {
      const int st = stream_of[c];
      const long long grid = block_grid(c, nq);
      if (sizeof(double) * (size_t)L->block_global_slots() * (size_t)grid > slice[st] ||
          off[st] + slice[st] > h->d_scratch.bytes)
        return fail(h, HFGPU_ERR_NOMEM, "Hessian scratch too small");
      gd.scratch = reinterpret_cast<double*>(h->d_scratch.as<unsigned char>() + off[st]);
      gd.scratch_threads = 0;
      if (form_of(c) == 2 && L->launch_warp(gd, o, h->pure, q + h->q_beg[c], (int)nq, h->aux[st])) {
        HF_CHECK_LAUNCH(h, "hess warp kernel");
        continue;
      }
      if (L->launch_block(gd, o, h->pure, q + h->q_beg[c], (int)nq, (int)grid, h->aux[st])) {
        HF_CHECK_LAUNCH(h, "hess block kernel");
        continue;
      }
      if (h->hess_form >= 1) return fail(h, HFGPU_ERR_UNSUPPORTED, "class without a Hessian block form");
    }
    const int slots = L->scratch_slots(h->pure);
    const long long thr = threads_of(slots, nq);
    const int st = stream_of[c];
    if ((size_t)slots * sizeof(double) * (size_t)thr > slice[st] || off[st] + slice[st] > h->d_scratch.bytes)
      return fail(h, HFGPU_ERR_NOMEM, "Hessian scratch too small");
    gd.scratch = reinterpret_cast<double*>(h->d_scratch.as<unsigned char>() + off[st]);
    gd.scratch_threads = (int)thr;
    L->launch(gd, o, h->pure, q + h->q_beg[c], (int)nq, (int)(thr / 128), o.smem ? (int)smem : 0, h->aux[st]);
    HF_CHECK_LAUNCH(h, "hess kernel");
  }
  return join_streams(h);
}

int hfgpu_set_hess_form(hfgpu_handle* h, int form) {
  if (!h || form < -1 || form > 3) return HFGPU_ERR_INVALID;
  h->hess_form = form;
  for (int c = 0; c < 21; ++c) h->hess_cls_form[c] = -1;
  return HFGPU_OK;
}

int hfgpu_set_hess_forms(hfgpu_handle* h, const int* forms) {
  if (!h || !forms) return HFGPU_ERR_INVALID;
  for (int c = 0; c < hfgpu::kNumClasses; ++c)
    if (forms[c] < -1 || forms[c] > 3) return HFGPU_ERR_INVALID;
  for (int c = 0; c < hfgpu::kNumClasses; ++c) h->hess_cls_form[c] = forms[c];
  return HFGPU_OK;
}

int hfgpu_hess2e_device(hfgpu_handle* h, const double* DJ, double cJ, int nK, const double* DK, double cK,
                        double* hess) {
  if (!h || !hess || nK < 0 || (nK > 0 && !DK)) return HFGPU_ERR_INVALID;
  DeviceGuard dev_guard(h);
  int rc = dev_guard.rc;
  if (rc) return rc;
  return hess_device_impl(h, DJ, cJ, nK, DK, cK, hess);
}

static int hess_host(hfgpu_handle* h, const double* DJ, double cJ, int nK, const double* const* DKs, double cK,
                     double scale, double* hess) {
  DeviceGuard dev_guard(h);
  int rc = dev_guard.rc;
  if (rc) return rc;
  const size_t nn = (size_t)h->n * h->n;
  const size_t n3 = 3 * (size_t)h->natoms;
  HF_CUDA(h, h->d_mats.ensure(sizeof(double) * (nn * (1 + nK) + n3 * n3)));
  double* dDJ = h->d_mats.as<double>();
  double* dDK = dDJ + nn;
  double* dH = dDK + nK * nn;
  HF_CUDA(h, cudaMemcpyAsync(dDJ, DJ, sizeof(double) * nn, cudaMemcpyHostToDevice, h->stream));
  for (int m = 0; m < nK; ++m)
    HF_CUDA(h, cudaMemcpyAsync(dDK + m * nn, DKs[m], sizeof(double) * nn, cudaMemcpyHostToDevice, h->stream));
  HF_CUDA(h, cudaMemsetAsync(dH, 0, sizeof(double) * n3 * n3, h->stream));
  if ((rc = hess_device_impl(h, dDJ, cJ, nK, dDK, cK, dH))) return rc;
  std::vector<double> H(n3 * n3);
  HF_CUDA(h, cudaMemcpyAsync(H.data(), dH, sizeof(double) * H.size(), cudaMemcpyDeviceToHost, h->stream));
  HF_CUDA(h, cudaStreamSynchronize(h->stream));
  for (size_t i = 0; i < H.size(); ++i) {
    if (!std::isfinite(H[i])) return fail(h, HFGPU_ERR_NONFINITE, "non-finite Hessian");
    hess[i] += scale * H[i];
  }
  return HFGPU_OK;
}

int hfgpu_hess2e(hfgpu_handle* h, const double* D, double scale, double* hess) {
  if (!h || !D || !hess) return HFGPU_ERR_INVALID;
  if (!h->have_geometry) return fail(h, HFGPU_ERR_STATE, "no geometry set");
  const double* dk[1] = {D};
  return hess_host(h, D, 2.0, 1, dk, 1.0, scale, hess);
}

int hfgpu_hess2e_uhf(hfgpu_handle* h, const double* Da, const double* Db, double scale, double* hess) {
  if (!h || !Da || !Db || !hess) return HFGPU_ERR_INVALID;
  if (!h->have_geometry) return fail(h, HFGPU_ERR_STATE, "no geometry set");
  const size_t nn = (size_t)h->n * h->n;
  std::vector<double> Dt(nn);
  for (size_t i = 0; i < nn; ++i) Dt[i] = Da[i] + Db[i];
  const double* dk[2] = {Da, Db};
  return hess_host(h, Dt.data(), 0.5, 2, dk, 0.5, scale, hess);
}

// Host-only basis view for the one-electron code (normalised coefficients).
struct OneEHost {
  std::vector<int> off, first;
  std::vector<double> coefs;
  OneEBasis b{};
};

static int onee_basis(const hfgpu_basis* in, OneEHost& o) {
  if (!in || in->nshell <= 0 || !in->L || !in->shell_atom || !in->nprim || !in->exps || !in->coefs)
    return HFGPU_ERR_INVALID;
  const int ns = in->nshell;
  o.off.assign(ns + 1, 0);
  o.first.assign(ns + 1, 0);
  for (int s = 0; s < ns; ++s) {
    if (in->L[s] < 0 || in->L[s] > 2 || in->nprim[s] < 1) return HFGPU_ERR_INVALID;
    o.off[s + 1] = o.off[s] + in->nprim[s];
    o.first[s + 1] = o.first[s] + (in->pure ? 2 * in->L[s] + 1 : (in->L[s] + 1) * (in->L[s] + 2) / 2);
  }
  o.coefs.resize(o.off[ns]);
  for (int s = 0; s < ns; ++s)
    normalise(in->L[s], in->nprim[s], &in->exps[o.off[s]], &in->coefs[o.off[s]], &o.coefs[o.off[s]]);
  o.b.nshell = ns;
  o.b.n = o.first[ns];
  o.b.pure = in->pure ? 1 : 0;
  o.b.L = in->L;
  o.b.atom = in->shell_atom;
  o.b.nprim = in->nprim;
  o.b.off = o.off.data();
  o.b.first = o.first.data();
  o.b.exps = in->exps;
  o.b.coefs = o.coefs.data();
  return HFGPU_OK;
}

int hfgpu_one_electron(const hfgpu_basis* basis, const double* xyz, const double* Z, double* S, double* T, double* V) {
  OneEHost o;
  if (!xyz || !Z || !S || !T || !V || onee_basis(basis, o)) return HFGPU_ERR_INVALID;
  hfgpu_onee_matrices(o.b, Z, xyz, basis->natoms, S, T, V);
  return HFGPU_OK;
}

int hfgpu_one_electron_grad(const hfgpu_basis* basis, const double* xyz, const double* Z, const double* D,
                            const double* W, double cH, double cS, double* grad) {
  OneEHost o;
  if (!xyz || !Z || !D || !W || !grad || onee_basis(basis, o)) return HFGPU_ERR_INVALID;
  hfgpu_onee_gradient(o.b, Z, xyz, basis->natoms, D, W, cH, cS, grad);
  return HFGPU_OK;
}

// Kernel arguments of the device one-electron kernels; uploads atoms and charges.
static int onee_setup(hfgpu_handle* h, const double* Z, onee::Args& a, long long& nitems) {
  if (!h->have_geometry) return fail(h, HFGPU_ERR_STATE, "no geometry set");
  const int na = h->natoms, nm = h->nmol;
  std::vector<int> mol_atom = h->batched ? h->mol_atom : std::vector<int>{0, na};
  int slots = 0;
  for (int m = 0; m < nm; ++m) slots = std::max(slots, mol_atom[m + 1] - mol_atom[m]);
  slots += 1;
  // layout: ylm [3][30] | atoms [na][4] | mol_atom [nm + 1] (ints)
  const size_t bytes = sizeof(double) * (90 + 4 * (size_t)na) + sizeof(int) * (nm + 1);
  std::vector<unsigned char> host(bytes, 0);
  double* y = reinterpret_cast<double*>(host.data());
  for (int L = 0; L <= 2; ++L) hfgpu_onee_ylm(L, y + 30 * L);
  double* at = y + 90;
  for (int i = 0; i < na; ++i) {
    if (!std::isfinite(Z[i])) return fail(h, HFGPU_ERR_INVALID, "non-finite nuclear charge");
    for (int d = 0; d < 3; ++d) at[4 * i + d] = h->xyz[3 * i + d];
    at[4 * i + 3] = Z[i];
  }
  std::memcpy(at + 4 * na, mol_atom.data(), sizeof(int) * (nm + 1));
  HF_CUDA(h, h->d_onee.ensure(bytes));
  HF_CUDA(h, cudaMemcpyAsync(h->d_onee.p, host.data(), bytes, cudaMemcpyHostToDevice, h->stream));
  const double* dy = h->d_onee.as<double>();
  const size_t np = std::max<size_t>(h->nprimpairs, 1);
  a = onee::Args{};
  a.pairs = h->d_pairs.as<PairInfo>();
  a.prims = h->d_prim_d.as<PrimPair<double>>();
  a.alpha_a = h->d_alpha_d.as<double>();
  a.alpha_b = h->d_alpha_d.as<double>() + np;
  a.npairs = (int)h->pairs.size();
  a.boys.tab = h->d_boys_d.as<double>();
  a.atoms.xyzZ = dy + 90;
  a.atoms.mol_atom = reinterpret_cast<const int*>(dy + 90 + 4 * na);
  a.atoms.slots = slots;
  a.ylm = dy;
  a.pure = h->pure;
  a.n = h->n;
  if (h->batched) {
    a.mol_off = h->d_mol.as<long long>();
    a.mol_n = reinterpret_cast<const int*>(a.mol_off + h->nmol);
  }
  nitems = (long long)a.npairs * slots;
  return HFGPU_OK;
}

int hfgpu_one_electron_device(hfgpu_handle* h, const double* Z, double* S, double* T, double* V) {
  if (!h || !Z || !S || !T || !V) return HFGPU_ERR_INVALID;
  DeviceGuard dev_guard(h);
  int rc = dev_guard.rc;
  if (rc) return rc;
  onee::Args a;
  long long nitems = 0;
  if ((rc = onee_setup(h, Z, a, nitems))) return rc;
  const size_t nn = h->batched ? (size_t)h->mat_total : (size_t)h->n * h->n;
  HF_CUDA(h, cudaMemsetAsync(V, 0, sizeof(double) * nn, h->stream));
  if (nitems > 0) {
    onee_matrices_kernel<<<(unsigned)((nitems + 127) / 128), 128, 0, h->stream>>>(a, nitems, S, T, V);
    HF_CHECK_LAUNCH(h, "one-electron matrices");
  }
  return HFGPU_OK;
}

int hfgpu_one_electron_grad_device(hfgpu_handle* h, const double* Z, const double* D, const double* W, double cH,
                                   double cS, double* grad) {
  if (!h || !Z || !D || !W || !grad) return HFGPU_ERR_INVALID;
  DeviceGuard dev_guard(h);
  int rc = dev_guard.rc;
  if (rc) return rc;
  onee::Args a;
  long long nitems = 0;
  if ((rc = onee_setup(h, Z, a, nitems))) return rc;
  if (nitems > 0) {
    onee_grad_kernel<<<(unsigned)((nitems + 127) / 128), 128, 0, h->stream>>>(a, nitems, D, W, cH, cS, grad);
    HF_CHECK_LAUNCH(h, "one-electron gradient");
  }
  return HFGPU_OK;
}

int hfgpu_batch_eigh(hfgpu_handle* h, const double* A, double* W, double* V, int* sweeps) {
  if (!h || !A || !W || !V) return HFGPU_ERR_INVALID;
  if (!h->batched) return fail(h, HFGPU_ERR_UNSUPPORTED, "hfgpu_batch_eigh needs a batched handle");
  const int nmax = h->n;
  if (nmax > kJacobiMaxN) return fail(h, HFGPU_ERR_UNSUPPORTED, "batched eigensolver: a molecule has more than 118 functions");
  DeviceGuard dev_guard(h);
  int rc = dev_guard.rc;
  if (rc) return rc;
  const size_t smem = jacobi_smem_bytes(nmax);
  HF_CUDA(h, cudaFuncSetAttribute(batch_jacobi_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int* mol_n = reinterpret_cast<const int*>(h->d_mol.as<long long>() + h->nmol);
  batch_jacobi_kernel<<<h->nmol, kJacobiThreads, smem, h->stream>>>(A, nmax, mol_n, W, V, 30, sweeps);
  HF_CHECK_LAUNCH(h, "batched eigensolver");
  return HFGPU_OK;
}

int hfgpu_batch_purify_device(hfgpu_handle* h, const double* Fo, const int* nocc, int max_steps, double* P,
                              double* err) {
  if (!h || !Fo || !nocc || !P || !err || max_steps <= 0 || max_steps > 256) return HFGPU_ERR_INVALID;
  if (!h->batched) return fail(h, HFGPU_ERR_UNSUPPORTED, "hfgpu_batch_purify_device needs a batched handle");
  const int nmax = h->n;
  if (nmax > kBatchPurifyMaxN)
    return fail(h, HFGPU_ERR_UNSUPPORTED, "batched purification: a molecule has more than 116 functions");
  DeviceGuard dev_guard(h);
  int rc = dev_guard.rc;
  if (rc) return rc;
  const size_t smem = batch_purify_smem_bytes(nmax);
  HF_CUDA(h, cudaFuncSetAttribute(batch_purify_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int* mol_n = reinterpret_cast<const int*>(h->d_mol.as<long long>() + h->nmol);
  batch_purify_kernel<<<h->nmol, kBatchPurifyThreads, smem, h->stream>>>(Fo, nmax, mol_n, nocc, max_steps, 1e-11, P,
                                                                          err);
  HF_CHECK_LAUNCH(h, "batched purification");
  return HFGPU_OK;
}

int hfgpu_set_timing(hfgpu_handle* h, int on) {
  if (!h) return HFGPU_ERR_INVALID;
  DeviceGuard dev_guard(h);
  int rc = dev_guard.rc;
  if (rc) return rc;
  if (on && !h->ev[0])
    for (auto& e : h->ev) HF_CUDA(h, cudaEventCreate(&e));
  h->timing = on != 0;
  return HFGPU_OK;
}

int hfgpu_class_stats(hfgpu_handle* h, int cls, long long* out) {
  if (!h || !out || cls < 0 || cls >= hfgpu::kNumClasses) return HFGPU_ERR_INVALID;
  const hfgpu::ClassLaunchers* L = hfgpu::kClassLaunchers[cls];
  out[0] = L->la;
  out[1] = L->lb;
  out[2] = L->lc;
  out[3] = L->ld;
  out[4] = h->q_end[cls] - h->q_beg[cls];
  out[5] = h->q_mid[cls] - h->q_beg[cls];
  out[6] = out[7] = out[8] = 0;
  if (h->d_counters.p) {
    unsigned long long c[3];
    HF_CUDA(h, cudaStreamSynchronize(h->stream));
    HF_CUDA(h, cudaMemcpy(c, h->d_counters.as<unsigned long long>() + 3 * cls, sizeof(c), cudaMemcpyDeviceToHost));
    out[6] = (long long)c[0];
    out[7] = (long long)c[1];
    out[8] = (long long)c[2];
  }
  return HFGPU_OK;
}

int hfgpu_set_partition(hfgpu_handle* h, int part, int nparts) {
  if (!h) return HFGPU_ERR_INVALID;
  if (nparts < 1 || nparts > 65536 || part < 0 || part >= nparts)
    return fail(h, HFGPU_ERR_INVALID, "partition needs 0 <= part < nparts <= 65536");
  h->part = part;
  h->nparts = nparts;
  return HFGPU_OK;
}

int hfgpu_class_work(const hfgpu_handle* h, int cls, long long* out) {
  if (!h || !out || cls < 0 || cls >= hfgpu::kNumClasses) return HFGPU_ERR_INVALID;
  out[0] = h->q_end[cls] - h->q_beg[cls];
  out[1] = h->q_prims[cls];
  return HFGPU_OK;
}

int hfgpu_setup_times(const hfgpu_handle* h, double* ms) {
  if (!h || !ms) return HFGPU_ERR_INVALID;
  for (int i = 0; i < 4; ++i) ms[i] = h->setup_ms[i];
  return HFGPU_OK;
}

int hfgpu_class_time(hfgpu_handle* h, int cls, float* ms) {
  if (!h || !ms || cls < 0 || cls >= hfgpu::kNumClasses) return HFGPU_ERR_INVALID;
  *ms = 0.f;
  if (!h->timing || !h->ev_used[cls]) return HFGPU_OK;
  HF_CUDA(h, cudaEventSynchronize(h->ev[2 * cls + 1]));
  HF_CUDA(h, cudaEventElapsedTime(ms, h->ev[2 * cls], h->ev[2 * cls + 1]));
  return HFGPU_OK;
}

int hfgpu_set_schedule(hfgpu_handle* h, const int* schedule) {
  if (!h || !schedule) return HFGPU_ERR_INVALID;
  for (int c = 0; c < hfgpu::kNumClasses; ++c) {
    const int bs = schedule[4 * c], pw = schedule[4 * c + 1], wp = schedule[4 * c + 2], cp = schedule[4 * c + 3];
    if ((bs != 32 && bs != 64 && bs != 128) || (pw != 0 && pw != 1 && pw != 4 && pw != 8 && pw != 16 && pw != 32) ||
        wp < -1 || wp > 2 || cp < 0 || cp > 3)
      return fail(h, HFGPU_ERR_INVALID, "schedule entry out of range");
  }
  for (int c = 0; c < hfgpu::kNumClasses; ++c) {
    h->sched_block[c] = schedule[4 * c];
    h->sched_primwarp[c] = schedule[4 * c + 1];
    h->sched_warp[c] = schedule[4 * c + 2];
    h->sched_cap[c] = schedule[4 * c + 3];
  }
  return HFGPU_OK;
}

int hfgpu_get_schedule(const hfgpu_handle* h, int* schedule) {
  if (!h || !schedule) return HFGPU_ERR_INVALID;
  for (int c = 0; c < hfgpu::kNumClasses; ++c) {
    schedule[4 * c] = h->sched_block[c];
    schedule[4 * c + 1] = h->sched_primwarp[c];
    schedule[4 * c + 2] = h->sched_warp[c];
    schedule[4 * c + 3] = h->sched_cap[c];
  }
  return HFGPU_OK;
}

// Tuner timing: the median device time of `repeats` runs of run() on the handle's stream, each
// after a write of the buffer `flush` (larger than L2, when it could be allocated), the way the
// bench times its steps; one untimed warm-up run first.  A median of separately timed runs
// rather than one total keeps a single slow run from deciding a comparison.
extern "C++" {
template <typename Run>
static int tuner_time(hfgpu_handle* h, Run&& run, int repeats, cudaEvent_t e0, cudaEvent_t e1, const DevBuf& flush,
                      float* ms) {
  int rc;
  if ((rc = run())) return rc;
  float t[100];
  repeats = std::max(1, std::min(repeats, 100));
  for (int r = 0; r < repeats; ++r) {
    if (flush.p) HF_CUDA(h, cudaMemsetAsync(flush.p, r & 0xff, flush.bytes, h->stream));
    HF_CUDA(h, cudaEventRecord(e0, h->stream));
    if ((rc = run())) return rc;
    HF_CUDA(h, cudaEventRecord(e1, h->stream));
    HF_CUDA(h, cudaEventSynchronize(e1));
    HF_CUDA(h, cudaEventElapsedTime(&t[r], e0, e1));
  }
  std::sort(t, t + repeats);
  *ms = repeats % 2 ? t[repeats / 2] : 0.5f * (t[repeats / 2 - 1] + t[repeats / 2]);
  return HFGPU_OK;
}
}  // extern "C++"
constexpr size_t kTunerFlushBytes = (size_t)256 << 20;  // 256 MiB > the 126 MB L2

// Per class, times every launch form the class has on the handle's current quartet lists
// and the given density, one class at a time on the handle's stream, and keeps the fastest.
int hfgpu_autotune(hfgpu_handle* h, const double* D, int precision, int repeats, int* schedule) {
  if (!h || !D) return HFGPU_ERR_INVALID;
  DeviceGuard dev_guard(h);
  int rc = dev_guard.rc;
  if (rc) return rc;
  if (!h->have_geometry) return fail(h, HFGPU_ERR_STATE, "no geometry set");
  repeats = std::max(1, std::min(repeats, 100));
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  HF_CUDA(h, cudaEventCreate(&e0));
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return fail(h, HFGPU_ERR_CUDA, "cudaEventCreate");
  }
  struct Restore {  // the mask goes back and the flush buffer is freed on every exit path
    hfgpu_handle* h;
    unsigned mask;
    cudaEvent_t a, b;
    DevBuf flush;
    ~Restore() {
      h->class_mask = mask;
      cudaEventDestroy(a);
      cudaEventDestroy(b);
      flush.release();
    }
  } restore{h, h->class_mask, e0, e1, DevBuf{}};
  if (restore.flush.ensure(kTunerFlushBytes) != cudaSuccess) {
    cudaGetLastError();  // no room for the flush buffer: time without it
    restore.flush = DevBuf{};
  }
  auto build = [&]() { return jk_device_impl(h, D, 1, D, nullptr, nullptr, precision); };
  int start[4 * 21];
  hfgpu_get_schedule(h, start);
  // best candidate per class and kind of form: 0 thread per quartet, 1 primitive-split for
  // the many-primitive segments, 2 warp per quartet
  struct Cand {
    float ms;
    int b, p, w, c;
  };
  std::vector<Cand> kind_best((size_t)4 * hfgpu::kNumClasses, Cand{1e30f, 0, 0, 0, 0});
  auto kind_of = [&](int c, int pw, int wp, int cap) {
    const hfgpu::ClassLaunchers* L = hfgpu::kClassLaunchers[c];
    return wp >= 1 ? 2 : (L->has_primwarp && pw > 0 ? 1 : (cap == 2 && L->has_staged ? 3 : 0));
  };
  for (int c = 0; c < hfgpu::kNumClasses; ++c) {
    if (h->q_end[c] <= h->q_beg[c]) continue;
    const hfgpu::ClassLaunchers* L = hfgpu::kClassLaunchers[c];
    h->class_mask = 1u << c;
    float best = 1e30f;
    int bb = h->sched_block[c], bp = h->sched_primwarp[c], bw = h->sched_warp[c], bc = h->sched_cap[c];
    const int warps[3] = {2, 1, 0};  // block per quartet, warp per quartet, thread forms
    for (int wi = 0; wi < (L->has_warp ? 3 : 1); ++wi) {
      const int wp = L->has_warp ? warps[wi] : -1;
      const int pws[5] = {32, 16, 8, 4, 0};
      for (int pi = (L->has_primwarp ? 0 : 4); pi < 5; ++pi) {
        const int pw = pws[pi];
        // thread-form variants: plain (0), register-capped (1), persistent with the Boys table
        // staged in shared memory (2), at most two blocks per SM (3, the classes that spill)
        for (int cand = 0; cand < 12; ++cand) {
          const int bs = 32 << (cand % 3), cap = cand / 3;
          if ((cap == 1 && !L->has_capped) || (cap == 2 && !L->has_staged) || (cap == 3 && !L->has_lowres))
            continue;
          if (wp >= 1 && (bs != 64 || cap)) continue;  // the warp and block forms have their own shape
          h->sched_block[c] = bs;
          h->sched_primwarp[c] = L->has_primwarp ? pw : 1;
          h->sched_warp[c] = wp;
          h->sched_cap[c] = cap;
          float ms = 0.f;
          if ((rc = tuner_time(h, build, repeats, e0, e1, restore.flush, &ms))) return rc;
          if (ms < best) {
            best = ms;
            bb = bs;
            bp = h->sched_primwarp[c];
            bw = wp;
            bc = cap;
          }
          Cand& kb = kind_best[(size_t)4 * c + kind_of(c, pw, wp, cap)];
          if (ms < kb.ms) kb = Cand{ms, bs, h->sched_primwarp[c], wp, cap};
        }
      }
    }
    h->sched_block[c] = bb;
    h->sched_primwarp[c] = bp;
    h->sched_warp[c] = bw;
    h->sched_cap[c] = bc;
  }
  // Classes were timed one at a time; in a build they run concurrently on several streams,
  // where a slower form that overlaps better can win.  Refinement on whole builds: per
  // class, the best candidate of each other kind replaces the current form if the build
  // gets at least 1% faster.
  h->class_mask = restore.mask;
  // whole builds: at least five runs per median
  auto time_builds = [&](float* ms) -> int {
    return tuner_time(h, build, std::max(repeats, 5), e0, e1, restore.flush, ms);
  };
  float cur = 0.f;
  if ((rc = time_builds(&cur))) return rc;
  for (int c = 0; c < hfgpu::kNumClasses; ++c) {
    if (h->q_end[c] <= h->q_beg[c]) continue;
    for (int k = 0; k < 4; ++k) {
      const Cand& cd = kind_best[(size_t)4 * c + k];
      if (cd.ms >= 1e30f || k == kind_of(c, h->sched_primwarp[c], h->sched_warp[c], h->sched_cap[c])) continue;
      const Cand keep{0.f, h->sched_block[c], h->sched_primwarp[c], h->sched_warp[c], h->sched_cap[c]};
      h->sched_block[c] = cd.b;
      h->sched_primwarp[c] = cd.p;
      h->sched_warp[c] = cd.w;
      h->sched_cap[c] = cd.c;
      float ms = 0.f;
      if ((rc = time_builds(&ms))) return rc;
      if (ms < 0.99f * cur) {
        cur = ms;
      } else {
        h->sched_block[c] = keep.b;
        h->sched_primwarp[c] = keep.p;
        h->sched_warp[c] = keep.w;
        h->sched_cap[c] = keep.c;
      }
    }
  }
  // Keep the tuned schedule only if whole builds with it beat whole builds with the schedule
  // we started from.
  int tuned[4 * 21];
  hfgpu_get_schedule(h, tuned);
  float t_tuned = 0.f, t_start = 0.f;
  for (int round = 0; round < 2; ++round)
    for (int which = 0; which < 2; ++which) {
      if ((rc = hfgpu_set_schedule(h, which ? start : tuned))) return rc;
      float ms = 0.f;
      if ((rc = time_builds(&ms))) return rc;
      (which ? t_start : t_tuned) += ms;
    }
  if ((rc = hfgpu_set_schedule(h, t_tuned <= t_start ? tuned : start))) return rc;
  // the classes concurrently on the auxiliary streams, or one after another
  {
    float t_conc = 0.f, t_ser = 0.f;
    for (int round = 0; round < 2; ++round)
      for (int ser = 0; ser < 2; ++ser) {
        h->jk_serial = ser;
        float ms = 0.f;
        if ((rc = time_builds(&ms))) return rc;
        (ser ? t_ser : t_conc) += ms;
      }
    h->jk_serial = t_ser < 0.99f * t_conc ? 1 : 0;
  }
  return schedule ? hfgpu_get_schedule(h, schedule) : HFGPU_OK;
}

int hfgpu_request_abort(hfgpu_handle* h, int on) {
  if (!h) return HFGPU_ERR_INVALID;
  DeviceGuard dev_guard(h);
  if (dev_guard.rc) return dev_guard.rc;
  if (!h->ctl_stream) HF_CUDA(h, cudaStreamCreateWithFlags(&h->ctl_stream, cudaStreamNonBlocking));
  // written on a stream of its own, so that it lands while the handle's stream is busy
  HF_CUDA(h, cudaMemsetAsync(h->d_abort.p, on ? 0x01 : 0x00, 1, h->ctl_stream));
  HF_CUDA(h, cudaStreamSynchronize(h->ctl_stream));
  return HFGPU_OK;
}

int hfgpu_set_grad_forms(hfgpu_handle* h, const int* forms) {
  if (!h || !forms) return HFGPU_ERR_INVALID;
  for (int c = 0; c < hfgpu::kNumClasses; ++c)
    if (forms[c] < -1 || forms[c] > kGradForms - 1) return fail(h, HFGPU_ERR_INVALID, "gradient form out of range");
  for (int c = 0; c < hfgpu::kNumClasses; ++c)
    h->grad_form[c] = hfgpu::kClassLaunchers[c]->has_grad_warp ? forms[c] : -1;
  return HFGPU_OK;
}

// Hessian form per class: each class alone, one thread (global scratch), one block or one warp
// per quartet, or one thread on straight-line code where the class has it, on RHF weights of the
// device density D; the fastest is kept.
int hfgpu_autotune_hess(hfgpu_handle* h, const double* D, int repeats, int* forms) {
  if (!h || !D) return HFGPU_ERR_INVALID;
  DeviceGuard dev_guard(h);
  int rc = dev_guard.rc;
  if (rc) return rc;
  if (!h->have_geometry) return fail(h, HFGPU_ERR_STATE, "no geometry set");
  if (h->batched) return fail(h, HFGPU_ERR_UNSUPPORTED, "the Hessian takes a single-molecule handle");
  repeats = std::max(1, std::min(repeats, 100));
  DevBuf hb;
  const size_t n3 = 3 * (size_t)std::max(h->natoms, 1);
  HF_CUDA(h, hb.ensure(sizeof(double) * n3 * n3));
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  HF_CUDA(h, cudaEventCreate(&e0));
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return fail(h, HFGPU_ERR_CUDA, "cudaEventCreate");
  }
  struct Restore {
    hfgpu_handle* h;
    cudaEvent_t a, b;
    DevBuf flush;
    ~Restore() {
      h->hess_class_mask = ~0u;
      cudaEventDestroy(a);
      cudaEventDestroy(b);
      flush.release();
    }
  } restore{h, e0, e1, DevBuf{}};
  if (restore.flush.ensure(kTunerFlushBytes) != cudaSuccess) {
    cudaGetLastError();
    restore.flush = DevBuf{};
  }
  auto hessian = [&]() { return hess_device_impl(h, D, 2.0, 1, D, 1.0, hb.as<double>()); };
  for (int c = 0; c < hfgpu::kNumClasses; ++c) {
    if (h->q_end[c] <= h->q_beg[c]) continue;
    h->hess_class_mask = 1u << c;
    float best = 1e30f;
    int best_form = 0;
    for (int form = 0; form < 4; ++form) {
      if (form == 3 && !hfgpu::kHessLaunchers[c]->has_line) continue;
      h->hess_cls_form[c] = form;
      float ms = 0.f;
      if ((rc = tuner_time(h, hessian, repeats, e0, e1, restore.flush, &ms))) return rc;
      if (ms < best) {
        best = ms;
        best_form = form;
      }
    }
    h->hess_cls_form[c] = best_form;
  }
  if (forms)
    for (int c = 0; c < hfgpu::kNumClasses; ++c) forms[c] = h->hess_cls_form[c];
  hb.release();
  return HFGPU_OK;
}

int hfgpu_autotune_grad(hfgpu_handle* h, const double* D, int precision, int repeats, int* forms) {
  if (!h || !D) return HFGPU_ERR_INVALID;
  DeviceGuard dev_guard(h);
  int rc = dev_guard.rc;
  if (rc) return rc;
  if (!h->have_geometry) return fail(h, HFGPU_ERR_STATE, "no geometry set");
  repeats = std::max(1, std::min(repeats, 100));
  DevBuf g;
  HF_CUDA(h, g.ensure(sizeof(double) * 3 * std::max(h->natoms, 1)));
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  HF_CUDA(h, cudaEventCreate(&e0));
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return fail(h, HFGPU_ERR_CUDA, "cudaEventCreate");
  }
  struct Restore {  // the class mask goes back and the flush buffer is freed on every exit path
    hfgpu_handle* h;
    cudaEvent_t a, b;
    DevBuf flush;
    ~Restore() {
      h->grad_class_mask = ~0u;
      cudaEventDestroy(a);
      cudaEventDestroy(b);
      flush.release();
    }
  } restore{h, e0, e1, DevBuf{}};
  if (restore.flush.ensure(kTunerFlushBytes) != cudaSuccess) {
    cudaGetLastError();  // no room for the flush buffer: time without it
    restore.flush = DevBuf{};
  }
  auto gradient = [&]() { return grad_device_impl(h, D, 2.0, 1, D, 1.0, g.as<double>(), precision); };
  // RHF weights (cJ = 2, cK = 1) on the given density, one class at a time, each form timed
  for (int c = 0; c < hfgpu::kNumClasses; ++c) {
    const hfgpu::ClassLaunchers* L = hfgpu::kClassLaunchers[c];
    if (!L->has_grad_warp || h->q_end[c] <= h->q_beg[c]) continue;
    h->grad_class_mask = 1u << c;
    float best = 1e30f;
    int best_form = 0;
    // thread, warp, warp split into four one-set passes, block of four or eight warps (whole, split)
    for (int form = 0; form < kGradForms; ++form) {
      h->grad_form[c] = form;
      float ms = 0.f;
      if ((rc = tuner_time(h, gradient, repeats, e0, e1, restore.flush, &ms))) return rc;
      if (ms < best) {
        best = ms;
        best_form = form;
      }
    }
    h->grad_form[c] = best_form;
  }
  // Classes were timed alone; in a gradient they run concurrently on several streams, where the
  // slower form of a class can overlap the others better.  Refinement on whole gradients: per
  // class the other form replaces the chosen one if the whole gradient gets at least 1% faster.
  h->grad_class_mask = ~0u;
  auto time_all = [&](float* ms) -> int {
    return tuner_time(h, gradient, std::max(repeats, 5), e0, e1, restore.flush, ms);
  };
  float cur = 0.f;
  if ((rc = time_all(&cur))) return rc;
  for (int c = 0; c < hfgpu::kNumClasses; ++c) {
    if (h->grad_form[c] < 0) continue;
    const int keep = h->grad_form[c];
    for (int form = 0; form < kGradForms; ++form) {
      if (form == keep) continue;
      const int before = h->grad_form[c];
      h->grad_form[c] = form;
      float ms = 0.f;
      if ((rc = time_all(&ms))) return rc;
      if (ms < 0.99f * cur)
        cur = ms;
      else
        h->grad_form[c] = before;
    }
  }
  // the classes concurrently on the auxiliary streams, or one after another
  {
    float t_conc = 0.f, t_ser = 0.f;
    for (int round = 0; round < 2; ++round)
      for (int ser = 0; ser < 2; ++ser) {
        h->grad_serial = ser;
        float ms = 0.f;
        if ((rc = time_all(&ms))) return rc;
        (ser ? t_ser : t_conc) += ms;
      }
    h->grad_serial = t_ser < 0.99f * t_conc ? 1 : 0;
  }
  if (forms)
    for (int c = 0; c < hfgpu::kNumClasses; ++c) forms[c] = h->grad_form[c];
  g.release();
  return HFGPU_OK;
}

int hfgpu_purify_device(hfgpu_handle* h, const double* Fo, int n, int nocc, int max_steps, double* P,
                        double* err) {
  if (!h || !Fo || !P || !err || n <= 0 || nocc < 0 || nocc > n || max_steps <= 0 || max_steps > 256)
    return fail(h, HFGPU_ERR_INVALID, "bad purification arguments");
  if (n > 4096) return fail(h, HFGPU_ERR_UNSUPPORTED, "purification: n > 4096");
  DeviceGuard dev_guard(h);
  if (dev_guard.rc) return dev_guard.rc;
  const size_t nn = (size_t)n * n;
  const int nslot = 3 * (max_steps + 1);
  HF_CUDA(h, h->d_purify.ensure(sizeof(double) * (nn + nslot + 2)));
  double* C = h->d_purify.as<double>();
  double* slots = C + nn;
  double* bounds = slots + nslot;
  // one cooperative launch when the device supports it and the grid fits at once
  if (h->purify_blocks < 0) {
    int coop = 0, sms = 0, per_sm = 0;
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, h->device);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device);
    if (coop && cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, purify_coop_kernel, kPurifyTile * kPurifyTile,
                                                              0) == cudaSuccess)
      h->purify_blocks = per_sm * sms;
    else
      h->purify_blocks = 0;
    cudaGetLastError();
  }
  if (h->purify_blocks > 0 && h->purify_coop) {
    const int nt = (n + kPurifyTile - 1) / kPurifyTile;
    int grid = std::min(nt * nt, h->purify_blocks);
    double tol = 1e-11;
    void* args[] = {(void*)&Fo, (void*)&n, (void*)&nocc, (void*)&max_steps, (void*)&tol, (void*)&P, (void*)&C,
                    (void*)&slots, (void*)&err};
    HF_CUDA(h, cudaLaunchCooperativeKernel((const void*)purify_coop_kernel, dim3(grid), dim3(kPurifyTile * kPurifyTile),
                                           args, 0, h->stream));
    HF_CHECK_LAUNCH(h, "cooperative purification");
    return HFGPU_OK;
  }
  purify_bounds_kernel<<<1, 1024, 0, h->stream>>>(Fo, n, slots, nslot, bounds);
  const int eb = (int)((nn + 255) / 256);
  purify_init_kernel<<<eb, 256, 0, h->stream>>>(Fo, n, bounds, P);
  const dim3 tiles((n + kPurifyTile - 1) / kPurifyTile, (n + kPurifyTile - 1) / kPurifyTile);
  for (int k = 0; k < max_steps; ++k) {
    purify_square_kernel<<<tiles, kPurifyTile * kPurifyTile, 0, h->stream>>>(P, n, C, slots + 3 * k);
    purify_update_kernel<<<eb, 256, 0, h->stream>>>(P, C, n, nocc, 1e-11, slots + 3 * k, slots + 3 * (k + 1), err);
  }
  HF_CHECK_LAUNCH(h, "purification");
  return HFGPU_OK;
}

int hfgpu_set_purify_mode(hfgpu_handle* h, int cooperative) {
  if (!h || cooperative < 0 || cooperative > 1) return HFGPU_ERR_INVALID;
  h->purify_coop = cooperative;
  return HFGPU_OK;
}

int hfgpu_device_status(hfgpu_handle* h, int* status) {
  if (!h || !status) return HFGPU_ERR_INVALID;
  DeviceGuard dev_guard(h);
  if (dev_guard.rc) return dev_guard.rc;
  int v = 0;
  HF_CUDA(h, cudaMemcpyAsync(&v, h->d_status.p, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  HF_CUDA(h, cudaMemsetAsync(h->d_status.p, 0, sizeof(int), h->stream));
  HF_CUDA(h, cudaStreamSynchronize(h->stream));
  *status = v;
  return HFGPU_OK;
}

int hfgpu_last_launches(const hfgpu_handle* h, int* kernels) {
  if (!h || !kernels) return HFGPU_ERR_INVALID;
  *kernels = h->last_kernels;
  return HFGPU_OK;
}

int hfgpu_boys(hfgpu_handle* h, int precision, int m, const double* T, long long count, double* F) {
  if (!h || !T || !F || count < 0 || m < 0 || m > BOYS_MMAX) return fail(h, HFGPU_ERR_INVALID, "bad Boys arguments");
  if (precision != HFGPU_FP64 && precision != HFGPU_MIXED) return fail(h, HFGPU_ERR_INVALID, "bad precision");
  for (long long i = 0; i < count; ++i)
    if (!(T[i] >= 0.0) || !std::isfinite(T[i])) return fail(h, HFGPU_ERR_INVALID, "T must be finite and >= 0");
  if (count == 0) return HFGPU_OK;
  DeviceGuard dev_guard(h);
  if (dev_guard.rc) return dev_guard.rc;
  DevBuf buf;
  const size_t nT = sizeof(double) * (size_t)count, nF = sizeof(double) * (size_t)count * (m + 1);
  HF_CUDA(h, buf.ensure(nT + nF));
  double* dT = buf.as<double>();
  double* dF = dT + count;
  int rc = HFGPU_OK;
  cudaError_t e = cudaMemcpyAsync(dT, T, nT, cudaMemcpyHostToDevice, h->stream);
  if (e == cudaSuccess) {
    if (precision == HFGPU_FP64)
      boys_eval_dispatch<double>(m, h->d_boys_d.as<double>(), dT, count, dF, h->stream);
    else
      boys_eval_dispatch<float>(m, h->d_boys_f.as<float>(), dT, count, dF, h->stream);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(F, dF, nF, cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) rc = cuda_fail(h, e, "Boys evaluation");
  buf.release();
  return rc;
}

int hfgpu_fp64_peak(int device, double* tflops) {
  if (!tflops) return HFGPU_ERR_INVALID;
  int prev = -1;
  if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
  struct Restore {
    int d;
    ~Restore() {
      if (d >= 0) cudaSetDevice(d);
    }
  } restore{prev};
  if (cudaSetDevice(device) != cudaSuccess) return HFGPU_ERR_CUDA;
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  double* out = nullptr;
  if (cudaMalloc(&out, sizeof(double)) != cudaSuccess) return HFGPU_ERR_NOMEM;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  const int iters = 20000, blocks = sms * 8, threads = 256;
  fp64_peak_kernel<<<blocks, threads>>>(out, 100, 1.0000001, 1e-7);
  double best = 0.0;
  for (int r = 0; r < 3; ++r) {
    cudaEventRecord(a);
    fp64_peak_kernel<<<blocks, threads>>>(out, iters, 1.0000001, 1e-7);
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    const double fl = 2.0 * 8.0 * iters * (double)blocks * threads;
    best = std::max(best, fl / (ms * 1e-3) / 1e12);
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(out);
  *tflops = best;
  return cudaGetLastError() == cudaSuccess ? HFGPU_OK : HFGPU_ERR_CUDA;
}

int hfgpu_batch_create(int nmol, const hfgpu_basis* bases, const double* const* xyz, const hfgpu_opts* opts,
                       hfgpu_handle** out) {
  if (nmol <= 0 || !bases || !xyz || !out) return HFGPU_ERR_INVALID;
  *out = nullptr;
  // concatenate the molecules into one basis; function indices stay local to each molecule
  std::vector<int> L, atom, nprim;
  std::vector<double> exps, coefs;
  std::vector<int> mol_shell(1, 0), mol_atom(1, 0);
  int natoms = 0;
  for (int m = 0; m < nmol; ++m) {
    const hfgpu_basis& b = bases[m];
    if (b.nshell <= 0 || b.natoms <= 0 || !b.L || !b.shell_atom || !b.nprim || !b.exps || !b.coefs || !xyz[m] ||
        b.pure)
      return HFGPU_ERR_INVALID;  // batched handles are Cartesian (s and p are identical either way)
    int np = 0;
    for (int s = 0; s < b.nshell; ++s) {
      L.push_back(b.L[s]);
      atom.push_back(b.shell_atom[s] + natoms);
      nprim.push_back(b.nprim[s]);
      np += b.nprim[s];
    }
    exps.insert(exps.end(), b.exps, b.exps + np);
    coefs.insert(coefs.end(), b.coefs, b.coefs + np);
    natoms += b.natoms;
    mol_shell.push_back((int)L.size());
    mol_atom.push_back(natoms);
  }
  hfgpu_opts o;
  if (opts) o = *opts; else hfgpu_default_opts(&o);
  o.density_tol = 0.0;  // the density bound is per molecule pair data; not used in batches
  hfgpu_basis all{(int)L.size(), natoms, 0, L.data(), atom.data(), nprim.data(), exps.data(), coefs.data()};
  hfgpu_handle* h = nullptr;
  int rc = hfgpu_create(&all, &o, &h);
  if (rc) return rc;
  h->batched = true;
  h->nmol = nmol;
  h->mol_shell = mol_shell;
  h->mol_atom = mol_atom;
  h->mol_n.assign(nmol, 0);
  h->mol_off.assign(nmol, 0);
  long long off = 0;
  for (int m = 0; m < nmol; ++m) {
    int f = 0;
    for (int s = mol_shell[m]; s < mol_shell[m + 1]; ++s) {
      h->first[s] = f;
      f += (L[s] + 1) * (L[s] + 2) / 2;
    }
    h->mol_n[m] = f;
    h->mol_off[m] = off;
    off += (long long)f * f;
  }
  h->first[h->nshell] = h->mol_n[nmol - 1];
  h->mat_total = off;
  h->n = *std::max_element(h->mol_n.begin(), h->mol_n.end());
  std::vector<unsigned char> mol_dev(sizeof(long long) * nmol + sizeof(int) * nmol);
  std::memcpy(mol_dev.data(), h->mol_off.data(), sizeof(long long) * nmol);
  std::memcpy(mol_dev.data() + sizeof(long long) * nmol, h->mol_n.data(), sizeof(int) * nmol);
  if (h->d_mol.ensure(mol_dev.size()) || cudaMemcpy(h->d_mol.p, mol_dev.data(), mol_dev.size(), cudaMemcpyHostToDevice)) {
    hfgpu_destroy(h);
    return HFGPU_ERR_CUDA;
  }
  std::vector<double> x;
  for (int m = 0; m < nmol; ++m) x.insert(x.end(), xyz[m], xyz[m] + 3 * bases[m].natoms);
  if ((rc = hfgpu_set_geometry(h, x.data(), natoms))) {
    hfgpu_destroy(h);
    return rc;
  }
  *out = h;
  return HFGPU_OK;
}

int hfgpu_batch_layout(const hfgpu_handle* h, int* nbf, long long* mat_off, long long* mat_total) {
  if (!h) return HFGPU_ERR_INVALID;
  for (int m = 0; m < h->nmol; ++m) {
    if (nbf) nbf[m] = h->mol_n[m];
    if (mat_off) mat_off[m] = h->mol_off[m];
  }
  if (mat_total) *mat_total = h->mat_total;
  return HFGPU_OK;
}

int hfgpu_batch_jk_device(hfgpu_handle* h, const double* D, double* J, double* K, int precision) {
  if (!h || !D || !J || !K) return HFGPU_ERR_INVALID;
  DeviceGuard dev_guard(h);
  int rc = dev_guard.rc;
  if (rc) return rc;
  return jk_device_impl(h, D, 1, D, J, K, precision);
}

int hfgpu_batch_grad2e_device(hfgpu_handle* h, const double* D, double* grad, int precision) {
  if (!h || !D || !grad) return HFGPU_ERR_INVALID;
  DeviceGuard dev_guard(h);
  int rc = dev_guard.rc;
  if (rc) return rc;
  return grad_device_impl(h, D, 2.0, 1, D, 1.0, grad, precision);
}

}  // extern "C"
