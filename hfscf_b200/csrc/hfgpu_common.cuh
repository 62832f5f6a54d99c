// Device-side data layout and helpers shared by the two-electron kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define PI_2_5 34.986836655249725  // 2 pi^(5/2), hfscfmath::PI_25 (src/math/hfscf_math.hpp:25)

// ---------------------------------------------------------------------------
// Primitive pair of a shell pair (a b): p = alpha_a + alpha_b, ip = 1/p, P,
// PA = P - A and Kp = K sqrt(2 pi^2.5) / p with K = exp(-alpha_a alpha_b / p |AB|^2) c_a c_b
// (BASIS::ShellPair::set_params, src/integrals/hfscf_shellpair.cpp:33-61).  Kp is
// scaled so that the [00|00] prefactor K_ab K_cd 2 pi^2.5 / (p q sqrt(p+q)) is
// Kp_ab Kp_cd / sqrt(p+q).  eb2 is the square of the ket exponent, used only by the
// kinetic-energy integrals (for a folded self pair, the mean over (i, j) and (j, i)).
// 80 bytes in FP64 (five 16-byte loads).
// ---------------------------------------------------------------------------
template <typename R>
struct __align__(sizeof(R) * 2) PrimPair {
  R p, ip, Px, Py, Pz, PAx, PAy, PAz, Kp, eb2;
};

// One canonical shell pair (La >= Lb after an optional swap of the two shells).
struct PairInfo {
  int sa, sb;        // shell indices
  int fa, fb;        // first function of each shell in the final (pure or Cartesian) basis
  int prim_off;      // first primitive pair
  int nprim;         // primitive pairs kept
  int cls;           // pair class: 0 ss, 1 ps, 2 pp, 3 ds, 4 dp, 5 dd
  int atom_a, atom_b;
  int mol;           // molecule of a batched handle (0 otherwise); fa, fb are local to it
  double ABx, ABy, ABz;  // A - B
  double schwarz;        // sqrt(max |(ab|ab)|) over the pair's functions
};

// Status word written by kernels that detect a problem (bad input seen on device).
enum : int { HFGPU_DEV_OK = 0, HFGPU_DEV_NONFINITE = 1 };

template <typename R>
__device__ __forceinline__ R sqrt_t(R x);
template <>
__device__ __forceinline__ double sqrt_t<double>(double x) { return sqrt(x); }
template <>
__device__ __forceinline__ float sqrt_t<float>(float x) { return sqrtf(x); }
// Exact value of a small non-negative int (0 <= k < 2^22) without an int -> float
// conversion instruction (those issue on the narrow XU pipe): k is written into the low
// mantissa bits of 1.5 * 2^52 (1.5 * 2^23 in FP32) and the offset subtracted.
template <typename R>
__device__ __forceinline__ R small_int(int k);
template <>
__device__ __forceinline__ double small_int<double>(int k) {
  return __hiloint2double(0x43380000, k) - 6755399441055744.0;
}
template <>
__device__ __forceinline__ float small_int<float>(int k) {
  return __int_as_float(0x4B400000 | k) - 12582912.0f;
}

template <typename R>
__device__ __forceinline__ R exp_t(R x);
template <>
__device__ __forceinline__ double exp_t<double>(double x) { return exp(x); }
template <>
__device__ __forceinline__ float exp_t<float>(float x) { return expf(x); }
template <typename R>
__device__ __forceinline__ R rsqrt_t(R x);
template <>
__device__ __forceinline__ double rsqrt_t<double>(double x) { return rsqrt(x); }
template <>
__device__ __forceinline__ float rsqrt_t<float>(float x) { return rsqrtf(x); }

// ---------------------------------------------------------------------------
// Boys function F_m(T), m = 0..M, scaled by `pre`.
//
// Method (Gill, Johnson & Pople, Int. J. Quantum Chem. 40, 745 (1991); Helgaker,
// Jorgensen & Olsen, "Molecular Electronic-Structure Theory", sec. 9.8.2):
//   T <  BOYS_TMAX: Taylor expansion of F_M about the nearest grid point T_k = k h
//                  (h = 0.1), F_M(T) = sum_j F_{M+j}(T_k) (-dT)^j / j!, j = 0..6 in FP64
//                  (0..3 in FP32), then the stable downward recursion
//                  F_{m-1} = (2T F_m + e^-T) / (2m - 1), where (FP64) e^-T = e^-T_k e^(T_k - T)
//                  with e^-T_k tabulated and e^d, |d| <= h/2, from its degree-8 Taylor
//                  polynomial (remainder below (h/2)^9 / 9! = 5e-18 relative);
//   T >= BOYS_TMAX: F_0 = sqrt(pi/T)/2 (erf(sqrt T) = 1 to double precision there)
//                  and the upward recursion F_{m+1} = ((2m+1) F_m - e^-T) / (2T).
// Table layout: one row of 8 values per (order M, grid point k), rows of one order
// contiguous.  FP64 row: F_{M+j}(T_k) / j!, j = 0..6, then e^-T_k (64 bytes, four 16-byte
// loads give the whole expansion); FP32 row: F_{M+j}(T_k) / j!, j = 0..3, then e^-T_k and
// padding (32 bytes).  The values F_m(T_k) are computed on the host from the convergent
// series F_m(T) = e^-T sum_i (2T)^i / ((2m+1)(2m+3)...(2m+2i+1)) in long double.
// ---------------------------------------------------------------------------
#define BOYS_H 0.1
#define BOYS_NGRID 361           // T_k = 0 .. 36
#define BOYS_TMAX 36.0
#define BOYS_MMAX 10             // orders M = 0 .. 10 have rows
#define BOYS_NM 18               // m = 0 .. 17 computed on the host (M <= 10 plus 7 Taylor terms)
#define BOYS_ROW 8               // values per row

template <typename R>
struct BoysTable {
  const R* __restrict__ tab;  // [BOYS_MMAX + 1][BOYS_NGRID][BOYS_ROW]

  template <int M>
  __device__ __forceinline__ void eval(R T, R pre, R* F) const {
    static_assert(M <= BOYS_MMAX, "Boys order beyond the table");
    if (T < R(BOYS_TMAX)) {
      int k;
      R d;  // -(T - T_k)
      if constexpr (sizeof(R) == 8) {
        // nearest grid index without int/float conversions (they go through the narrow XU
        // pipe): adding 1.5 * 2^52 leaves round(T / h) in the low mantissa bits
        const double sh = T * 10.0 + 6755399441055744.0;
        k = __double2loint(sh);
        d = (sh - 6755399441055744.0) * BOYS_H - T;
      } else {
        k = __float2int_rn(T * R(10));
        d = R(k) * R(BOYS_H) - T;
      }
      const R* row = tab + ((size_t)M * BOYS_NGRID + k) * BOYS_ROW;
      R f;
      R ek;  // e^-T_k
      if constexpr (sizeof(R) == 8) {
        const double2* r = reinterpret_cast<const double2*>(row);
        const double2 r0 = r[0], r1 = r[1], r2 = r[2], r3 = r[3];
        f = r3.x;
        f = r2.y + f * d;
        f = r2.x + f * d;
        f = r1.y + f * d;
        f = r1.x + f * d;
        f = r0.y + f * d;
        f = r0.x + f * d;
        ek = r3.y;
      } else {
        const float4* r = reinterpret_cast<const float4*>(row);
        const float4 r0 = r[0];
        f = r0.w;
        f = r0.z + f * d;
        f = r0.y + f * d;
        f = r0.x + f * d;
        ek = R(0);
      }
      F[M] = f;
      if constexpr (M > 0) {
        R e;
        if constexpr (sizeof(R) == 8) {
          R x = R(1.0 / 40320.0);
          x = R(1.0 / 5040.0) + d * x;
          x = R(1.0 / 720.0) + d * x;
          x = R(1.0 / 120.0) + d * x;
          x = R(1.0 / 24.0) + d * x;
          x = R(1.0 / 6.0) + d * x;
          x = R(0.5) + d * x;
          x = R(1.0) + d * x;
          x = R(1.0) + d * x;
          e = ek * x;
        } else {
          (void)ek;
          e = exp_t<R>(-T);
        }
        const R t2 = T + T;
#pragma unroll
        for (int m = M; m > 0; --m) F[m - 1] = (t2 * F[m] + e) * R(1.0 / (2 * m - 1));
      }
    } else {
      const R rt = rsqrt_t<R>(T);
      const R it = rt * rt;
      F[0] = R(0.88622692545275801365) * rt;  // sqrt(pi)/2 / sqrt(T)
      if constexpr (M > 0) {
        const R e = exp_t<R>(-T);
        const R h = R(0.5) * it;
#pragma unroll
        for (int m = 0; m < M; ++m) F[m + 1] = (R(2 * m + 1) * F[m] - e) * h;
      }
    }
#pragma unroll
    for (int m = 0; m <= M; ++m) F[m] *= pre;
  }
};

__host__ __device__ constexpr int ncart_of(int L) { return (L + 1) * (L + 2) / 2; }
__host__ __device__ constexpr int npure_of(int L) { return 2 * L + 1; }

// ---------------------------------------------------------------------------
// Boys table of one order staged in shared memory.
//
// The same expansion as BoysTable::eval, reading the table of the kernel's single order MS
// from shared memory, where a block puts it once with one bulk copy (stage_boys_table).  The
// rows are stored as planes: FP64 plane j (j = 0..3) holds the 16-byte pair (value 2j, value
// 2j+1) of every grid point, so the four 16-byte loads of one evaluation go to four planes and
// the lanes of a warp, holding different T, spread over the banks by grid point instead of all
// hitting the same four banks of their 64-byte rows; FP32 has one plane of float4 (values
// 0..3).  Global layout: per order, the planes back to back (BOYS_PLANE_BYTES(R) bytes).
// ---------------------------------------------------------------------------
#define BOYS_PLANES_D 4
#define BOYS_PLANE_BYTES_D (BOYS_PLANES_D * BOYS_NGRID * 16)  // 23104 bytes per FP64 order
#define BOYS_PLANE_BYTES_F (BOYS_NGRID * 16)                  // 5776 bytes per FP32 order

template <typename R>
__host__ __device__ constexpr int boys_plane_bytes() {
  return sizeof(R) == 8 ? BOYS_PLANE_BYTES_D : BOYS_PLANE_BYTES_F;
}

template <typename R, int MS>
struct BoysShared {
  const R* tab;  // shared memory: the planes of order MS

  template <int M>
  __device__ __forceinline__ void eval(R T, R pre, R* F) const {
    static_assert(M == MS, "the staged table holds one order");
    if (T < R(BOYS_TMAX)) {
      int k;
      R d;
      if constexpr (sizeof(R) == 8) {
        const double sh = T * 10.0 + 6755399441055744.0;
        k = __double2loint(sh);
        d = (sh - 6755399441055744.0) * BOYS_H - T;
      } else {
        k = __float2int_rn(T * R(10));
        d = R(k) * R(BOYS_H) - T;
      }
      R f, ek;
      if constexpr (sizeof(R) == 8) {
        const double2* P = reinterpret_cast<const double2*>(tab);
        const double2 r0 = P[k], r1 = P[BOYS_NGRID + k], r2 = P[2 * BOYS_NGRID + k], r3 = P[3 * BOYS_NGRID + k];
        f = r3.x;
        f = r2.y + f * d;
        f = r2.x + f * d;
        f = r1.y + f * d;
        f = r1.x + f * d;
        f = r0.y + f * d;
        f = r0.x + f * d;
        ek = r3.y;
      } else {
        const float4 r0 = reinterpret_cast<const float4*>(tab)[k];
        f = r0.w;
        f = r0.z + f * d;
        f = r0.y + f * d;
        f = r0.x + f * d;
        ek = R(0);
      }
      F[M] = f;
      if constexpr (M > 0) {
        R e;
        if constexpr (sizeof(R) == 8) {
          R x = R(1.0 / 40320.0);
          x = R(1.0 / 5040.0) + d * x;
          x = R(1.0 / 720.0) + d * x;
          x = R(1.0 / 120.0) + d * x;
          x = R(1.0 / 24.0) + d * x;
          x = R(1.0 / 6.0) + d * x;
          x = R(0.5) + d * x;
          x = R(1.0) + d * x;
          x = R(1.0) + d * x;
          e = ek * x;
        } else {
          (void)ek;
          e = exp_t<R>(-T);
        }
        const R t2 = T + T;
#pragma unroll
        for (int m = M; m > 0; --m) F[m - 1] = (t2 * F[m] + e) * R(1.0 / (2 * m - 1));
      }
    } else {
      const R rt = rsqrt_t<R>(T);
      const R it = rt * rt;
      F[0] = R(0.88622692545275801365) * rt;
      if constexpr (M > 0) {
        const R e = exp_t<R>(-T);
        const R h = R(0.5) * it;
#pragma unroll
        for (int m = 0; m < M; ++m) F[m + 1] = (R(2 * m + 1) * F[m] - e) * h;
      }
    }
#pragma unroll
    for (int m = 0; m <= M; ++m) F[m] *= pre;
  }
};

// Status codes a kernel leaves in its status word (device int, 0 = fine).
enum : int { HFGPU_DEV_STAGE_TIMEOUT = 2, HFGPU_DEV_ABORTED = 3 };
// Polls of a bounded mbarrier wait (each followed by a short sleep): about 0.1 s in all.
#define HFGPU_STAGE_MAX_POLLS (1 << 20)

// Copies `bytes` (a multiple of 16; both addresses 16-byte aligned) from global memory into
// this block's shared memory with one bulk copy of the TMA unit (cp.async.bulk, completing on
// the mbarrier `mbar` in shared memory), called by every thread of the block.  The wait for the
// copy is bounded: after HFGPU_STAGE_MAX_POLLS polls the block records
// HFGPU_DEV_STAGE_TIMEOUT in *status and the function returns false (every thread gets the same
// answer).  issue = false arms the barrier for `bytes` without issuing any copy, so that the
// wait runs out: the bounded-wait test, never used by a build.
__device__ __forceinline__ bool stage_to_shared(void* smem_dst, const void* gmem_src, unsigned bytes,
                                                unsigned long long* mbar, int* status, bool issue = true) {
  const unsigned mb = (unsigned)__cvta_generic_to_shared(mbar);
  const unsigned dst = (unsigned)__cvta_generic_to_shared(smem_dst);
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mb) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mb), "r"(bytes) : "memory");
    if (issue)
      asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                   "l"(gmem_src), "r"(bytes), "r"(mb)
                   : "memory");
  }
  unsigned done = 0;
  for (int i = 0; i < HFGPU_STAGE_MAX_POLLS; ++i) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.test_wait.parity.shared::cta.b64 p, [%1], 0;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(mb)
        : "memory");
    if (done) break;
    __nanosleep(64);
  }
  const int ok = __syncthreads_and(done != 0);
  if (!ok) {
    if (threadIdx.x == 0 && status != nullptr) atomicExch(status, HFGPU_DEV_STAGE_TIMEOUT);
    // a copy that was issued may still be in flight: give it one more bounded wait before the
    // block leaves (and its shared memory goes to another block)
    if (issue) {
      for (int i = 0; i < HFGPU_STAGE_MAX_POLLS && !done; ++i) {
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.test_wait.parity.shared::cta.b64 p, [%1], 0;\n\tselp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(mb)
            : "memory");
        if (!done) __nanosleep(64);
      }
    }
    __syncthreads();
  }
  return ok != 0;
}
