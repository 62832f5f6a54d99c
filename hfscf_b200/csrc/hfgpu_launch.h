// Host-visible launchers of the per-class kernels (one translation unit per class).
#pragma once
#include <cuda_runtime.h>

template <typename R>
struct QuartetArgs;
template <typename R>
struct GradArgs;

namespace hfgpu {

struct ClassLaunchers {
  int la, lb, lc, ld;
  void (*quartet_d)(const QuartetArgs<double>&, const int2*, int, cudaStream_t);
  void (*quartet_f)(const QuartetArgs<float>&, const int2*, int, cudaStream_t);
  void (*grad_d)(const GradArgs<double>&, int pure, const int2*, int, int grid, cudaStream_t);
  void (*grad_f)(const GradArgs<float>&, int pure, const int2*, int, int grid, cudaStream_t);
  int (*grad_scratch_slots)(int pure);  // per-thread scratch of table-mode gradient classes (0 otherwise)
  bool has_primwarp;                     // warp-over-primitives kernel for high-contraction quartets
  bool (*primwarp_d)(const QuartetArgs<double>&, const int2*, int, cudaStream_t);
  bool (*primwarp_f)(const QuartetArgs<float>&, const int2*, int, cudaStream_t);
  bool has_warp;                         // warp-per-quartet form with levelised tables
  bool warp_default;                     // ... used unless the schedule or opts say otherwise
  bool has_grad_warp;                    // warp-per-quartet adjoint gradient (shared memory, no scratch)
  bool (*grad_warp_d)(const GradArgs<double>&, int pure, const int2*, int, cudaStream_t);
  bool (*grad_warp_f)(const GradArgs<float>&, int pure, const int2*, int, cudaStream_t);
  int (*grad_warp_bytes)(int fp32);      // shared memory of one warp-form block (0: no warp form)
  bool has_capped;                       // register-capped variant of the thread-per-quartet form
  bool has_staged;                       // persistent thread form with the Boys table in shared memory
  bool has_lowres;                       // low-residency variant of the thread form (classes that spill)
};

extern const ClassLaunchers* const kClassLaunchers[];
extern const int kNumClasses;

}  // namespace hfgpu
