// Host-visible launchers of the per-class adjoint Hessian kernels (one translation unit per class,
// generated by gen_eri.py next to the J/K and gradient units).
#pragma once
#include <cuda_runtime.h>

template <typename R>
struct GradArgs;
struct HessOut;

namespace hfgpu {

struct HessLaunchers {
  int la, lb, lc, ld;
  // hess_kernel over quartets q[0, nq) with grid blocks of 128 threads and smem bytes of
  // dynamic shared memory (0: atomics straight into the output)
  void (*launch)(const GradArgs<double>&, const HessOut&, int pure, const int2* q, int nq, int grid, int smem,
                 cudaStream_t);
  int (*scratch_slots)(int pure);  // doubles of scratch per thread
  // block form (hess_block_kernel, one block of 128 threads per quartet, grid-stride); false when
  // the class's tables do not fit one block's shared memory
  bool (*launch_block)(const GradArgs<double>&, const HessOut&, int pure, const int2* q, int nq, int grid,
                       cudaStream_t);
  int (*block_global_slots)();  // doubles of global scratch per block of the block form (0: none)
  // warp form (hess_block_kernel with one warp per quartet, four per block); false when four
  // quartets' tables do not fit one block's shared memory
  bool (*launch_warp)(const GradArgs<double>&, const HessOut&, int pure, const int2* q, int nq, cudaStream_t);
  // straight-line form (hess_line_kernel, one thread per quartet on register code, grid blocks of
  // 128 threads; smem as for launch, to which the launcher adds the threads' 45-entry slices);
  // false when the class has none
  bool has_line;
  bool (*launch_line)(const GradArgs<double>&, const HessOut&, int pure, const int2* q, int nq, int grid, int smem,
                      cudaStream_t);
};

extern const HessLaunchers* const kHessLaunchers[];
extern const int kNumHessClasses;

}  // namespace hfgpu
