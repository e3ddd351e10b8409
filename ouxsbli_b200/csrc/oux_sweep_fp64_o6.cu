// FP64 sweep instantiations for convective order 6 (compiled without FMA
// contraction so the arithmetic matches the reference operation by operation).
#include "oux_dispatch.h"
#include "oux_launch.cuh"

namespace oux {
int launch_sweeps_fp64_o6(int dim, int vk, bool les, const StepArgs<double>& A, cudaStream_t s) {
#define OUX_CASE(D, V, L) \
  if (dim == D && vk == V && les == L) return launch_stage_sweeps<D, 6, V, L, double>(A, s);
  OUX_CASE(3, VK_EULER, false) OUX_CASE(3, VK_C6, false) OUX_CASE(3, VK_C4, false) OUX_CASE(3, VK_ME4, false)
  OUX_CASE(3, VK_C6W, false) OUX_CASE(3, VK_C4W, false) OUX_CASE(3, VK_ME4W, false)
  OUX_CASE(3, VK_C6W, true) OUX_CASE(3, VK_C4W, true) OUX_CASE(3, VK_ME4W, true)
  OUX_CASE(3, VK_C6, true) OUX_CASE(3, VK_C4, true) OUX_CASE(3, VK_ME4, true)
  OUX_CASE(2, VK_EULER, false) OUX_CASE(2, VK_2D4, false) OUX_CASE(2, VK_GV2, false)
#undef OUX_CASE
  return 2;
}

int launch_sweep_dir_fp64_o6(int dim, int vk, bool les, int dir, const StepArgs<double>& A, cudaStream_t s) {
#define OUX_CASE(D, V, L) \
  if (dim == D && vk == V && les == L) return launch_stage_sweep_dir<D, 6, V, L, double>(A, dir, s);
  OUX_CASE(3, VK_EULER, false) OUX_CASE(3, VK_C6, false) OUX_CASE(3, VK_C4, false) OUX_CASE(3, VK_ME4, false)
  OUX_CASE(3, VK_C6W, false) OUX_CASE(3, VK_C4W, false) OUX_CASE(3, VK_ME4W, false)
  OUX_CASE(3, VK_C6W, true) OUX_CASE(3, VK_C4W, true) OUX_CASE(3, VK_ME4W, true)
  OUX_CASE(3, VK_C6, true) OUX_CASE(3, VK_C4, true) OUX_CASE(3, VK_ME4, true)
  OUX_CASE(2, VK_EULER, false) OUX_CASE(2, VK_2D4, false) OUX_CASE(2, VK_GV2, false)
#undef OUX_CASE
  return 2;
}
}  // namespace oux
