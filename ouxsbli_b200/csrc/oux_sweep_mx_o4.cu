// Mixed-form sweep instantiations for convective order 4: FP32 fields and face
// fluxes, FP64 flux differences and stage combinations (FMA contraction allowed).
#include "oux_dispatch.h"
#include "oux_launch.cuh"

namespace oux {
int launch_sweeps_mx_o4(int dim, int vk, bool les, int dir, const StepArgs<float>& A, cudaStream_t s) {
#define OUX_CASE(D, V, L)                                                                     \
  if (dim == D && vk == V && les == L)                                                        \
    return dir < 0 ? launch_stage_sweeps<D, 4, V, L, float>(A, s)                            \
                   : launch_stage_sweep_dir<D, 4, V, L, float>(A, dir, s);
  OUX_CASE(3, VK_EULER, false) OUX_CASE(3, VK_C4, false) OUX_CASE(3, VK_GV2, false)
  OUX_CASE(3, VK_C4W, false) OUX_CASE(3, VK_GV2W, false) OUX_CASE(3, VK_C4W, true) OUX_CASE(3, VK_GV2W, true)
  OUX_CASE(3, VK_C4, true) OUX_CASE(3, VK_GV2, true)
  OUX_CASE(2, VK_EULER, false) OUX_CASE(2, VK_2D4, false) OUX_CASE(2, VK_GV2, false)
#undef OUX_CASE
  return 2;
}
}  // namespace oux
