// Mixed-form batched-step instantiations for convective order 2.
#include "oux_batch_dispatch.h"
#include "oux_batch_launch.cuh"

namespace oux {
int batch_launch_mx_o2(int dim, int vk, bool les, const BatchArgs<float>& B, int bps, int nsm, int* grid,
                       cudaStream_t s, int dry, bool konly) {
#define OUX_CASE(D, V, L) \
  if (dim == D && vk == V && les == L) return konly ? batch_launch_t<D, 2, V, L, float, true>(B, bps, nsm, grid, s, dry) \
                 : batch_launch_t<D, 2, V, L, float, false>(B, bps, nsm, grid, s, dry);
  OUX_CASE(3, VK_EULER, false) OUX_CASE(3, VK_GV2, false) OUX_CASE(3, VK_GV2, true)
  OUX_CASE(2, VK_EULER, false) OUX_CASE(2, VK_GV2, false) OUX_CASE(2, VK_2D4, false)
#undef OUX_CASE
  return 2;
}
}  // namespace oux
