// Launch of the batched step kernel: grid = SMs x resident blocks per SM (or the
// caller's cap), never more blocks than work items.
#pragma once
#include "oux_batch.cuh"

namespace oux {

// dry != 0: set the kernel's shared-memory attribute, size the grid into *grid
// and launch nothing (done once, outside any stream capture).  dry == 0: launch
// with the grid sized before.
template <int DIM, int ORDER, int VK, bool LES, class T, bool KONLY>
int batch_launch_t(const BatchArgs<T>& B, int blocks_per_sm, int nsm, int* grid, cudaStream_t s, int dry) {
  constexpr size_t smem = batch_smem<ORDER, T>();
  auto kern = k_batch_step<DIM, ORDER, VK, LES, T, KONLY>;
  if (dry) {
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
      return 1;
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, BATCH_THREADS, smem) != cudaSuccess || occ < 1)
      return 1;
    const int bps = (blocks_per_sm > 0 && blocks_per_sm < occ) ? blocks_per_sm : occ;
    int g = nsm * bps;
    if (g > B.nitems) g = B.nitems > 0 ? B.nitems : 1;
    *grid = g;
    return 0;
  }
  kern<<<*grid, BATCH_THREADS, smem, s>>>(B);
  return cudaPeekAtLastError() == cudaSuccess ? 0 : 1;
}

}  // namespace oux
