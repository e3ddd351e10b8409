// Batched-step launch entry points, one translation unit per order and precision.
#pragma once
#include <cuda_runtime.h>
#include "oux_batch.cuh"

namespace oux {
int batch_launch_fp64_o2(int dim, int vk, bool les, const BatchArgs<double>& B, int bps, int nsm, int* grid,
                         cudaStream_t s, int dry, bool konly);
int batch_launch_fp64_o4(int dim, int vk, bool les, const BatchArgs<double>& B, int bps, int nsm, int* grid,
                         cudaStream_t s, int dry, bool konly);
int batch_launch_fp64_o6(int dim, int vk, bool les, const BatchArgs<double>& B, int bps, int nsm, int* grid,
                         cudaStream_t s, int dry, bool konly);
int batch_launch_mx_o2(int dim, int vk, bool les, const BatchArgs<float>& B, int bps, int nsm, int* grid,
                       cudaStream_t s, int dry, bool konly);
int batch_launch_mx_o4(int dim, int vk, bool les, const BatchArgs<float>& B, int bps, int nsm, int* grid,
                       cudaStream_t s, int dry, bool konly);
int batch_launch_mx_o6(int dim, int vk, bool les, const BatchArgs<float>& B, int bps, int nsm, int* grid,
                       cudaStream_t s, int dry, bool konly);

// 0 = launched (or sized), 1 = CUDA error, 2 = no kernel built for the configuration
inline int batch_launch(int dim, int order, int vk, bool les, const BatchArgs<double>& B, int bps, int nsm,
                        int* grid, cudaStream_t s, int dry, bool konly) {
  if (order == 6) return batch_launch_fp64_o6(dim, vk, les, B, bps, nsm, grid, s, dry, konly);
  if (order == 4) return batch_launch_fp64_o4(dim, vk, les, B, bps, nsm, grid, s, dry, konly);
  return batch_launch_fp64_o2(dim, vk, les, B, bps, nsm, grid, s, dry, konly);
}
inline int batch_launch(int dim, int order, int vk, bool les, const BatchArgs<float>& B, int bps, int nsm,
                        int* grid, cudaStream_t s, int dry, bool konly) {
  if (order == 6) return batch_launch_mx_o6(dim, vk, les, B, bps, nsm, grid, s, dry, konly);
  if (order == 4) return batch_launch_mx_o4(dim, vk, les, B, bps, nsm, grid, s, dry, konly);
  return batch_launch_mx_o2(dim, vk, les, B, bps, nsm, grid, s, dry, konly);
}
}  // namespace oux
