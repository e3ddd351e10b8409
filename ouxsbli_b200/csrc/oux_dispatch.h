// Sweep-launch entry points, one translation unit per convective order so the
// template instantiations compile in parallel.
#pragma once
#include <cuda_runtime.h>
#include "oux_kernels.cuh"

namespace oux {
int launch_sweeps_fp64_o2(int dim, int vk, bool les, const StepArgs<double>& A, cudaStream_t s);
int launch_sweeps_fp64_o4(int dim, int vk, bool les, const StepArgs<double>& A, cudaStream_t s);
int launch_sweeps_fp64_o6(int dim, int vk, bool les, const StepArgs<double>& A, cudaStream_t s);

int launch_sweep_dir_fp64_o2(int dim, int vk, bool les, int dir, const StepArgs<double>& A, cudaStream_t s);
int launch_sweep_dir_fp64_o4(int dim, int vk, bool les, int dir, const StepArgs<double>& A, cudaStream_t s);
int launch_sweep_dir_fp64_o6(int dim, int vk, bool les, int dir, const StepArgs<double>& A, cudaStream_t s);

// one sweep direction (used when per-kernel timing is on)
inline int launch_sweep_dir_fp64(int dim, int order, int vk, bool les, int dir, const StepArgs<double>& A,
                                 cudaStream_t s) {
  if (order == 6) return launch_sweep_dir_fp64_o6(dim, vk, les, dir, A, s);
  if (order == 4) return launch_sweep_dir_fp64_o4(dim, vk, les, dir, A, s);
  return launch_sweep_dir_fp64_o2(dim, vk, les, dir, A, s);
}

inline int launch_sweeps_fp64(int dim, int order, int vk, bool les, const StepArgs<double>& A, cudaStream_t s) {
  if (order == 6) return launch_sweeps_fp64_o6(dim, vk, les, A, s);
  if (order == 4) return launch_sweeps_fp64_o4(dim, vk, les, A, s);
  return launch_sweeps_fp64_o2(dim, vk, les, A, s);
}
// mixed form (FP32 fields and face fluxes)
int launch_sweeps_mx_o2(int dim, int vk, bool les, int dir, const StepArgs<float>& A, cudaStream_t s);
int launch_sweeps_mx_o4(int dim, int vk, bool les, int dir, const StepArgs<float>& A, cudaStream_t s);
int launch_sweeps_mx_o6(int dim, int vk, bool les, int dir, const StepArgs<float>& A, cudaStream_t s);
inline int launch_sweep_dir_mx(int dim, int order, int vk, bool les, int dir, const StepArgs<float>& A,
                               cudaStream_t s) {
  if (order == 6) return launch_sweeps_mx_o6(dim, vk, les, dir, A, s);
  if (order == 4) return launch_sweeps_mx_o4(dim, vk, les, dir, A, s);
  return launch_sweeps_mx_o2(dim, vk, les, dir, A, s);
}
inline int launch_sweeps_mx(int dim, int order, int vk, bool les, const StepArgs<float>& A, cudaStream_t s) {
  return launch_sweep_dir_mx(dim, order, vk, les, -1, A, s);
}
}  // namespace oux
