// Grid/block/shared-memory setup for the three sweeps of one stage.
#pragma once
#include <cstring>
#include "oux_sweep.cuh"

namespace oux {

template <int DIM, int DIR, int ORDER, int VK, bool LES, class T, bool SHARE = false>
int launch_one(const StepArgs<T>& A, int last, cudaStream_t s) {
  // ME4 on an axis of uniform spacing: the shared-position variant of the x and y
  // sweeps (measured on B200 at 512^3: y 9.98 -> 9.66 ms, x unchanged; the z sweep,
  // whose operand prefetch already holds 82 KB of shared memory per block, lost L1
  // capacity to the extra 20 KB and ran slower, 11.1 -> 14.3 ms)
  if constexpr (VK == VK_ME4 && !SHARE && DIR < 2) {
    if ((A.G.uni >> DIR) & 1) return launch_one<DIM, DIR, ORDER, VK, LES, T, true>(A, last, s);
  }
  constexpr size_t smem = sweep_smem<ORDER, DIR, T, default_rows<DIR>(), sweep_tma<DIM, DIR, VK>()>() +
                          sweep_pf_bytes<DIR, T>(sweep_pf_mode<DIM, DIR, T>()) +
                          (SHARE ? me4_share_bytes<DIR, T, LES>() : 0);
  constexpr bool TM = sweep_tma<DIM, DIR, VK>();
  const void* fn;
  if constexpr (TM) fn = (const void*)k_sweep_tm<DIM, DIR, ORDER, VK, LES, T, SHARE>;
  else fn = (const void*)k_sweep<DIM, DIR, ORDER, VK, LES, T, SHARE>;
  static const cudaError_t attr_rc = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (attr_rc != cudaSuccess) return 1;
  const Geo& G = A.G;
  const int g = G.g;
  const int Nx = G.nx - 2 * G.gx, Ny = G.ny - 2 * G.gy, Nz = DIM == 3 ? G.sk1 - G.sk0 : 1;
  if (Nz <= 0) return 0;  // an empty part of a split stage
  dim3 block(sweep_threads<DIR>(), 1, 1);
  dim3 grid;
  if (DIR == 0) grid = dim3((Nx + 31) / 32, (Ny + SWEEP_BR - 1) / SWEEP_BR, Nz);
  else if (DIR == 1) grid = dim3((Nx + 31) / 32, (Ny + SWEEP_BF - 1) / SWEEP_BF, Nz);
  else grid = dim3((Nx + 31) / 32, (Nz + SWEEP_BZ - 1) / SWEEP_BZ, Ny);
  if constexpr (TM) {
    // this direction's tile tensor maps from the handle (A.tmaps, a host address)
    SweepMaps maps;
    if (A.tmaps) std::memcpy(&maps, static_cast<const unsigned char*>(A.tmaps) + DIR * sizeof(SweepMaps),
                             sizeof(SweepMaps));
    else std::memset(&maps, 0, sizeof(SweepMaps));
    k_sweep_tm<DIM, DIR, ORDER, VK, LES, T, SHARE><<<grid, block, smem, s>>>(A, last, maps, A.tmaps ? 1 : 0);
  } else {
    k_sweep<DIM, DIR, ORDER, VK, LES, T, SHARE><<<grid, block, smem, s>>>(A, last);
  }
  return cudaPeekAtLastError() == cudaSuccess ? 0 : 1;
}

template <int DIM, int ORDER, int VK, bool LES, class T>
int launch_stage_sweeps(const StepArgs<T>& A, cudaStream_t s) {
  if (launch_one<DIM, 0, ORDER, VK, LES, T>(A, 0, s)) return 1;
  if constexpr (DIM == 3) {
    if (launch_one<DIM, 1, ORDER, VK, LES, T>(A, 0, s)) return 1;
    return launch_one<DIM, 2, ORDER, VK, LES, T>(A, 1, s);
  } else {
    return launch_one<DIM, 1, ORDER, VK, LES, T>(A, 1, s);
  }
}

template <int DIM, int ORDER, int VK, bool LES, class T>
int launch_stage_sweep_dir(const StepArgs<T>& A, int dir, cudaStream_t s) {
  if (dir == 0) return launch_one<DIM, 0, ORDER, VK, LES, T>(A, 0, s);
  if constexpr (DIM == 3) {
    if (dir == 1) return launch_one<DIM, 1, ORDER, VK, LES, T>(A, 0, s);
    return launch_one<DIM, 2, ORDER, VK, LES, T>(A, 1, s);
  } else {
    return launch_one<DIM, 1, ORDER, VK, LES, T>(A, 1, s);
  }
}

}  // namespace oux
