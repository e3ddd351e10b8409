// Batched time step: many independent periodic solves (uneven grids, one
// physics configuration) advanced by ONE persistent kernel per time step.
//
// Work list.  A step is a fixed sequence of phases (per stage: primitives,
// [sensor], [SGS viscosity, its edge copy], x / y / [z] sweeps, ghost fill).
// The host enumerates items phase-major: for every phase, for every solve, the
// solve's tiles of that phase grouped `pencil` (sweeps) or `chunk` cells
// (point-wise phases) per item.  Blocks claim items in list order from one
// atomic counter.
//
// Dependencies.  Within a solve the phases form a chain: an item of phase p
// may start once every item of the solve's previous non-empty phase is done
// (a per-(solve, phase) completion counter).  Different solves never wait on
// each other, so a block rarely waits: by the time it claims phase p of solve
// i, phase p-1 of every solve has been claimed and mostly finished.
//
// Progress.  An item only waits on items earlier in the list, which were
// claimed earlier by blocks that are running, so every wait ends.  Each wait is
// still bounded: after spin_limit polls (OUX_BATCH_SPIN_LIMIT unless the batch
// sets another) the block sets OUX_FAULT_TIMEOUT in the batch status word and
// returns.
//
// Memory ordering.  A block publishes an item with __syncthreads, a gpu-scope
// fence and a relaxed atomic add (release); a waiting block polls with
// ld.acquire.gpu and then __syncthreads, so its later ordinary loads see the
// producer's stores.  Nothing produced inside the kernel is read through the
// non-coherent read-only path.
#pragma once
#include "oux_sweep.cuh"

namespace oux {

enum PhaseKind {
  PH_PRIM = 0,      // primitives of Q^n (src_qs = 0) or of the stage state (src_qs = 1)
  PH_SENSOR = 1,    // Ducros sensor
  PH_MUT = 2,       // SMS SGS viscosity
  PH_MUT_EDGES = 3, // its ghost-layer copy
  PH_SWEEP_X = 4,
  PH_SWEEP_Y = 5,
  PH_SWEEP_Z = 6,
  PH_GHOST_QS = 7,  // periodic fill of the stage state
  PH_GHOST_QN = 8   // periodic fill of Q^n (end of the step)
};

constexpr int BATCH_MAX_PHASES = 40;
constexpr int BATCH_THREADS = 288;   // 32 x 9: the y/z sweep tile shape
constexpr int BATCH_ROWS_X = 7;      // x-sweep tile 33 x 7 (231 of the 288 threads): its 38 x 7 cells
                                      // load in one pass of the block
constexpr int BATCH_ROWS_YZ = 8;     // y/z-sweep tile 32 x (8 + 1)
static_assert(32 * (BATCH_ROWS_YZ + 1) == BATCH_THREADS, "y/z tile shape must fill the batch block");
static_assert(33 * BATCH_ROWS_X <= BATCH_THREADS, "x tile shape must fit the batch block");
static_assert(38 * BATCH_ROWS_X <= BATCH_THREADS, "the x tile should load in one pass");
#ifndef OUX_BATCH_SPIN_LIMIT
#define OUX_BATCH_SPIN_LIMIT (1 << 22)  // polls of >= 64 ns each: a few seconds at most
#endif
constexpr int BATCH_FAULT_TIMEOUT = 4;  // OUX_FAULT_TIMEOUT of the C ABI
#ifndef OUX_BATCH_MINB
#define OUX_BATCH_MINB 2  // resident blocks per SM the 3D register budget is sized for
#endif
// 2D steps fit 3 resident blocks per SM without spills (measured: the 64-vortex
// FP64 ensemble runs 1.39x faster than at 2); 3D sweeps need the larger budget.
constexpr int batch_minb(int dim) { return dim == 2 ? 3 : OUX_BATCH_MINB; }

struct PhaseDesc {
  int kind;
  int src_qs;  // PH_PRIM, PH_SENSOR: 1 = the stage state (else Q^n)
  int last;    // sweeps: 1 = last sweep of the stage (applies the combination)
};

struct BatchItem {
  int phase, inst, first, count;  // units [first, first + count) of (phase, inst)
};

// dependency of (inst, phase): wait until done[inst * nphases + dep_phase] == dep_count
struct BatchDep {
  int dep_phase, dep_count;
};

template <class T> struct BatchArgs {
  const StepArgs<T>* args;   // [inst * nphases + phase]: the solve's arguments for that phase
  const PhaseDesc* phases;   // [nphases]
  const BatchItem* items;    // [nitems]
  const BatchDep* deps;      // [inst * nphases + phase]
  int* done;                 // [ninst * nphases] completion counters (zeroed before each step)
  int* head;                 // item counter (zeroed before each step)
  int* status;               // OUX_FAULT_TIMEOUT on a wait that gave up
  int nitems, nphases;
  int chunk;                 // cells per point-wise unit
  int spin_limit;            // polls of a dependency wait before it gives up (OUX_BATCH_SPIN_LIMIT)
};

__device__ __forceinline__ int ld_acquire_gpu(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

template <int ORDER, class T>
__host__ __device__ constexpr size_t batch_smem() {
  constexpr size_t a = sweep_smem<ORDER, 0, T, BATCH_ROWS_X>();
  constexpr size_t b = sweep_smem<ORDER, 1, T, BATCH_ROWS_YZ>();
  return a > b ? a : b;
}

// Tile counts of a sweep direction (launch_one's grid, with the batch's x rows).
template <int DIR>
__host__ __device__ inline void sweep_grid(const Geo& G, int n[3]) {
  const int g = G.g;
  const int Nx = G.nx - 2 * G.gx, Ny = G.ny - 2 * G.gy, Nz = G.dim == 3 ? G.nz - 2 * G.gz : 1;
  if (DIR == 0) { n[0] = (Nx + 31) / 32; n[1] = (Ny + BATCH_ROWS_X - 1) / BATCH_ROWS_X; n[2] = Nz; }
  else if (DIR == 1) { n[0] = (Nx + 31) / 32; n[1] = (Ny + BATCH_ROWS_YZ - 1) / BATCH_ROWS_YZ; n[2] = Nz; }
  else { n[0] = (Nx + 31) / 32; n[1] = (Nz + BATCH_ROWS_YZ - 1) / BATCH_ROWS_YZ; n[2] = Ny; }
}

template <int DIM, int DIR, int ORDER, int VK, bool LES, class T, bool KONLY>
__device__ __forceinline__ void batch_sweep(const StepArgs<T>& A, int last, int first, int count,
                                            unsigned char* smraw) {
  constexpr int ROWS = DIR == 0 ? BATCH_ROWS_X : BATCH_ROWS_YZ;
  int n[3];
  sweep_grid<DIR>(A.G, n);
  for (int t = first; t < first + count; ++t) {
    int b0, b1, b2;
    if (DIR == 0) { b0 = t % n[0]; b1 = (t / n[0]) % n[1]; b2 = t / (n[0] * n[1]); }
    else { b1 = t % n[1]; b0 = (t / n[1]) % n[0]; b2 = t / (n[0] * n[1]); }  // pencil along the sweep
    sweep_tile<DIM, DIR, ORDER, VK, LES, T, ROWS, false, KONLY>(A, last, b0, b1, b2, smraw, threadIdx.x,
                                                              BATCH_THREADS);
    __syncthreads();
  }
}

// [c0, c1) of a point-wise phase whose units hold `chunk` cells each
__device__ __forceinline__ int64_t batch_end(int64_t c0, int count, int chunk, int64_t n) {
  const int64_t e = c0 + (int64_t)count * chunk;
  return e < n ? e : n;
}

// KONLY: every member uses KEEP (no sensor phase, KEEP flux only).
template <int DIM, int ORDER, int VK, bool LES, class T, bool KONLY>
__global__ void __launch_bounds__(BATCH_THREADS, batch_minb(DIM)) k_batch_step(BatchArgs<T> B) {
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ int s_item, s_abort;
  const int tid = threadIdx.x;
  constexpr bool VISC = VK != VK_EULER;
  for (;;) {
    if (tid == 0) {
      const int it = atomicAdd(B.head, 1);
      int abort = 0;
      if (it < B.nitems) {
        const BatchItem bi = B.items[it];
        const BatchDep d = B.deps[bi.inst * B.nphases + bi.phase];
        if (d.dep_phase >= 0) {
          const int* ctr = B.done + bi.inst * B.nphases + d.dep_phase;
          int spins = 0;
          while (ld_acquire_gpu(ctr) < d.dep_count) {
            if (++spins > B.spin_limit) {
              atomicOr(B.status, BATCH_FAULT_TIMEOUT);
              abort = 1;
              break;
            }
            __nanosleep(64);
          }
        }
      }
      s_item = it;
      s_abort = abort;
    }
    __syncthreads();
    const int it = s_item;
    if (it >= B.nitems || s_abort) return;
    const BatchItem bi = B.items[it];
    const StepArgs<T>& A = B.args[bi.inst * B.nphases + bi.phase];
    const PhaseDesc ph = B.phases[bi.phase];
    const Geo& G = A.G;
    const int64_t c0 = (int64_t)bi.first * B.chunk;
    const int64_t ncell = (int64_t)G.nx * G.ny * G.nz;
    switch (ph.kind) {
      case PH_PRIM: {
        const int64_t c1 = batch_end(c0, bi.count, B.chunk, ncell);
        if constexpr (sizeof(T) < sizeof(double)) {
          const float* dQ = ph.src_qs ? reinterpret_cast<const float*>(A.Qs) : nullptr;
          for (int64_t t = c0 + tid; t < c1; t += BATCH_THREADS)
            prim_mx_cell<DIM, VISC>(A.Qn, dQ, G, A.W, A.M.jac, A.K, t);
        } else {
          if (ph.src_qs) {
            for (int64_t t = c0 + tid; t < c1; t += BATCH_THREADS)
              prim_cell<DIM, VISC, T, T>(A.Qs, G, A.W, A.M.jac, A.K, t);
          } else {
            for (int64_t t = c0 + tid; t < c1; t += BATCH_THREADS)
              prim_cell<DIM, VISC, double, T>(A.Qn, G, A.W, A.M.jac, A.K, t);
          }
        }
        break;
      }
      case PH_SENSOR: {
        if constexpr (!KONLY) {
          const int64_t c1 = batch_end(c0, bi.count, B.chunk, ncell);
          if constexpr (sizeof(T) < sizeof(double)) {
            const float* dQ = ph.src_qs ? reinterpret_cast<const float*>(A.Qs) : nullptr;
            for (int64_t t = c0 + tid; t < c1; t += BATCH_THREADS) sensor_mx_cell<DIM>(G, A.Qn, dQ, A.W, A.M, t);
          } else {
            for (int64_t t = c0 + tid; t < c1; t += BATCH_THREADS) sensor_cell<DIM, T>(G, A.W, A.M, t);
          }
        }
        break;
      }
      case PH_MUT: {
        if constexpr (LES && DIM == 3) {
          const int mx = G.nx - 2, my = G.ny - 2;
          const int64_t c1 = batch_end(c0, bi.count, B.chunk, (int64_t)mx * my * (G.nz - 2));
          for (int64_t t = c0 + tid; t < c1; t += BATCH_THREADS) {
            const int i = (int)(t % mx) + 1;
            const int64_t r = t / mx;
            mut_cell<T>(G, A.W, A.M, A.K, i, (int)(r % my) + 1, (int)(r / my) + 1);
          }
        }
        break;
      }
      case PH_MUT_EDGES: {
        if constexpr (LES && DIM == 3) {
          const int64_t c1 = batch_end(c0, bi.count, B.chunk, ncell);
          for (int64_t t = c0 + tid; t < c1; t += BATCH_THREADS) mut_edge_cell<T>(G, A.W, t);
        }
        break;
      }
      case PH_SWEEP_X:
        batch_sweep<DIM, 0, ORDER, VK, LES, T, KONLY>(A, ph.last, bi.first, bi.count, smraw);
        break;
      case PH_SWEEP_Y:
        batch_sweep<DIM, 1, ORDER, VK, LES, T, KONLY>(A, ph.last, bi.first, bi.count, smraw);
        break;
      case PH_SWEEP_Z:
        if constexpr (DIM == 3) batch_sweep<DIM, 2, ORDER, VK, LES, T, KONLY>(A, ph.last, bi.first, bi.count, smraw);
        break;
      case PH_GHOST_QS:
      case PH_GHOST_QN: {
        const int64_t c1 = batch_end(c0, bi.count, B.chunk, ghost_cells(G));
        if (ph.kind == PH_GHOST_QS) {
          for (int64_t t = c0 + tid; t < c1; t += BATCH_THREADS)
            ghost_cell<T>(A.Qs, G, DIM + 2, t, sizeof(T) < sizeof(double) ? A.Qn : nullptr);
        } else {
          for (int64_t t = c0 + tid; t < c1; t += BATCH_THREADS) ghost_cell<double>(A.Qn, G, DIM + 2, t);
        }
        break;
      }
      default: break;
    }
    __syncthreads();
    if (tid == 0) {
      __threadfence();
      atomicAdd(B.done + bi.inst * B.nphases + bi.phase, 1);
    }
  }
}

}  // namespace oux
