// Internal host-side declarations shared by the C-ABI translation units
// (oux_api.cu: single solves; oux_batch_api.cu: batched solves).
#pragma once
#include <cuda_runtime.h>
#include <string>
#include <vector>
#include "oux.h"
#include "oux_kernels.cuh"

// Sets the thread-local message oux_last_error() returns; returns `code`.
int oux_internal_fail(int code, const std::string& msg);

// nsteps time steps of a bound handle on `s` (the body of oux_step).
int oux_internal_run_steps(oux_handle* h, int nsteps, cudaStream_t s);

struct oux_handle {
  oux_config cfg;
  oux::Geo G;
  int nv;
  int vk;
  bool les;
  oux::PhysConst K;
  std::vector<double> inv_dx, inv_dy, inv_dz, jac, dtdxdy, dtdydz, dtdzdx, dtdx, dtdy;
  // bound buffers
  double* Q = nullptr;
  unsigned char* scratch = nullptr;
  size_t scratch_bytes = 0;
  bool mixed = false;           // FP32 stage states/fields, FP64 Q^n and accumulations
  oux::Fields<double> W{};           // FP64 form
  oux::Fields<float> Wf{};           // mixed form
  double *Racc = nullptr, *Rs = nullptr, *partials = nullptr;
  void* Qs = nullptr;           // stage state (double or float)
  int* status = nullptr;
  // tensor maps of the x and y sweeps' tiles, [sweep direction][tile field] (CUtensorMap
  // bytes, encoded by oux_bind); tmaps points at them once they are valid
  alignas(64) unsigned char tmap_host[2][14][128] = {};
  const void* tmaps = nullptr;
  oux::Metrics M{};
  int64_t launches = 0;
  int diag_blocks = 0;
  // optional per-kernel timing (oux_profile): CUDA events recorded around each
  // launch on the launching stream
  bool profiling = false;
  struct Rec { int kind; cudaEvent_t a, b; };
  std::vector<Rec> recs;
};

namespace oux {
template <class T> inline Fields<T>& fields_of(oux_handle* h);
template <> inline Fields<double>& fields_of<double>(oux_handle* h) { return h->W; }
template <> inline Fields<float>& fields_of<float>(oux_handle* h) { return h->Wf; }

// Step arguments of a bound handle (combination mode and coefficients left at 0).
template <class T>
inline StepArgs<T> base_args(oux_handle* h) {
  StepArgs<T> A{};
  A.G = h->G;
  A.W = fields_of<T>(h);
  A.M = h->M;
  A.K = h->K;
  A.scheme = h->cfg.scheme;
  A.tvd = h->cfg.tvd;
  A.slau = h->cfg.slau;
  A.Racc = h->Racc;
  A.Rs = h->Rs;
  A.Qn = h->Q;
  A.Qs = reinterpret_cast<T*>(h->Qs);
  A.tmaps = h->tmaps;
  A.status = h->status;
  return A;
}
}  // namespace oux
