// C ABI of batched solves (include/oux.h, "batched solves"): builds the phase
// list and the phase-major work list of a set of bound handles, uploads them to
// a caller-owned workspace, and launches one persistent k_batch_step per time
// step, optionally as the replay of one captured CUDA graph.
#include <cuda_runtime.h>
#include <cstdint>
#include <string>
#include <vector>
#include "oux_internal.h"
#include "oux_batch_dispatch.h"

using namespace oux;

namespace {
int fail(int code, const std::string& msg) { return oux_internal_fail(code, msg); }
#define OUX_CUDA(call)                                                                    \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess)                                                                \
      return fail(OUX_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));        \
  } while (0)

size_t align256(size_t a) { return (a + 255) / 256 * 256; }

// Stage combinations of one time step, as run_steps sequences them
// (calc_time_dev.f90.fypp:81-101 RK3, :264-287 RK4).
struct StageParams { int mode; double coef, c1, c2, c4; };
std::vector<StageParams> stage_params(int rk) {
  if (rk == 3)
    return {{CM_RK3_1, 1.0, 0.0, 0.0, 0.0}, {CM_RK3_2, 0.25, 0.75, 0.25, 1.0}, {CM_RK3_3, 2.0, 2.0, 1.0, 1.0 / 3.0}};
  return {{CM_RK4_S, 1.0, 0.5, 1.0, 0.0}, {CM_RK4_S, 1.0, 0.5, 2.0, 0.0}, {CM_RK4_S, 1.0, 1.0, 2.0, 0.0},
          {CM_RK4_4, 1.0, 1.0, 2.0, 0.0}};
}

int64_t cdiv(int64_t a, int64_t b) { return (a + b - 1) / b; }
}  // namespace

struct oux_batch {
  std::vector<oux_handle*> members;
  oux_batch_tuning tune{};
  int dim = 0, order = 0, vk = 0, rk = 0;
  bool les = false, mixed = false;
  bool keep_only = false;  // every member uses KEEP: the KEEP-only kernel
  std::vector<PhaseDesc> phases;
  std::vector<int> phase_stage;
  std::vector<BatchItem> items;
  std::vector<BatchDep> deps;
  size_t args_elem = 0;
  size_t off_args = 0, off_phases = 0, off_items = 0, off_deps = 0, off_ctr = 0, ctr_bytes = 0, off_status = 0,
         total = 0;
  unsigned char* ws = nullptr;
  BatchArgs<double> B64{};
  BatchArgs<float> B32{};
  int nsm = 0, grid = 0;
  int spin_limit = OUX_BATCH_SPIN_LIMIT;
  cudaStream_t cap = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  // OUX_BATCH_GRAPH: one capture branch (stream + join event) per member
  std::vector<cudaStream_t> branch;
  std::vector<cudaEvent_t> joined;
  cudaEvent_t fork = nullptr;
};

namespace {

bool is_sweep(int kind) { return kind == PH_SWEEP_X || kind == PH_SWEEP_Y || kind == PH_SWEEP_Z; }

// Work units of (member, phase): chunks of `chunk` cells for the point-wise
// phases, sweep tiles for the sweeps.
int64_t phase_units(const oux_batch* b, const oux_handle* h, const PhaseDesc& ph) {
  const Geo& G = h->G;
  const int64_t ncell = (int64_t)G.nx * G.ny * G.nz;
  const int64_t ch = b->tune.chunk;
  int n[3];
  switch (ph.kind) {
    case PH_PRIM: case PH_MUT_EDGES: return cdiv(ncell, ch);
    case PH_SENSOR: return h->cfg.scheme != OUX_KEEP ? cdiv(ncell, ch) : 0;
    case PH_MUT: return cdiv((int64_t)(G.nx - 2) * (G.ny - 2) * (G.nz - 2), ch);
    case PH_SWEEP_X: sweep_grid<0>(G, n); return (int64_t)n[0] * n[1] * n[2];
    case PH_SWEEP_Y: sweep_grid<1>(G, n); return (int64_t)n[0] * n[1] * n[2];
    case PH_SWEEP_Z: sweep_grid<2>(G, n); return (int64_t)n[0] * n[1] * n[2];
    case PH_GHOST_QS: case PH_GHOST_QN: return cdiv(ghost_cells(G), ch);
    default: return 0;
  }
}

int build_lists(oux_batch* b) {
  const int stages = b->rk == 3 ? 3 : 4;
  bool any_sensor = false;
  for (auto* h : b->members) any_sensor |= h->cfg.scheme != OUX_KEEP;
  b->keep_only = !any_sensor;
  b->phases.clear();
  b->phase_stage.clear();
  auto add = [&](int kind, int src_qs, int last, int st) {
    b->phases.push_back({kind, src_qs, last});
    b->phase_stage.push_back(st);
  };
  for (int s = 0; s < stages; ++s) {
    add(PH_PRIM, s > 0, 0, s);
    if (any_sensor) add(PH_SENSOR, s > 0, 0, s);
    if (b->les) { add(PH_MUT, 0, 0, s); add(PH_MUT_EDGES, 0, 0, s); }
    add(PH_SWEEP_X, 0, 0, s);
    if (b->dim == 3) { add(PH_SWEEP_Y, 0, 0, s); add(PH_SWEEP_Z, 0, 1, s); }
    else add(PH_SWEEP_Y, 0, 1, s);
    add(s + 1 < stages ? PH_GHOST_QS : PH_GHOST_QN, 0, 0, s);
  }
  const int np = (int)b->phases.size();
  if (np > BATCH_MAX_PHASES) return fail(OUX_E_INVALID, "too many phases per step");
  const int ni = (int)b->members.size();
  std::vector<int> nit((size_t)ni * np, 0);
  b->items.clear();
  for (int p = 0; p < np; ++p)
    for (int i = 0; i < ni; ++i) {
      const int64_t units = phase_units(b, b->members[i], b->phases[p]);
      const int64_t per = is_sweep(b->phases[p].kind) ? b->tune.pencil : 1;
      if (units > INT32_MAX) return fail(OUX_E_INVALID, "work list too large");
      int cnt = 0;
      for (int64_t f = 0; f < units; f += per) {
        const int64_t c = units - f < per ? units - f : per;
        b->items.push_back({p, i, (int)f, (int)c});
        ++cnt;
      }
      nit[(size_t)i * np + p] = cnt;
    }
  if (b->items.size() > (size_t)INT32_MAX) return fail(OUX_E_INVALID, "work list too large");
  b->deps.assign((size_t)ni * np, BatchDep{-1, 0});
  for (int i = 0; i < ni; ++i)
    for (int p = 0; p < np; ++p)
      for (int q = p - 1; q >= 0; --q)
        if (nit[(size_t)i * np + q] > 0) {
          b->deps[(size_t)i * np + p] = {q, nit[(size_t)i * np + q]};
          break;
        }
  return OUX_OK;
}

template <class T>
std::vector<StepArgs<T>> build_args(oux_batch* b) {
  const std::vector<StageParams> sp = stage_params(b->rk);
  const int np = (int)b->phases.size();
  std::vector<StepArgs<T>> v;
  v.reserve(b->members.size() * np);
  for (auto* h : b->members)
    for (int p = 0; p < np; ++p) {
      StepArgs<T> A = base_args<T>(h);
      const StageParams& s = sp[b->phase_stage[p]];
      A.mode = s.mode; A.coef = s.coef; A.c1 = s.c1; A.c2 = s.c2; A.c4 = s.c4;
      v.push_back(A);
    }
  return v;
}

template <class T>
void fill_args(oux_batch* b, BatchArgs<T>& B) {
  B.args = reinterpret_cast<const StepArgs<T>*>(b->ws + b->off_args);
  B.phases = reinterpret_cast<const PhaseDesc*>(b->ws + b->off_phases);
  B.items = reinterpret_cast<const BatchItem*>(b->ws + b->off_items);
  B.deps = reinterpret_cast<const BatchDep*>(b->ws + b->off_deps);
  B.done = reinterpret_cast<int*>(b->ws + b->off_ctr);
  B.head = B.done + b->members.size() * b->phases.size();
  B.status = reinterpret_cast<int*>(b->ws + b->off_status);
  B.nitems = (int)b->items.size();
  B.nphases = (int)b->phases.size();
  B.chunk = b->tune.chunk;
  B.spin_limit = b->spin_limit;
}

int launch(oux_batch* b, cudaStream_t s, int dry) {
  int rc = b->mixed ? batch_launch(b->dim, b->order, b->vk, b->les, b->B32, b->tune.blocks_per_sm, b->nsm,
                                   &b->grid, s, dry, b->keep_only)
                    : batch_launch(b->dim, b->order, b->vk, b->les, b->B64, b->tune.blocks_per_sm, b->nsm,
                                   &b->grid, s, dry, b->keep_only);
  if (rc == 2) return fail(OUX_E_INVALID, "no batched kernel built for this configuration");
  if (rc) return fail(OUX_E_CUDA, std::string("batched step launch: ") + cudaGetErrorString(cudaGetLastError()));
  return OUX_OK;
}

int one_step(oux_batch* b, cudaStream_t s) {
  OUX_CUDA(cudaMemsetAsync(b->ws + b->off_ctr, 0, b->ctr_bytes, s));
  return launch(b, s, 0);
}

void release_graph(oux_batch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
}

// OUX_BATCH_GRAPH capture of one step: fork every member onto its own branch,
// run the member's stage kernels there, join all branches back.
int capture_branches(oux_batch* b) {
  OUX_CUDA(cudaEventRecord(b->fork, b->cap));
  for (size_t i = 0; i < b->members.size(); ++i) {
    OUX_CUDA(cudaStreamWaitEvent(b->branch[i], b->fork, 0));
    int rc = oux_internal_run_steps(b->members[i], 1, b->branch[i]);
    if (rc) return rc;
    OUX_CUDA(cudaEventRecord(b->joined[i], b->branch[i]));
    OUX_CUDA(cudaStreamWaitEvent(b->cap, b->joined[i], 0));
  }
  return OUX_OK;
}

void release_branches(oux_batch* b) {
  for (auto s : b->branch) cudaStreamDestroy(s);
  for (auto e : b->joined) cudaEventDestroy(e);
  if (b->fork) cudaEventDestroy(b->fork);
  b->branch.clear();
  b->joined.clear();
  b->fork = nullptr;
}

}  // namespace

extern "C" {

int oux_batch_create(oux_handle* const* members, int32_t n, const oux_batch_tuning* tuning, oux_batch** out) {
  if (!members || !out || n < 1) return fail(OUX_E_INVALID, "need at least one member and an output");
  oux_batch_tuning t{4, 4 * BATCH_THREADS, 0, 1, OUX_BATCH_PERSISTENT};
  if (tuning) t = *tuning;
  if (t.pencil < 1 || t.chunk < 1 || t.blocks_per_sm < 0)
    return fail(OUX_E_INVALID, "tuning: pencil >= 1, chunk >= 1, blocks_per_sm >= 0");
  if (t.mode != OUX_BATCH_PERSISTENT && t.mode != OUX_BATCH_GRAPH) return fail(OUX_E_INVALID, "unknown batch mode");
  if (t.mode == OUX_BATCH_GRAPH) t.use_graph = 1;
  oux_handle* h0 = members[0];
  if (h0 && vk_wall(h0->vk))
    return fail(OUX_E_INVALID, "batches of 3D Navier-Stokes solves with non-periodic boundaries are not built");
  for (int i = 0; i < n; ++i) {
    const oux_handle* h = members[i];
    if (!h) return fail(OUX_E_INVALID, "null member");
    if (!h->Q) return fail(OUX_E_UNBOUND, "member " + std::to_string(i) + " has no device buffers bound");
    if (h->cfg.dim != h0->cfg.dim || h->cfg.order != h0->cfg.order || h->vk != h0->vk || h->les != h0->les ||
        h->mixed != h0->mixed || h->cfg.rk != h0->cfg.rk)
      return fail(OUX_E_INVALID, "member " + std::to_string(i) +
                                     " differs in dim, order, viscous stencil, LES, precision or rk");
  }
  oux_batch* b = new (std::nothrow) oux_batch();
  if (!b) return fail(OUX_E_INVALID, "host allocation failed");
  b->members.assign(members, members + n);
  b->tune = t;
  b->dim = h0->cfg.dim; b->order = h0->cfg.order; b->vk = h0->vk; b->rk = h0->cfg.rk;
  b->les = h0->les; b->mixed = h0->mixed;
  int rc = build_lists(b);
  if (rc) { delete b; return rc; }
  const size_t np = b->phases.size(), ni = b->members.size();
  b->args_elem = b->mixed ? sizeof(StepArgs<float>) : sizeof(StepArgs<double>);
  size_t off = 0;
  b->off_args = off; off = align256(off + ni * np * b->args_elem);
  b->off_phases = off; off = align256(off + np * sizeof(PhaseDesc));
  b->off_items = off; off = align256(off + b->items.size() * sizeof(BatchItem));
  b->off_deps = off; off = align256(off + ni * np * sizeof(BatchDep));
  b->off_ctr = off; b->ctr_bytes = (ni * np + 1) * sizeof(int); off = align256(off + b->ctr_bytes);
  b->off_status = off; off = align256(off + sizeof(int));
  b->total = off;
  *out = b;
  return OUX_OK;
}

int oux_batch_workspace_bytes(const oux_batch* b, size_t* bytes) {
  if (!b || !bytes) return fail(OUX_E_INVALID, "null argument");
  *bytes = b->total;
  return OUX_OK;
}

int oux_batch_bind(oux_batch* b, void* workspace_dev, size_t bytes, void* stream) {
  if (!b || !workspace_dev) return fail(OUX_E_INVALID, "null argument");
  if (bytes < b->total) return fail(OUX_E_TOO_SMALL, "workspace smaller than oux_batch_workspace_bytes()");
  if ((uintptr_t)workspace_dev & 255) return fail(OUX_E_INVALID, "workspace must be 256-byte aligned");
  cudaStream_t s = (cudaStream_t)stream;
  release_graph(b);
  b->ws = static_cast<unsigned char*>(workspace_dev);
  int dev = 0;
  OUX_CUDA(cudaGetDevice(&dev));
  OUX_CUDA(cudaDeviceGetAttribute(&b->nsm, cudaDevAttrMultiProcessorCount, dev));
  // host vectors stay alive until the synchronisation below
  std::vector<StepArgs<double>> a64;
  std::vector<StepArgs<float>> a32;
  if (b->mixed) {
    a32 = build_args<float>(b);
    OUX_CUDA(cudaMemcpyAsync(b->ws + b->off_args, a32.data(), a32.size() * sizeof(a32[0]), cudaMemcpyHostToDevice, s));
    fill_args(b, b->B32);
  } else {
    a64 = build_args<double>(b);
    OUX_CUDA(cudaMemcpyAsync(b->ws + b->off_args, a64.data(), a64.size() * sizeof(a64[0]), cudaMemcpyHostToDevice, s));
    fill_args(b, b->B64);
  }
  OUX_CUDA(cudaMemcpyAsync(b->ws + b->off_phases, b->phases.data(), b->phases.size() * sizeof(PhaseDesc),
                           cudaMemcpyHostToDevice, s));
  OUX_CUDA(cudaMemcpyAsync(b->ws + b->off_items, b->items.data(), b->items.size() * sizeof(BatchItem),
                           cudaMemcpyHostToDevice, s));
  OUX_CUDA(cudaMemcpyAsync(b->ws + b->off_deps, b->deps.data(), b->deps.size() * sizeof(BatchDep),
                           cudaMemcpyHostToDevice, s));
  OUX_CUDA(cudaMemsetAsync(b->ws + b->off_status, 0, sizeof(int), s));
  OUX_CUDA(cudaStreamSynchronize(s));
  // size the persistent grid and set the kernel attribute before any capture
  if (b->tune.mode == OUX_BATCH_PERSISTENT) {
    int rc = launch(b, s, 1);
    if (rc) return rc;
  }
  if (b->tune.use_graph && !b->cap) OUX_CUDA(cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking));
  if (b->tune.mode == OUX_BATCH_GRAPH && b->branch.empty()) {
    OUX_CUDA(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming));
    for (size_t i = 0; i < b->members.size(); ++i) {
      cudaStream_t st = nullptr;
      cudaEvent_t ev = nullptr;
      OUX_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
      b->branch.push_back(st);
      OUX_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
      b->joined.push_back(ev);
    }
  }
  return OUX_OK;
}

int oux_batch_step(oux_batch* b, int32_t nsteps, void* stream) {
  if (!b) return fail(OUX_E_INVALID, "null batch");
  if (!b->ws) return fail(OUX_E_UNBOUND, "no workspace bound");
  if (nsteps < 0) return fail(OUX_E_INVALID, "nsteps must be >= 0");
  cudaStream_t s = (cudaStream_t)stream;
  if (b->tune.use_graph) {
    if (!b->exec) {
      // relaxed: the members' kernels may set their shared-memory attribute on
      // their first launch, which happens inside this capture
      const bool branches = b->tune.mode == OUX_BATCH_GRAPH;
      OUX_CUDA(cudaStreamBeginCapture(b->cap, branches ? cudaStreamCaptureModeRelaxed
                                                       : cudaStreamCaptureModeThreadLocal));
      int rc = branches ? capture_branches(b) : one_step(b, b->cap);
      cudaGraph_t g = nullptr;
      cudaError_t e = cudaStreamEndCapture(b->cap, &g);
      if (rc) { if (g) cudaGraphDestroy(g); return rc; }
      if (e != cudaSuccess) return fail(OUX_E_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
      b->graph = g;
      e = cudaGraphInstantiate(&b->exec, b->graph, 0);
      if (e != cudaSuccess) {
        release_graph(b);
        return fail(OUX_E_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
      }
    }
    for (int k = 0; k < nsteps; ++k) OUX_CUDA(cudaGraphLaunch(b->exec, s));
    return OUX_OK;
  }
  for (int k = 0; k < nsteps; ++k) {
    int rc = one_step(b, s);
    if (rc) return rc;
  }
  return OUX_OK;
}

int oux_batch_status(oux_batch* b, int32_t* fault_bits) {
  if (!b || !fault_bits) return fail(OUX_E_INVALID, "null argument");
  if (!b->ws) return fail(OUX_E_UNBOUND, "no workspace bound");
  int v = 0;
  OUX_CUDA(cudaMemcpy(&v, b->ws + b->off_status, sizeof(int), cudaMemcpyDeviceToHost));
  *fault_bits = v;
  return OUX_OK;
}

int oux_batch_info(const oux_batch* b, int64_t* items, int32_t* phases, int32_t* grid) {
  if (!b) return fail(OUX_E_INVALID, "null batch");
  if (items) *items = (int64_t)b->items.size();
  if (phases) *phases = (int32_t)b->phases.size();
  if (grid) *grid = b->grid;
  return OUX_OK;
}

int oux_batch_set_spin_limit(oux_batch* b, int32_t polls) {
  if (!b) return fail(OUX_E_INVALID, "null batch");
  if (polls < 1) return fail(OUX_E_INVALID, "the spin limit must be at least 1 poll");
  b->spin_limit = polls;
  b->B64.spin_limit = polls;
  b->B32.spin_limit = polls;
  release_graph(b);  // a captured step holds the kernel's arguments: capture anew
  return OUX_OK;
}

int oux_batch_dep_offset(const oux_batch* b, int32_t member, int32_t phase, size_t* offset) {
  if (!b || !offset) return fail(OUX_E_INVALID, "null argument");
  const int np = (int)b->phases.size();
  if (member < 0 || member >= (int)b->members.size() || phase < 0 || phase >= np)
    return fail(OUX_E_INVALID, "member or phase out of range");
  *offset = b->off_deps + ((size_t)member * np + phase) * sizeof(BatchDep);
  return OUX_OK;
}

int oux_batch_destroy(oux_batch* b) {
  if (!b) return OUX_OK;
  release_graph(b);
  release_branches(b);
  if (b->cap) cudaStreamDestroy(b->cap);
  delete b;
  return OUX_OK;
}

}  // extern "C"
