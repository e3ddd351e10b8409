// Host side of liboux: configuration checks, metric tables, scratch carving,
// the stage driver that sequences the kernels of oux_kernels.cuh /
// oux_sweep.cuh, and the C ABI declared in include/oux.h.
#include <cuda.h>
#include <cuda_runtime.h>
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>
#include "oux.h"
#include "oux_sweep.cuh"
#include "oux_dispatch.h"
#include "oux_internal.h"

using namespace oux;

namespace {
thread_local std::string g_last_error;
}  // namespace

int oux_internal_fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

namespace {
int fail(int code, const std::string& msg) { return oux_internal_fail(code, msg); }
#define OUX_CUDA(call)                                                                    \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess)                                                                \
      return fail(OUX_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));        \
  } while (0)

int64_t round_up(int64_t a, int64_t b) { return (a + b - 1) / b * b; }
}  // namespace

namespace {

// ---- configuration -------------------------------------------------------------
int validate(const oux_config* c, std::string& why) {
  if (!c) { why = "null config"; return OUX_E_INVALID; }
  if (c->dim != 2 && c->dim != 3) { why = "dim must be 2 or 3"; return OUX_E_INVALID; }
  if (c->order != 2 && c->order != 4 && c->order != 6) { why = "order must be 2, 4 or 6"; return OUX_E_INVALID; }
  int g = c->order / 2;
  int nzc = c->dim == 3 ? c->nz : 1;
  // a periodic axis keeps g ghost cells a side, a non-periodic one a single boundary
  // cell (and at least two interior cells for the boundary faces' fallback stencils)
  auto too_small = [&](int n, bool nonper) { return nonper ? n < 4 : n < 2 * g + 1; };
  const bool zb = c->dim == 3 && (c->bc_z == 1 || c->bc_z == 3 || c->bc_z == 4);
  if (too_small(c->nx, c->bc_x == 1) || too_small(c->ny, c->bc_y == 1) ||
      (c->dim == 3 && too_small(c->nz, zb)) || c->nx < 4) {
    why = "grid too small for the stencil (need at least 1 interior cell per axis)";
    return OUX_E_INVALID;
  }
  if ((int64_t)c->nx * c->ny * nzc > (int64_t)1 << 34) { why = "grid too large"; return OUX_E_INVALID; }
  if ((int64_t)c->nx * c->ny > ((int64_t)1 << 31) - 256 || nzc > 65535) {
    why = "grid too large (an x-y plane must hold fewer than 2^31 - 256 points, nz at most 65535)";
    return OUX_E_INVALID;
  }
  if (c->scheme < 0 || c->scheme > 3) { why = "unknown scheme"; return OUX_E_INVALID; }
  if (c->dim == 2 && c->scheme == OUX_ROE) { why = "the 2D solver has no Roe scheme"; return OUX_E_INVALID; }
  if (c->visc < 0 || c->visc > 2) { why = "unknown visc"; return OUX_E_INVALID; }
  if (c->dim == 2 && c->visc == OUX_LES) { why = "the 2D solver has no LES model"; return OUX_E_INVALID; }
  if (c->tvd < 0 || c->tvd > 2) { why = "unknown tvd mode"; return OUX_E_INVALID; }
  if (c->slau < 0 || c->slau > 1) { why = "unknown SLAU variant"; return OUX_E_INVALID; }
  if (c->rk != 3 && c->rk != 4) { why = "rk must be 3 or 4"; return OUX_E_INVALID; }
  if ((c->dim == 3 && (c->bc_z < 0 || c->bc_z > 4)) || c->bc_x < 0 || c->bc_x > 1 || c->bc_y < 0 ||
      c->bc_y > 1) {
    why = "boundaries: bc_x, bc_y = 0 (periodic) or 1 (non-periodic); bc_z = 0 (periodic), 1 (non-periodic) "
          "or a z slab (2: halo planes at both ends, 3: at the upper end, 4: at the lower end)";
    return OUX_E_INVALID;
  }
  if (c->dim == 3 && c->bc_z >= 2) {
    if (c->visc == OUX_LES) {
      why = "z slabs (bc_z >= 2): the SGS viscosity's edge layers wrap z, so LES runs are not built as slabs";
      return OUX_E_INVALID;
    }
    if (c->nz < 3 * g) { why = "z slab (bc_z >= 2) needs at least g interior planes (nz >= 3g)"; return OUX_E_INVALID; }
  }
  if (c->dim == 3 && (c->bc_z == 3 || c->bc_z == 4) && c->order != 2) {
    why = "a z slab with a boundary end (bc_z = 3, 4) is built for order 2";
    return OUX_E_INVALID;
  }
  if (c->bc_y == 1 && c->ny < 4) { why = "non-periodic y (bc_y = 1) needs ny >= 4"; return OUX_E_INVALID; }
  if (c->precision != OUX_FP64 && c->precision != OUX_MIXED) { why = "unknown precision"; return OUX_E_INVALID; }
  if (!c->dx || !c->dy || (c->dim == 3 && !c->dz)) { why = "dx/dy/dz host arrays required"; return OUX_E_INVALID; }
  if (!(c->gamma > 1.0) || !(c->R > 0.0) || !(c->dt > 0.0)) { why = "gamma > 1, R > 0, dt > 0 required"; return OUX_E_INVALID; }
  if (c->visc != OUX_EULER) {
    if (!(c->Pr > 0.0)) { why = "Pr > 0 required for viscous runs"; return OUX_E_INVALID; }
    if (c->visc == OUX_LES && !(c->Prt > 0.0)) { why = "Prt > 0 required for LES"; return OUX_E_INVALID; }
  }
  return OUX_OK;
}

// Viscous kernel family the reference selects for (dim, order, visc_order, stencil):
// calc_flux_base.f90.fypp:161-177 (3D) and 2D_solver/src/calc_flux_base.f90.fypp:108-132.
int visc_kind_base(const oux_config* c, std::string& why);

// 3D Navier-Stokes grids with a non-periodic direction take the walled variants
// (order fallback of the convective faces, 2nd-order fallback of the viscous faces
// outside the high-order guard); at order 2 neither applies and the periodic
// kernels serve unchanged.
int visc_kind(const oux_config* c, std::string& why) {
  const int vk = visc_kind_base(c, why);
  const bool walls = c->dim == 3 && (c->bc_x == 1 || c->bc_y == 1 || c->bc_z == 1 || c->bc_z == 3 || c->bc_z == 4);
  if (vk <= VK_EULER || !walls || c->order == 2) return vk;
  switch (vk) {
    case VK_C6: return VK_C6W;
    case VK_C4: return VK_C4W;
    case VK_ME4: return VK_ME4W;
    case VK_GV2: return VK_GV2W;
    default: return vk;
  }
}

int visc_kind_base(const oux_config* c, std::string& why) {
  if (c->visc == OUX_EULER) return VK_EULER;
  // unset visc_order: the order in 3D (calc_visc_high.f90.fypp:2-4), 4 if the order
  // is at least 4 else 2 in 2D (2D_solver/src/calc_flux_base.f90.fypp:2-4)
  int vo = c->visc_order ? c->visc_order : (c->dim == 2 ? (c->order >= 4 ? 4 : 2) : c->order);
  if (c->dim == 2) {
    // calc_Ev4 / calc_Fv4 guard their 4th-order stencil by absolute indices, so
    // any convective order works (2D_solver/BL: ORDER 2, VISC_ORDER 4)
    if (vo == 4) return VK_2D4;
    return VK_GV2;
  }
  if (vo == 2) {
    if (c->order == 6) { why = "order 6 with visc_order 2 has no reference kernel (calc_Ev2_in)"; return -1; }
    return VK_GV2;
  }
  if (vo == 4) {
    if (c->order < 4) { why = "visc_order 4 needs order >= 4"; return -1; }
    return VK_C4;
  }
  if (vo == 6) {
    if (c->order != 6) { why = "visc_order 6 is built for order 6 only"; return -1; }
    return c->visc_stencil == OUX_ME4 ? VK_ME4 : VK_C6;
  }
  why = "visc_order must be 2, 4 or 6";
  return -1;
}

void build_tables(oux_handle* h) {
  const oux_config& c = h->cfg;
  const double* dx = c.dx;
  const double* dy = c.dy;
  const double* dz = c.dz;
  int nx = c.nx, ny = c.ny, nz = c.dim == 3 ? c.nz : 1;
  h->inv_dx.resize(nx - 1);
  h->inv_dy.resize(ny - 1);
  for (int i = 0; i < nx - 1; ++i) h->inv_dx[i] = 1.0 / dx[i];
  for (int j = 0; j < ny - 1; ++j) h->inv_dy[j] = 1.0 / dy[j];
  if (c.dim == 3) {
    h->inv_dz.resize(nz - 1);
    for (int k = 0; k < nz - 1; ++k) h->inv_dz[k] = 1.0 / dz[k];
  } else {
    h->inv_dz.assign(1, 0.0);
  }
  // Jacobian: src/set_coordinate.f90:80-117 (1/cell volume, edges copied)
  h->jac.assign((size_t)nx * ny, 0.0);
  auto J = [&](int i, int j) -> double& { return h->jac[(size_t)j * nx + i]; };
  for (int j = 1; j <= ny - 2; ++j)
    for (int i = 1; i <= nx - 2; ++i) {
      if (c.dim == 3)
        J(i, j) = 8.0 / ((dx[i - 1] + dx[i]) * (dy[j - 1] + dy[j]) * 2.0 * dz[0]);
      else
        J(i, j) = 4.0 / ((dx[i - 1] + dx[i]) * (dy[j - 1] + dy[j]));
    }
  for (int i = 0; i < nx; ++i) { J(i, 0) = J(i, 1); J(i, ny - 1) = J(i, ny - 2); }
  for (int j = 0; j < ny; ++j) { J(0, j) = J(1, j); J(nx - 1, j) = J(nx - 2, j); }
  const double dt = c.dt;
  if (c.dim == 3) {  // 3D_solver/src/preprocess.f90.fypp:76-87
    h->dtdxdy.resize((size_t)(nx - 2) * (ny - 2));
    h->dtdydz.resize((size_t)(ny - 2) * (nz - 2));
    h->dtdzdx.resize((size_t)(nx - 2) * (nz - 2));
    for (int j = 0; j < ny - 2; ++j)
      for (int i = 0; i < nx - 2; ++i)
        h->dtdxdy[(size_t)j * (nx - 2) + i] = 0.25 * dt * (dx[i] + dx[i + 1]) * (dy[j] + dy[j + 1]);
    for (int k = 0; k < nz - 2; ++k)
      for (int j = 0; j < ny - 2; ++j)
        h->dtdydz[(size_t)k * (ny - 2) + j] = 0.25 * dt * (dy[j] + dy[j + 1]) * (dz[k] + dz[k + 1]);
    for (int k = 0; k < nz - 2; ++k)
      for (int i = 0; i < nx - 2; ++i)
        h->dtdzdx[(size_t)k * (nx - 2) + i] = 0.25 * dt * (dz[k] + dz[k + 1]) * (dx[i] + dx[i + 1]);
  } else {  // 2D_solver/src/preprocess.f90.fypp:96-101
    h->dtdx.resize(nx - 2);
    h->dtdy.resize(ny - 2);
    for (int i = 0; i < nx - 2; ++i) h->dtdx[i] = 0.5 * dt * (dx[i] + dx[i + 1]);
    for (int j = 0; j < ny - 2; ++j) h->dtdy[j] = 0.5 * dt * (dy[j] + dy[j + 1]);
  }
  // derived constants: src/mod_constant.f90.fypp:18-32
  PhysConst& K = h->K;
  K.gamma = c.gamma; K.R = c.R; K.Pr = c.Pr; K.Prt = c.Prt; K.threshold = c.threshold;
  K.gamma_1 = c.gamma - 1.0;
  K.over_gamma_1 = 1.0 / (c.gamma - 1.0);
  K.R_over_gamma_1 = c.R / (c.gamma - 1.0);
  K.Cp = c.gamma * c.R / (c.gamma - 1.0);
  K.Cp_over_Pr = c.visc != OUX_EULER ? K.Cp / c.Pr : 0.0;
  K.sutherland = 1.716e-5 * 384.2 * std::pow(273.2, -1.5);
  K.gamma_over_gamma_1 = c.gamma * K.over_gamma_1;
  K.p_ref = 0.0;
  K.T_ref = 0.0;
  double t10 = std::tan(10.0 * std::acos(-1.0) / 180.0);
  K.tan10deg2 = t10 * t10;
}

Geo make_geo(const oux_config& c) {
  Geo G;
  G.dim = c.dim; G.nx = c.nx; G.ny = c.ny; G.nz = c.dim == 3 ? c.nz : 1; G.g = c.order / 2;
  G.bcx = c.bc_x;
  G.gx = c.bc_x ? 1 : G.g;
  G.bcy = c.bc_y;
  G.gy = c.bc_y ? 1 : G.g;
  G.bcz = c.dim == 3 ? c.bc_z : 0;
  G.gz = (G.bcz == 1 || G.bcz == 3 || G.bcz == 4) ? 1 : G.g;
  G.bkind = 0;  // zero-gradient boundary cells until oux_set_boundary says otherwise
  for (int f = 0; f < 4; ++f) G.bfix[f] = nullptr;
  G.gamma_1 = c.gamma - 1.0;  // mod_constant.f90.fypp gamma_1, over_gamma_1, over_gamma
  G.over_gamma_1 = 1.0 / (c.gamma - 1.0);
  G.gamma = c.gamma;
  G.over_gamma = 1.0 / c.gamma;
  for (int f = 0; f < 4; ++f) {
    G.bkinds[f] = nullptr;
    for (int q = 0; q < 4; ++q) G.bpar[f][q] = 0.0;
  }
  G.ylast = 0;
  G.bjac = nullptr;
  for (int f = 0; f < 6; ++f) G.bfix3[f] = nullptr;
  G.pk0 = 0;
  G.pk1 = G.nz;
  G.gk0 = 0;
  G.gk1 = G.nz;
  G.sk0 = c.dim == 3 ? G.gz : 0;
  G.sk1 = c.dim == 3 ? G.nz - G.gz : 1;
  G.uni = 0;
  const double* d[3] = {c.dx, c.dy, c.dim == 3 ? c.dz : nullptr};
  const int n[3] = {c.nx, c.ny, c.dim == 3 ? c.nz : 1};
  for (int a = 0; a < 3; ++a) {
    if (!d[a] || n[a] < 2) continue;
    bool same = true;
    for (int i = 1; i < n[a] - 1 && same; ++i) same = std::memcmp(&d[a][i], &d[a][0], sizeof(double)) == 0;
    if (same) G.uni |= 1 << a;
  }
  G.sx = round_up(c.nx, 4);
  G.plane = G.sx * c.ny;
  G.vs = round_up(G.plane * G.nz, 32);
  return G;
}

struct ScratchPlan {
  size_t fields = 0, racc = 0, q2 = 0, rs = 0, metrics = 0, partials = 0, status = 0, total = 0;
  int nfield_arrays = 0;
};

constexpr int DIAG_BLOCKS = 1184;  // 8 blocks per SM on 148 SMs; fixed for a deterministic sum

// Whether a configuration's sweeps read the node velocity gradients from fields
// (k_grad writes them; sweep_uses_grads): 3D grids with Central-4/6 or ME4 viscous
// stencils, periodic or walled.
bool uses_grads(const oux_config& c) {
  std::string why;
  const int vk = visc_kind(&c, why);
  if (vk < 0) return false;
  const int vb = vk_base(vk);
  return c.dim == 3 && (vb == VK_C6 || vb == VK_C4 || vb == VK_ME4);
}

ScratchPlan plan_scratch(const oux_config& c) {
  Geo G = make_geo(c);
  int nv = c.dim + 2;
  ScratchPlan P;
  size_t vsb = (size_t)G.vs * sizeof(double);
  size_t vse = (size_t)G.vs * (c.precision == OUX_MIXED ? sizeof(float) : sizeof(double));
  // rho,u,v,w,p,T,mu,sensor,mut,qc2 [+ the 9 velocity gradients]
  P.nfield_arrays = uses_grads(c) ? 19 : 10;
  size_t off = 0;
  P.fields = off; off += round_up((size_t)P.nfield_arrays * vse, 256);
  P.racc = off; off += (size_t)nv * vsb;
  P.q2 = off; off += round_up((size_t)nv * vse, 256);
  P.rs = off; off += (c.rk == 4 ? (size_t)nv * vsb : 0);
  P.metrics = off;
  int nx = c.nx, ny = c.ny, nz = c.dim == 3 ? c.nz : 1;
  size_t mcount = (size_t)(nx - 1) + (ny - 1) + (c.dim == 3 ? nz - 1 : 1) + (size_t)nx * ny;
  if (c.dim == 3) mcount += (size_t)(nx - 2) * (ny - 2) + (size_t)(ny - 2) * (nz - 2) + (size_t)(nx - 2) * (nz - 2);
  else mcount += (size_t)(nx - 2) + (ny - 2);
  off += round_up(mcount * sizeof(double), 256);
  P.partials = off; off += round_up((size_t)3 * DIAG_BLOCKS * sizeof(double) + 3 * sizeof(double), 256);
  P.status = off; off += 256;
  P.total = off;
  return P;
}

// ---- small kernels ---------------------------------------------------------------
// reference order ref[((k*ny + j)*nv + l)*nx + i]  <->  SoA Q[l*vs + k*plane + j*sx + i]
template <class T>
__global__ void k_ref_to_soa(const double* __restrict__ ref, T* __restrict__ Q, Geo G, int nv) {
  int64_t n = (int64_t)G.nx * G.ny * G.nz * nv;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    int i = (int)(t % G.nx);
    int64_t r = t / G.nx;
    int l = (int)(r % nv); r /= nv;
    int j = (int)(r % G.ny);
    int k = (int)(r / G.ny);
    Q[G.at(i, j, k) + l * G.vs] = (T)ref[t];
  }
}
template <class T>
__global__ void k_soa_to_ref(const T* __restrict__ Q, double* __restrict__ ref, Geo G, int nv) {
  int64_t n = (int64_t)G.nx * G.ny * G.nz * nv;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    int i = (int)(t % G.nx);
    int64_t r = t / G.nx;
    int l = (int)(r % nv); r /= nv;
    int j = (int)(r % G.ny);
    int k = (int)(r / G.ny);
    ref[t] = (double)Q[G.at(i, j, k) + l * G.vs];
  }
}

__device__ __forceinline__ double block_sum(double v, double* sm) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) sm[wid] = v;
  __syncthreads();
  int nw = (blockDim.x + 31) >> 5;
  v = (threadIdx.x < nw) ? sm[threadIdx.x] : 0.0;
  if (wid == 0)
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  __syncthreads();
  return v;
}

// FP64 domain integrals over interior cells (ke, entropy, enstrophy) of the FP64
// state Q (= conservative / J): primitives as in calc_quantities_3D, vorticity by
// the central difference of the solve's order (6th: load_smem_visc_cent.f90.fypp:67).
__global__ void k_diag(Geo G, const double* __restrict__ Q, Metrics M, double gamma_1, double gamma, int order,
                       double* partials) {
  __shared__ double sm[32];
  const int g = G.g;
  const int Nx = G.nx - 2 * g, Ny = G.ny - 2 * g, Nz = (G.dim == 3) ? G.nz - 2 * g : 1;
  int64_t n = (int64_t)Nx * Ny * Nz;
  double ke = 0.0, en = 0.0, ens = 0.0;
  auto vel = [&](int c, int64_t o) -> double { return Q[o + (1 + c) * G.vs] * (1.0 / Q[o]); };
  auto dd = [&](int c, int64_t o, int64_t st, double inv) -> double {
    if (order == 6)
      return ((1.0 / 60.0) * (-vel(c, o - 3 * st) + vel(c, o + 3 * st)) +
              0.15 * (vel(c, o - 2 * st) - vel(c, o + 2 * st)) + 0.75 * (-vel(c, o - st) + vel(c, o + st))) * inv;
    if (order == 4)
      return ((2.0 / 3.0) * (-vel(c, o - st) + vel(c, o + st)) -
              (1.0 / 12.0) * (-vel(c, o - 2 * st) + vel(c, o + 2 * st))) * inv;
    return 0.5 * (-vel(c, o - st) + vel(c, o + st)) * inv;
  };
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    int i = (int)(t % Nx) + g;
    int64_t r = t / Nx;
    int j = (int)(r % Ny) + g;
    int k = (G.dim == 3) ? (int)(r / Ny) + g : 0;
    int64_t o = G.at(i, j, k);
    double Jv = M.jac[(int64_t)j * G.nx + i];
    double q1 = Q[o], over = 1.0 / q1, rho = Jv * q1;
    double u = Q[o + G.vs] * over, v = Q[o + 2 * G.vs] * over;
    double w = (G.dim == 3) ? Q[o + 3 * G.vs] * over : 0.0;
    double p = gamma_1 * (Jv * Q[o + (G.dim + 1) * G.vs] - 0.5 * rho * (u * u + v * v + w * w));
    ke += 0.5 * rho * (u * u + v * v + w * w);
    en += rho * log(p * pow(rho, -gamma));
    double ix = M.inv_dx[i], iy = M.inv_dy[j];
    double dvdx = dd(1, o, 1, ix), dudy = dd(0, o, G.sx, iy);
    double om2;
    if (G.dim == 3) {
      double iz = M.inv_dz[k];
      double dwdy = dd(2, o, G.sx, iy), dvdz = dd(1, o, G.plane, iz);
      double dudz = dd(0, o, G.plane, iz), dwdx = dd(2, o, 1, ix);
      double a = dwdy - dvdz, b = dudz - dwdx, c = dvdx - dudy;
      om2 = a * a + b * b + c * c;
    } else {
      double c = dvdx - dudy;
      om2 = c * c;
    }
    ens += 0.5 * rho * om2;
  }
  ke = block_sum(ke, sm);
  en = block_sum(en, sm);
  ens = block_sum(ens, sm);
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = ke;
    partials[gridDim.x + blockIdx.x] = en;
    partials[2 * gridDim.x + blockIdx.x] = ens;
  }
}
__global__ void k_diag_final(const double* partials, int nb, double inv_n, double* out) {
  __shared__ double sm[32];
  for (int q = 0; q < 3; ++q) {
    double s = 0.0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) s += partials[q * nb + b];
    s = block_sum(s, sm);
    if (threadIdx.x == 0) out[q] = s * inv_n;
  }
}

// status scan: NaN / non-positive density or pressure in interior cells
__global__ void k_check(const double* __restrict__ Q, Geo G, const double* __restrict__ jac, double gamma_1,
                        int* status) {
  const int g = G.g;
  const int Nx = G.nx - 2 * G.gx, Ny = G.ny - 2 * G.gy, Nz = (G.dim == 3) ? G.nz - 2 * G.gz : 1;
  int64_t n = (int64_t)Nx * Ny * Nz;
  int bits = 0;
  (void)g;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    int i = (int)(t % Nx) + G.gx;
    int64_t r = t / Nx;
    int j = (int)(r % Ny) + G.gy;
    int k = (G.dim == 3) ? (int)(r / Ny) + G.gz : 0;
    int64_t o = G.at(i, j, k);
    double Jv = jac[(int64_t)j * G.nx + i];
    double q1 = Q[o], rho = Jv * q1;
    double ke = 0.0;
    for (int l = 1; l <= G.dim; ++l) { double vv = Q[o + l * G.vs] / q1; ke += vv * vv; }
    double p = gamma_1 * (Jv * Q[o + (G.dim + 1) * G.vs] - 0.5 * rho * ke);
    if (!(rho == rho) || !(p == p)) bits |= OUX_FAULT_NAN;
    if (!(rho > 0.0) || !(p > 0.0)) bits |= OUX_FAULT_NONPOSITIVE;
  }
  if (bits) atomicOr(status, bits);
}

inline int grid_for(int64_t n, int threads) {
  int64_t b = (n + threads - 1) / threads;
  if (b > 148 * 16) b = 148 * 16;
  if (b < 1) b = 1;
  return (int)b;
}

void carve(oux_handle* h) {
  ScratchPlan P = plan_scratch(h->cfg);
  size_t vsb = (size_t)h->G.vs;
  if (!h->mixed) {
    double* f = reinterpret_cast<double*>(h->scratch + P.fields);
    double** fp[10] = {&h->W.rho, &h->W.u, &h->W.v, &h->W.w, &h->W.p, &h->W.T_, &h->W.mu, &h->W.sensor, &h->W.mut, &h->W.qc2};
    for (int q = 0; q < 10; ++q) *fp[q] = f + q * vsb;
    for (int q = 0; q < 9; ++q) h->W.grad[q] = P.nfield_arrays == 19 ? f + (10 + q) * vsb : nullptr;
  } else {
    float* f = reinterpret_cast<float*>(h->scratch + P.fields);
    float** fp[10] = {&h->Wf.rho, &h->Wf.u, &h->Wf.v, &h->Wf.w, &h->Wf.p, &h->Wf.T_, &h->Wf.mu, &h->Wf.sensor, &h->Wf.mut, &h->Wf.qc2};
    for (int q = 0; q < 10; ++q) *fp[q] = f + q * vsb;
    for (int q = 0; q < 9; ++q) h->Wf.grad[q] = P.nfield_arrays == 19 ? f + (10 + q) * vsb : nullptr;
  }
  h->Racc = reinterpret_cast<double*>(h->scratch + P.racc);
  h->Qs = h->scratch + P.q2;
  h->Rs = h->cfg.rk == 4 ? reinterpret_cast<double*>(h->scratch + P.rs) : nullptr;
  double* m = reinterpret_cast<double*>(h->scratch + P.metrics);
  auto take = [&](const std::vector<double>& v) {
    double* p = m;
    m += v.size();
    return (const double*)p;
  };
  h->M.inv_dx = take(h->inv_dx);
  h->M.inv_dy = take(h->inv_dy);
  h->M.inv_dz = take(h->inv_dz);
  h->M.jac = take(h->jac);
  h->G.bjac = h->M.jac;
  if (h->cfg.dim == 3) {
    h->M.dtdxdy = take(h->dtdxdy);
    h->M.dtdydz = take(h->dtdydz);
    h->M.dtdzdx = take(h->dtdzdx);
    h->M.dtdx = h->M.dtdy = nullptr;
  } else {
    h->M.dtdx = take(h->dtdx);
    h->M.dtdy = take(h->dtdy);
    h->M.dtdxdy = h->M.dtdydz = h->M.dtdzdx = nullptr;
  }
  h->partials = reinterpret_cast<double*>(h->scratch + P.partials);
  h->status = reinterpret_cast<int*>(h->scratch + P.status);
}

// kinds reported by oux_profile_read
enum KernelKind { KK_PRIM = 0, KK_SENSOR, KK_MUT, KK_MUT_EDGES, KK_SWEEP_X, KK_SWEEP_Y, KK_SWEEP_Z, KK_GHOST,
                  KK_PRIM_FUSED, KK_GRAD, KK_COUNT };

struct Timed {
  oux_handle* h;
  int kind;
  cudaStream_t s;
  cudaEvent_t b = nullptr;
  Timed(oux_handle* h_, int kind_, cudaStream_t s_) : h(h_), kind(kind_), s(s_) {
    if (!h->profiling) return;
    cudaEvent_t a;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, s);
    h->recs.push_back({kind, a, b});
  }
  ~Timed() {
    if (b) cudaEventRecord(b, s);
  }
};

template <class T>
int launch_sweeps_t(int dim, int order, int vk, bool les, int dir, const StepArgs<T>& A, cudaStream_t s);
template <>
int launch_sweeps_t<double>(int dim, int order, int vk, bool les, int dir, const StepArgs<double>& A, cudaStream_t s) {
  return dir < 0 ? launch_sweeps_fp64(dim, order, vk, les, A, s) : launch_sweep_dir_fp64(dim, order, vk, les, dir, A, s);
}
template <>
int launch_sweeps_t<float>(int dim, int order, int vk, bool les, int dir, const StepArgs<float>& A, cudaStream_t s) {
  return dir < 0 ? launch_sweeps_mx(dim, order, vk, les, A, s) : launch_sweep_dir_mx(dim, order, vk, les, dir, A, s);
}

// k_prim_fused (primitives + sensor) on `q` (FP64 form: the stage source; mixed form:
// Q^n, with the FP32 increment of the stage source unless that is Q^n itself).
template <bool VISC, class TQ, class T, class TS>
int launch_prim_fused(const TQ* q, const TS* src, const Geo& G, Fields<T>& W, oux_handle* h, cudaStream_t s) {
  constexpr bool MX = sizeof(T) < sizeof(double);
  const float* inc = nullptr;
  if constexpr (MX) {
    if (!std::is_same<TS, double>::value) inc = reinterpret_cast<const float*>(src);
  }
  constexpr size_t smem = prim_fused_smem<1>();
  auto kern = k_prim_fused<1, true, VISC, MX, TQ, T>;
  static const cudaError_t attr = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (attr != cudaSuccess) return 1;
  kern<<<prim_fused_grid(G), PS_TX * PS_TY, smem, s>>>(q, inc, G, W, h->M, h->K);
  return cudaPeekAtLastError() == cudaSuccess ? 0 : 1;
}

// One stage: primitives of `src` (FP64 Q^n or the stage state), sensor, SGS
// viscosity, then the sweeps.
template <class T, class TS>
int run_stage(oux_handle* h, const TS* src, StepArgs<T> A, cudaStream_t s) {
  const Geo& G = h->G;
  const oux_config& c = h->cfg;
  Fields<T>& W = fields_of<T>(h);
  int64_t ncell = (int64_t)G.nx * G.ny * G.nz;
  bool visc = c.visc != OUX_EULER;
  const bool sens = c.scheme != OUX_KEEP;
  // FP64 with gradient fields: the plain primitive pass, and the sensor in the gradient
  // pass (which reads the neighbour velocities anyway); otherwise a 3D sensor scheme
  // takes the fused primitive + sensor pass (the mixed form's sensor from FP64 velocities)
  const bool sens_in_grad = sens && W.grad[0] != nullptr && sizeof(T) == sizeof(double);
  if (G.dim == 3 && sens && !sens_in_grad) {
    // primitives and sensor in one z-marching pass
    Timed tm(h, KK_PRIM_FUSED, s);
    int rc;
    if constexpr (sizeof(T) < sizeof(double)) {
      rc = visc ? launch_prim_fused<true>(h->Q, src, G, W, h, s) : launch_prim_fused<false>(h->Q, src, G, W, h, s);
    } else {
      rc = visc ? launch_prim_fused<true>(src, src, G, W, h, s) : launch_prim_fused<false>(src, src, G, W, h, s);
    }
    if (rc) return fail(OUX_E_CUDA, std::string("primitive + sensor pass: ") + cudaGetErrorString(cudaGetLastError()));
    h->launches++;
  } else {
    Timed tm(h, KK_PRIM, s);
    const dim3 gb = plane_grid(G);
    if constexpr (sizeof(T) < sizeof(double)) {
      // mixed form: Q^(s) = Q^n + FP32 increment (no increment for the first stage)
      const float* dQ = std::is_same<TS, double>::value ? nullptr : reinterpret_cast<const float*>(src);
      if (G.dim == 3) {
        if (visc) k_prim_mx<3, true><<<gb, PLANE_THREADS, 0, s>>>(h->Q, dQ, G, h->Wf, h->M.jac, h->K);
        else k_prim_mx<3, false><<<gb, PLANE_THREADS, 0, s>>>(h->Q, dQ, G, h->Wf, h->M.jac, h->K);
      } else {
        if (visc) k_prim_mx<2, true><<<gb, PLANE_THREADS, 0, s>>>(h->Q, dQ, G, h->Wf, h->M.jac, h->K);
        else k_prim_mx<2, false><<<gb, PLANE_THREADS, 0, s>>>(h->Q, dQ, G, h->Wf, h->M.jac, h->K);
      }
    } else {
      if (G.dim == 3) {
        if (visc) k_prim<3, true, TS, T><<<gb, PLANE_THREADS, 0, s>>>(src, G, W, h->M.jac, h->K);
        else k_prim<3, false, TS, T><<<gb, PLANE_THREADS, 0, s>>>(src, G, W, h->M.jac, h->K);
      } else {
        if (visc) k_prim<2, true, TS, T><<<gb, PLANE_THREADS, 0, s>>>(src, G, W, h->M.jac, h->K);
        else k_prim<2, false, TS, T><<<gb, PLANE_THREADS, 0, s>>>(src, G, W, h->M.jac, h->K);
      }
    }
    h->launches++;
  }
  if (G.dim == 2 && c.scheme != OUX_KEEP) {  // Ducros sensor (3D: fused into another pass)
    Timed tm(h, KK_SENSOR, s);
    const dim3 gb = plane_grid(G);
    if constexpr (sizeof(T) < sizeof(double)) {
      const float* dQ = std::is_same<TS, double>::value ? nullptr : reinterpret_cast<const float*>(src);
      if (G.dim == 3) k_sensor_mx<3><<<gb, PLANE_THREADS, 0, s>>>(G, h->Q, dQ, h->Wf, h->M);
      else k_sensor_mx<2><<<gb, PLANE_THREADS, 0, s>>>(G, h->Q, dQ, h->Wf, h->M);
    } else {
      if (G.dim == 3) k_sensor<3, T><<<gb, PLANE_THREADS, 0, s>>>(G, W, h->M);
      else k_sensor<2, T><<<gb, PLANE_THREADS, 0, s>>>(G, W, h->M);
    }
    h->launches++;
  }
  if (W.grad[0]) {  // node velocity gradients of the high-order viscous stencils
    Timed tm(h, KK_GRAD, s);
    if (G.gk1 > G.gk0) {
      if (sens_in_grad) {
        if (vk_base(h->vk) == VK_C6) k_grad<true, T, true><<<grad_grid(G), PLANE_THREADS, 0, s>>>(G, W, h->M);
        else k_grad<false, T, true><<<grad_grid(G), PLANE_THREADS, 0, s>>>(G, W, h->M);
      } else {
        if (vk_base(h->vk) == VK_C6) k_grad<true, T><<<grad_grid(G), PLANE_THREADS, 0, s>>>(G, W, h->M);
        else k_grad<false, T><<<grad_grid(G), PLANE_THREADS, 0, s>>>(G, W, h->M);
      }
      h->launches++;
    }
  }
  if (h->les) {
    dim3 b(32, 4, 1), gr((G.nx - 2 + 31) / 32, (G.ny - 2 + 3) / 4, G.nz - 2);
    {
      Timed tm(h, KK_MUT, s);
      k_mut<T><<<gr, b, 0, s>>>(G, W, h->M, h->K);
    }
    {
      Timed tm(h, KK_MUT_EDGES, s);
      k_mut_edges<T><<<grid_for(ncell, 256), 256, 0, s>>>(G, W);
    }
    h->launches += 2;
  }
  int rc;
  if (h->profiling) {
    // one direction at a time so each sweep gets its own event pair
    rc = 0;
    for (int d = 0; d < G.dim && !rc; ++d) {
      Timed tm(h, KK_SWEEP_X + d, s);
      rc = launch_sweeps_t<T>(G.dim, c.order, h->vk, h->les, d, A, s);
    }
  } else {
    rc = launch_sweeps_t<T>(G.dim, c.order, h->vk, h->les, -1, A, s);
  }
  if (rc == 2) return fail(OUX_E_INVALID, "no sweep kernel is built for this configuration");
  if (rc) return fail(OUX_E_CUDA, std::string("sweep launch: ") + cudaGetErrorString(cudaGetLastError()));
  h->launches += G.dim;
  return OUX_OK;
}

// Ghost / boundary fill of a full FP64 state, or (T = float) of the mixed form's
// stage increments over h->Q.
template <class T>
int ghost(oux_handle* h, T* Q, cudaStream_t s) {
  const Geo& G = h->G;
  int64_t n = (int64_t)G.nx * G.ny * G.nz;
  Timed tm(h, KK_GHOST, s);
  const double* Qn = sizeof(T) < sizeof(double) ? h->Q : nullptr;
  k_ghost<T><<<grid_for(n / 4 + 1, 256), 256, 0, s>>>(Q, G, h->nv, Qn);
  h->launches++;
  return OUX_OK;
}

// Stage st (0-based) of one time step with compute type T (double: plain FP64 form;
// float: mixed form), followed by the ghost / boundary fill of the array it wrote.
template <class T>
int run_stage_n(oux_handle* h, int st, cudaStream_t s, int part = 0) {
  double* Qn = h->Q;
  T* Qs = reinterpret_cast<T*>(h->Qs);
  const int nst = h->cfg.rk == 3 ? 3 : 4;
  // the stage's combination: calc_time_dev.f90.fypp:81-101 (RK3), 264-287 (RK4)
  auto args = [&]() {
    StepArgs<T> A = base_args<T>(h);
    if (h->cfg.rk == 3) {
      if (st == 0) {
        A.mode = CM_RK3_1; A.coef = 1.0;
      } else if (st == 1) {
        A.mode = CM_RK3_2; A.coef = 0.25; A.c1 = 0.75; A.c2 = 0.25; A.c4 = 1.0;
      } else {
        A.mode = CM_RK3_3; A.coef = 2.0; A.c1 = 2.0; A.c2 = 1.0; A.c4 = 1.0 / 3.0;
      }
    } else {
      const double c1[3] = {0.5, 0.5, 1.0}, c2[3] = {1.0, 2.0, 2.0};
      if (st < 3) {
        A.mode = CM_RK4_S; A.coef = 1.0; A.c1 = c1[st]; A.c2 = c2[st];
      } else {
        A.mode = CM_RK4_4; A.coef = 1.0;
      }
    }
    return A;
  };
  // per-cell passes and sweeps over the plane ranges h->G holds
  auto body = [&]() -> int {
    StepArgs<T> A = args();
    return st == 0 ? run_stage<T, double>(h, Qn, A, s) : run_stage<T, T>(h, Qs, A, s);
  };
  int rc = 0;
  if (part == 0) {
    if ((rc = body())) return rc;
  } else {
    // A z slab's stage in two parts (the reference's overlap of the COMMZ exchange,
    // calc_time_dev.f90.fypp:465-470): part 1 updates the cells of planes [2g, nz-2g),
    // whose stencils (g planes deep) do not reach the ghost planes, so it can run while
    // the halo of its source is in flight; part 2, once the halo is unpacked, redoes
    // the per-cell passes next to both ends (their ghost-plane inputs are now valid)
    // and updates the cells of planes [g, 2g) and [nz-2g, nz-g), then fills the ghosts.
    // Only a slab with halo planes at both ends (bc_z = 2), a halo of at least 2 planes
    // and an interior part is split; otherwise part 1 does nothing and part 2 is the
    // whole stage.
    const Geo keep = h->G;
    const int g = keep.g, nz = keep.nz;
    const int hd = vk_base(h->vk) == VK_C6 ? 3 : 2;  // reach of the gradient pass along z
    const bool split = keep.bcz == 2 && g >= 2 && nz - 2 * g > 2 * g;
    auto narrow = [&](int p0, int p1, int q0, int q1, int c0, int c1) {
      h->G.pk0 = p0; h->G.pk1 = p1; h->G.gk0 = q0; h->G.gk1 = q1; h->G.sk0 = c0; h->G.sk1 = c1;
    };
    if (!split) {
      if (part == 2) rc = body();
    } else if (part == 1) {
      // per-cell passes over every plane (the values that read stale ghost planes are
      // redone in part 2), the sweeps for the cells of [2g, nz-2g)
      narrow(0, nz, 0, nz, 2 * g, nz - 2 * g);
      rc = body();
    } else {
      // Part 1 has overwritten the cells of [2g, nz-2g) of the stage's output, which for
      // an in-place stage is its source, so part 2 redoes only the per-cell values whose
      // inputs reached the ghost planes, all of them computed from planes below 2g (above
      // nz-2g): the primitives and sensor of planes [0, g+1) (their velocities reach g+2
      // <= 2g-1... the sensor's ring one plane further) and the gradients of [0, g+hd)
      // (they read the velocity fields, which the sweeps do not write).  Then it updates
      // the cells of [g, 2g) and [nz-2g, nz-g).
      narrow(0, g + 1, 0, g + hd, g, 2 * g);
      rc = body();
      if (!rc) {
        narrow(nz - g - 1, nz, nz - g - hd, nz, nz - 2 * g, nz - g);
        rc = body();
      }
    }
    h->G = keep;
    if (rc) return rc;
    if (part == 1) return OUX_OK;
  }
  // ghost / boundary fill of the array the stage wrote
  if (st == nst - 1) ghost<double>(h, Qn, s);
  else ghost<T>(h, Qs, s);
  return OUX_OK;
}

// nsteps time steps
template <class T>
int run_steps(oux_handle* h, int nsteps, cudaStream_t s) {
  const int nst = h->cfg.rk == 3 ? 3 : 4;
  for (int n = 0; n < nsteps; ++n)
    for (int st = 0; st < nst; ++st) {
      int rc = run_stage_n<T>(h, st, s);
      if (rc) return rc;
    }
  return OUX_OK;
}

// The array stage st writes (Q^n after the last stage, else the stage state) and
// its element size.
void stage_array(oux_handle* h, int st, unsigned char** base, size_t* elem) {
  const int nst = h->cfg.rk == 3 ? 3 : 4;
  if (st == nst - 1) {
    *base = reinterpret_cast<unsigned char*>(h->Q);
    *elem = sizeof(double);
  } else {
    *base = reinterpret_cast<unsigned char*>(h->Qs);
    *elem = h->mixed ? sizeof(float) : sizeof(double);
  }
}

// ---- allocation-free residual (oux_rhs_noalloc) ------------------------------------
// Scratch for oux_rhs_noalloc: a fixed array in the library's own device image,
// created when the library's module is loaded on a device and held until the
// process exits.  Every oux_rhs_noalloc call on a device uses the same bytes.
static __device__ __align__(256) unsigned char g_noalloc_scratch[OUX_NOALLOC_SCRATCH_BYTES];

constexpr int NOALLOC_MAX_DEVICES = 64;
// Per device: the context the address was looked up in (its driver-assigned id) and
// the address.  A context made anew on the device (after cudaDeviceReset, or after
// the primary context was released and retained again) reloads the library's device
// code, and the array may then sit elsewhere, so a changed id means a new lookup.
struct NoallocSlot {
  std::atomic<unsigned long long> ctx{0};
  std::atomic<unsigned char*> ptr{nullptr};
};
NoallocSlot g_noalloc[NOALLOC_MAX_DEVICES];

// cuCtxGetCurrent / cuCtxGetId through the runtime's driver entry points (no link
// against libcuda): the id of the current context, 0 if it cannot be had.
unsigned long long current_ctx_id() {
  using GetCurrent = int (*)(void**);
  using GetId = int (*)(void*, unsigned long long*);
  static GetCurrent get_current = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return reinterpret_cast<GetCurrent>(f);
  }();
  static GetId get_id = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return reinterpret_cast<GetId>(f);
  }();
  void* ctx = nullptr;
  unsigned long long id = 0;
  if (!get_current || !get_id || get_current(&ctx) != 0 || !ctx || get_id(ctx, &id) != 0) return 0;
  return id;
}

// cuTensorMapEncodeTiled through the runtime's driver entry points (no link against
// libcuda); null when the driver does not offer it.
using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiled encode_tiled() {
  static EncodeTiled fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return reinterpret_cast<EncodeTiled>(f);
  }();
  return fn;
}
static_assert(sizeof(CUtensorMap) == TMA_MAP_BYTES, "tensor map size");

// Tensor maps of the x and y sweeps' tiles (sweep_tma, the TMA tile layout), direction-
// major then tile field: a 3D map of the field (nx x ny x nz cells; the padded layout's
// row and plane strides) whose box is tma_row x-cells by tma_box_rows rows (x: the
// pencil rows; y: the tile's cells along the sweep).  The gradient slots D0..D3 hold the
// four gradients the sweep's viscous stencil reads (the same choice as the cp.async
// tile load).  False if a map cannot be encoded; the sweeps then stage their tiles with
// cp.async.
template <class T>
bool encode_tile_maps(const Geo& G, const Fields<T>& W, CUtensorMap* out) {
  EncodeTiled enc = encode_tiled();
  if (!enc) return false;
  const CUtensorMapDataType dt = sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  const cuuint64_t dims[3] = {(cuuint64_t)G.nx, (cuuint64_t)G.ny, (cuuint64_t)G.nz};
  const cuuint64_t strides[2] = {(cuuint64_t)G.sx * sizeof(T), (cuuint64_t)G.plane * sizeof(T)};
  const cuuint32_t estr[3] = {1, 1, 1};
  for (int dir = 0; dir <= 1; ++dir) {
    const int n = dir, a1 = (n + 1) % 3, a2 = (n + 2) % 3, ca = n == 0 ? 1 : 0, cb = 2;
    const T* f[TF_COUNT] = {};
    f[TF_RHO] = W.rho; f[TF_U] = W.u; f[TF_V] = W.v; f[TF_W] = W.w; f[TF_P] = W.p; f[TF_T] = W.T_;
    f[TF_MU] = W.mu; f[TF_MUT] = W.mut; f[TF_QC2] = W.qc2; f[TF_SEN] = W.sensor;
    f[TF_D0] = W.grad[3 * a1 + a1]; f[TF_D1] = W.grad[3 * a2 + a2];
    f[TF_D2] = W.grad[3 * n + ca]; f[TF_D3] = W.grad[3 * n + cb];
    const cuuint32_t box[3] = {
        (cuuint32_t)(dir == 0 ? tma_row<0>() : tma_row<1>()),
        (cuuint32_t)(dir == 0 ? tma_box_rows<6, 0, default_rows<0>()>() : tma_box_rows<6, 1, default_rows<1>()>()),
        1u};
    for (int q = 0; q < TF_COUNT; ++q) {
      CUtensorMap* m = out + dir * TF_COUNT + q;
      std::memset(m, 0, sizeof(CUtensorMap));
      if (!f[q]) continue;
      if ((uintptr_t)f[q] & 15) return false;
      if (enc(m, dt, 3, (void*)f[q], dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
              CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return false;
    }
  }
  return true;
}

// Device address of g_noalloc_scratch on the current device, looked up once per
// device context (cudaGetSymbolAddress with that device current) and cached.
int noalloc_scratch(unsigned char** out) {
  int dev = -1;
  OUX_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return fail(OUX_E_INVALID, "device ordinal out of range");
  // the runtime makes the device's primary context current on its first call above
  const unsigned long long id = current_ctx_id();
  NoallocSlot& slot = g_noalloc[dev];
  unsigned char* p = slot.ptr.load(std::memory_order_acquire);
  if (!p || id == 0 || slot.ctx.load(std::memory_order_acquire) != id) {
    void* a = nullptr;
    OUX_CUDA(cudaGetSymbolAddress(&a, g_noalloc_scratch));
    p = static_cast<unsigned char*>(a);
    slot.ptr.store(p, std::memory_order_release);
    slot.ctx.store(id, std::memory_order_release);
  }
  *out = p;
  return OUX_OK;
}

// Physical constants of a configuration (src/mod_constant.f90.fypp:18-32),
// without the host metric tables.
PhysConst consts_of(const oux_config& c) {
  PhysConst K{};
  K.gamma = c.gamma; K.R = c.R; K.Pr = c.Pr; K.Prt = c.Prt; K.threshold = c.threshold;
  K.gamma_1 = c.gamma - 1.0;
  K.over_gamma_1 = 1.0 / (c.gamma - 1.0);
  K.R_over_gamma_1 = c.R / (c.gamma - 1.0);
  K.Cp = c.gamma * c.R / (c.gamma - 1.0);
  K.Cp_over_Pr = c.visc != OUX_EULER ? K.Cp / c.Pr : 0.0;
  K.sutherland = 1.716e-5 * 384.2 * std::pow(273.2, -1.5);
  K.gamma_over_gamma_1 = c.gamma * K.over_gamma_1;
  K.p_ref = 0.0;
  K.T_ref = 0.0;
  double t10 = std::tan(10.0 * std::acos(-1.0) / 180.0);
  K.tan10deg2 = t10 * t10;
  return K;
}

// Metric tables on the device from the raw spacings d = [dx | dy | dz] (same
// arithmetic and order of operations as build_tables, so the values are the
// same bits): 1/d, the Jacobian with clamped edges, and the dt * face-area
// tables of preprocess.f90.fypp.
__global__ void k_noalloc_tables(const double* __restrict__ d, Geo G, double dt, Metrics M) {
  const int nx = G.nx, ny = G.ny, nz = G.nz;
  const double* dx = d;
  const double* dy = d + (nx - 1);
  const double* dz = dy + (ny - 1);
  double* inv_dx = const_cast<double*>(M.inv_dx);
  double* inv_dy = const_cast<double*>(M.inv_dy);
  double* inv_dz = const_cast<double*>(M.inv_dz);
  double* jac = const_cast<double*>(M.jac);
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t t0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  for (int64_t t = t0; t < nx - 1; t += stride) inv_dx[t] = 1.0 / dx[t];
  for (int64_t t = t0; t < ny - 1; t += stride) inv_dy[t] = 1.0 / dy[t];
  if (G.dim == 3) {
    for (int64_t t = t0; t < nz - 1; t += stride) inv_dz[t] = 1.0 / dz[t];
  } else if (t0 == 0) {
    inv_dz[0] = 0.0;
  }
  for (int64_t t = t0; t < (int64_t)nx * ny; t += stride) {
    int i = (int)(t % nx), j = (int)(t / nx);
    i = i < 1 ? 1 : (i > nx - 2 ? nx - 2 : i);
    j = j < 1 ? 1 : (j > ny - 2 ? ny - 2 : j);
    if (G.dim == 3)
      jac[t] = 8.0 / ((dx[i - 1] + dx[i]) * (dy[j - 1] + dy[j]) * 2.0 * dz[0]);
    else
      jac[t] = 4.0 / ((dx[i - 1] + dx[i]) * (dy[j - 1] + dy[j]));
  }
  if (G.dim == 3) {
    double* dtdxdy = const_cast<double*>(M.dtdxdy);
    double* dtdydz = const_cast<double*>(M.dtdydz);
    double* dtdzdx = const_cast<double*>(M.dtdzdx);
    for (int64_t t = t0; t < (int64_t)(nx - 2) * (ny - 2); t += stride) {
      int i = (int)(t % (nx - 2)), j = (int)(t / (nx - 2));
      dtdxdy[t] = 0.25 * dt * (dx[i] + dx[i + 1]) * (dy[j] + dy[j + 1]);
    }
    for (int64_t t = t0; t < (int64_t)(ny - 2) * (nz - 2); t += stride) {
      int j = (int)(t % (ny - 2)), k = (int)(t / (ny - 2));
      dtdydz[t] = 0.25 * dt * (dy[j] + dy[j + 1]) * (dz[k] + dz[k + 1]);
    }
    for (int64_t t = t0; t < (int64_t)(nx - 2) * (nz - 2); t += stride) {
      int i = (int)(t % (nx - 2)), k = (int)(t / (nx - 2));
      dtdzdx[t] = 0.25 * dt * (dz[k] + dz[k + 1]) * (dx[i] + dx[i + 1]);
    }
  } else {
    double* dtdx = const_cast<double*>(M.dtdx);
    double* dtdy = const_cast<double*>(M.dtdy);
    for (int64_t t = t0; t < nx - 2; t += stride) dtdx[t] = 0.5 * dt * (dx[t] + dx[t + 1]);
    for (int64_t t = t0; t < ny - 2; t += stride) dtdy[t] = 0.5 * dt * (dy[t] + dy[t + 1]);
  }
}

}  // namespace

int oux_internal_run_steps(oux_handle* h, int nsteps, cudaStream_t s) {
  return h->mixed ? run_steps<float>(h, nsteps, s) : run_steps<double>(h, nsteps, s);
}

// ================================ C ABI =========================================
extern "C" {

const char* oux_last_error(void) { return g_last_error.c_str(); }
int oux_abi_version(void) { return OUX_ABI_VERSION; }

int oux_state_bytes(const oux_config* cfg, size_t* bytes) {
  std::string why;
  int rc = validate(cfg, why);
  if (rc) return fail(rc, why);
  if (!bytes) return fail(OUX_E_INVALID, "null output");
  Geo G = make_geo(*cfg);
  *bytes = (size_t)(cfg->dim + 2) * G.vs * sizeof(double);
  return OUX_OK;
}

int oux_scratch_bytes(const oux_config* cfg, size_t* bytes) {
  std::string why;
  int rc = validate(cfg, why);
  if (rc) return fail(rc, why);
  if (!bytes) return fail(OUX_E_INVALID, "null output");
  *bytes = plan_scratch(*cfg).total;
  return OUX_OK;
}

int oux_create(const oux_config* cfg, oux_handle** out) {
  std::string why;
  int rc = validate(cfg, why);
  if (rc) return fail(rc, why);
  if (!out) return fail(OUX_E_INVALID, "null output");
  int vk = visc_kind(cfg, why);
  if (vk < 0) return fail(OUX_E_INVALID, why);
  oux_handle* h = new (std::nothrow) oux_handle();
  if (!h) return fail(OUX_E_INVALID, "host allocation failed");
  h->cfg = *cfg;
  if (h->cfg.dim == 2) { h->cfg.nz = 1; h->cfg.bc_z = 0; }
  h->G = make_geo(h->cfg);
  h->nv = cfg->dim + 2;
  h->vk = vk;
  h->les = cfg->visc == OUX_LES;
  h->mixed = cfg->precision == OUX_MIXED;
  build_tables(h);
  h->cfg.dx = h->cfg.dy = h->cfg.dz = nullptr;  // host arrays are not retained
  *out = h;
  return OUX_OK;
}

int oux_destroy(oux_handle* h) {
  if (h) oux_profile(h, 0);
  delete h;
  return OUX_OK;
}

int oux_layout_of(const oux_handle* h, oux_layout* out) {
  if (!h || !out) return fail(OUX_E_INVALID, "null argument");
  out->nv = h->nv;
  out->row_stride = h->G.sx;
  out->plane_stride = h->G.plane;
  out->var_stride = h->G.vs;
  out->elem_bytes = sizeof(double);
  return OUX_OK;
}

int oux_bind(oux_handle* h, void* state_dev, void* scratch_dev, size_t scratch_bytes, void* stream) {
  if (!h || !state_dev || !scratch_dev) return fail(OUX_E_INVALID, "null argument");
  ScratchPlan P = plan_scratch(h->cfg);
  if (scratch_bytes < P.total)
    return fail(OUX_E_TOO_SMALL, "scratch buffer smaller than oux_scratch_bytes()");
  if (((uintptr_t)state_dev & 255) || ((uintptr_t)scratch_dev & 255))
    return fail(OUX_E_INVALID, "device buffers must be 256-byte aligned");
  cudaStream_t s = (cudaStream_t)stream;
  h->Q = (double*)state_dev;
  h->scratch = (unsigned char*)scratch_dev;
  h->scratch_bytes = scratch_bytes;
  carve(h);
  // the x and y sweep tiles' tensor maps (kept null where a map cannot be made)
  h->tmaps = nullptr;
  if (uses_grads(h->cfg)) {
    static_assert(sizeof(h->tmap_host) == 2 * TF_COUNT * sizeof(CUtensorMap), "tensor map storage");
    CUtensorMap* maps = reinterpret_cast<CUtensorMap*>(h->tmap_host);
    const bool ok = h->mixed ? encode_tile_maps<float>(h->G, h->Wf, maps) : encode_tile_maps<double>(h->G, h->W, maps);
    if (ok) h->tmaps = h->tmap_host;
  }
  // upload metric tables (contiguous block, same order as carve())
  std::vector<double> m;
  auto put = [&](const std::vector<double>& v) { m.insert(m.end(), v.begin(), v.end()); };
  put(h->inv_dx); put(h->inv_dy); put(h->inv_dz); put(h->jac);
  if (h->cfg.dim == 3) { put(h->dtdxdy); put(h->dtdydz); put(h->dtdzdx); }
  else { put(h->dtdx); put(h->dtdy); }
  OUX_CUDA(cudaMemcpyAsync((void*)h->M.inv_dx, m.data(), m.size() * sizeof(double), cudaMemcpyHostToDevice, s));
  OUX_CUDA(cudaMemsetAsync(h->status, 0, sizeof(int), s));
  if (h->Rs) OUX_CUDA(cudaMemsetAsync(h->Rs, 0, (size_t)h->nv * h->G.vs * sizeof(double), s));
  // the metric upload reads a host vector that goes out of scope: finish it now
  OUX_CUDA(cudaStreamSynchronize(s));
  return OUX_OK;
}

int oux_set_state(oux_handle* h, const double* host_qj, void* stream) {
  if (!h || !host_qj) return fail(OUX_E_INVALID, "null argument");
  if (!h->Q) return fail(OUX_E_UNBOUND, "no device buffers bound");
  cudaStream_t s = (cudaStream_t)stream;
  const Geo& G = h->G;
  int64_t n = (int64_t)G.nx * G.ny * G.nz * h->nv;
  {
    // mixed form references: p and T of the first interior cell (any value of
    // the field's magnitude keeps the FP32 deviations small)
    const int g = G.g, nv = h->nv;
    const int kk = G.dim == 3 ? g : 0;
    auto at = [&](int l) { return host_qj[(((int64_t)kk * G.ny + g) * nv + l) * G.nx + g]; };
    const double Jv = h->jac[(size_t)g * G.nx + g];
    const double q1 = at(0), rho = Jv * q1, over = 1.0 / q1;
    double ke = 0.0;
    for (int l = 1; l <= G.dim; ++l) { double vv = at(l) * over; ke += vv * vv; }
    const double p = h->K.gamma_1 * (Jv * at(nv - 1) - 0.5 * rho * ke);
    h->K.p_ref = h->mixed ? p : 0.0;
    h->K.T_ref = h->mixed ? p / (h->K.R * rho) : 0.0;
  }
  OUX_CUDA(cudaMemcpyAsync(h->Racc, host_qj, n * sizeof(double), cudaMemcpyHostToDevice, s));
  k_ref_to_soa<double><<<grid_for(n, 256), 256, 0, s>>>(h->Racc, h->Q, G, h->nv);
  OUX_CUDA(cudaGetLastError());
  return OUX_OK;
}

int oux_get_state(oux_handle* h, double* host_qj, void* stream) {
  if (!h || !host_qj) return fail(OUX_E_INVALID, "null argument");
  if (!h->Q) return fail(OUX_E_UNBOUND, "no device buffers bound");
  cudaStream_t s = (cudaStream_t)stream;
  const Geo& G = h->G;
  int64_t n = (int64_t)G.nx * G.ny * G.nz * h->nv;
  k_soa_to_ref<double><<<grid_for(n, 256), 256, 0, s>>>(h->Q, h->Racc, G, h->nv);
  OUX_CUDA(cudaGetLastError());
  OUX_CUDA(cudaMemcpyAsync(host_qj, h->Racc, n * sizeof(double), cudaMemcpyDeviceToHost, s));
  OUX_CUDA(cudaStreamSynchronize(s));
  return OUX_OK;
}

int oux_get_state_async(oux_handle* h, double* host_qj, void* stream) {
  if (!h || !host_qj) return fail(OUX_E_INVALID, "null argument");
  if (!h->Q) return fail(OUX_E_UNBOUND, "no device buffers bound");
  cudaStream_t s = (cudaStream_t)stream;
  const Geo& G = h->G;
  int64_t n = (int64_t)G.nx * G.ny * G.nz * h->nv;
  k_soa_to_ref<double><<<grid_for(n, 256), 256, 0, s>>>(h->Q, h->Racc, G, h->nv);
  OUX_CUDA(cudaGetLastError());
  OUX_CUDA(cudaMemcpyAsync(host_qj, h->Racc, n * sizeof(double), cudaMemcpyDeviceToHost, s));
  return OUX_OK;
}

int oux_pack_state(const oux_handle* h, const double* ref_qj, void* dev_layout_host) {
  if (!h || !ref_qj || !dev_layout_host) return fail(OUX_E_INVALID, "null argument");
  const Geo& G = h->G;
  double* Q = (double*)dev_layout_host;
  for (int k = 0; k < G.nz; ++k)
    for (int j = 0; j < G.ny; ++j)
      for (int l = 0; l < h->nv; ++l)
        for (int i = 0; i < G.nx; ++i)
          Q[G.at(i, j, k) + l * G.vs] = ref_qj[(((int64_t)k * G.ny + j) * h->nv + l) * G.nx + i];
  return OUX_OK;
}

int oux_unpack_state(const oux_handle* h, const void* dev_layout_host, double* ref_qj) {
  if (!h || !ref_qj || !dev_layout_host) return fail(OUX_E_INVALID, "null argument");
  const Geo& G = h->G;
  const double* Q = (const double*)dev_layout_host;
  for (int k = 0; k < G.nz; ++k)
    for (int j = 0; j < G.ny; ++j)
      for (int l = 0; l < h->nv; ++l)
        for (int i = 0; i < G.nx; ++i)
          ref_qj[(((int64_t)k * G.ny + j) * h->nv + l) * G.nx + i] = Q[G.at(i, j, k) + l * G.vs];
  return OUX_OK;
}

int oux_fill_ghosts(oux_handle* h, void* stream) {
  if (!h) return fail(OUX_E_INVALID, "null handle");
  if (!h->Q) return fail(OUX_E_UNBOUND, "no device buffers bound");
  ghost<double>(h, h->Q, (cudaStream_t)stream);
  OUX_CUDA(cudaGetLastError());
  return OUX_OK;
}

int oux_stage(oux_handle* h, int32_t stage, void* stream) {
  if (!h) return fail(OUX_E_INVALID, "null handle");
  if (!h->Q) return fail(OUX_E_UNBOUND, "no device buffers bound");
  const int nst = h->cfg.rk == 3 ? 3 : 4;
  if (stage < 0 || stage >= nst) return fail(OUX_E_INVALID, "stage out of range (0..2 for RK3, 0..3 for RK4)");
  cudaStream_t s = (cudaStream_t)stream;
  int rc = h->mixed ? run_stage_n<float>(h, stage, s) : run_stage_n<double>(h, stage, s);
  if (rc) return rc;
  OUX_CUDA(cudaGetLastError());
  return OUX_OK;
}

int oux_stage_part(oux_handle* h, int32_t stage, int32_t part, void* stream) {
  if (!h) return fail(OUX_E_INVALID, "null handle");
  const int nst = h->cfg.rk == 3 ? 3 : 4;
  if (stage < 0 || stage >= nst) return fail(OUX_E_INVALID, "stage out of range (0..2 for RK3, 0..3 for RK4)");
  if (part < 0 || part > 2) return fail(OUX_E_INVALID, "part must be 0 (whole stage), 1 (interior) or 2 (ends)");
  if (part != 0 && (h->cfg.dim != 3 || h->les))
    return fail(OUX_E_INVALID, "stage parts are built for 3D Euler / Navier-Stokes grids");
  if (!h->Q) return fail(OUX_E_UNBOUND, "no device buffers bound");
  cudaStream_t s = (cudaStream_t)stream;
  int rc = h->mixed ? run_stage_n<float>(h, stage, s, part) : run_stage_n<double>(h, stage, s, part);
  if (rc) return rc;
  OUX_CUDA(cudaGetLastError());
  return OUX_OK;
}

int oux_halo_bytes(const oux_handle* h, int32_t stage, size_t* bytes) {
  if (!h || !bytes) return fail(OUX_E_INVALID, "null argument");
  const int nst = h->cfg.rk == 3 ? 3 : 4;
  if (stage < 0 || stage >= nst) return fail(OUX_E_INVALID, "stage out of range");
  size_t elem = stage == nst - 1 ? sizeof(double) : (h->mixed ? sizeof(float) : sizeof(double));
  *bytes = (size_t)h->nv * h->G.g * h->G.plane * elem;
  return OUX_OK;
}

// g planes of every variable of the array `stage` writes, between the state and a
// packed buffer [nv][g][plane]: pack (to_buf) copies planes k0..k0+g-1 into buf,
// unpack copies buf into them.
static int halo_copy(oux_handle* h, int stage, int k0, void* buf, bool to_buf, cudaStream_t s) {
  unsigned char* base;
  size_t elem;
  stage_array(h, stage, &base, &elem);
  const Geo& G = h->G;
  const size_t chunk = (size_t)G.g * G.plane * elem;
  for (int l = 0; l < h->nv; ++l) {
    unsigned char* st = base + ((size_t)l * G.vs + (size_t)k0 * G.plane) * elem;
    unsigned char* bf = static_cast<unsigned char*>(buf) + (size_t)l * chunk;
    OUX_CUDA(cudaMemcpyAsync(to_buf ? bf : st, to_buf ? st : bf, chunk, cudaMemcpyDeviceToDevice, s));
  }
  return OUX_OK;
}

int oux_halo_pack(oux_handle* h, int32_t stage, void* lo_dev, void* hi_dev, void* stream) {
  if (!h || !lo_dev || !hi_dev) return fail(OUX_E_INVALID, "null argument");
  if (!h->Q) return fail(OUX_E_UNBOUND, "no device buffers bound");
  if (h->G.dim != 3 || h->G.bcz < 2) return fail(OUX_E_INVALID, "halo exchange needs a z slab (bc_z >= 2)");
  const int nst = h->cfg.rk == 3 ? 3 : 4;
  if (stage < 0 || stage >= nst) return fail(OUX_E_INVALID, "stage out of range");
  const int g = h->G.g, nz = h->G.nz;
  cudaStream_t s = (cudaStream_t)stream;
  int rc = halo_copy(h, stage, g, lo_dev, true, s);  // lowest interior planes -> the rank below
  if (!rc) rc = halo_copy(h, stage, nz - 2 * g, hi_dev, true, s);  // highest -> the rank above
  return rc;
}

int oux_halo_unpack(oux_handle* h, int32_t stage, const void* lo_dev, const void* hi_dev, void* stream) {
  if (!h || !lo_dev || !hi_dev) return fail(OUX_E_INVALID, "null argument");
  if (!h->Q) return fail(OUX_E_UNBOUND, "no device buffers bound");
  if (h->G.dim != 3 || h->G.bcz < 2) return fail(OUX_E_INVALID, "halo exchange needs a z slab (bc_z >= 2)");
  const int nst = h->cfg.rk == 3 ? 3 : 4;
  if (stage < 0 || stage >= nst) return fail(OUX_E_INVALID, "stage out of range");
  const int g = h->G.g, nz = h->G.nz;
  cudaStream_t s = (cudaStream_t)stream;
  // only the halo ends: a slab end on the grid's boundary keeps its boundary cells
  int rc = OUX_OK;
  if (!z_fill_lo(h->G)) rc = halo_copy(h, stage, 0, const_cast<void*>(lo_dev), false, s);  // from below
  if (!rc && !z_fill_hi(h->G)) rc = halo_copy(h, stage, nz - g, const_cast<void*>(hi_dev), false, s);  // above
  return rc;
}

int oux_set_boundary(oux_handle* h, int32_t face, int32_t kind, const double* fixed_dev) {
  if (!h) return fail(OUX_E_INVALID, "null handle");
  const int nfaces = h->G.dim == 3 ? 6 : 4;
  if (face < 0 || face >= nfaces)
    return fail(OUX_E_INVALID, "face must be 0..3 (x low, x high, y low, y high), 4..5 (z low, z high) in 3D");
  if (kind < OUX_BC_ZERO_GRADIENT || kind > OUX_BC_NEUMANN || kind == OUX_BC_FARFIELD)
    return fail(OUX_E_INVALID, "unknown boundary rule (far-field faces: oux_set_boundary_farfield)");
  bool open;
  if (face < 2) open = h->G.bcx;
  else if (face < 4) open = h->G.bcy;
  else open = face == 4 ? z_bnd_lo(h->G) : z_bnd_hi(h->G);
  if (!open) return fail(OUX_E_INVALID, "the face is periodic or a slab's halo end");
  if (kind == OUX_BC_FIXED && !fixed_dev) return fail(OUX_E_INVALID, "a fixed rule needs its device values");
  if (kind == OUX_BC_FIXED && (reinterpret_cast<uintptr_t>(fixed_dev) & 7))
    return fail(OUX_E_INVALID, "fixed values must be 8-byte aligned");
  h->G.bkind = (h->G.bkind & ~(15 << (4 * face))) | (kind << (4 * face));
  if (h->G.dim == 3) h->G.bfix3[face] = kind == OUX_BC_FIXED ? fixed_dev : nullptr;
  else h->G.bfix[face] = kind == OUX_BC_FIXED ? fixed_dev : nullptr;
  return OUX_OK;
}

int oux_set_boundary_farfield(oux_handle* h, int32_t face, double rho_inf, double u_tangential,
                              double u_normal, double c_inf) {
  if (!h) return fail(OUX_E_INVALID, "null handle");
  if (face != OUX_FACE_X_HI && face != OUX_FACE_Y_HI)
    return fail(OUX_E_INVALID, "the far-field rule is built for the high faces (x high, y high)");
  if (!(face < 2 ? h->G.bcx : h->G.bcy))
    return fail(OUX_E_INVALID, "the face's direction is periodic (set bc_x / bc_y = 1)");
  if (!(rho_inf > 0.0) || !(c_inf > 0.0)) return fail(OUX_E_INVALID, "far field needs rho > 0 and c > 0");
  h->G.bkind = (h->G.bkind & ~(15 << (4 * face))) | (OUX_BC_FARFIELD << (4 * face));
  h->G.bpar[face][0] = rho_inf;
  h->G.bpar[face][1] = u_tangential;
  h->G.bpar[face][2] = u_normal;
  h->G.bpar[face][3] = c_inf;
  return OUX_OK;
}

int oux_set_boundary_cells(oux_handle* h, int32_t face, const int8_t* kinds_dev) {
  if (!h) return fail(OUX_E_INVALID, "null handle");
  if (h->G.dim != 2) return fail(OUX_E_INVALID, "per-position rules are built for 2D solves");
  if (face < 0 || face > 3) return fail(OUX_E_INVALID, "face must be 0..3 (x low, x high, y low, y high)");
  if (kinds_dev && !(face < 2 ? h->G.bcx : h->G.bcy))
    return fail(OUX_E_INVALID, "the face's direction is periodic (set bc_x / bc_y = 1)");
  h->G.bkinds[face] = reinterpret_cast<const signed char*>(kinds_dev);
  return OUX_OK;
}

int oux_set_boundary_order(oux_handle* h, int32_t y_last) {
  if (!h) return fail(OUX_E_INVALID, "null handle");
  h->G.ylast = y_last ? 1 : 0;
  return OUX_OK;
}

int oux_rhs(oux_handle* h, double* rhs_dev, void* stream) {
  if (!h || !rhs_dev) return fail(OUX_E_INVALID, "null argument");
  if (!h->Q) return fail(OUX_E_UNBOUND, "no device buffers bound");
  cudaStream_t s = (cudaStream_t)stream;
  const Geo& G = h->G;
  size_t n = (size_t)h->nv * (G.nx - 2) * (G.ny - 2) * (G.dim == 3 ? G.nz - 2 : 1);
  OUX_CUDA(cudaMemsetAsync(rhs_dev, 0, n * sizeof(double), s));
  int rc;
  if (h->mixed) {
    StepArgs<float> A = base_args<float>(h);
    A.mode = CM_R_OUT; A.coef = 1.0; A.Rout = rhs_dev;
    rc = run_stage<float, double>(h, h->Q, A, s);
  } else {
    StepArgs<double> A = base_args<double>(h);
    A.mode = CM_R_OUT; A.coef = 1.0; A.Rout = rhs_dev;
    rc = run_stage<double, double>(h, h->Q, A, s);
  }
  if (rc) return rc;
  OUX_CUDA(cudaGetLastError());
  return OUX_OK;
}

int oux_step(oux_handle* h, int32_t nsteps, void* stream) {
  if (!h) return fail(OUX_E_INVALID, "null handle");
  if (!h->Q) return fail(OUX_E_UNBOUND, "no device buffers bound");
  if (nsteps < 0) return fail(OUX_E_INVALID, "nsteps must be >= 0");
  cudaStream_t s = (cudaStream_t)stream;
  h->launches = 0;
  int rc = h->mixed ? run_steps<float>(h, nsteps, s) : run_steps<double>(h, nsteps, s);
  if (rc) return rc;
  OUX_CUDA(cudaGetLastError());
  return OUX_OK;
}

int oux_diagnostics(oux_handle* h, double out[3], void* stream) {
  if (!h || !out) return fail(OUX_E_INVALID, "null argument");
  if (!h->Q) return fail(OUX_E_UNBOUND, "no device buffers bound");
  cudaStream_t s = (cudaStream_t)stream;
  const Geo& G = h->G;
  int64_t ncell = (int64_t)G.nx * G.ny * G.nz;
  (void)ncell;
  k_diag<<<DIAG_BLOCKS, 256, 0, s>>>(G, h->Q, h->M, h->K.gamma_1, h->K.gamma, h->cfg.order, h->partials);
  int64_t nint = (int64_t)(G.nx - 2 * G.g) * (G.ny - 2 * G.g) * (G.dim == 3 ? G.nz - 2 * G.g : 1);
  double* res = h->partials + 3 * DIAG_BLOCKS;
  k_diag_final<<<1, 256, 0, s>>>(h->partials, DIAG_BLOCKS, 1.0 / (double)nint, res);
  OUX_CUDA(cudaGetLastError());
  OUX_CUDA(cudaMemcpyAsync(out, res, 3 * sizeof(double), cudaMemcpyDeviceToHost, s));
  OUX_CUDA(cudaStreamSynchronize(s));
  return OUX_OK;
}

int oux_check_state(oux_handle* h, int32_t* fault_bits, void* stream) {
  if (!h || !fault_bits) return fail(OUX_E_INVALID, "null argument");
  if (!h->Q) return fail(OUX_E_UNBOUND, "no device buffers bound");
  cudaStream_t s = (cudaStream_t)stream;
  const Geo& G = h->G;
  int64_t n = (int64_t)(G.nx - 2 * G.g) * (G.ny - 2 * G.g) * (G.dim == 3 ? G.nz - 2 * G.g : 1);
  OUX_CUDA(cudaMemsetAsync(h->status, 0, sizeof(int), s));
  k_check<<<grid_for(n, 256), 256, 0, s>>>(h->Q, G, h->M.jac, h->K.gamma_1, h->status);
  OUX_CUDA(cudaGetLastError());
  int v = 0;
  OUX_CUDA(cudaMemcpyAsync(&v, h->status, sizeof(int), cudaMemcpyDeviceToHost, s));
  OUX_CUDA(cudaStreamSynchronize(s));
  *fault_bits = v;
  return v ? fail(OUX_E_DEVICE_FAULT, "device status word reports a fault") : OUX_OK;
}

int oux_status(oux_handle* h, int32_t* fault_bits) {
  if (!h || !fault_bits) return fail(OUX_E_INVALID, "null argument");
  if (!h->status) return fail(OUX_E_UNBOUND, "no device buffers bound");
  int v = 0;
  OUX_CUDA(cudaMemcpy(&v, h->status, sizeof(int), cudaMemcpyDeviceToHost));
  *fault_bits = v;
  return OUX_OK;
}

int oux_profile(oux_handle* h, int32_t enable) {
  if (!h) return fail(OUX_E_INVALID, "null handle");
  for (auto& r : h->recs) { cudaEventDestroy(r.a); cudaEventDestroy(r.b); }
  h->recs.clear();
  h->profiling = enable != 0;
  return OUX_OK;
}

int oux_profile_read(oux_handle* h, double* ms, int64_t* count, int32_t nkinds) {
  if (!h || !ms || !count) return fail(OUX_E_INVALID, "null argument");
  for (int k = 0; k < nkinds; ++k) { ms[k] = 0.0; count[k] = 0; }
  for (auto& r : h->recs) {
    OUX_CUDA(cudaEventSynchronize(r.b));
    float t = 0.f;
    OUX_CUDA(cudaEventElapsedTime(&t, r.a, r.b));
    if (r.kind < nkinds) { ms[r.kind] += t; count[r.kind] += 1; }
  }
  return OUX_OK;
}

int oux_host_ref_diagnostics(int32_t nx, int32_t ny, int32_t nz, int32_t order, double gamma,
                              const float* rho_flat, const float* p_flat, const float* vel_flat,
                              double out[2]) {
  if (!rho_flat || !p_flat || !vel_flat || !out) return fail(OUX_E_INVALID, "null argument");
  if (order != 2 && order != 4 && order != 6) return fail(OUX_E_INVALID, "order must be 2, 4 or 6");
  const int off = order / 2;
  float ent = 0.0f, ke = 0.0f;
  for (int k = 1 + off; k <= nz - off; ++k)
    for (int j = 1 + off; j <= ny - off; ++j)
      for (int i = 1 + off; i <= nx - off; ++i) {
        const size_t l = (size_t)(i - 1) + (size_t)(j - 1) * nx + (size_t)(k - 1) * nx * ny;
        const size_t m = 3 * l;
        const double r = rho_flat[l];
        ent = (float)((double)ent + r * std::log((double)p_flat[l] * std::pow(r, -gamma)));
        const double a = vel_flat[m], b = vel_flat[m + 1], c = vel_flat[m + 2];
        ke = (float)((double)ke + 0.5 * r * (a * a + b * b + c * c));
      }
  const double cnt = (double)((int64_t)(nx - order) * (ny - order) * (nz - order));
  out[0] = (double)(float)((double)ke / cnt);
  out[1] = (double)(float)((double)ent / cnt);
  return OUX_OK;
}

int oux_launch_count(const oux_handle* h, int64_t* launches) {
  if (!h || !launches) return fail(OUX_E_INVALID, "null argument");
  *launches = h->launches;
  return OUX_OK;
}

int oux_rhs_noalloc(const oux_config* cfg, const double* state_dev, double* rhs_dev, void* stream) {
  std::string why;
  int rc = validate(cfg, why);
  if (rc) return fail(rc, why);
  if (!state_dev || !rhs_dev) return fail(OUX_E_INVALID, "null argument");
  if (cfg->precision != OUX_FP64) return fail(OUX_E_INVALID, "oux_rhs_noalloc computes the FP64 form only");
  if ((uintptr_t)state_dev & 255) return fail(OUX_E_INVALID, "state buffer must be 256-byte aligned");
  int vk = visc_kind(cfg, why);
  if (vk < 0) return fail(OUX_E_INVALID, why);
  // The call has no handle and so no boundary rules: LES on a grid with a
  // non-periodic face would give the wall cells' SGS viscosity from the default rule
  // instead of the rule a handle carries (0 on a no-slip wall), so it is refused.
  if (cfg->visc == OUX_LES && (cfg->bc_x || cfg->bc_y || (cfg->dim == 3 && cfg->bc_z)))
    return fail(OUX_E_INVALID, "oux_rhs_noalloc: LES needs periodic x, y and z (no boundary rules without a handle)");
  // a handle on the stack: its host tables stay empty (nothing is allocated)
  oux_handle h;
  h.cfg = *cfg;
  if (h.cfg.dim == 2) { h.cfg.nz = 1; h.cfg.bc_z = 0; }
  const ScratchPlan P = plan_scratch(h.cfg);
  if (P.total > (size_t)OUX_NOALLOC_SCRATCH_BYTES)
    return fail(OUX_E_TOO_SMALL, "oux_rhs_noalloc: this grid needs " + std::to_string(P.total) +
                                     " scratch bytes, more than the fixed OUX_NOALLOC_SCRATCH_BYTES = " +
                                     std::to_string((size_t)OUX_NOALLOC_SCRATCH_BYTES));
  h.G = make_geo(h.cfg);
  h.nv = h.cfg.dim + 2;
  h.vk = vk;
  h.les = h.cfg.visc == OUX_LES;
  h.mixed = false;
  h.K = consts_of(h.cfg);
  unsigned char* scratch = nullptr;
  if ((rc = noalloc_scratch(&scratch))) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  h.Q = const_cast<double*>(state_dev);  // read only: the residual mode writes no state
  h.scratch = scratch;
  h.scratch_bytes = OUX_NOALLOC_SCRATCH_BYTES;
  carve(&h);
  // metric tables: same carve order as oux_bind's upload (1/dx, 1/dy, 1/dz, J, dt*area)
  const Geo& G = h.G;
  const int nx = G.nx, ny = G.ny, nz = G.nz;
  double* m = reinterpret_cast<double*>(scratch + P.metrics);
  h.M.inv_dx = m; m += nx - 1;
  h.M.inv_dy = m; m += ny - 1;
  h.M.inv_dz = m; m += (G.dim == 3 ? nz - 1 : 1);
  h.M.jac = m; m += (size_t)nx * ny;
  if (G.dim == 3) {
    h.M.dtdxdy = m; m += (size_t)(nx - 2) * (ny - 2);
    h.M.dtdydz = m; m += (size_t)(ny - 2) * (nz - 2);
    h.M.dtdzdx = m;
    h.M.dtdx = h.M.dtdy = nullptr;
  } else {
    h.M.dtdx = m; m += nx - 2;
    h.M.dtdy = m;
    h.M.dtdxdy = h.M.dtdydz = h.M.dtdzdx = nullptr;
  }
  h.G.bjac = h.M.jac;
  // raw spacings staged in the (unused here) stage-state region, then expanded on the device
  double* d = reinterpret_cast<double*>(scratch + P.q2);
  OUX_CUDA(cudaMemcpyAsync(d, cfg->dx, (size_t)(nx - 1) * sizeof(double), cudaMemcpyHostToDevice, s));
  OUX_CUDA(cudaMemcpyAsync(d + (nx - 1), cfg->dy, (size_t)(ny - 1) * sizeof(double), cudaMemcpyHostToDevice, s));
  if (G.dim == 3)
    OUX_CUDA(cudaMemcpyAsync(d + (nx - 1) + (ny - 1), cfg->dz, (size_t)(nz - 1) * sizeof(double),
                             cudaMemcpyHostToDevice, s));
  k_noalloc_tables<<<grid_for((int64_t)nx * ny, 256), 256, 0, s>>>(d, G, h.cfg.dt, h.M);
  OUX_CUDA(cudaGetLastError());
  // what must start at zero: the status word and the output (ghost entries stay 0)
  OUX_CUDA(cudaMemsetAsync(h.status, 0, sizeof(int), s));
  const size_t n = (size_t)h.nv * (nx - 2) * (ny - 2) * (G.dim == 3 ? nz - 2 : 1);
  OUX_CUDA(cudaMemsetAsync(rhs_dev, 0, n * sizeof(double), s));
  StepArgs<double> A = base_args<double>(&h);
  A.mode = CM_R_OUT; A.coef = 1.0; A.Rout = rhs_dev;
  if ((rc = run_stage<double, double>(&h, h.Q, A, s))) return rc;
  OUX_CUDA(cudaGetLastError());
  return OUX_OK;
}

}  // extern "C"
