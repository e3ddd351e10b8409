// Kernels of one explicit stage on the ghost-padded SoA layout.
//
// Per stage (3D): prim -> [sensor] -> [SGS mut/qc2 + their edge copy] ->
//   x sweep (faces -> dt*S*dE into Racc) -> y sweep (+= dt*S*dF) ->
//   z sweep (+= dt*S*dG, then the RK combination) -> ghost fill.
// Face fluxes never touch HBM: each sweep block computes the 2*ORDER/2 + 32
// cell tile of its pencil rows into shared memory, evaluates every face of the
// tile once, and differences neighbouring faces in shared memory.
#pragma once
#include <cstdint>
#include "oux_math.cuh"

namespace oux {

enum ViscKind { VK_EULER = 0, VK_C6 = 1, VK_C4 = 2, VK_ME4 = 3, VK_GV2 = 4, VK_2D4 = 5,
                // 3D Navier-Stokes grids with a non-periodic direction: the same stencils
                // with the convective order lowered next to a boundary and the viscous
                // faces outside the high-order guard on the 2nd-order fallback
                VK_C6W = 6, VK_C4W = 7, VK_ME4W = 8, VK_GV2W = 9 };
__host__ __device__ constexpr int vk_base(int vk) {
  return vk == VK_C6W ? VK_C6 : vk == VK_C4W ? VK_C4 : vk == VK_ME4W ? VK_ME4 : vk == VK_GV2W ? VK_GV2 : vk;
}
__host__ __device__ constexpr bool vk_wall(int vk) { return vk >= VK_C6W; }
// Stage combinations of 3D_solver/src/calc_steps.f90 with Qn = the FP64 state
// Q^n and Qs = the stage state (FP64 in the plain form, FP32 in the mixed form);
// all arithmetic of the combinations is FP64.
enum CombineMode {
  CM_ACCUM = 0,   // first/middle sweep: Racc (=|+=) c * dF
  CM_R_OUT = 1,   // last sweep: write R to an output buffer (reference Rs order)
  CM_RK3_1 = 2,   // Qs = Qn - R                                (calc_step1)
  CM_RK3_2 = 3,   // Qs = (c1*Qn + c2*Qs - R) * c4              (calc_step2_3, stage 2)
  CM_RK3_3 = 4,   // Qn = (c1*Qs + c2*Qn - R) * c4              (calc_step2_3, stage 3)
  CM_RK4_S = 5,   // Qs = Qn - c1*R ; Rs = Rs + c2*R            (calc_step)
  CM_RK4_4 = 6    // R = Rs + R ; Qn = Qn - R/6 ; Rs = 0        (calc_step4)
};

struct Geo {
  int dim, nx, ny, nz, g;     // padded extents, ghost width
  int gx, bcx;                // x ghost width of the cell ranges (g, or 1 for a non-periodic x), bc_x
  int gy, bcy;                // the same for y
  int gz;                     // z ghost width of the cell ranges (g, or 1 for a non-periodic z)
  int bcz;                    // enum oux_bc_z: 0 periodic; 1 non-periodic (both ends); slabs whose
                              // z ghost planes come from the neighbours: 2 both ends, 3 / 4 the
                              // upper / lower end only (the other end is the grid's boundary)
  int bkind;                  // boundary-cell rule of face f (enum oux_bc_kind) in bits 4f..4f+3;
                              // faces 0..5: x low, x high, y low, y high, z low, z high
  int64_t sx, plane, vs;      // row stride, plane stride, variable stride (elements)
  const double* bfix[4];      // OUX_BC_FIXED faces: nv x (ny for x faces, nx for y faces) values of Q/J
  double gamma_1, over_gamma_1;  // gamma - 1 and 1 / (gamma - 1), for the wall and far-field rules
  double gamma, over_gamma;
  const signed char* bkinds[4];  // per-position rule of a face (overrides its kind), or null
  double bpar[4][4];          // far-field state of a face: rho, tangential and normal velocity, c
  int ylast;                  // 1: y faces applied after x faces (corners take their y rule)
  const double* bjac;         // J(nx, ny), for the far-field and Neumann rules
  const double* bfix3[6];     // 3D: fixed values of the faces x lo .. z hi
  int pk0, pk1;               // z planes [pk0, pk1) the primitive (+ sensor) pass of a stage covers
  int gk0, gk1;               // z planes [gk0, gk1) the gradient pass covers
  int sk0, sk1;               // z planes [sk0, sk1) of the cells the sweeps update
                              // (defaults: every plane / every plane / every interior plane; a z
                              // slab's stage split into an interior part and the parts next to
                              // its ends narrows them, oux_stage_part)
  int uni;                    // bit a: every spacing along axis a is the same double (so are
                              // the inverse spacings), which lets the ME4 sweeps share the
                              // values of a face position between the three faces using it
  __host__ __device__ int64_t at(int i, int j, int k) const { return (int64_t)k * plane + (int64_t)j * sx + i; }
};

template <class T> struct Fields {
  // primitive / auxiliary arrays (each vs elements)
  T *rho, *u, *v, *w, *p, *T_, *mu, *sensor, *mut, *qc2;
  // node velocity gradient d(vel_c)/d(x_a) at index 3*c + a (3D: 9, 2D: c,a < 2)
  T* grad[9];
};

struct Metrics {
  const double *inv_dx, *inv_dy, *inv_dz;   // 1/dx, n-1 each
  const double *jac;                        // (nx,ny)
  const double *dtdxdy, *dtdydz, *dtdzdx;   // 3D: (nx-2)(ny-2), (ny-2)(nz-2), (nx-2)(nz-2)
  const double *dtdx, *dtdy;                // 2D: nx-2, ny-2
};

template <class T> struct StepArgs {
  Geo G;
  Fields<T> W;
  Metrics M;
  PhysConst K;
  int scheme, tvd, slau;
  // state (conservative / J) and accumulators, nv * vs each
  double* Qn;   // Q^n, FP64
  T* Qs;        // stage state Q^(1), Q^(2) (RK3) / Q^(s) (RK4)
  double* Rs;   // RK4 accumulator, FP64
  double* Racc; // running flux difference (FP64)
  double* Rout; // CM_R_OUT destination
  double coef;  // metric scale (RK3 coef3 or 1)
  double c1, c2, c4;
  int mode;
  // single solves: HOST address of the handle's x / y sweep tile tensor maps, which the
  // launch passes to the sweep kernels by value (null: the tiles are staged with
  // cp.async; never dereferenced on the device), and the status word a TMA wait that
  // runs out marks with OUX_FAULT_TIMEOUT
  const void* tmaps;
  int* status;
};

// Load through the read-only data path when the caller guarantees the array is
// not written during the kernel (RO = true: the single-solve kernels); plain
// coherent load otherwise (the batched kernel, where other blocks of the same
// launch produce the fields).
template <bool RO, class T>
__device__ __forceinline__ T ldro(const T* p) {
  if constexpr (RO) return __ldg(p);
  else return *p;
}

// Padded cell (i, j, k) of a flat index t (x fastest over nx, then ny, then nz).
__device__ __forceinline__ void cell_of(const Geo& G, int64_t t, int& i, int& j, int& k) {
  i = (int)(t % G.nx);
  const int64_t r = t / G.nx;
  j = (int)(r % G.ny);
  k = (int)(r / G.ny);
}

// Plane-flattened launch of a per-cell kernel: blockIdx.y is the z plane, and a
// block's 256 threads cover 256 consecutive cells of the plane (x fastest), so the
// cell follows from one 32-bit division per thread.
constexpr int PLANE_THREADS = 256;
__device__ __forceinline__ bool plane_cell(const Geo& G, int& i, int& j, int& k) {
  const int t = blockIdx.x * PLANE_THREADS + threadIdx.x;
  if (t >= G.nx * G.ny) return false;
  j = t / G.nx;
  i = t - j * G.nx;
  k = G.pk0 + blockIdx.y;
  return true;
}
inline dim3 plane_grid(const Geo& G) {
  return dim3((unsigned)((G.nx * G.ny + PLANE_THREADS - 1) / PLANE_THREADS), (unsigned)(G.pk1 - G.pk0), 1);
}

// ---- prim: src/calc_physical_quantities.f90:60-116 (3D), :7-57 (2D) -------
template <int DIM, bool VISC, class TS, class T, bool RO = false>
__device__ __forceinline__ void prim_cell(const TS* Q, const Geo& G, const Fields<T>& W, const double* jac,
                                          const PhysConst& K, int i, int j, int k) {
  int64_t o = G.at(i, j, k);
  T Jv = (T)ldro<RO>(jac + (int64_t)j * G.nx + i);
  T q1 = (T)ldro<RO>(Q + o);
  T over_Q1 = T(1) / q1;
  T rho = Jv * q1;
  T u = (T)ldro<RO>(Q + o + G.vs) * over_Q1;
  T v = (T)ldro<RO>(Q + o + 2 * G.vs) * over_Q1;
  T w = T(0), p;
  if constexpr (DIM == 3) {
    w = (T)ldro<RO>(Q + o + 3 * G.vs) * over_Q1;
    p = T(K.gamma_1) * (Jv * (T)ldro<RO>(Q + o + 4 * G.vs) - T(0.5) * rho * (u * u + v * v + w * w));
  } else {
    p = T(K.gamma_1) * (Jv * (T)ldro<RO>(Q + o + 3 * G.vs) - T(0.5) * rho * (u * u + v * v));
  }
  W.rho[o] = rho; W.u[o] = u; W.v[o] = v;
  if constexpr (DIM == 3) W.w[o] = w;
  W.p[o] = p;
  T temp = p / (T(K.R) * rho);
  W.T_[o] = temp;
  if constexpr (VISC) W.mu[o] = T(K.sutherland) / (temp + T(111)) * (temp * sqrt(temp));
}

template <int DIM, bool VISC, class TS, class T, bool RO = false>
__device__ __forceinline__ void prim_cell(const TS* Q, const Geo& G, const Fields<T>& W, const double* jac,
                                          const PhysConst& K, int64_t t) {
  int i, j, k;
  cell_of(G, t, i, j, k);
  prim_cell<DIM, VISC, TS, T, RO>(Q, G, W, jac, K, i, j, k);
}

template <int DIM, bool VISC, class TS, class T>
__global__ void __launch_bounds__(PLANE_THREADS) k_prim(const TS* __restrict__ Q, Geo G, Fields<T> W,
                                                        const double* __restrict__ jac, PhysConst K) {
  int i, j, k;
  if (plane_cell(G, i, j, k)) prim_cell<DIM, VISC, TS, T, true>(Q, G, W, jac, K, i, j, k);
}

// ---- mixed-form primitives: Q = Q^n (FP64) + dQ (FP32 stage increment, may be
// null), evaluated in FP64 like k_prim, stored in FP32 with p and T as deviations
// from the per-solve references K.p_ref, K.T_ref.
template <int DIM, bool VISC, bool RO = false>
__device__ __forceinline__ void prim_mx_cell(const double* Qn, const float* dQ, const Geo& G,
                                             const Fields<float>& W, const double* jac, const PhysConst& K,
                                             int i, int j, int k) {
  int64_t o = G.at(i, j, k);
  double q[5];
#pragma unroll
  for (int l = 0; l < DIM + 2; ++l)
    q[l] = ldro<RO>(Qn + o + l * G.vs) + (dQ ? (double)ldro<RO>(dQ + o + l * G.vs) : 0.0);
  double Jv = ldro<RO>(jac + (int64_t)j * G.nx + i);
  double over = 1.0 / q[0], rho = Jv * q[0];
  double u = q[1] * over, v = q[2] * over, w = 0.0, p;
  if constexpr (DIM == 3) {
    w = q[3] * over;
    p = K.gamma_1 * (Jv * q[4] - 0.5 * rho * (u * u + v * v + w * w));
  } else {
    p = K.gamma_1 * (Jv * q[3] - 0.5 * rho * (u * u + v * v));
  }
  double temp = p / (K.R * rho);
  W.rho[o] = (float)rho; W.u[o] = (float)u; W.v[o] = (float)v;
  if constexpr (DIM == 3) W.w[o] = (float)w;
  W.p[o] = (float)(p - K.p_ref);
  W.T_[o] = (float)(temp - K.T_ref);
  if constexpr (VISC) W.mu[o] = (float)(K.sutherland / (temp + 111.0) * (temp * sqrt(temp)));
}

template <int DIM, bool VISC, bool RO = false>
__device__ __forceinline__ void prim_mx_cell(const double* Qn, const float* dQ, const Geo& G,
                                             const Fields<float>& W, const double* jac, const PhysConst& K,
                                             int64_t t) {
  int i, j, k;
  cell_of(G, t, i, j, k);
  prim_mx_cell<DIM, VISC, RO>(Qn, dQ, G, W, jac, K, i, j, k);
}

template <int DIM, bool VISC>
__global__ void __launch_bounds__(PLANE_THREADS) k_prim_mx(const double* __restrict__ Qn,
                                                           const float* __restrict__ dQ, Geo G, Fields<float> W,
                                                           const double* __restrict__ jac, PhysConst K) {
  int i, j, k;
  if (plane_cell(G, i, j, k)) prim_mx_cell<DIM, VISC, true>(Qn, dQ, G, W, jac, K, i, j, k);
}

// ---- Ducros sensor: calc_Ducros (3D_solver/src/calc_hybrid.f90:11-72; 2D twin
// :11-55) on cells 1..n-2, with the reference's copies to the outer faces.
// sensor_of_diffs takes the raw central differences df(c, a) = -vel_c(o - st_a) +
// vel_c(o + st_a) of velocity component c along axis a (the caller has checked that
// the cell lies in 1..n-2 on every axis), so that a pass which has loaded those
// neighbours already (k_grad) reuses them.
// The sensor value from the summed divergence and the rotation components, stored
// with the reference's copies to the outer faces (3D: r1, r2, r3; 2D: r3 = rot).
template <int DIM, class T>
__device__ __forceinline__ void ducros_store(const Geo& G, const Fields<T>& W, int i, int j, int k, T div, T r1,
                                             T r2, T r3) {
  const T eps = T(1.0e-12);
  T f;
  if constexpr (DIM == 3) f = (div * div) / (div * div + (r1 * r1 + r2 * r2 + r3 * r3) + eps);
  else f = (div * div) / (div * div + r3 * r3 + eps);
  f = fmin_f(T(1), f);
  W.sensor[G.at(i, j, k)] = f;
  if (i == 1) W.sensor[G.at(0, j, k)] = f; else if (i == G.nx - 2) W.sensor[G.at(G.nx - 1, j, k)] = f;
  if (j == 1) W.sensor[G.at(i, 0, k)] = f; else if (j == G.ny - 2) W.sensor[G.at(i, G.ny - 1, k)] = f;
  if constexpr (DIM == 3) {
    if (k == 1) W.sensor[G.at(i, j, 0)] = f; else if (k == G.nz - 2) W.sensor[G.at(i, j, G.nz - 1)] = f;
  }
}

// Central difference scale of the sensor along an axis at cell c.
template <class T>
__device__ __forceinline__ T ducros_scale(const double* inv, int c) {
  return T(0.25) * ((T)inv[c - 1] + (T)inv[c]);
}

template <int DIM, class T, class DF>
__device__ __forceinline__ void sensor_of_diffs(const Geo& G, const Fields<T>& W, const Metrics& M, int i, int j,
                                                int k, DF df) {
  T dxt = ducros_scale<T>(M.inv_dx, i);
  T dyt = ducros_scale<T>(M.inv_dy, j);
  if constexpr (DIM == 3) {
    T dzt = ducros_scale<T>(M.inv_dz, k);
    T dudx = df(0, 0) * dxt;
    T dvdx = df(1, 0) * dxt;
    T dwdx = df(2, 0) * dxt;
    T dudy = df(0, 1) * dyt;
    T dvdy = df(1, 1) * dyt;
    T dwdy = df(2, 1) * dyt;
    T dudz = df(0, 2) * dzt;
    T dvdz = df(1, 2) * dzt;
    T dwdz = df(2, 2) * dzt;
    T div = dudx + dvdy + dwdz;
    ducros_store<3, T>(G, W, i, j, k, div, dwdy - dvdz, dudz - dwdx, dvdx - dudy);
  } else {
    T dudx = df(0, 0) * dxt;
    T dvdx = df(1, 0) * dxt;
    T dudy = df(0, 1) * dyt;
    T dvdy = df(1, 1) * dyt;
    ducros_store<2, T>(G, W, i, j, k, dudx + dvdy, T(0), T(0), dvdx - dudy);
  }
}

template <int DIM, class T, bool RO = false>
__device__ __forceinline__ void sensor_cell(const Geo& G, const Fields<T>& W, const Metrics& M, int i, int j,
                                            int k) {
  if (i < 1 || i > G.nx - 2 || j < 1 || j > G.ny - 2) return;
  if (DIM == 3 && (k < 1 || k > G.nz - 2)) return;
  const int64_t o = G.at(i, j, k);
  const T* vel[3] = {W.u, W.v, W.w};
  const int64_t st[3] = {1, G.sx, G.plane};
  sensor_of_diffs<DIM, T>(G, W, M, i, j, k, [&](int c, int a) -> T {
    return -ldro<RO>(vel[c] + o - st[a]) + ldro<RO>(vel[c] + o + st[a]);
  });
}

template <int DIM, class T, bool RO = false>
__device__ __forceinline__ void sensor_cell(const Geo& G, const Fields<T>& W, const Metrics& M, int64_t t) {
  int i, j, k;
  cell_of(G, t, i, j, k);
  sensor_cell<DIM, T, RO>(G, W, M, i, j, k);
}

template <int DIM, class T>
__global__ void __launch_bounds__(PLANE_THREADS) k_sensor(Geo G, Fields<T> W, Metrics M) {
  int i, j, k;
  if (plane_cell(G, i, j, k)) sensor_cell<DIM, T, false>(G, W, M, i, j, k);
}

// Mixed form: the sensor from FP64 velocities decoded from Q^n + the FP32 stage
// increment (dQ, null for the first stage) the way prim_mx_cell decodes them, with the
// FP64 sensor's arithmetic, rounded once when stored.  The FP32 velocity fields carry
// relative rounding errors of 6e-8, and the velocity differences of the sensor cancel
// them into much larger relative errors of the divergence; this way the sensor is the
// FP64 solve's value for the same state to within one FP32 rounding, so the hybrid
// threshold and the TVD switch flip only where a face value lies that close to 0.4.
template <int DIM, bool RO = false>
__device__ __forceinline__ void sensor_mx_cell(const Geo& G, const double* Qn, const float* dQ,
                                               const Fields<float>& W, const Metrics& M, int i, int j, int k) {
  if (i < 1 || i > G.nx - 2 || j < 1 || j > G.ny - 2) return;
  if (DIM == 3 && (k < 1 || k > G.nz - 2)) return;
  const int64_t o = G.at(i, j, k);
  auto q = [&](int64_t c, int l) -> double {
    const int64_t a = c + l * G.vs;
    return ldro<RO>(Qn + a) + (dQ ? (double)ldro<RO>(dQ + a) : 0.0);
  };
  // velocities of cell c (prim_mx_cell: over = 1 / q0, u = q1 * over)
  auto vel = [&](int64_t c, double (&v)[3]) {
    const double over = 1.0 / q(c, 0);
    v[0] = q(c, 1) * over;
    v[1] = q(c, 2) * over;
    v[2] = DIM == 3 ? q(c, 3) * over : 0.0;
  };
  const double eps = 1.0e-12;
  const double dxt = 0.25 * (M.inv_dx[i - 1] + M.inv_dx[i]);
  const double dyt = 0.25 * (M.inv_dy[j - 1] + M.inv_dy[j]);
  double f;
  double xm[3], xp[3], ym[3], yp[3];
  vel(o - 1, xm);
  vel(o + 1, xp);
  vel(o - G.sx, ym);
  vel(o + G.sx, yp);
  if constexpr (DIM == 3) {
    double zm[3], zp[3];
    vel(o - G.plane, zm);
    vel(o + G.plane, zp);
    const double dzt = 0.25 * (M.inv_dz[k - 1] + M.inv_dz[k]);
    const double dudx = (-xm[0] + xp[0]) * dxt, dvdx = (-xm[1] + xp[1]) * dxt, dwdx = (-xm[2] + xp[2]) * dxt;
    const double dudy = (-ym[0] + yp[0]) * dyt, dvdy = (-ym[1] + yp[1]) * dyt, dwdy = (-ym[2] + yp[2]) * dyt;
    const double dudz = (-zm[0] + zp[0]) * dzt, dvdz = (-zm[1] + zp[1]) * dzt, dwdz = (-zm[2] + zp[2]) * dzt;
    const double div = dudx + dvdy + dwdz;
    const double r1 = dwdy - dvdz, r2 = dudz - dwdx, r3 = dvdx - dudy;
    f = (div * div) / (div * div + (r1 * r1 + r2 * r2 + r3 * r3) + eps);
  } else {
    const double dudx = (-xm[0] + xp[0]) * dxt, dvdx = (-xm[1] + xp[1]) * dxt;
    const double dudy = (-ym[0] + yp[0]) * dyt, dvdy = (-ym[1] + yp[1]) * dyt;
    const double div = dudx + dvdy;
    const double rot = dvdx - dudy;
    f = (div * div) / (div * div + rot * rot + eps);
  }
  const float fs = (float)fmin_f(1.0, f);
  W.sensor[o] = fs;
  if (i == 1) W.sensor[G.at(0, j, k)] = fs; else if (i == G.nx - 2) W.sensor[G.at(G.nx - 1, j, k)] = fs;
  if (j == 1) W.sensor[G.at(i, 0, k)] = fs; else if (j == G.ny - 2) W.sensor[G.at(i, G.ny - 1, k)] = fs;
  if constexpr (DIM == 3) {
    if (k == 1) W.sensor[G.at(i, j, 0)] = fs; else if (k == G.nz - 2) W.sensor[G.at(i, j, G.nz - 1)] = fs;
  }
}

template <int DIM, bool RO = false>
__device__ __forceinline__ void sensor_mx_cell(const Geo& G, const double* Qn, const float* dQ,
                                               const Fields<float>& W, const Metrics& M, int64_t t) {
  int i, j, k;
  cell_of(G, t, i, j, k);
  sensor_mx_cell<DIM, RO>(G, Qn, dQ, W, M, i, j, k);
}

template <int DIM>
__global__ void __launch_bounds__(PLANE_THREADS) k_sensor_mx(Geo G, const double* __restrict__ Qn,
                                                             const float* __restrict__ dQ, Fields<float> W,
                                                             Metrics M) {
  int i, j, k;
  if (plane_cell(G, i, j, k)) sensor_mx_cell<DIM, true>(G, Qn, dQ, W, M, i, j, k);
}

// ---- primitives and Ducros sensor in one pass (3D) --------------------------------
// A block owns a PS_TX x PS_TY column of cells (x, y) over PS_PLANES z planes and
// marches along z.  For every plane it decodes the velocities of its cells and of a
// one-cell ring around them into shared memory (the last three planes are kept),
// writes its own cells' primitive fields (prim_cell / prim_mx_cell), and evaluates the
// previous plane's sensor from shared memory with the FP64 sensor's arithmetic
// (calc_Ducros, 3D_solver/src/calc_hybrid.f90:11-72, with the reference's copies to
// the outer faces).  Q is read once per cell plus the ring (mostly from L2), and the
// sensor's neighbour velocities never leave the SM.
//   FP64 form: the same bits as k_prim then k_sensor (the same expressions on the
//   same values).
//   Mixed form (MX): velocities decoded in FP64 from Q^n + the FP32 increment dQ, so
//   the sensor is sensor_mx_cell's value, rounded once when stored.
constexpr int PS_TX = 32, PS_TY = 8, PS_PLANES = 32;

template <int HD> __host__ __device__ constexpr size_t prim_fused_smem() {
  return sizeof(double) * (2 * HD + 1) * 3 * (PS_TY + 2 * HD) * (PS_TX + 2 * HD);
}

inline dim3 prim_fused_grid(const Geo& G) {
  return dim3((unsigned)((G.nx + PS_TX - 1) / PS_TX), (unsigned)((G.ny + PS_TY - 1) / PS_TY),
              (unsigned)((G.pk1 - G.pk0 + PS_PLANES - 1) / PS_PLANES));
}

template <int HD, bool SENSOR, bool VISC, bool MX, class TS, class T>
__global__ void __launch_bounds__(PS_TX * PS_TY) k_prim_fused(const TS* __restrict__ Q, const float* __restrict__ dQ,
                                                              Geo G, Fields<T> W, Metrics M, PhysConst K) {
  static_assert(HD == 1, "the sensor's ring is one cell wide");
  constexpr int NW = 2 * HD + 1;                      // planes kept
  constexpr int RX = PS_TX + 2 * HD, RY = PS_TY + 2 * HD;
  extern __shared__ __align__(16) unsigned char smraw[];
  double* vel = reinterpret_cast<double*>(smraw);     // [plane slot][component][ry][rx]
  auto V = [&](int slot, int c, int y, int x) -> double& { return vel[((slot * 3 + c) * RY + y) * RX + x]; };
  const int tid = threadIdx.x;
  const int bx = blockIdx.x * PS_TX, by = blockIdx.y * PS_TY;
  const int k0 = G.pk0 + blockIdx.z * PS_PLANES, k1 = min(G.pk1, k0 + PS_PLANES);
  const int tx = tid % PS_TX, ty = tid / PS_TX;
  const int oi = bx + tx, oj = by + ty;  // this thread's own cell
  const bool own = oi < G.nx && oj < G.ny;
  const int rx = tx + HD, ry = ty + HD;  // and its place in the ring
  auto slot_of = [](int k) { return (k % NW + NW) % NW; };
  for (int kk = k0 - HD; kk < k1 + HD; ++kk) {
    // 1. velocities of plane kk (block cells and ring)
    if (kk >= 0 && kk < G.nz) {
      const int slot = slot_of(kk);
      for (int c = tid; c < RX * RY; c += PS_TX * PS_TY) {
        const int cx = c % RX, cy = c / RX;
        const int i = bx - HD + cx, j = by - HD + cy;
        if (i < 0 || i >= G.nx || j < 0 || j >= G.ny) continue;
        const int64_t o = G.at(i, j, kk);
        double q0, q1, q2, q3;
        if constexpr (MX) {
          const double* Qd = reinterpret_cast<const double*>(Q);
          q0 = __ldg(Qd + o) + (dQ ? (double)__ldg(dQ + o) : 0.0);
          q1 = __ldg(Qd + o + G.vs) + (dQ ? (double)__ldg(dQ + o + G.vs) : 0.0);
          q2 = __ldg(Qd + o + 2 * G.vs) + (dQ ? (double)__ldg(dQ + o + 2 * G.vs) : 0.0);
          q3 = __ldg(Qd + o + 3 * G.vs) + (dQ ? (double)__ldg(dQ + o + 3 * G.vs) : 0.0);
        } else {
          q0 = (double)__ldg(Q + o);
          q1 = (double)__ldg(Q + o + G.vs);
          q2 = (double)__ldg(Q + o + 2 * G.vs);
          q3 = (double)__ldg(Q + o + 3 * G.vs);
        }
        const double over = 1.0 / q0;  // prim_cell / prim_mx_cell: u = q1 * (1 / q0)
        V(slot, 0, cy, cx) = q1 * over;
        V(slot, 1, cy, cx) = q2 * over;
        V(slot, 2, cy, cx) = q3 * over;
      }
      // 2. the block's own cells: every primitive field
      if (own && kk >= k0 && kk < k1) {
        if constexpr (MX) prim_mx_cell<3, VISC, true>(reinterpret_cast<const double*>(Q), dQ, G, W, M.jac, K, oi, oj, kk);
        else prim_cell<3, VISC, TS, T, true>(Q, G, W, M.jac, K, oi, oj, kk);
      }
    }
    __syncthreads();
    // 3. the sensor of plane k = kk - 1 from the planes k - 1, k, k + 1
    if constexpr (SENSOR) {
      const int k = kk - 1;
      if (own && k >= k0 && k < k1 && oi >= 1 && oi <= G.nx - 2 && oj >= 1 && oj <= G.ny - 2 && k >= 1 &&
          k <= G.nz - 2) {
        const int sm = slot_of(k - 1), s0 = slot_of(k), sp = slot_of(k + 1);
        const double dxt = 0.25 * (M.inv_dx[oi - 1] + M.inv_dx[oi]);
        const double dyt = 0.25 * (M.inv_dy[oj - 1] + M.inv_dy[oj]);
        const double dzt = 0.25 * (M.inv_dz[k - 1] + M.inv_dz[k]);
        const double dudx = (-V(s0, 0, ry, rx - 1) + V(s0, 0, ry, rx + 1)) * dxt;
        const double dvdx = (-V(s0, 1, ry, rx - 1) + V(s0, 1, ry, rx + 1)) * dxt;
        const double dwdx = (-V(s0, 2, ry, rx - 1) + V(s0, 2, ry, rx + 1)) * dxt;
        const double dudy = (-V(s0, 0, ry - 1, rx) + V(s0, 0, ry + 1, rx)) * dyt;
        const double dvdy = (-V(s0, 1, ry - 1, rx) + V(s0, 1, ry + 1, rx)) * dyt;
        const double dwdy = (-V(s0, 2, ry - 1, rx) + V(s0, 2, ry + 1, rx)) * dyt;
        const double dudz = (-V(sm, 0, ry, rx) + V(sp, 0, ry, rx)) * dzt;
        const double dvdz = (-V(sm, 1, ry, rx) + V(sp, 1, ry, rx)) * dzt;
        const double dwdz = (-V(sm, 2, ry, rx) + V(sp, 2, ry, rx)) * dzt;
        const double div = dudx + dvdy + dwdz;
        const double r1 = dwdy - dvdz, r2 = dudz - dwdx, r3 = dvdx - dudy;
        double f = (div * div) / (div * div + (r1 * r1 + r2 * r2 + r3 * r3) + 1.0e-12);
        f = fmin_f(1.0, f);
        const T fs = (T)f;
        const int i = oi, j = oj;
        W.sensor[G.at(i, j, k)] = fs;
        if (i == 1) W.sensor[G.at(0, j, k)] = fs; else if (i == G.nx - 2) W.sensor[G.at(G.nx - 1, j, k)] = fs;
        if (j == 1) W.sensor[G.at(i, 0, k)] = fs; else if (j == G.ny - 2) W.sensor[G.at(i, G.ny - 1, k)] = fs;
        if (k == 1) W.sensor[G.at(i, j, 0)] = fs; else if (k == G.nz - 2) W.sensor[G.at(i, j, G.nz - 1)] = fs;
      }
    }
    __syncthreads();
  }
}

// ---- node velocity gradients (3D, the high-order viscous stencils) ----------------
// grad[3c + a] = d(velocity c)/d(axis a) by the 6th-order (SIXTH: Central-6) or 4th-order
// (Central-4, ME4) central node derivative of the viscous loaders
// (load_smem_visc_cent.f90.fypp:51-70, load_smem_visc_me4_base.f90:120-127), at every
// cell whose stencil fits in the grid (else 0: no sweep reads those), on the z planes
// [gk0, gk1).  Plane-flattened like k_prim: the neighbours come through L1 / L2.
// Measured slower on B200 at 518^3: a z-marching variant with a shared-memory ring of
// the velocities filled by cp.async one plane ahead (3.78 against 2.96 ms without the
// sensor), and 32 x 8 tiles of one plane staged in shared memory with their x / y
// ring, the z neighbours from L2 (FP64 with the sensor 4.76 against 3.84 ms; FP32
// without it 2.06 against 2.17).
template <bool SIXTH, class T>
__device__ __forceinline__ T node_deriv_of(T m3, T m2, T m1, T p1, T p2, T p3, T inv) {
  if constexpr (SIXTH)
    return (T(1.0 / 60.0) * (-m3 + p3) + T(0.15) * (m2 - p2) + T(0.75) * (-m1 + p1)) * inv;
  else
    return (T(2.0 / 3.0) * (-m1 + p1) - T(1.0 / 12.0) * (-m2 + p2)) * inv;
}

inline dim3 grad_grid(const Geo& G) {
  return dim3((unsigned)((G.nx * G.ny + PLANE_THREADS - 1) / PLANE_THREADS), (unsigned)(G.gk1 - G.gk0), 1);
}

// SENSOR: the same pass also writes the Ducros sensor of its cells from the +-1
// neighbours it loads for the gradients (the arithmetic of sensor_of_diffs), so that
// the primitive pass before it can be the plain per-cell k_prim.  Every neighbour value
// is loaded once and feeds both.  Bounded to 8 blocks per SM (32 registers; the FP64
// sensor pass spills 24 B): measured on B200 at 518^3 faster than its 40 registers at
// 6 blocks per SM, 3.79 against 4.06 ms (this latency-bound pass wants resident warps).
template <bool SIXTH, class T, bool SENSOR = false>
__global__ void __launch_bounds__(PLANE_THREADS, 8) k_grad(Geo G, Fields<T> W, Metrics M) {
  const int t = blockIdx.x * PLANE_THREADS + threadIdx.x;
  if (t >= G.nx * G.ny) return;
  int c[3];
  c[1] = t / G.nx;
  c[0] = t - c[1] * G.nx;
  c[2] = G.gk0 + blockIdx.y;
  constexpr int HD = SIXTH ? 3 : 2;
  const int n[3] = {G.nx, G.ny, G.nz};
  const int64_t st[3] = {1, G.sx, G.plane};
  const double* invd[3] = {M.inv_dx, M.inv_dy, M.inv_dz};
  const T* vel[3] = {W.u, W.v, W.w};
  const int64_t o = G.at(c[0], c[1], c[2]);
  // the sensor's cells: 1..n-2 on every axis
  const bool sens = SENSOR && c[0] >= 1 && c[0] <= n[0] - 2 && c[1] >= 1 && c[1] <= n[1] - 2 && c[2] >= 1 &&
                    c[2] <= n[2] - 2;
  // the sensor's terms, summed axis by axis in the order sensor_of_diffs sums them, so
  // that few of them are live at once
  T div = T(0), r1 = T(0), r2 = T(0), r3 = T(0), dwdx = T(0), dwdy = T(0);
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const bool fits = c[a] >= HD && c[a] + HD < n[a];
    const T inv = fits ? (T)invd[a][c[a]] : T(0);
    const T sc = sens ? ducros_scale<T>(invd[a], c[a]) : T(0);
    T d[3];  // (-vel_q(o - st_a) + vel_q(o + st_a)) times the sensor's scale
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const T* f = vel[q] + o;
      T gq = T(0);
      d[q] = T(0);
      if (fits) {
        const T m1 = __ldg(f - st[a]), p1 = __ldg(f + st[a]);
        const T m2 = __ldg(f - 2 * st[a]), p2 = __ldg(f + 2 * st[a]);
        T m3 = T(0), p3 = T(0);
        if constexpr (SIXTH) { m3 = __ldg(f - 3 * st[a]); p3 = __ldg(f + 3 * st[a]); }
        gq = node_deriv_of<SIXTH, T>(m3, m2, m1, p1, p2, p3, inv);
        if (sens) d[q] = (-m1 + p1) * sc;
      } else if (sens) {
        d[q] = (-__ldg(f - st[a]) + __ldg(f + st[a])) * sc;
      }
      W.grad[3 * q + a][o] = gq;
    }
    if constexpr (SENSOR) {
      if (a == 0) { div = d[0]; r3 = d[1]; dwdx = d[2]; }                  // dudx, dvdx, dwdx
      else if (a == 1) { div = div + d[1]; r3 = r3 - d[0]; dwdy = d[2]; }  // + dvdy; dvdx - dudy
      else { div = div + d[2]; r1 = dwdy - d[1]; r2 = d[0] - dwdx; }      // + dwdz; dwdy - dvdz; dudz - dwdx
    }
  }
  if constexpr (SENSOR) {
    if (sens) ducros_store<3, T>(G, W, c[0], c[1], c[2], div, r1, r2, r3);
  }
}

// ---- SMS sub-grid model: 3D_solver/src/calc_les.f90:30-125 -------------------
template <class T>
__device__ __forceinline__ void grad3(const T (&u)[3][3][3], const T (&v)[3][3][3], const T (&w)[3][3][3],
                                      T dx, T dy, T dz, T d[9]) {  // calc_differential :11-27
  d[0] = T(0.5) * (-u[1][1][0] + u[1][1][2]) * dx;
  d[1] = T(0.5) * (-u[1][0][1] + u[1][2][1]) * dy;
  d[2] = T(0.5) * (-u[0][1][1] + u[2][1][1]) * dz;
  d[3] = T(0.5) * (-v[1][1][0] + v[1][1][2]) * dx;
  d[4] = T(0.5) * (-v[1][0][1] + v[1][2][1]) * dy;
  d[5] = T(0.5) * (-v[0][1][1] + v[2][1][1]) * dz;
  d[6] = T(0.5) * (-w[1][1][0] + w[1][1][2]) * dx;
  d[7] = T(0.5) * (-w[1][0][1] + w[1][2][1]) * dy;
  d[8] = T(0.5) * (-w[0][1][1] + w[2][1][1]) * dz;
}

template <class T>
__device__ __forceinline__ T filt(const T* a, int64_t o, int64_t sx, int64_t pl) {  // test_filter :74-80
  T c = a[o];
  return c + T(0.25) * (a[o - 1] - T(2) * c + a[o + 1] + a[o - sx] - T(2) * c + a[o + sx] + a[o - pl] -
                        T(2) * c + a[o + pl]);
}

// One cell (i, j, k) of calc_mut, 1 <= i,j,k <= n-2.
template <class T>
__device__ __forceinline__ void mut_cell(const Geo& G, const Fields<T>& W, const Metrics& M, const PhysConst& K,
                                         int i, int j, int k) {
  const int64_t sx = G.sx, pl = G.plane;
  int64_t o = G.at(i, j, k);
  T u3[3][3][3], v3[3][3][3], w3[3][3][3], ut[3][3][3], vt[3][3][3], wt[3][3][3];
  bool inner = (2 <= i && i <= G.nx - 3 && 2 <= j && j <= G.ny - 3 && 2 <= k && k <= G.nz - 3);
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int b = 0; b < 3; ++b)
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        int64_t q = o + (a - 1) + (b - 1) * sx + (c - 1) * pl;
        u3[c][b][a] = W.u[q]; v3[c][b][a] = W.v[q]; w3[c][b][a] = W.w[q];
        if (inner) {
          ut[c][b][a] = filt(W.u, q, sx, pl);
          vt[c][b][a] = filt(W.v, q, sx, pl);
          wt[c][b][a] = filt(W.w, q, sx, pl);
        } else {
          ut[c][b][a] = u3[c][b][a]; vt[c][b][a] = v3[c][b][a]; wt[c][b][a] = w3[c][b][a];
        }
      }
  T du = u3[1][1][1] - ut[1][1][1], dv = v3[1][1][1] - vt[1][1][1], dw = w3[1][1][1] - wt[1][1][1];
  T qc2 = T(0.5) * (du * du + dv * dv + dw * dw);
  // SMS :30-71
  T dx = (T)M.inv_dx[i], dy = (T)M.inv_dy[j], dz = (T)M.inv_dz[k];
  T a[9], h[9];
  grad3(u3, v3, w3, dx, dy, dz, a);
  grad3(ut, vt, wt, dx, dy, dz, h);
  T vo1 = a[7] - a[5], vo2 = a[2] - a[6], vo3 = a[3] - a[1];
  T vh1 = h[7] - h[5], vh2 = h[2] - h[6], vh3 = h[3] - h[1];
  T vd1 = vo1 - vh1, vd2 = vo2 - vh2, vd3 = vo3 - vh3;
  T vor2 = vo1 * vo1 + vo2 * vo2 + vo3 * vo3;
  T vorh2 = vh1 * vh1 + vh2 * vh2 + vh3 * vh3;
  T vdif2 = vd1 * vd1 + vd2 * vd2 + vd3 * vd3;
  T svor2 = T(2) * sqrt(vor2) * sqrt(vorh2) + vorh2 + vor2 - vdif2;
  T tan2 = (fabs(svor2) < T(1.0e-30)) ? T(0)
                                       : (T(2) * sqrt(vorh2) * sqrt(vor2) - vorh2 - vor2 + vdif2) / svor2;
  T rth = tan2 / T(K.tan10deg2);
  T fth = fmin_f(T(1), rth * rth);
  T S2 = T(2) * (a[0] * a[0] + a[4] * a[4] + a[8] * a[8]) +
         ((a[3] + a[1]) * (a[3] + a[1]) + (a[7] + a[5]) * (a[7] + a[5]) + (a[2] + a[6]) * (a[2] + a[6]));
  T mn = fmin_f(fmin_f(dx, dy), dz);
  T a1 = mn / dx, a2 = mn / dy;
  T l1 = log(a1), l2 = log(a2);
  T delta = cosh(sqrt(T(4) * (l1 * l1 - l1 * l2 + l2 * l2) / T(27))) * pow(dx * dy * dz, T(-1.0 / 3.0));
  const T Cm = T(0.06), alpha = T(0.5);
  T nut = fth * Cm * pow(S2, T(0.5) * alpha) * pow(qc2, T(0.5) * (T(1) - alpha)) * pow(delta, T(1) + alpha);
  W.qc2[o] = qc2;
  W.mut[o] = W.rho[o] * nut;
}

template <class T>
__global__ void k_mut(Geo G, Fields<T> W, Metrics M, PhysConst K) {
  int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
  int k = blockIdx.z * blockDim.z + threadIdx.z + 1;
  if (i > G.nx - 2 || j > G.ny - 2 || k > G.nz - 2) return;
  mut_cell<T>(G, W, M, K, i, j, k);
}

// set_bc_mut_common (3D_solver/src/set_bc_common.f90:296-335): one ghost layer,
// images taken at distance n-2 (the reference's composite copy order).  On a
// non-periodic face the boundary cell takes its neighbour's value, or 0 on a no-slip
// wall (set_bc_mut of 3D_solver/TBL/set.f90 and SBLI/set.f90: wall 0, top and
// outlet copies).  Applying the faces one after the other, x, y, z, as those routines
// do, gives the same as this per-cell rule: 0 if the cell lies on a no-slip face,
// else the value of its source cell in every edge direction at once.
template <class T>
__device__ __forceinline__ void mut_edge_cell(const Geo& G, const Fields<T>& W, int64_t t) {
  const int c[3] = {(int)(t % G.nx), (int)((t / G.nx) % G.ny), (int)(t / ((int64_t)G.nx * G.ny))};
  const int n[3] = {G.nx, G.ny, G.nz};
  const bool per[3] = {!G.bcx, !G.bcy, G.bcz == 0};
  int s[3];
  bool edge = false, zero = false;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    s[a] = c[a];
    const bool lo = c[a] == 0, hi = c[a] == n[a] - 1;
    if (!lo && !hi) continue;
    edge = true;
    if (per[a]) {
      s[a] = lo ? n[a] - 2 : 1;
    } else {
      s[a] = lo ? 1 : n[a] - 2;
      const int f = 2 * a + (hi ? 1 : 0);
      if (((G.bkind >> (4 * f)) & 15) == 3) zero = true;
    }
  }
  if (!edge) return;
  const int64_t o = G.at(c[0], c[1], c[2]), src = G.at(s[0], s[1], s[2]);
  W.mut[o] = zero ? T(0) : W.mut[src];
  W.qc2[o] = zero ? T(0) : W.qc2[src];
}

template <class T>
__global__ void k_mut_edges(Geo G, Fields<T> W) {
  int64_t n = (int64_t)G.nx * G.ny * G.nz;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
       t += (int64_t)gridDim.x * blockDim.x)
    mut_edge_cell<T>(G, W, t);
}

// ---- ghost / boundary-cell fill ------------------------------------------------
// Periodic directions: every ghost cell takes its interior image (set_bc_cyclic{2,4,6},
// set_bc_common.f90:101-273).  Non-periodic directions (2D): one boundary cell on
// each side, set by the face's rule from the adjacent interior cell -- the roles of a
// case's set_bc (2D_solver/ST/set.f90, 2D_solver/OS/set.f90:50-90):
//   OUX_BC_ZERO_GRADIENT  copy of the neighbour
//   OUX_BC_SLIP_WALL      copy with the normal momentum negated
//   OUX_BC_FIXED          caller-given Q/J values
//   OUX_BC_NOSLIP_WALL    the neighbour's density and pressure, zero momentum (the
//                         wall rows of 2D_solver/ST/set.f90 and 2D_solver/BL0/set.f90)
//   OUX_BC_FARFIELD       (high faces) the boundary state from the Riemann invariants
//                         of the neighbour and of a far-field state (the top row of
//                         2D_solver/BL0/set.f90; 3D: 3D_solver/src/set_bc_tbl_sbli.f90)
//   OUX_BC_NEUMANN        the neighbour's primitive state through the two cells'
//                         Jacobians (3D_solver/src/set_bc_tbl_sbli.f90:6-36)
// A face may carry a rule per position (bkinds).  By default y faces are applied
// first and x faces last (2D_solver/OS/set.f90), so a corner takes its x rule of the
// y-boundary value beside it; with ylast the order is reversed (2D_solver/BL0/set.f90).
// With both x and y non-periodic the y faces are set first for every column and the
// x faces after them for every row (2D_solver/OS/set.f90 order), so a corner takes
// its x rule applied to the y-boundary value next to it.  Every value is computed
// from interior cells only, so the cells can be filled in any order.
// The three groups enumerate z-ghost planes, y-ghost rows of interior planes and
// x-ghost cells of interior rows without touching interior cells.
// z ends whose ghost planes the fill writes (the others come from the halo exchange)
__host__ __device__ inline bool z_fill_lo(const Geo& G) { return G.bcz == 0 || G.bcz == 1 || G.bcz == 3; }
__host__ __device__ inline bool z_fill_hi(const Geo& G) { return G.bcz == 0 || G.bcz == 1 || G.bcz == 4; }
__host__ __device__ inline bool z_bnd_lo(const Geo& G) { return G.bcz == 1 || G.bcz == 3; }
__host__ __device__ inline bool z_bnd_hi(const Geo& G) { return G.bcz == 1 || G.bcz == 4; }

// A z slab leaves the ghost planes of its halo ends to the halo exchange.
__host__ __device__ inline int64_t ghost_cells(const Geo& G) {
  const int gy = G.gy;
  const int Ny = G.ny - 2 * gy, Nz = (G.dim == 3) ? G.nz - 2 * G.gz : 1;
  const int gz = (G.dim == 3) ? G.gz * ((int)z_fill_lo(G) + (int)z_fill_hi(G)) : 0;
  return (int64_t)gz * G.ny * G.nx + (int64_t)Nz * (2 * gy) * G.nx + (int64_t)Nz * Ny * (2 * G.gx);
}

// Apply face f's rule to the neighbour state v (in place); pos: position along the
// face (j for x faces, i for y faces); jb / jn: the J(nx, ny) offsets of the boundary
// cell and of its neighbour.
__device__ __forceinline__ void bc_rule(const Geo& G, int f, int pos, int nv, double (&v)[5], int64_t jb,
                                        int64_t jn) {
  const int kind = G.bkinds[f] ? (int)G.bkinds[f][pos] : (G.bkind >> (4 * f)) & 15;
  if (kind == 1) {  // slip wall: normal momentum (rho u for x faces, rho v for y faces) negated
    const int n = f < 2 ? 1 : 2;
    v[n] = -v[n];
  } else if (kind == 2) {  // fixed
    const int len = f < 2 ? G.ny : G.nx;
    for (int l = 0; l < nv; ++l) v[l] = G.bfix[f][(int64_t)l * len + pos];
  } else if (kind == 3) {  // no-slip wall (2D): p_wall from the neighbour, momenta 0
    const double p_wall = G.gamma_1 * (v[3] - 0.5 * (v[1] * v[1] + v[2] * v[2]) / v[0]);
    v[1] = 0.0;
    v[2] = 0.0;
    v[3] = p_wall * G.over_gamma_1;
  } else if (kind == 4) {  // far field (2D, high faces): Riemann invariants along the normal
    const double* P = G.bpar[f];
    const int n = f < 2 ? 1 : 2, t = 3 - n;
    const double Jn = G.bjac[jn], Jt = 1.0 / G.bjac[jb];
    const double pin = G.gamma_1 * (v[3] - 0.5 * (v[1] * v[1] + v[2] * v[2]) / v[0]) * Jn;
    const double rhoin = v[0] * Jn;
    const double cin = sqrt(G.gamma * pin / rhoin);
    const double vin = v[n] / v[0];
    const double Rp = vin + 2.0 * cin * G.over_gamma_1;
    const double Rm = P[2] - 2.0 * P[3] * G.over_gamma_1;
    const double vb = 0.5 * (Rp + Rm);
    const double cb = 0.25 * G.gamma_1 * (Rp - Rm);
    const double rhob = pow(cb * (1.0 / P[3]), 2.0 * G.over_gamma_1) * P[0];
    const double pb = (rhob * (cb * cb)) * G.over_gamma;
    v[0] = rhob * Jt;
    v[t] = rhob * P[1] * Jt;
    v[n] = rhob * vb * Jt;
    v[3] = (pb * G.over_gamma_1 + 0.5 * rhob * (P[1] * P[1] + vb * vb)) * Jt;
  } else if (kind == 5) {  // Neumann: the neighbour's primitive state through the two cells' Jacobians
    const double Jn = G.bjac[jn], Jt = 1.0 / G.bjac[jb];
    const double o1 = 1.0 / v[0];
    const double rhob = v[0] * Jn, ub = v[1] * o1, vb = v[2] * o1;
    const double pb = G.gamma_1 * (v[3] * Jn - 0.5 * rhob * (ub * ub + vb * vb));
    v[0] = rhob * Jt;
    v[1] = rhob * ub * Jt;
    v[2] = rhob * vb * Jt;
    v[3] = (pb * G.over_gamma_1 + 0.5 * rhob * (ub * ub + vb * vb)) * Jt;
  }
}

// 3D grids with non-periodic directions (order 2: one boundary cell a side): the
// rules of the x, y and z faces applied in that order, each to the value the
// previous ones left beside it (2D_solver-style zero gradient / slip / no-slip /
// fixed values; the order of 3D_solver/STZ/set.f90 set_bc).  Periodic directions
// take their images; the ghost planes of a slab's halo ends are not enumerated.
// Faces 4 / 5 are z low / high; fixed values are indexed by the face's position
// (x faces j + ny k, y faces i + nx k, z faces i + nx j).
template <class T>
__device__ __forceinline__ void ghost_cell_3d_bnd(T* Q, const Geo& G, int nv, int i, int j, int k,
                                                  const double* Qn) {
  const int n[3] = {G.nx, G.ny, G.nz};
  const int c[3] = {i, j, k};
  const bool per[3] = {!G.bcx, !G.bcy, G.bcz == 0};
  const bool blo[3] = {(bool)G.bcx, (bool)G.bcy, z_bnd_lo(G)};
  const bool bhi[3] = {(bool)G.bcx, (bool)G.bcy, z_bnd_hi(G)};
  int src[3], cur[3];
  bool bnd[3];
  for (int a = 0; a < 3; ++a) {
    const int g = G.g;
    src[a] = c[a];
    bnd[a] = false;
    if (per[a]) {
      if (c[a] < g || c[a] >= n[a] - g) src[a] = (c[a] - g + (n[a] - 2 * g)) % (n[a] - 2 * g) + g;
    } else if ((c[a] == 0 && blo[a]) || (c[a] == n[a] - 1 && bhi[a])) {
      bnd[a] = true;
      src[a] = c[a] == 0 ? 1 : n[a] - 2;
    }
    cur[a] = src[a];
  }
  double v[5];
  const int64_t s = G.at(src[0], src[1], src[2]);
  for (int l = 0; l < nv; ++l) {
    const int64_t q = s + l * G.vs;
    v[l] = Qn ? Qn[q] + (double)Q[q] : (double)Q[q];
  }
  for (int a = 0; a < 3; ++a) {
    if (!bnd[a]) continue;
    cur[a] = c[a];
    const int f = 2 * a + (c[a] == 0 ? 0 : 1);
    const int kind = (G.bkind >> (4 * f)) & 15;
    if (kind == 1) {  // slip wall: the normal momentum negated
      v[1 + a] = -v[1 + a];
    } else if (kind == 2) {  // fixed values of the face position
      const int64_t pos = a == 0 ? cur[1] + (int64_t)G.ny * cur[2]
                                 : (a == 1 ? cur[0] + (int64_t)G.nx * cur[2] : cur[0] + (int64_t)G.nx * cur[1]);
      const int64_t len = a == 0 ? (int64_t)G.ny * G.nz : (a == 1 ? (int64_t)G.nx * G.nz : (int64_t)G.nx * G.ny);
      for (int l = 0; l < nv; ++l) v[l] = G.bfix3[f][l * len + pos];
    } else if (kind == 3) {  // no-slip wall: the neighbour's density and pressure, zero momentum
      const double p_wall = G.gamma_1 * (v[4] - 0.5 * (v[1] * v[1] + v[2] * v[2] + v[3] * v[3]) / v[0]);
      v[1] = 0.0;
      v[2] = 0.0;
      v[3] = 0.0;
      v[4] = p_wall * G.over_gamma_1;
    } else if (kind == 4 || kind == 5) {
      // the x-y Jacobian table (uniform z) at the boundary cell and at the cell its
      // value came from (3D_solver/src/set_bc_tbl_sbli.f90: Jacobian(i,ny), (i,ny-1))
      int nb[2] = {cur[0], cur[1]};
      if (a < 2) nb[a] = src[a];
      const double Jn = G.bjac[(int64_t)nb[1] * G.nx + nb[0]];
      const double Jt = 1.0 / G.bjac[(int64_t)cur[1] * G.nx + cur[0]];
      if (kind == 4) {
        // far field (x / y high; set_bc_Riemann_tbl_top_down, :38-76): Riemann invariants
        // along the normal, the first tangential velocity the far field's, the second 0
        const double* P = G.bpar[f];
        const int n = 1 + a, t1 = a == 0 ? 2 : 1, t2 = 3;
        const double pin = G.gamma_1 * (v[4] - 0.5 * (v[1] * v[1] + v[2] * v[2] + v[3] * v[3]) / v[0]) * Jn;
        const double rhoin = v[0] * Jn;
        const double cin = sqrt(G.gamma * pin / rhoin);
        const double vin = v[n] / v[0];
        const double Rp = vin + 2.0 * cin * G.over_gamma_1;
        const double Rm = P[2] - 2.0 * P[3] * G.over_gamma_1;
        const double vb = 0.5 * (Rp + Rm);
        const double cb = 0.25 * G.gamma_1 * (Rp - Rm);
        const double rhob = pow(cb * (1.0 / P[3]), 2.0 * G.over_gamma_1) * P[0];
        const double pb = (rhob * (cb * cb)) * G.over_gamma;
        v[0] = rhob * Jt;
        v[t1] = rhob * P[1] * Jt;
        v[n] = rhob * vb * Jt;
        v[t2] = 0.0;
        v[4] = (pb * G.over_gamma_1 + 0.5 * rhob * (P[1] * P[1] + vb * vb)) * Jt;
      } else {
        // Neumann (set_bc_Neumann_tbl_top_down, :6-36): the neighbour's primitive state
        const double o1 = 1.0 / v[0];
        const double rhob = v[0] * Jn, ub = v[1] * o1, vb = v[2] * o1, wb = v[3] * o1;
        const double pb = G.gamma_1 * (v[4] * Jn - 0.5 * rhob * (ub * ub + vb * vb + wb * wb));
        v[0] = rhob * Jt;
        v[1] = rhob * ub * Jt;
        v[2] = rhob * vb * Jt;
        v[3] = rhob * wb * Jt;
        v[4] = (pb * G.over_gamma_1 + 0.5 * rhob * (ub * ub + vb * vb + wb * wb)) * Jt;
      }
    }
  }
  const int64_t o = G.at(i, j, k);
  for (int l = 0; l < nv; ++l) {
    const int64_t q = o + l * G.vs;
    Q[q] = Qn ? (T)(v[l] - Qn[q]) : (T)v[l];
  }
}

// Qn: null for a full state Q; in the mixed form Q holds FP32 stage increments over
// the FP64 state Qn, and a boundary rule is applied to Qn + Q (the increment stored
// is the rule's state minus Qn), so it acts as on a full state.
template <class T>
__device__ __forceinline__ void ghost_cell(T* Q, const Geo& G, int nv, int64_t t, const double* Qn = nullptr) {
  const int g = G.g, gx = G.gx, gy = G.gy;
  const int Nx = G.nx - 2 * gx, Ny = G.ny - 2 * gy, Nz = (G.dim == 3) ? G.nz - 2 * G.gz : 1;
  const int glo = (G.dim == 3 && z_fill_lo(G)) ? G.gz : 0, ghi = (G.dim == 3 && z_fill_hi(G)) ? G.gz : 0;
  const int gz = glo + ghi;
  int64_t nA = (int64_t)gz * G.ny * G.nx;            // z ghost planes
  int64_t nB = (int64_t)Nz * (2 * gy) * G.nx;        // y ghost rows
  int zo = (G.dim == 3) ? G.gz : 0;
  int i, j, k;
  if (t < nA) {
    i = (int)(t % G.nx); int64_t r = t / G.nx; j = (int)(r % G.ny); int kk = (int)(r / G.ny);
    k = kk < glo ? kk : G.nz - gz + kk;
  } else if (t < nA + nB) {
    int64_t s = t - nA;
    i = (int)(s % G.nx); int64_t r = s / G.nx; int jj = (int)(r % (2 * gy)); k = (int)(r / (2 * gy)) + zo;
    j = jj < gy ? jj : G.ny - 2 * gy + jj;
  } else {
    int64_t s = t - nA - nB;
    int ii = (int)(s % (2 * gx)); int64_t r = s / (2 * gx); j = (int)(r % Ny) + gy; k = (int)(r / Ny) + zo;
    i = ii < gx ? ii : G.nx - 2 * gx + ii;
  }
  const int64_t o = G.at(i, j, k);
  if (G.dim == 3 && (G.bcx || G.bcy || z_bnd_lo(G) || z_bnd_hi(G))) {
    ghost_cell_3d_bnd<T>(Q, G, nv, i, j, k, Qn);
    return;
  }
  const bool xb = G.bcx && (i == 0 || i == G.nx - 1);  // x boundary cell
  const bool yb = G.bcy && (j == 0 || j == G.ny - 1);  // y boundary cell
  if (!xb && !yb) {  // periodic images only
    int si = (i - gx + Nx) % Nx + gx;
    int sj = (j - gy + Ny) % Ny + gy;
    int sk = (G.dim == 3) ? (k - g + Nz) % Nz + g : 0;
    int64_t s = G.at(si, sj, sk);
    for (int l = 0; l < nv; ++l) Q[o + l * G.vs] = Q[s + l * G.vs];
    return;
  }
  double v[5];
  auto load = [&](int64_t s) {
    for (int l = 0; l < nv; ++l) {
      const int64_t q = s + l * G.vs;
      v[l] = Qn ? Qn[q] + (double)Q[q] : (double)Q[q];
    }
  };
  const int sk = (G.dim == 3) ? (k - g + Nz) % Nz + g : 0;
  const int64_t nx = G.nx;
  if (xb && yb) {
    // corner: the rule applied last, to the other direction's boundary value beside it
    const int fx = i == 0 ? 0 : 1, in = i == 0 ? 1 : G.nx - 2;
    const int fy = j == 0 ? 2 : 3, jn = j == 0 ? 1 : G.ny - 2;
    load(G.at(in, jn, sk));
    if (!G.ylast) {
      bc_rule(G, fy, in, nv, v, j * nx + in, jn * nx + in);
      bc_rule(G, fx, j, nv, v, j * nx + i, j * nx + in);
    } else {
      bc_rule(G, fx, jn, nv, v, jn * nx + i, jn * nx + in);
      bc_rule(G, fy, i, nv, v, j * nx + i, jn * nx + i);
    }
  } else if (xb) {
    // x face: the neighbour column's value in this row (a periodic image of an
    // interior row when y is periodic)
    const int fx = i == 0 ? 0 : 1, in = i == 0 ? 1 : G.nx - 2;
    const int sj = G.bcy ? j : (j - gy + Ny) % Ny + gy;
    load(G.at(in, sj, sk));
    bc_rule(G, fx, j, nv, v, sj * nx + i, sj * nx + in);
  } else {
    // y face of an interior column (or a periodic-x ghost column's image)
    const int fy = j == 0 ? 2 : 3, jn = j == 0 ? 1 : G.ny - 2;
    const int si = G.bcx ? i : (i - gx + Nx) % Nx + gx;
    load(G.at(si, jn, sk));
    bc_rule(G, fy, i, nv, v, j * nx + si, jn * nx + si);
  }
  for (int l = 0; l < nv; ++l) {
    const int64_t q = o + l * G.vs;
    Q[q] = Qn ? (T)(v[l] - Qn[q]) : (T)v[l];
  }
}

template <class T>
__global__ void k_ghost(T* Q, Geo G, int nv, const double* Qn) {
  const int64_t tot = ghost_cells(G);
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < tot;
       t += (int64_t)gridDim.x * blockDim.x)
    ghost_cell<T>(Q, G, nv, t, Qn);
}

}  // namespace oux
