// Directional flux sweeps: face fluxes (convective + viscous) of a pencil tile
// evaluated in shared memory and differenced into the stage residual, with the
// Runge-Kutta combination fused into the last sweep of the stage.
//
// Block shapes (cells per block along the sweep, pencil rows):
//   x sweep: 32 cells x BR rows, threads (33, BR): thread tx owns face tx-1.
//   y/z sweep: 32 x-cells x BF cells along the sweep, threads (32, BF+1).
// Tile = the block's cells plus H = ORDER/2 halo cells on each side along the
// sweep; it holds rho,u,v,w,p,T,mu,mut,qc2,sensor and the four transverse
// velocity derivatives the viscous stencils need.
#pragma once
#include "oux_kernels.cuh"

namespace oux {

#ifndef OUX_SWEEP_BR
#define OUX_SWEEP_BR 4
#endif
// y / z tiles of 7 cells (8 face rows, 256 threads): two blocks of 8 warps per SM leave
// the FP64 ME4 z sweep 128 registers and no spills, where 8 cells (288 threads, 96
// registers) spilled 120 B per thread; measured on B200 at 512^3 (Hybrid-6 / ME4): z
// 9.64 -> 9.44 ms, and the mixed form's y sweep 6.12 -> 5.38 ms
#ifndef OUX_SWEEP_BF
#define OUX_SWEEP_BF 7
#endif
#ifndef OUX_SWEEP_BZ
#define OUX_SWEEP_BZ OUX_SWEEP_BF
#endif
constexpr int SWEEP_BR = OUX_SWEEP_BR;  // x sweep rows per block
constexpr int SWEEP_BF = OUX_SWEEP_BF;  // y sweep cells per block along the sweep
constexpr int SWEEP_BZ = OUX_SWEEP_BZ;  // z sweep cells per block along the sweep

enum TileField { TF_RHO = 0, TF_U, TF_V, TF_W, TF_P, TF_T, TF_MU, TF_MUT, TF_QC2, TF_SEN, TF_D0, TF_D1, TF_D2, TF_D3, TF_COUNT };

// ROWS: pencil rows per x-sweep tile, or cells along the sweep per y/z tile.
template <int DIR> __host__ __device__ constexpr int default_rows() {
  return DIR == 0 ? SWEEP_BR : DIR == 1 ? SWEEP_BF : SWEEP_BZ;
}
template <int DIR, int ROWS = default_rows<DIR>()> struct SweepShape {
  static constexpr int TX = (DIR == 0) ? 33 : 32;
  static constexpr int TY = (DIR == 0) ? ROWS : ROWS + 1;
};

// The tile halo is 3 cells for every order: the widest stencils (6-point
// convective, Central-6 / ME4 / 2D 4th-order viscous) reach 2 cells left and
// 3 cells right of a face's left cell.
constexpr int TILE_HALO = 3;
template <int ORDER, int DIR, int ROWS = default_rows<DIR>()> __host__ __device__ constexpr int tile_len() {
  return DIR == 0 ? 32 + 2 * TILE_HALO : ROWS + 2 * TILE_HALO;
}
template <int ORDER, int DIR, int ROWS = default_rows<DIR>()> __host__ __device__ constexpr int tile_cells() {
  return DIR == 0 ? tile_len<ORDER, DIR, ROWS>() * ROWS : tile_len<ORDER, DIR, ROWS>() * 32;
}
// TMA-staged tiles (TM: 3D single solves whose tile fields are all plain copies;
// sweep_tma picks the sweeps): every tile field is one box copy into rows of tma_row
// cells, whose x origin is 16-byte aligned for 4- and 8-byte elements, as a tiled
// tensor copy needs (tma_row x 4 B and x 8 B are multiples of 16 B):
//  - y / z: TMA_ROW x cells by tile_len cells along the sweep, from x = 32 b (the
//    block's first owned cell minus the x ghost width); the 32 owned cells start at
//    column gx (gx <= 3);
//  - x: TMA_ROW_X x cells by ROWS rows, from x = 32 b - 4; the tile's tile_len cells
//    start at column gx + 1.
// Each field's slab is rounded up to 128 bytes of shared memory.
constexpr int TMA_ROW = 36;
constexpr int TMA_ROW_X = 44;
constexpr int TMA_MAP_BYTES = 128;  // one tensor map (CUtensorMap)
template <int DIR> __host__ __device__ constexpr int tma_row() { return DIR == 0 ? TMA_ROW_X : TMA_ROW; }
// rows of a tile field's box: the pencil rows (x) or the cells along the sweep (y / z)
template <int ORDER, int DIR, int ROWS> __host__ __device__ constexpr int tma_box_rows() {
  return DIR == 0 ? ROWS : tile_len<ORDER, DIR, ROWS>();
}
template <int ORDER, int DIR, class T, int ROWS, bool TM>
__host__ __device__ constexpr int tile_fstride() {
  if constexpr (TM) {
    constexpr size_t b = sizeof(T) * tma_row<DIR>() * tma_box_rows<ORDER, DIR, ROWS>();
    return (int)(((b + 127) / 128) * 128 / sizeof(T));
  } else {
    return tile_cells<ORDER, DIR, ROWS>();
  }
}
template <int ORDER, int DIR, class T, int ROWS = default_rows<DIR>(), bool TM = false>
__host__ __device__ constexpr size_t sweep_smem() {
  // TF_COUNT tile fields + 5 face-flux components per face thread (FP64) [+ the
  // tile's mbarrier, 16 bytes]
  return sizeof(T) * TF_COUNT * tile_fstride<ORDER, DIR, T, ROWS, TM>() +
         sizeof(double) * 5 * SweepShape<DIR, ROWS>::TX * SweepShape<DIR, ROWS>::TY + (TM ? 16 : 0);
}

// Terms of one shared ME4 face position (me4_position).
template <bool LES> __host__ __device__ constexpr int me4_terms() { return LES ? 9 : 7; }
// Shared ME4 face positions (me4_position): per pencil row 35 positions in the x sweep
// (the 33 faces' neighbours), 32 x (ROWS + 3) in the y / z sweeps.
template <int DIR, int ROWS = default_rows<DIR>()> __host__ __device__ constexpr int me4_positions() {
  return DIR == 0 ? (SweepShape<DIR, ROWS>::TX + 2) * ROWS : 32 * (ROWS + 3);
}
template <int DIR, class T, bool LES, int ROWS = default_rows<DIR>()>
__host__ __device__ constexpr size_t me4_share_bytes() {
  return sizeof(T) * me4_terms<LES>() * me4_positions<DIR, ROWS>();
}

// Operand prefetch of a y/z sweep, PF = bit mask: 1 = the combination operands
// (nv values of Q^n and of Qs or Rs, never needed together), 2 = the accumulator
// Racc; copied into shared memory when the tile starts.
template <int DIR, class T, int ROWS = default_rows<DIR>()>
__host__ __device__ constexpr size_t sweep_pf_bytes(int pf) {
  return DIR == 0 ? 0 : (size_t)5 * 32 * ROWS * sizeof(double) * ((pf & 1 ? 2 : 0) + (pf & 2 ? 1 : 0));
}

// Which prefetch k_sweep uses (measured on B200, 256^3 Hybrid-6 / NS C6):
//  - last sweep of a stage (applies the RK combination): Q^n / Qs / Rs, which moves
//    their latency under the face fluxes (FP64 z sweep 1.79 -> 1.37 ms);
//  - the mixed form, whose FP32 tile is half as large, also prefetches the
//    accumulator, in every y/z sweep (y 0.89 -> 0.85 ms);
//  - in FP64 the accumulator prefetch costs more L1 hits than it saves (y 1.20 ->
//    1.24 ms), so FP64 y sweeps in 3D prefetch nothing.
template <int DIM, int DIR, class T>
__host__ __device__ constexpr int sweep_pf_mode() {
  constexpr bool mx = sizeof(T) < sizeof(double);
  return DIR == 0 ? 0 : (DIR != DIM - 1 ? (mx ? 2 : 0) : (mx ? 3 : 1));
}

// asynchronous global -> shared copies (the issuing thread waits for its own)
template <int BYTES>
__device__ __forceinline__ void cp_async(void* smem, const void* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(sa), "l"(gmem), "n"(BYTES) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait_group() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// mbarrier and tiled tensor copy (TMA, no multicast) for the sweep tiles
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long* bar, int count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// box of the 3D tensor map `map` (in global memory) at (x, y, z) into shared `dst`;
// completes `bar`'s transaction bytes
__device__ __forceinline__ void tma_load_3d(void* dst, const void* map, int x, int y, int z,
                                            unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];\n" ::"r"(smem_u32(dst)),
      "l"(map), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}
// The tensor maps of the TMA-staged sweep's tile fields, passed to the kernel by value
// (a __grid_constant__ parameter: the copies read them from the parameter space, with
// no fence, where maps in global memory would need a tensor-map proxy fence per use).
struct SweepMaps {
  alignas(64) unsigned char m[TF_COUNT][TMA_MAP_BYTES];
};
// polls of a tile's mbarrier before the block gives up with OUX_FAULT_TIMEOUT
constexpr int TMA_WAIT_LIMIT = 1 << 20;

// transverse node derivative of `a` along axis `ax` at offset o (4th/6th order)
template <bool SIXTH, bool RO, class T>
__device__ __forceinline__ T node_d(const T* a, int64_t o, int64_t st, T inv) {
  auto A = [&](int64_t q) { return ldro<RO>(a + q); };
  if constexpr (SIXTH)
    return (T(1.0 / 60.0) * (-A(o - 3 * st) + A(o + 3 * st)) + T(0.15) * (A(o - 2 * st) - A(o + 2 * st)) +
            T(0.75) * (-A(o - st) + A(o + st))) * inv;
  else
    return (T(2.0 / 3.0) * (-A(o - st) + A(o + st)) - T(1.0 / 12.0) * (-A(o - 2 * st) + A(o + 2 * st))) * inv;
}

// ---- convective face flux: calc_{keep,slau,hybrid,roe}_{x,y,z}_in ---------------
// s(f,m) reads tile field f at stencil point m (0 .. 2io+1).
// KONLY: every solve of the launch uses KEEP (compile-time; the other schemes'
// code and registers drop out).
template <int ORDER, bool KONLY, class T, class Acc>
__device__ __forceinline__ void conv_flux(const StepArgs<T>& A, const Acc& s, T fd, int nd, T F[5]) {
  constexpr int NS = ORDER;  // 2io+2 stencil points
  T rho[NS], u[NS], v[NS], w[NS], p[NS], Tt[NS];
#pragma unroll
  for (int m = 0; m < NS; ++m) {
    rho[m] = s(TF_RHO, m); u[m] = s(TF_U, m); v[m] = s(TF_V, m); w[m] = s(TF_W, m);
    p[m] = s(TF_P, m); Tt[m] = s(TF_T, m);
  }
  const T* un = nd == 0 ? u : (nd == 1 ? v : w);
  const int scheme = A.scheme;
  // mixed form: the tile's p and T are deviations from the per-solve references
  constexpr bool MX = sizeof(T) < sizeof(double);
  const T pr = MX ? T(A.K.p_ref) : T(0), tr = MX ? T(A.K.T_ref) : T(0);
  if (KONLY || scheme == 0 || (scheme == 3 && fd <= T(A.K.threshold))) {
    keep_flux<ORDER, T, MX>(rho, u, v, w, un, p, Tt, nd, T(A.K.R_over_gamma_1), F, pr, tr);
    return;
  }
  T Lr, Rr, Lu, Ru, Lv, Rv, Lw, Rw, Lp, Rp;
  const T thr = T(A.K.threshold);
  reconstruct<ORDER>(A.tvd, thr, fd, rho, Lr, Rr);
  reconstruct<ORDER>(A.tvd, thr, fd, u, Lu, Ru);
  reconstruct<ORDER>(A.tvd, thr, fd, v, Lv, Rv);
  reconstruct<ORDER>(A.tvd, thr, fd, w, Lw, Rw);
  reconstruct<ORDER>(A.tvd, thr, fd, p, Lp, Rp);
  if (scheme == 1 || scheme == 3) {
    T HR;
    if (scheme == 3 || ORDER == 2) HR = T(1);
    else if constexpr (ORDER == 6) HR = wiggle(p[1], p[2], p[3], p[4]);
    else HR = wiggle(p[0], p[1], p[2], p[3]);
    T un1 = nd == 0 ? Lu : (nd == 1 ? Lv : Lw);
    T un2 = nd == 0 ? Ru : (nd == 1 ? Rv : Rw);
    slau_flux<T, MX>(A.slau == 1, Lr, Rr, Lu, Ru, Lv, Rv, Lw, Rw, un1, un2, Lp, Rp, nd, HR, T(A.K.gamma),
                     T(A.K.gamma_over_gamma_1), F, pr);
  } else {  // Roe with the normal velocity first (calc_roe_{y,z}_in permutations)
    // rotate so the normal velocity leads: x (u,v,w), y (v,w,u), z (w,u,v)
    T a1 = nd == 0 ? Lu : (nd == 1 ? Lv : Lw), b1 = nd == 0 ? Ru : (nd == 1 ? Rv : Rw);
    T a2 = nd == 0 ? Lv : (nd == 1 ? Lw : Lu), b2 = nd == 0 ? Rv : (nd == 1 ? Rw : Ru);
    T a3 = nd == 0 ? Lw : (nd == 1 ? Lu : Lv), b3 = nd == 0 ? Rw : (nd == 1 ? Ru : Rv);
    T Fr[5];
    bool wide = false;
    if constexpr (sizeof(T) < sizeof(double)) {
      // mixed form: the eigen-decomposition stays FP64 where |u_n| or |u_n| - c is
      // small against c (stagnation / sonic points), where FP32 |lambda| loses digits
      T cl = sqrt(T(A.K.gamma) * (Lp + pr) / Lr), cr = sqrt(T(A.K.gamma) * (Rp + pr) / Rr);
      T un = T(0.5) * (a1 + b1), cm = T(0.5) * (cl + cr);
      wide = fabs(un) < T(0.05) * cm || fabs(fabs(un) - cm) < T(0.05) * cm;
    }
    if (wide) {
      double Fd[5];
      roe_flux<double, MX>(Lr, Rr, a1, b1, a2, b2, a3, b3, Lp, Rp, A.K.gamma_1, A.K.over_gamma_1,
                           A.K.gamma_over_gamma_1, Fd, A.K.p_ref);
#pragma unroll
      for (int q = 0; q < 5; ++q) Fr[q] = (T)Fd[q];
    } else {
      roe_flux<T, MX>(Lr, Rr, a1, b1, a2, b2, a3, b3, Lp, Rp, T(A.K.gamma_1), T(A.K.over_gamma_1),
                      T(A.K.gamma_over_gamma_1), Fr, pr);
    }
    if (nd == 0) {
      F[0] = Fr[0]; F[1] = Fr[1]; F[2] = Fr[2]; F[3] = Fr[3]; F[4] = Fr[4];
    } else if (nd == 1) {
      F[0] = Fr[0]; F[2] = Fr[1]; F[3] = Fr[2]; F[1] = Fr[3]; F[4] = Fr[4];
    } else {
      F[0] = Fr[0]; F[3] = Fr[1]; F[1] = Fr[2]; F[2] = Fr[3]; F[4] = Fr[4];
    }
  }
}

// ---- high-order viscous face terms: calc_visc_high_internal.f90.fypp ----------
// Stencil points m = 0..5 (C6, ME4) or 0..3 (C4) start at face cell - 2 (- 1).
// D0,D1 = straight-stress derivatives (cyclic pair), D2,D3 = normal velocity
// along the two tangential axes in increasing axis order.
template <int VK, bool LES, class T, class Acc>
__device__ __forceinline__ void visc_high(const StepArgs<T>& A, const Acc& s, int nd, T inv, T out[4]) {
  const T two3 = T(2.0 / 3.0);
  const int ca = nd == 0 ? 1 : 0, cb = nd == 2 ? 1 : 2;
  const int fn = TF_U + nd, fa = TF_U + ca, fb = TF_U + cb;
  T tn, ta, tb, wn, wa, wb, kT, Hs = T(0);
  if constexpr (VK == VK_C6 || VK == VK_C4) {
    constexpr int N = (VK == VK_C6) ? 6 : 4;
    T mu[N], mut[N], un[N], ua[N], ub[N], s0[N], s1[N], c0[N], c1[N], Tt[N];
#pragma unroll
    for (int m = 0; m < N; ++m) {
      mu[m] = s(TF_MU, m); un[m] = s(fn, m); ua[m] = s(fa, m); ub[m] = s(fb, m);
      s0[m] = s(TF_D0, m); s1[m] = s(TF_D1, m); c0[m] = s(TF_D2, m); c1[m] = s(TF_D3, m);
      Tt[m] = s(TF_T, m);
      if constexpr (LES) mut[m] = s(TF_MUT, m);
    }
    T mui = v_interp<N>(mu);
    kT = T(A.K.Cp_over_Pr) * mui * v_diff<N>(inv, Tt);
    // calc_tau_straight(_LES) / calc_tau_cross(_LES), calc_visc_cent.f90.fypp:23-91
    {
      T s0i = v_interp<N>(s0), s1i = v_interp<N>(s1), dn = v_diff<N>(inv, un);
      tn = two3 * mui * (T(2) * dn - s0i - s1i);
      wn = v_interp<N>(un) * tn;
      if constexpr (LES) {
        T m2 = T(0.5) * (mui + v_interp<N>(mut));
        tn = two3 * m2 * (T(2) * dn - s0i - s1i);
      }
    }
    {
      T ci = v_interp<N>(c0), dv = v_diff<N>(inv, ua);
      ta = mui * (ci + dv);
      wa = v_interp<N>(ua) * ta;
      if constexpr (LES) { T m2 = T(0.5) * (mui + v_interp<N>(mut)); ta = m2 * (ci + dv); }
    }
    {
      T ci = v_interp<N>(c1), dv = v_diff<N>(inv, ub);
      tb = mui * (ci + dv);
      wb = v_interp<N>(ub) * tb;
      if constexpr (LES) { T m2 = T(0.5) * (mui + v_interp<N>(mut)); tb = m2 * (ci + dv); }
    }
    if constexpr (LES) {
      T H[N];
#pragma unroll
      for (int m = 0; m < N; ++m) {
        T uu = s(TF_U, m), vv = s(TF_V, m), ww = s(TF_W, m);
        H[m] = T(A.K.Cp) * Tt[m] + T(0.5) * (uu * uu + vv * vv + ww * ww) + s(TF_QC2, m);
      }
      Hs = -v_interp<N>(mut) * v_diff<N>(inv, H) / T(A.K.Prt);
    }
  } else {  // VK_ME4: calc_visc_me4_base.f90:4-111 on a 6-point stencil
    T mu3[3], mut3[3], k3[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      mu3[q] = T(0.0625) * (T(9) * (s(TF_MU, q + 1) + s(TF_MU, q + 2)) - (s(TF_MU, q) + s(TF_MU, q + 3)));
      if constexpr (LES)
        mut3[q] = T(0.0625) * (T(9) * (s(TF_MUT, q + 1) + s(TF_MUT, q + 2)) - (s(TF_MUT, q) + s(TF_MUT, q + 3)));
    }
#pragma unroll
    for (int q = 0; q < 3; ++q)
      k3[q] = T(A.K.Cp_over_Pr) * mu3[q] *
              (T(1.125) * (-s(TF_T, q + 1) + s(TF_T, q + 2)) - (-s(TF_T, q) + s(TF_T, q + 3)) * T(1.0 / 24.0)) * inv;
    kT = flux4(k3[0], k3[1], k3[2]);
    // straight
    {
      T t1[3], t2[3];
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        T a0 = s(fn, q), a1 = s(fn, q + 1), a2 = s(fn, q + 2), a3 = s(fn, q + 3);
        T y0 = s(TF_D0, q), y1 = s(TF_D0, q + 1), y2 = s(TF_D0, q + 2), y3 = s(TF_D0, q + 3);
        T z0 = s(TF_D1, q), z1 = s(TF_D1, q + 1), z2 = s(TF_D1, q + 2), z3 = s(TF_D1, q + 3);
        T dd = (T(2.25) * (-a1 + a2) - (-a0 + a3) * T(1.0 / 12.0)) * inv;
        if constexpr (!LES) {
          t1[q] = two3 * mu3[q] * (dd - T(0.0625) * (-y0 + T(9) * (y1 + y2) - y3) -
                                   T(0.0625) * (-z0 + T(9) * (z1 + z2) - z3));
        } else {
          t1[q] = dd;
          t1[q] = t1[q] - T(0.0625) * (-y0 + T(9) * (y1 + y2) - y3);
          t1[q] = t1[q] - T(0.0625) * (-z0 + T(9) * (z1 + z2) - z3);
        }
      }
      if constexpr (!LES) {
        tn = flux4(t1[0], t1[1], t1[2]);
#pragma unroll
        for (int q = 0; q < 3; ++q)
          t2[q] = T(0.0625) * (-s(fn, q) + T(9) * (s(fn, q + 1) + s(fn, q + 2)) - s(fn, q + 3)) * t1[q];
        wn = flux4(t2[0], t2[1], t2[2]);
      } else {
#pragma unroll
        for (int q = 0; q < 3; ++q) t2[q] = two3 * mu3[q] * t1[q];
#pragma unroll
        for (int q = 0; q < 3; ++q)
          t2[q] = T(0.0625) * (-s(fn, q) + T(9) * (s(fn, q + 1) + s(fn, q + 2)) - s(fn, q + 3)) * t2[q];
        wn = flux4(t2[0], t2[1], t2[2]);
#pragma unroll
        for (int q = 0; q < 3; ++q) t2[q] = two3 * (mu3[q] + mut3[q]) * t1[q];
        tn = flux4(t2[0], t2[1], t2[2]);
      }
    }
    // cross terms (component fa with derivative D2, component fb with D3)
#pragma unroll
    for (int side = 0; side < 2; ++side) {
      const int fv = side == 0 ? fa : fb, fd_ = side == 0 ? TF_D2 : TF_D3;
      T t1[3], t2[3], tt, ww;
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        T a0 = s(fv, q), a1 = s(fv, q + 1), a2 = s(fv, q + 2), a3 = s(fv, q + 3);
        T y0 = s(fd_, q), y1 = s(fd_, q + 1), y2 = s(fd_, q + 2), y3 = s(fd_, q + 3);
        T dd = (T(1.125) * (-a1 + a2) - (-a0 + a3) * T(1.0 / 24.0)) * inv;
        if constexpr (!LES) t1[q] = mu3[q] * (dd + T(0.0625) * (-y0 + T(9) * (y1 + y2) - y3));
        else { t1[q] = dd; t1[q] = t1[q] + T(0.0625) * (-y0 + T(9) * (y1 + y2) - y3); }
      }
      if constexpr (!LES) {
        tt = flux4(t1[0], t1[1], t1[2]);
#pragma unroll
        for (int q = 0; q < 3; ++q)
          t2[q] = T(0.0625) * (-s(fv, q) + T(9) * (s(fv, q + 1) + s(fv, q + 2)) - s(fv, q + 3)) * t1[q];
        ww = flux4(t2[0], t2[1], t2[2]);
      } else {
#pragma unroll
        for (int q = 0; q < 3; ++q) t2[q] = mu3[q] * t1[q];
#pragma unroll
        for (int q = 0; q < 3; ++q)
          t2[q] = T(0.0625) * (-s(fv, q) + T(9) * (s(fv, q + 1) + s(fv, q + 2)) - s(fv, q + 3)) * t2[q];
        ww = flux4(t2[0], t2[1], t2[2]);
#pragma unroll
        for (int q = 0; q < 3; ++q) t2[q] = (mu3[q] + mut3[q]) * t1[q];
        tt = flux4(t2[0], t2[1], t2[2]);
      }
      if (side == 0) { ta = tt; wa = ww; } else { tb = tt; wb = ww; }
    }
    if constexpr (LES) {
      T H[4];
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        T uu = s(TF_U, m + 1), vv = s(TF_V, m + 1), ww = s(TF_W, m + 1);
        H[m] = T(A.K.Cp) * s(TF_T, m + 1) + T(0.5) * (uu * uu + vv * vv + ww * ww) + s(TF_QC2, m + 1);
      }
      Hs = -flux4(mut3[0], mut3[1], mut3[2]) * (T(1.125) * (-H[1] + H[2]) - (-H[0] + H[3]) * T(1.0 / 24.0)) *
           inv / T(A.K.Prt);
    }
  }
  T t[3], wk[3];
  t[nd] = tn; t[ca] = ta; t[cb] = tb;
  wk[nd] = wn; wk[ca] = wa; wk[cb] = wb;
  out[0] = t[0]; out[1] = t[1]; out[2] = t[2];
  T e = wk[0] + wk[1] + wk[2] + kT;
  if constexpr (LES) e = e + Hs;
  out[3] = e;
}

// ---- ME4 with shared face positions ----------------------------------------------
// ME4 evaluates 4th-order stresses at three face positions (the faces with left cells
// f-1, f, f+1) and combines them with flux4 (calc_visc_me4_base.f90:4-111); each
// position serves three neighbouring faces.  On an axis whose spacings are all the
// same double, a position's terms are the same bits whichever face asks for them, so
// the sweep evaluates each position once into shared memory and every face combines
// its three.  me4_position gives the terms of one position from its stencil cells
// s(field, 0..3) (the position's left cell - 1 .. + 2), with the expression trees of
// visc_high<VK_ME4> so that the results are bit for bit the same:
//   0 heat flux k3, 1 normal stress, 2 its work term, 3 / 4 first cross stress and
//   work term, 5 / 6 second cross stress and work term; LES: 7 mut3, 8 the position's
//   total-enthalpy difference (used by the face at this position only).

template <bool LES, class T, class Acc>
__device__ __forceinline__ void me4_position(const StepArgs<T>& A, const Acc& s, int nd, T inv, T v[9]) {
  const T two3 = T(2.0 / 3.0);
  const int ca = nd == 0 ? 1 : 0, cb = nd == 2 ? 1 : 2;
  const int fn = TF_U + nd, fa = TF_U + ca, fb = TF_U + cb;
  const T mu3 = T(0.0625) * (T(9) * (s(TF_MU, 1) + s(TF_MU, 2)) - (s(TF_MU, 0) + s(TF_MU, 3)));
  T mut3 = T(0);
  if constexpr (LES) mut3 = T(0.0625) * (T(9) * (s(TF_MUT, 1) + s(TF_MUT, 2)) - (s(TF_MUT, 0) + s(TF_MUT, 3)));
  v[0] = T(A.K.Cp_over_Pr) * mu3 *
         (T(1.125) * (-s(TF_T, 1) + s(TF_T, 2)) - (-s(TF_T, 0) + s(TF_T, 3)) * T(1.0 / 24.0)) * inv;
  {  // straight
    const T a0 = s(fn, 0), a1 = s(fn, 1), a2 = s(fn, 2), a3 = s(fn, 3);
    const T y0 = s(TF_D0, 0), y1 = s(TF_D0, 1), y2 = s(TF_D0, 2), y3 = s(TF_D0, 3);
    const T z0 = s(TF_D1, 0), z1 = s(TF_D1, 1), z2 = s(TF_D1, 2), z3 = s(TF_D1, 3);
    const T dd = (T(2.25) * (-a1 + a2) - (-a0 + a3) * T(1.0 / 12.0)) * inv;
    const T un4 = T(0.0625) * (-a0 + T(9) * (a1 + a2) - a3);
    if constexpr (!LES) {
      const T t1 = two3 * mu3 * (dd - T(0.0625) * (-y0 + T(9) * (y1 + y2) - y3) -
                                 T(0.0625) * (-z0 + T(9) * (z1 + z2) - z3));
      v[1] = t1;
      v[2] = un4 * t1;
    } else {
      T t1 = dd;
      t1 = t1 - T(0.0625) * (-y0 + T(9) * (y1 + y2) - y3);
      t1 = t1 - T(0.0625) * (-z0 + T(9) * (z1 + z2) - z3);
      v[2] = un4 * (two3 * mu3 * t1);
      v[1] = two3 * (mu3 + mut3) * t1;
    }
  }
#pragma unroll
  for (int side = 0; side < 2; ++side) {  // cross terms: fa with D2, fb with D3
    const int fv = side == 0 ? fa : fb, fd_ = side == 0 ? TF_D2 : TF_D3;
    const T a0 = s(fv, 0), a1 = s(fv, 1), a2 = s(fv, 2), a3 = s(fv, 3);
    const T y0 = s(fd_, 0), y1 = s(fd_, 1), y2 = s(fd_, 2), y3 = s(fd_, 3);
    const T dd = (T(1.125) * (-a1 + a2) - (-a0 + a3) * T(1.0 / 24.0)) * inv;
    const T v4 = T(0.0625) * (-a0 + T(9) * (a1 + a2) - a3);
    if constexpr (!LES) {
      const T t1 = mu3 * (dd + T(0.0625) * (-y0 + T(9) * (y1 + y2) - y3));
      v[3 + 2 * side] = t1;
      v[4 + 2 * side] = v4 * t1;
    } else {
      T t1 = dd;
      t1 = t1 + T(0.0625) * (-y0 + T(9) * (y1 + y2) - y3);
      v[4 + 2 * side] = v4 * (mu3 * t1);
      v[3 + 2 * side] = (mu3 + mut3) * t1;
    }
  }
  if constexpr (LES) {
    v[7] = mut3;
    T H[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      const T uu = s(TF_U, m), vv = s(TF_V, m), ww = s(TF_W, m);
      H[m] = T(A.K.Cp) * s(TF_T, m) + T(0.5) * (uu * uu + vv * vv + ww * ww) + s(TF_QC2, m);
    }
    v[8] = T(1.125) * (-H[1] + H[2]) - (-H[0] + H[3]) * T(1.0 / 24.0);
  }
}

// The four viscous terms of a face from the terms of its three positions:
// P(k, q) = term k of position q (0: left cell f-1, 1: f, 2: f+1).
template <bool LES, class T, class PosAcc>
__device__ __forceinline__ void me4_face(const StepArgs<T>& A, const PosAcc& P, int nd, T inv, T out[4]) {
  const int ca = nd == 0 ? 1 : 0, cb = nd == 2 ? 1 : 2;
  const T kT = flux4(P(0, 0), P(0, 1), P(0, 2));
  const T tn = flux4(P(1, 0), P(1, 1), P(1, 2)), wn = flux4(P(2, 0), P(2, 1), P(2, 2));
  const T ta = flux4(P(3, 0), P(3, 1), P(3, 2)), wa = flux4(P(4, 0), P(4, 1), P(4, 2));
  const T tb = flux4(P(5, 0), P(5, 1), P(5, 2)), wb = flux4(P(6, 0), P(6, 1), P(6, 2));
  T t[3], wk[3];
  t[nd] = tn; t[ca] = ta; t[cb] = tb;
  wk[nd] = wn; wk[ca] = wa; wk[cb] = wb;
  out[0] = t[0]; out[1] = t[1]; out[2] = t[2];
  T e = wk[0] + wk[1] + wk[2] + kT;
  if constexpr (LES) e = e + -flux4(P(7, 0), P(7, 1), P(7, 2)) * P(8, 1) * inv / T(A.K.Prt);
  out[3] = e;
}

// ---- Gaitonde-Visbal 2nd order: 3D_solver/src/calc_visc2.f90.fypp (2D :10-103) ----
// Reads global arrays directly: face between o and o + st[nd].
template <int DIM, bool LES, bool RO, class T>
__device__ __forceinline__ void visc_gv2(const StepArgs<T>& A, int nd, int64_t o, const int64_t st[3],
                                         const T invs[3], T out[4]) {
  // read-only view of the fields: W.f[q] loads through ldro<RO>
  struct RoField {
    const T* p;
    __device__ T operator[](int64_t q) const { return ldro<RO>(p + q); }
  };
  struct {
    RoField u, v, w, mu, T_, mut, qc2;
  } W{{A.W.u}, {A.W.v}, {A.W.w}, {A.W.mu}, {A.W.T_}, {A.W.mut}, {A.W.qc2}};
  const int64_t o2 = o + st[nd];
  const T inv = invs[nd];
  auto vel = [&](int c, int64_t q) -> T { return c == 0 ? W.u[q] : (c == 1 ? W.v[q] : (DIM == 3 ? W.w[q] : T(0))); };
  T md = T(0.5) * (W.mu[o] + W.mu[o2]) * inv;
  T vw = T(A.K.Cp_over_Pr) * md * (-W.T_[o] + W.T_[o2]);
  T dn[3], sg[3] = {T(0), T(0), T(0)}, Hs = T(0);
#pragma unroll
  for (int c = 0; c < 3; ++c) dn[c] = md * (-vel(c, o) + vel(c, o2));
  if constexpr (LES) {
    T msd = T(0.5) * (W.mut[o] + W.mut[o2]) * inv;
    auto Hf = [&](int64_t q) {
      T uu = W.u[q], vv = W.v[q], ww = W.w[q];
      return T(A.K.Cp) * W.T_[q] + T(0.5) * (uu * uu + vv * vv + ww * ww) + W.qc2[q];
    };
    T H1 = Hf(o), H2 = Hf(o2);
    Hs = -msd * (-H1 + H2) / T(A.K.Prt);
#pragma unroll
    for (int c = 0; c < 3; ++c) sg[c] = msd * (-vel(c, o) + vel(c, o2));
  }
  auto cross = [&](bool sgs, int c, int t) -> T {
    const RoField m = sgs ? W.mut : W.mu;
    const int64_t s = st[t];
    T m1 = T(0.0625) * (m[o - s] + m[o] + m[o2 - s] + m[o2]);
    T m2 = T(0.0625) * (m[o] + m[o + s] + m[o2] + m[o2 + s]);
    return (m1 * (-vel(c, o - s) - vel(c, o2 - s)) + (m1 - m2) * (vel(c, o) + vel(c, o2)) +
            m2 * (vel(c, o + s) + vel(c, o2 + s))) * invs[t];
  };
  T uS = W.u[o] + W.u[o2], vS = W.v[o] + W.v[o2];
  T wS = (DIM == 3) ? (W.w[o] + W.w[o2]) : T(0);
  const T two3 = T(2.0 / 3.0);
  T s1, s2, s3 = T(0);
  if constexpr (DIM == 3) {
    if (nd == 0) {
      T txx = two3 * (T(2) * dn[0] - cross(false, 1, 1) - cross(false, 2, 2));
      T txy = cross(false, 0, 1) + dn[1];
      T txz = dn[2] + cross(false, 0, 2);
      vw = vw + T(0.5) * (uS * txx + vS * txy + wS * txz);
      if constexpr (LES) {
        txx = txx + two3 * (T(2) * sg[0] - cross(true, 1, 1) - cross(true, 2, 2));
        txy = txy + cross(true, 0, 1) + sg[1];
        txz = txz + sg[2] + cross(true, 0, 2);
      }
      s1 = txx; s2 = txy; s3 = txz;
    } else if (nd == 1) {
      T tyx = dn[0] + cross(false, 1, 0);
      T tyy = two3 * (T(2) * dn[1] - cross(false, 2, 2) - cross(false, 0, 0));
      T tyz = cross(false, 1, 2) + dn[2];
      vw = vw + T(0.5) * (uS * tyx + vS * tyy + wS * tyz);
      if constexpr (LES) {
        tyx = tyx + sg[0] + cross(true, 1, 0);
        tyy = tyy + two3 * (T(2) * sg[1] - cross(true, 2, 2) - cross(true, 0, 0));
        tyz = tyz + cross(true, 1, 2) + sg[2];
      }
      s1 = tyx; s2 = tyy; s3 = tyz;
    } else {
      T tzx = cross(false, 2, 0) + dn[0];
      T tzy = dn[1] + cross(false, 2, 1);
      T tzz = two3 * (T(2) * dn[2] - cross(false, 0, 0) - cross(false, 1, 1));
      vw = vw + T(0.5) * (uS * tzx + vS * tzy + wS * tzz);
      if constexpr (LES) {
        tzx = tzx + cross(true, 2, 0) + sg[0];
        tzy = tzy + sg[1] + cross(true, 2, 1);
        tzz = tzz + two3 * (T(2) * sg[2] - cross(true, 0, 0) - cross(true, 1, 1));
      }
      s1 = tzx; s2 = tzy; s3 = tzz;
    }
  } else {
    if (nd == 0) {
      T txx = two3 * (T(2) * dn[0] - cross(false, 1, 1));
      T txy = cross(false, 0, 1) + dn[1];
      vw = vw + T(0.5) * (uS * txx + vS * txy);
      s1 = txx; s2 = txy;
    } else {
      T tyx = dn[0] + cross(false, 1, 0);
      T tyy = two3 * (T(2) * dn[1] - cross(false, 0, 0));
      vw = vw + T(0.5) * (uS * tyx + vS * tyy);
      s1 = tyx; s2 = tyy;
    }
  }
  out[0] = s1; out[1] = s2; out[2] = s3;
  out[3] = LES ? (vw + Hs) : vw;
}

// ---- 2D 4th-order viscous face with its 2nd-order fallback: 2D_solver/src/calc_visc4.f90.fypp ----
template <class T, class Acc>
__device__ __forceinline__ void visc_2d4(const StepArgs<T>& A, const Acc& s, int nd, bool inner,
                                         int64_t o, const int64_t st[2], const T invs[2], T out[4]) {
  const T two3 = T(2.0 / 3.0);
  const int fn = TF_U + nd, fa = TF_U + (1 - nd);
  const T inv = invs[nd];
  T tn, ta, wn, wa, kT;
  if (inner) {
    T mu3[3], k3[3], t1[3];
#pragma unroll
    for (int q = 0; q < 3; ++q)
      mu3[q] = T(0.0625) * (T(9) * (s(TF_MU, q + 1) + s(TF_MU, q + 2)) - (s(TF_MU, q) + s(TF_MU, q + 3)));
#pragma unroll
    for (int q = 0; q < 3; ++q)
      k3[q] = T(A.K.Cp_over_Pr) * mu3[q] *
              (T(1.125) * (-s(TF_T, q + 1) + s(TF_T, q + 2)) - (-s(TF_T, q) + s(TF_T, q + 3)) * T(1.0 / 24.0)) * inv;
    kT = flux4(k3[0], k3[1], k3[2]);
#pragma unroll
    for (int q = 0; q < 3; ++q) {  // 2D calc_tau_straight: one transverse derivative (D0)
      T a0 = s(fn, q), a1 = s(fn, q + 1), a2 = s(fn, q + 2), a3 = s(fn, q + 3);
      T y0 = s(TF_D0, q), y1 = s(TF_D0, q + 1), y2 = s(TF_D0, q + 2), y3 = s(TF_D0, q + 3);
      t1[q] = two3 * mu3[q] * ((T(2.25) * (-a1 + a2) - (-a0 + a3) * T(1.0 / 12.0)) * inv -
                               T(0.0625) * (-y0 + T(9) * (y1 + y2) - y3));
    }
    tn = flux4(t1[0], t1[1], t1[2]);
#pragma unroll
    for (int q = 0; q < 3; ++q)
      t1[q] = T(0.0625) * (-s(fn, q) + T(9) * (s(fn, q + 1) + s(fn, q + 2)) - s(fn, q + 3)) * t1[q];
    wn = flux4(t1[0], t1[1], t1[2]);
#pragma unroll
    for (int q = 0; q < 3; ++q) {  // cross: tangential velocity with D2 (normal velocity along tangent)
      T a0 = s(fa, q), a1 = s(fa, q + 1), a2 = s(fa, q + 2), a3 = s(fa, q + 3);
      T y0 = s(TF_D2, q), y1 = s(TF_D2, q + 1), y2 = s(TF_D2, q + 2), y3 = s(TF_D2, q + 3);
      t1[q] = mu3[q] * ((T(1.125) * (-a1 + a2) - (-a0 + a3) * T(1.0 / 24.0)) * inv +
                        T(0.0625) * (-y0 + T(9) * (y1 + y2) - y3));
    }
    ta = flux4(t1[0], t1[1], t1[2]);
#pragma unroll
    for (int q = 0; q < 3; ++q)
      t1[q] = T(0.0625) * (-s(fa, q) + T(9) * (s(fa, q + 1) + s(fa, q + 2)) - s(fa, q + 3)) * t1[q];
    wa = flux4(t1[0], t1[1], t1[2]);
  } else {
    const Fields<T>& W = A.W;
    const int64_t o2 = o + st[nd];
    const int64_t sa = st[1 - nd];
    const T inva = invs[1 - nd];
    T mn = T(0.5) * (W.mu[o] + W.mu[o2]);
    kT = T(A.K.Cp_over_Pr) * mn * (-W.T_[o] + W.T_[o2]) * inv;
    T m1 = T(0.25) * (W.mu[o - sa] + W.mu[o] + W.mu[o2 - sa] + W.mu[o2]);
    T m2 = T(0.25) * (W.mu[o] + W.mu[o + sa] + W.mu[o2] + W.mu[o2 + sa]);
    auto tder = [&](const T* a) {
      return T(0.25) * (m1 * (-a[o - sa] + a[o] - a[o2 - sa] + a[o2]) + m2 * (-a[o] + a[o + sa] - a[o2] + a[o2 + sa])) * inva;
    };
    const T* vn = nd == 0 ? W.u : W.v;
    const T* va = nd == 0 ? W.v : W.u;
    T dnn = mn * (-vn[o] + vn[o2]) * inv;   // mux (x) / mvy (y)
    T dan = mn * (-va[o] + va[o2]) * inv;   // mvx (x) / muy (y)
    T dna = tder(vn);                       // muy (x) / mvx (y)
    T daa = tder(va);                       // mvy (x) / mux (y)
    tn = two3 * (T(2) * dnn - daa);
    ta = (nd == 0) ? (dna + dan) : (dan + dna);
    wn = T(0.5) * (vn[o] + vn[o2]) * tn;
    wa = T(0.5) * (va[o] + va[o2]) * ta;
  }
  // energy in (u, v) order
  T wu = nd == 0 ? wn : wa, wv = nd == 0 ? wa : wn;
  out[nd] = tn; out[1 - nd] = ta; out[2] = T(0);
  out[3] = wu + wv + kT;
}

// ---- 3D 2nd-order fallback of the high-order viscous faces (Navier-Stokes) -------
// The branch of calc_Ev / calc_Fv / calc_Gv taken outside their high-order guard
// (3D_solver/src/calc_visc_high.f90.fypp:194-260, 432-497, 674-739): face viscosity
// and normal derivatives from the face's two cells; tangential derivatives from the
// two cell pairs on either side weighted by their 4-point viscosity averages.
// D[c][a] is mu * d(velocity c) / d(axis a) as the reference names them (mux, mvy ...);
// LES adds the same stresses with the SGS viscosity (Ds, muxsgs ...) after the work
// terms, and the SGS enthalpy flux.
template <bool LES, class T>
__device__ __forceinline__ void visc_fb3(const StepArgs<T>& A, int nd, int64_t o, const int64_t st[3],
                                         const T invs[3], T out[4]) {
  const Fields<T>& W = A.W;
  const T* vel[3] = {W.u, W.v, W.w};
  const int64_t o2 = o + st[nd];
  const T inv = invs[nd];
  const T mn = T(0.5) * (W.mu[o] + W.mu[o2]);
  const T kT = T(A.K.Cp_over_Pr) * mn * (-W.T_[o] + W.T_[o2]) * inv;
  // mu * derivatives with viscosity field m (mu, or mut for the SGS part)
  auto derivs = [&](const T* m, T D[3][3]) {
    const T mf = T(0.5) * (m[o] + m[o2]);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      if (a == nd) continue;
      const int64_t s = st[a];
      const T m1 = T(0.25) * (m[o - s] + m[o] + m[o2 - s] + m[o2]);
      const T m2 = T(0.25) * (m[o] + m[o + s] + m[o2] + m[o2 + s]);
      auto tder = [&](const T* q) {
        return T(0.25) * (m1 * (-q[o - s] + q[o] - q[o2 - s] + q[o2]) + m2 * (-q[o] + q[o + s] - q[o2] + q[o2 + s])) *
               invs[a];
      };
      D[nd][a] = tder(vel[nd]);  // normal velocity along the tangent (cross stress)
      D[a][a] = tder(vel[a]);    // tangential velocity along itself (normal stress)
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) D[c][nd] = mf * (-vel[c][o] + vel[c][o2]) * inv;
  };
  const T two3 = T(2.0 / 3.0);
  // the stresses of the face in the reference's operand order; `t` starts from base
  auto stresses = [&](const T D[3][3], const T base[3], T t[3]) {
    if (nd == 0) {
      t[0] = base[0] + two3 * (T(2) * D[0][0] - D[1][1] - D[2][2]);  // txx
      t[1] = base[1] + D[0][1] + D[1][0];                             // txy: muy + mvx
      t[2] = base[2] + D[2][0] + D[0][2];                             // txz: mwx + muz
    } else if (nd == 1) {
      t[0] = base[0] + D[0][1] + D[1][0];                             // tyx: muy + mvx
      t[1] = base[1] + two3 * (T(2) * D[1][1] - D[2][2] - D[0][0]);  // tyy
      t[2] = base[2] + D[1][2] + D[2][1];                             // tyz: mvz + mwy
    } else {
      t[0] = base[0] + D[2][0] + D[0][2];                             // tzx: mwx + muz
      t[1] = base[1] + D[1][2] + D[2][1];                             // tzy: mvz + mwy
      t[2] = base[2] + two3 * (T(2) * D[2][2] - D[0][0] - D[1][1]);  // tzz
    }
  };
  T D[3][3], t[3];
  derivs(W.mu, D);
  if (nd == 0) {
    t[0] = two3 * (T(2) * D[0][0] - D[1][1] - D[2][2]);
    t[1] = D[0][1] + D[1][0];
    t[2] = D[2][0] + D[0][2];
  } else if (nd == 1) {
    t[0] = D[0][1] + D[1][0];
    t[1] = two3 * (T(2) * D[1][1] - D[2][2] - D[0][0]);
    t[2] = D[1][2] + D[2][1];
  } else {
    t[0] = D[2][0] + D[0][2];
    t[1] = D[1][2] + D[2][1];
    t[2] = two3 * (T(2) * D[2][2] - D[0][0] - D[1][1]);
  }
  T e = T(0.5) * (vel[0][o] + vel[0][o2]) * t[0];
  e = e + T(0.5) * (vel[1][o] + vel[1][o2]) * t[1];
  e = e + T(0.5) * (vel[2][o] + vel[2][o2]) * t[2];
  e = e + kT;
  if constexpr (LES) {
    T Ds[3][3], ts[3];
    derivs(W.mut, Ds);
    stresses(Ds, t, ts);
    t[0] = ts[0]; t[1] = ts[1]; t[2] = ts[2];
    auto Hf = [&](int64_t q) {
      const T uu = W.u[q], vv = W.v[q], ww = W.w[q];
      return T(A.K.Cp) * W.T_[q] + T(0.5) * (uu * uu + vv * vv + ww * ww) + W.qc2[q];
    };
    const T msf = T(0.5) * (W.mut[o] + W.mut[o2]);
    e = e + -msf * (-Hf(o) + Hf(o2)) * inv / T(A.K.Prt);
  }
  out[0] = t[0]; out[1] = t[1]; out[2] = t[2];
  out[3] = e;
}

}  // namespace oux

namespace oux {

// ---- the sweep kernel -----------------------------------------------------------
// VK: viscous kind; LES: add the SGS terms.  `last` selects the combination.
// minimum resident blocks per SM (caps registers; measured on B200: 3 / 2 beat 1 / 1 by 1.5x)
#ifndef OUX_SWEEP_MINB_X
#define OUX_SWEEP_MINB_X 3
#endif
#ifndef OUX_SWEEP_MINB_YZ
#define OUX_SWEEP_MINB_YZ 2
#endif
// One sweep tile: block-tile indices (b0, b1, b2) as the grid of launch_one
// enumerates them; `tid` / `nthr_all` are the calling block's linear thread index
// and size (>= TX*TY: threads beyond the tile shape only help load the tile).
// PF: prefetch the cell operands of the combination (Q^n, Qs / Rs; PF = 2: and the
// accumulator) into shared memory when the tile starts, so their latency overlaps
// the face fluxes; needs sweep_pf_bytes(PF) more dynamic shared memory.
// SHARE (ME4 on an axis of uniform spacing): the viscous terms of every face position
// are evaluated once into shared memory (me4_position) and combined per face
// (me4_face); needs me4_share_bytes() more dynamic shared memory after the prefetch.
// GR: the transverse node derivatives are staged from the gradient fields W.grad
// (written by k_grad) instead of being differenced from the velocities in the tile
// load.
// AT: the tile's plain fields (and, with GR, the gradients) are staged with
// asynchronous global -> shared copies (cp.async): no register staging, and every
// copy of the tile is in flight at once; derivatives differenced in the load (no GR)
// are computed while the copies fly.
// TM (sweeps whose tile fields are all plain copies, sweep_tma): the TMA tile layout
// (tma_row-wide rows, 128-byte field slabs); given `tmaps` (the sweep's SweepMaps),
// one thread stages every field by a tensor copy completing one mbarrier, else the
// threads fill the same layout with cp.async.
template <int DIM, int DIR, int ORDER, int VK, bool LES, class T, int ROWS = default_rows<DIR>(),
          bool RO = false, bool KONLY = false, int PF = 0, bool SHARE = false, bool GR = false, bool AT = false,
          bool TM = false>
__device__ __forceinline__ void sweep_tile(const StepArgs<T>& A, int last, int b0, int b1, int b2,
                                           unsigned char* smraw, int tid, int nthr_all,
                                           const SweepMaps* tmaps = nullptr) {
  constexpr int H = ORDER / 2;
  constexpr int TL = tile_len<ORDER, DIR, ROWS>();
  constexpr int NC = tile_cells<ORDER, DIR, ROWS>();
  constexpr int TX = SweepShape<DIR, ROWS>::TX, TY = SweepShape<DIR, ROWS>::TY;
  constexpr int VB = vk_base(VK);      // stencil family
  constexpr bool WALL = vk_wall(VK);   // 3D viscous grid with a non-periodic direction
  constexpr bool HIGH = (VB == VK_C6 || VB == VK_C4 || VB == VK_ME4 || VB == VK_2D4);
  constexpr bool SIXTH = (VB == VK_C6);
  constexpr bool TMA = TM;
  static_assert(!TMA || (AT && DIM == 3), "TMA tiles hold plain copies of 3D fields");
  constexpr int FS = tile_fstride<ORDER, DIR, T, ROWS, TM>();  // tile field stride
  constexpr int TW = TMA ? tma_row<DIR>() : (DIR == 0 ? TL : 32);  // tile row width
  T* tile = reinterpret_cast<T*>(smraw);
  double* Fs = reinterpret_cast<double*>(smraw + sizeof(T) * TF_COUNT * FS);
  const Geo& G = A.G;
  const int g = G.g, gx = G.gx, gy = G.gy;  // gx / gy: 1 with a non-periodic x / y
  // column of a row's first tile cell (x) or first owned cell (y / z)
  const int TOFF = TMA ? (DIR == 0 ? gx + 1 : gx) : 0;
  const int Nx = G.nx - 2 * gx, Ny = G.ny - 2 * gy;
  const int gz = G.gz;                        // 1 with a non-periodic z
  const int Nz = (DIM == 3) ? G.nz - 2 * gz : 1;
  const bool act = tid < TX * TY;  // thread owns a face / cell slot of the tile shape
  const int tx = tid % TX, ty = tid / TX;
  const int nthr = nthr_all;
  // block origin (first owned cell) in padded coordinates
  int bx0, by0, bz0;
  // z: the cells of planes [sk0, sk1) (every interior plane unless a stage part narrows it)
  if constexpr (DIR == 0) {
    bx0 = gx + 32 * b0; by0 = gy + ROWS * b1; bz0 = (DIM == 3) ? G.sk0 + b2 : 0;
  } else if constexpr (DIR == 1) {
    bx0 = gx + 32 * b0; by0 = gy + ROWS * b1; bz0 = (DIM == 3) ? G.sk0 + b2 : 0;
  } else {
    bx0 = gx + 32 * b0; bz0 = G.sk0 + ROWS * b1; by0 = gy + b2;
  }
  const int64_t stv[3] = {1, G.sx, G.plane};
  const int nsweep = DIR == 0 ? G.nx : (DIR == 1 ? G.ny : G.nz);
  const int ext[3] = {gx + Nx, gy + Ny, DIM == 3 ? G.sk1 : gz + Nz};

  // ---- operand prefetch (y/z sweeps): the thread that owns a cell copies it ----
  constexpr bool PF_ON = PF > 0 && DIR != 0;
  constexpr bool PF_C = PF_ON && (PF & 1);  // combination operands
  constexpr bool PF_R = PF_ON && (PF & 2);  // accumulator
  constexpr bool MXC = sizeof(T) < sizeof(double);
  constexpr int PFC = 32 * ROWS;  // owned cells per tile
  double* pfQn = reinterpret_cast<double*>(smraw + sweep_smem<ORDER, DIR, T, ROWS, TM>());
  double* pfX = pfQn + 5 * PFC;             // Qs (as T) or Rs
  T* pfQs = reinterpret_cast<T*>(pfX);
  double* pfRs = pfX;
  double* pfR = pfQn + (PF_C ? 10 : 0) * PFC;
  static_assert(!SHARE || VK == VK_ME4, "shared face positions are built for the periodic ME4 stencil");
  constexpr int NPOS = me4_positions<DIR, ROWS>();
  constexpr int PSTEP = DIR == 0 ? 1 : 32;                // next position along the sweep
  constexpr int TSTEP = DIR == 0 ? 1 : TW;                // next tile cell along the sweep
  constexpr int PROW = DIR == 0 ? TX + 2 : 32;            // x sweep: positions per pencil row
  T* Vs = reinterpret_cast<T*>(smraw + sweep_smem<ORDER, DIR, T, ROWS, TM>() + sweep_pf_bytes<DIR, T, ROWS>(PF));
  const int md = last ? A.mode : CM_ACCUM;
  const bool needQn = (!MXC && (md == CM_RK3_1 || md == CM_RK3_2 || md == CM_RK4_S)) || md == CM_RK3_3 ||
                      md == CM_RK4_4;
  const bool needQs = md == CM_RK3_2 || md == CM_RK3_3;
  const bool needRs = md == CM_RK4_S || md == CM_RK4_4;
  const int slot = ty * 32 + tx;
  // the prefetch is one cp.async group; with AT it is issued after the tile's group, so
  // that waiting for the tile (wait_group 1) leaves the prefetch in flight
  auto issue_prefetch = [&]() {
    if (act && ty < TY - 1) {
      int pc[3];
      pc[0] = bx0 + tx;
      pc[DIR] = (DIR == 1 ? by0 : bz0) + ty;
      if (DIR == 1) pc[2] = bz0; else pc[1] = by0;
      if (pc[0] < ext[0] && pc[1] < ext[1] && (DIM == 2 || pc[2] < ext[2])) {
        const int64_t po = G.at(pc[0], pc[1], DIM == 3 ? pc[2] : 0);
#pragma unroll
        for (int l = 0; l < DIM + 2; ++l) {
          const int64_t q = po + l * G.vs;
          if (PF_R) cp_async<8>(pfR + l * PFC + slot, A.Racc + q);
          if (PF_C && needQn) cp_async<8>(pfQn + l * PFC + slot, A.Qn + q);
          if (PF_C && needRs) cp_async<8>(pfRs + l * PFC + slot, A.Rs + q);
          else if (PF_C && needQs) cp_async<sizeof(T)>(pfQs + l * PFC + slot, A.Qs + q);
        }
      }
    }
    cp_async_commit();
  };
  if constexpr (PF_ON && !AT) issue_prefetch();

  // ---- tile load: tensor copies (TMA layout with maps) ----
  bool use_tma = false;
  unsigned long long* tbar = nullptr;
  if constexpr (TMA) {
    tbar = reinterpret_cast<unsigned long long*>(smraw + sizeof(T) * TF_COUNT * FS +
                                                 sizeof(double) * 5 * TX * TY);
    use_tma = tmaps != nullptr && (smem_u32(smraw) & 127u) == 0;
    if (use_tma && tid == 0) {
      const bool sen = !KONLY && A.scheme != 0;
      const unsigned nf = 6u + (sen ? 1u : 0u) + (VK != VK_EULER ? 1u : 0u) + (LES ? 2u : 0u) + (GR ? 4u : 0u);
      mbar_init(tbar, 1);
      mbar_fence_init();
      constexpr unsigned BOX = (unsigned)(sizeof(T) * TW * tma_box_rows<ORDER, DIR, ROWS>());
      mbar_expect_tx(tbar, BOX * nf);
      // box origin: x = the row's first cell (32 b, or 32 b - 4 in the x sweep), the
      // tile's first cell along the sweep
      const int x0 = DIR == 0 ? bx0 - gx - 4 : bx0 - gx;
      const int y0 = DIR == 1 ? by0 - TILE_HALO : by0;
      const int z0 = DIR == 2 ? bz0 - TILE_HALO : bz0;
      auto copy = [&](int field) { tma_load_3d(tile + field * FS, tmaps->m[field], x0, y0, z0, tbar); };
      copy(TF_RHO); copy(TF_U); copy(TF_V); copy(TF_W); copy(TF_P); copy(TF_T);
      if (sen) copy(TF_SEN);
      if constexpr (VK != VK_EULER) copy(TF_MU);
      if constexpr (LES) { copy(TF_MUT); copy(TF_QC2); }
      if constexpr (GR) { copy(TF_D0); copy(TF_D1); copy(TF_D2); copy(TF_D3); }
    }
  }

  // ---- tile load (cooperative) ----
  for (int c = use_tma ? NC : tid; c < NC; c += nthr) {
    int ci[3];
    int along;
    int sl = c;  // the cell's slot in a field's slab
    if constexpr (DIR == 0) {
      int t = c % TL, r = c / TL;
      along = bx0 - TILE_HALO + t; ci[0] = along; ci[1] = by0 + r; ci[2] = bz0;
      sl = r * TW + TOFF + t;
    } else {
      int x = c % 32, t = c / 32;
      along = (DIR == 1 ? by0 : bz0) - TILE_HALO + t;
      ci[0] = bx0 + x;
      ci[1] = (DIR == 1) ? along : by0;
      ci[2] = (DIR == 2) ? along : bz0;
      sl = t * TW + TOFF + x;
    }
    bool ok = along >= 0 && along < nsweep;
#pragma unroll
    for (int a = 0; a < 3; ++a)
      if (a != DIR && (a < DIM) && ci[a] >= ext[a]) ok = false;
    if (!ok) continue;
    const int64_t o = G.at(ci[0], ci[1], DIM == 3 ? ci[2] : 0);
    if constexpr (AT) {
      cp_async<sizeof(T)>(&tile[TF_RHO * FS + sl], A.W.rho + o);
      cp_async<sizeof(T)>(&tile[TF_U * FS + sl], A.W.u + o);
      cp_async<sizeof(T)>(&tile[TF_V * FS + sl], A.W.v + o);
      if constexpr (DIM == 3) cp_async<sizeof(T)>(&tile[TF_W * FS + sl], A.W.w + o);
      else tile[TF_W * FS + sl] = T(0);
      cp_async<sizeof(T)>(&tile[TF_P * FS + sl], A.W.p + o);
      cp_async<sizeof(T)>(&tile[TF_T * FS + sl], A.W.T_ + o);
      if (!KONLY && A.scheme != 0) cp_async<sizeof(T)>(&tile[TF_SEN * FS + sl], A.W.sensor + o);
      if constexpr (VK != VK_EULER) cp_async<sizeof(T)>(&tile[TF_MU * FS + sl], A.W.mu + o);
      if constexpr (LES) {
        cp_async<sizeof(T)>(&tile[TF_MUT * FS + sl], A.W.mut + o);
        cp_async<sizeof(T)>(&tile[TF_QC2 * FS + sl], A.W.qc2 + o);
      }
      if constexpr (HIGH && GR) {
        constexpr int n = DIR, a1 = (n + 1) % 3, a2 = (n + 2) % 3;
        constexpr int ca = n == 0 ? 1 : 0, cb = n == 2 ? 1 : 2;
        cp_async<sizeof(T)>(&tile[TF_D0 * FS + sl], A.W.grad[3 * a1 + a1] + o);
        cp_async<sizeof(T)>(&tile[TF_D1 * FS + sl], A.W.grad[3 * a2 + a2] + o);
        cp_async<sizeof(T)>(&tile[TF_D2 * FS + sl], A.W.grad[3 * n + ca] + o);
        cp_async<sizeof(T)>(&tile[TF_D3 * FS + sl], A.W.grad[3 * n + cb] + o);
      }
      // without gradient fields the derivatives are differenced below, while the
      // copies above are in flight
      if constexpr (!HIGH || GR) continue;
    }
    if constexpr (!AT) {
      tile[TF_RHO * FS + sl] = ldro<RO>(A.W.rho + o);
      tile[TF_U * FS + sl] = ldro<RO>(A.W.u + o);
      tile[TF_V * FS + sl] = ldro<RO>(A.W.v + o);
      tile[TF_W * FS + sl] = (DIM == 3) ? ldro<RO>(A.W.w + o) : T(0);
      tile[TF_P * FS + sl] = ldro<RO>(A.W.p + o);
      tile[TF_T * FS + sl] = ldro<RO>(A.W.T_ + o);
      if (!KONLY && A.scheme != 0) tile[TF_SEN * FS + sl] = ldro<RO>(A.W.sensor + o);
      if constexpr (VK != VK_EULER) tile[TF_MU * FS + sl] = ldro<RO>(A.W.mu + o);
      if constexpr (LES) {
        tile[TF_MUT * FS + sl] = ldro<RO>(A.W.mut + o);
        tile[TF_QC2 * FS + sl] = ldro<RO>(A.W.qc2 + o);
      }
    }
    if constexpr (HIGH && GR) {  // transverse node derivatives from the gradient fields
      static_assert(DIM == 3, "gradient fields are built for 3D grids");
      constexpr int n = DIR, a1 = (n + 1) % 3, a2 = (n + 2) % 3;
      constexpr int ca = n == 0 ? 1 : 0, cb = n == 2 ? 1 : 2;
      tile[TF_D0 * FS + sl] = ldro<RO>(A.W.grad[3 * a1 + a1] + o);
      tile[TF_D1 * FS + sl] = ldro<RO>(A.W.grad[3 * a2 + a2] + o);
      tile[TF_D2 * FS + sl] = ldro<RO>(A.W.grad[3 * n + ca] + o);
      tile[TF_D3 * FS + sl] = ldro<RO>(A.W.grad[3 * n + cb] + o);
    } else if constexpr (HIGH) {  // transverse node derivatives (the viscous loaders' stencils)
      const T* vel[3] = {A.W.u, A.W.v, A.W.w};
      const double* invd[3] = {A.M.inv_dx, A.M.inv_dy, A.M.inv_dz};
      if constexpr (DIM == 3) {
        const int n = DIR, a1 = (n + 1) % 3, a2 = (n + 2) % 3;
        const int ca = n == 0 ? 1 : 0, cb = n == 2 ? 1 : 2;
        // with a non-periodic direction, only where the stencil stays inside the grid:
        // the other cells lie outside the high-order guard, whose 2nd-order fallback
        // does not read these values
        constexpr int HD = SIXTH ? 3 : 2;
        const int na[3] = {G.nx, G.ny, G.nz};
        auto nd = [&](const T* f, int ax) -> T {
          if (WALL && !(ci[ax] >= HD && ci[ax] + HD < na[ax])) return T(0);
          return node_d<SIXTH, RO>(f, o, stv[ax], (T)invd[ax][ci[ax]]);
        };
        tile[TF_D0 * FS + sl] = nd(vel[a1], a1);
        tile[TF_D1 * FS + sl] = nd(vel[a2], a2);
        tile[TF_D2 * FS + sl] = nd(vel[n], ca);
        tile[TF_D3 * FS + sl] = nd(vel[n], cb);
      } else {
        // 2D: only where the stencil stays inside the grid; the other cells lie
        // outside the 4th-order guard of calc_Ev4 / calc_Fv4, whose 2nd-order
        // fallback does not read these values (non-periodic edges, order 2 grids)
        const int n = DIR, t = 1 - DIR;
        constexpr int HD = SIXTH ? 3 : 2;
        if (ci[t] >= HD && ci[t] + HD < (t == 0 ? G.nx : G.ny)) {
          tile[TF_D0 * FS + sl] = node_d<SIXTH, RO>(vel[t], o, stv[t], (T)invd[t][ci[t]]);
          tile[TF_D2 * FS + sl] = node_d<SIXTH, RO>(vel[n], o, stv[t], (T)invd[t][ci[t]]);
        } else {
          tile[TF_D0 * FS + sl] = T(0);
          tile[TF_D2 * FS + sl] = T(0);
        }
      }
    }
  }
  if constexpr (AT) {
    cp_async_commit();
    if constexpr (PF_ON) {
      issue_prefetch();
      cp_async_wait_group<1>();  // this thread's tile copies have landed; the prefetch may not have
    } else {
      cp_async_wait_all();
    }
  }
  __syncthreads();  // (also orders the mbarrier's initialisation before the waits below)
  if constexpr (TMA) {
    if (use_tma) {
      bool done = false;
      for (int it = 0; it < TMA_WAIT_LIMIT && !done; ++it) done = mbar_try_wait(tbar, 0);
      // a tile whose copies never complete ends the whole block, flagged on the host's
      // status word (the block's threads decide together)
      if (!__syncthreads_and(done)) {
        if (tid == 0 && A.status) atomicOr(A.status, 4 /* OUX_FAULT_TIMEOUT */);
        return;
      }
    }
  }

  // ---- shared ME4 face positions (every thread, strided) ----
  if constexpr (SHARE) {
    const double* invd[3] = {A.M.inv_dx, A.M.inv_dy, A.M.inv_dz};
    const T inv = (T)invd[DIR][0];  // the axis' spacings are all the same double
    for (int c = tid; c < NPOS; c += nthr) {
      // tile index of the position's first stencil cell (its left cell - 1)
      const int t0 = DIR == 0 ? (c / PROW) * TW + TOFF + c % PROW : (c / 32) * TW + TOFF + c % 32;
      auto sp = [&](int field, int m) -> T { return tile[field * FS + t0 + m * TSTEP]; };
      T v[9];
      me4_position<LES>(A, sp, DIR, inv, v);
#pragma unroll
      for (int q = 0; q < me4_terms<LES>(); ++q) Vs[q * NPOS + c] = v[q];
    }
  }

  // ---- faces ----
  bool face_valid = false;
  int face_pos = 0;  // SHARE: position index of the face's left neighbour position
  {
    int fc[3] = {bx0, by0, bz0};  // left cell of this thread's face
    int base, step;
    bool rowok;
    if constexpr (DIR == 0) {
      fc[0] = bx0 - 1 + tx; fc[1] = by0 + ty;
      base = ty * TW + TOFF + tx; step = 1;
      rowok = fc[1] < ext[1];
    } else {
      fc[0] = bx0 + tx;
      fc[DIR] = (DIR == 1 ? by0 : bz0) - 1 + ty;
      base = ty * TW + TOFF + tx; step = TW;
      rowok = fc[0] < ext[0];
    }
    const int f = fc[DIR];
    const bool valid = act && rowok && f >= (DIR == 0 ? gx : DIR == 1 ? gy : gz) - 1 && f <= ext[DIR] - 1;
    face_valid = valid;
    face_pos = DIR == 0 ? ty * PROW + tx : ty * 32 + tx;
    if (valid) {
      T F[5];
      // tile position of cell f + off is base + (2 + off) * step
      auto st0 = [&](int field, int m) -> T { return tile[field * FS + base + m * step]; };
      const int cb = base + (TILE_HALO - H) * step;
      auto sc = [&](int field, int m) -> T { return tile[field * FS + cb + m * step]; };
      T fd = T(0);
      if (!KONLY && A.scheme != 0) fd = T(0.5) * (st0(TF_SEN, 2) + st0(TF_SEN, 3));
      if constexpr (DIM == 2 || VK == VK_EULER || WALL) {
        // non-periodic x / y (/ z): every face, the stencil order lowered next to the
        // boundary as the reference's boundary kernels do (2D_solver/src/calc_{slau,
        // keep,hybrid}_kernel.f90.fypp, calc_*_x and calc_*_y; 3D_solver/src/calc_*
        // _kernel.f90.fypp): 6th for 2 <= f <= n-4, 4th for 1 <= f <= n-3, else 2nd /
        // first order (f: 0-based left cell of the face).  Compiled out of the periodic
        // 3D viscous sweeps (their walled variants carry it).
        int lo = ORDER;
        const int nn = DIR == 0 ? G.nx : (DIR == 1 ? G.ny : G.nz);
        const bool nonper = DIR == 0 ? (bool)G.bcx : (DIR == 1 ? (bool)G.bcy : G.bcz == 1);
        if (nonper)
          lo = (ORDER == 6 && f >= 2 && f <= nn - 4) ? 6 : (ORDER >= 4 && f >= 1 && f <= nn - 3) ? 4 : 2;
        if (lo == ORDER) {
          conv_flux<ORDER, KONLY>(A, sc, fd, DIR, F);
        } else if (lo == 4) {
          auto s4 = [&](int field, int m) -> T { return tile[field * FS + base + (TILE_HALO - 2 + m) * step]; };
          conv_flux<4, KONLY>(A, s4, fd, DIR, F);
        } else {
          auto s2 = [&](int field, int m) -> T { return tile[field * FS + base + (TILE_HALO - 1 + m) * step]; };
          conv_flux<2, KONLY>(A, s2, fd, DIR, F);
        }
      } else {
        conv_flux<ORDER, KONLY>(A, sc, fd, DIR, F);
      }
      if constexpr (VK != VK_EULER && !SHARE) {
        T vo[4];
        const double* invd[3] = {A.M.inv_dx, A.M.inv_dy, A.M.inv_dz};
        const T inv = (T)invd[DIR][f];
        if constexpr (VB == VK_GV2) {
          const int64_t o = G.at(fc[0], fc[1], DIM == 3 ? fc[2] : 0);
          T invs[3] = {(T)A.M.inv_dx[fc[0]], (T)A.M.inv_dy[fc[1]], DIM == 3 ? (T)A.M.inv_dz[fc[2]] : T(0)};
          visc_gv2<DIM, LES, RO>(A, DIR, o, stv, invs, vo);
        } else if constexpr (VK == VK_2D4) {
          // inner guard of calc_Ev4 / calc_Fv4 (2D): face 2..n-4, transverse 2..n-3
          const int nt = DIR == 0 ? G.ny : G.nx;
          const int tr = fc[1 - DIR];
          const int nn = DIR == 0 ? G.nx : G.ny;
          bool inner = (f >= 2 && f <= nn - 4 && tr >= 2 && tr <= nt - 3);
          const int64_t o = G.at(fc[0], fc[1], 0);
          T invs[2] = {(T)A.M.inv_dx[fc[0]], (T)A.M.inv_dy[fc[1]]};
          invs[DIR] = inv;
          auto sv = [&](int field, int m) -> T { return tile[field * FS + base + m * step]; };
          visc_2d4(A, sv, DIR, inner, o, stv, invs, vo);
        } else {
          constexpr int off0 = (VB == VK_C4) ? -1 : -2;
          const int vb = base + (2 + off0) * step;
          auto sv = [&](int field, int m) -> T { return tile[field * FS + vb + m * step]; };
          if constexpr (WALL) {
            // high-order guard of calc_{E,F,G}v (calc_visc_high.f90.fypp:114/139/169,
            // 350/376/406, 592/618/648), 0-based: C4 faces 1..n-3 and transverse cells
            // 2..n-3, ME4 faces 2..n-4 and cells 2..n-3, C6 faces 2..n-4 and cells 3..n-4
            constexpr int FA = (VB == VK_C4) ? 1 : 2, TA = (VB == VK_C6) ? 3 : 2;
            const int na[3] = {G.nx, G.ny, G.nz};
            bool inner = f >= FA && f <= na[DIR] - 2 - FA;
#pragma unroll
            for (int a = 0; a < 3; ++a)
              if (a != DIR) inner = inner && fc[a] >= TA && fc[a] <= na[a] - 1 - TA;
            if (inner) {
              visc_high<VB, LES>(A, sv, DIR, inv, vo);
            } else {
              const int64_t o = G.at(fc[0], fc[1], fc[2]);
              T invs[3] = {(T)A.M.inv_dx[fc[0]], (T)A.M.inv_dy[fc[1]], (T)A.M.inv_dz[fc[2]]};
              invs[DIR] = inv;
              visc_fb3<LES>(A, DIR, o, stv, invs, vo);
            }
          } else {
            visc_high<VB, LES>(A, sv, DIR, inv, vo);
          }
        }
        if constexpr (DIM == 3) {
          F[1] = F[1] - vo[0]; F[2] = F[2] - vo[1]; F[3] = F[3] - vo[2]; F[4] = F[4] - vo[3];
        } else {
          F[1] = F[1] - vo[0]; F[2] = F[2] - vo[1]; F[4] = F[4] - vo[3];
        }
      }
#pragma unroll
      for (int l = 0; l < 5; ++l) Fs[l * (TX * TY) + tid] = (double)F[l];
    }
  }
  __syncthreads();

  // ---- shared ME4: each face combines its three positions ----
  if constexpr (SHARE) {
    if (face_valid) {
      const double* invd[3] = {A.M.inv_dx, A.M.inv_dy, A.M.inv_dz};
      const T inv = (T)invd[DIR][0];
      auto P = [&](int k, int q) -> T { return Vs[k * NPOS + face_pos + q * PSTEP]; };
      T vo[4];
      me4_face<LES>(A, P, DIR, inv, vo);
      // F[l] - vo in the compute type, as the unshared path does
      Fs[1 * (TX * TY) + tid] = (double)((T)Fs[1 * (TX * TY) + tid] - vo[0]);
      Fs[2 * (TX * TY) + tid] = (double)((T)Fs[2 * (TX * TY) + tid] - vo[1]);
      if constexpr (DIM == 3) Fs[3 * (TX * TY) + tid] = (double)((T)Fs[3 * (TX * TY) + tid] - vo[2]);
      Fs[4 * (TX * TY) + tid] = (double)((T)Fs[4 * (TX * TY) + tid] - vo[3]);
    }
    __syncthreads();
  }

  // ---- cells: difference, accumulate, combine ----
  if (!act) return;
  {
    int cc[3];
    bool ok;
    int lo, hi;  // flux slots of the left / right faces
    if constexpr (DIR == 0) {
      if (tx >= 32) return;
      cc[0] = bx0 + tx; cc[1] = by0 + ty; cc[2] = bz0;
      lo = ty * TX + tx; hi = lo + 1;
    } else {
      if (ty >= TY - 1) return;
      cc[0] = bx0 + tx;
      cc[DIR] = (DIR == 1 ? by0 : bz0) + ty;
      if (DIR == 1) cc[2] = bz0; else cc[1] = by0;
      lo = ty * TX + tx; hi = lo + TX;
    }
    ok = cc[0] < ext[0] && cc[1] < ext[1] && (DIM == 2 || cc[2] < ext[2]);
    if (!ok) return;
    const int i = cc[0], j = cc[1], k = (DIM == 3) ? cc[2] : 0;
    const int64_t o = G.at(i, j, k);
    if constexpr (PF_ON) cp_async_wait_all();
    // operands of the difference / combination: prefetched copy or global
    auto RACC = [&](int l) -> double {
      if constexpr (PF_R) return pfR[l * PFC + slot];
      else return A.Racc[o + l * G.vs];
    };
    auto QN = [&](int l) -> double {
      if constexpr (PF_C) return pfQn[l * PFC + slot];
      else return A.Qn[o + l * G.vs];
    };
    auto QS = [&](int l) -> T {
      if constexpr (PF_C) return pfQs[l * PFC + slot];
      else return A.Qs[o + l * G.vs];
    };
    auto RS = [&](int l) -> double {
      if constexpr (PF_C) return pfRs[l * PFC + slot];
      else return A.Rs[o + l * G.vs];
    };
    // dt * S metric for this direction, scaled by coef (calc_steps.f90 calc_R)
    double met;
    if constexpr (DIM == 3) {
      if (DIR == 0) met = A.M.dtdydz[(int64_t)(k - 1) * (G.ny - 2) + (j - 1)];
      else if (DIR == 1) met = A.M.dtdzdx[(int64_t)(k - 1) * (G.nx - 2) + (i - 1)];
      else met = A.M.dtdxdy[(int64_t)(j - 1) * (G.nx - 2) + (i - 1)];
    } else {
      met = (DIR == 0) ? A.M.dtdy[j - 1] : A.M.dtdx[i - 1];
    }
    const double cm = A.coef * met;
    constexpr int NV = DIM + 2;
    double R[NV];
#pragma unroll
    for (int l = 0; l < NV; ++l) {
      const int fl = (DIM == 2 && l == 3) ? 4 : l;  // 2D: energy is flux slot 4
      double d = cm * (-Fs[fl * (TX * TY) + lo] + Fs[fl * (TX * TY) + hi]);
      if (DIR == 0) R[l] = d;
      else R[l] = RACC(l) + d;
    }
    if (!last) {
#pragma unroll
      for (int l = 0; l < NV; ++l) A.Racc[o + l * G.vs] = R[l];
      return;
    }
    // mixed form: the stage state holds the FP32 increment Q^(s) - Q^n
    switch (A.mode) {
      case CM_R_OUT: {
        // reference Rs(nx-2, nv, ny-2, nz-2) order, cell (i,j,k) -> (i-1, l, j-1, k-1)
        int64_t base = (((int64_t)(DIM == 3 ? k - 1 : 0) * (G.ny - 2) + (j - 1)) * NV) * (G.nx - 2) + (i - 1);
#pragma unroll
        for (int l = 0; l < NV; ++l) A.Rout[base + (int64_t)l * (G.nx - 2)] = R[l];
        break;
      }
      case CM_RK3_1: {
#pragma unroll
        for (int l = 0; l < NV; ++l) {
          const int64_t q = o + l * G.vs;
          if constexpr (MXC) A.Qs[q] = (T)(-R[l]);  // stage increment Q1 - Qn
          else A.Qs[q] = (T)(QN(l) - R[l]);
        }
        break;
      }
      case CM_RK3_2: {
#pragma unroll
        for (int l = 0; l < NV; ++l) {
          const int64_t q = o + l * G.vs;
          if constexpr (MXC) A.Qs[q] = (T)((A.c2 * (double)QS(l) - R[l]) * A.c4);  // c1 + c2 = 1
          else A.Qs[q] = (T)((A.c1 * QN(l) + A.c2 * (double)QS(l) - R[l]) * A.c4);
        }
        break;
      }
      case CM_RK3_3: {
#pragma unroll
        for (int l = 0; l < NV; ++l) {
          const int64_t q = o + l * G.vs;
          if constexpr (MXC) A.Qn[q] = QN(l) + (A.c1 * (double)QS(l) - R[l]) * A.c4;  // (c1 + c2) c4 = 1
          else A.Qn[q] = (A.c1 * (double)QS(l) + A.c2 * QN(l) - R[l]) * A.c4;
        }
        break;
      }
      case CM_RK4_S: {
#pragma unroll
        for (int l = 0; l < NV; ++l) {
          const int64_t q = o + l * G.vs;
          if constexpr (MXC) A.Qs[q] = (T)(-A.c1 * R[l]);
          else A.Qs[q] = (T)(QN(l) - A.c1 * R[l]);
          A.Rs[q] = RS(l) + A.c2 * R[l];
        }
        break;
      }
      case CM_RK4_4: {
#pragma unroll
        for (int l = 0; l < NV; ++l) {
          const int64_t q = o + l * G.vs;
          double r = RS(l) + R[l];
          A.Qn[q] = QN(l) - r * (1.0 / 6.0);
          A.Rs[q] = 0.0;
        }
        break;
      }
      default: break;
    }
  }
}

// Threads of a k_sweep block (1D): the tile shape rounded up to whole warps.  For the
// x sweep (33 x 4 face threads) the 28 extra threads load tile cells only, so the
// 38 x 4 tile loads in one pass.
template <int DIR> __host__ __device__ constexpr int sweep_threads() {
  return (SweepShape<DIR>::TX * SweepShape<DIR>::TY + 31) / 32 * 32;
}

// Single-solve sweeps of 3D grids with a high-order viscous stencil read the transverse
// node derivatives from the gradient fields (k_grad writes them).  On walled grids too:
// k_grad writes 0 where a stencil leaves the grid, as the walled tile load does, and
// the viscous faces read tile derivatives only inside the high-order guard, whose
// cells' stencils all fit.
template <int DIM, int VK> __host__ __device__ constexpr bool sweep_uses_grads() {
  return DIM == 3 && (vk_base(VK) == VK_C6 || vk_base(VK) == VK_C4 || vk_base(VK) == VK_ME4);
}
// Their tiles are then all plain copies; the x and y sweeps' are staged by TMA (the
// TMA tile layout).  Measured on B200 at 512^3 (Hybrid-6 / ME4, ms per launch, TMA
// against cp.async): x 8.12 / 8.18 (FP64) and 5.52 / 5.48 (mixed); y 8.74 / 8.80 and
// 4.89 / 5.30; z 9.46 / 9.11 and 6.39 / 6.24, where a box is 13 rows from 13 planes
// 2 MB apart; so z keeps cp.async.
template <int DIM, int DIR, int VK> __host__ __device__ constexpr bool sweep_tma() {
  return DIR <= 1 && sweep_uses_grads<DIM, VK>();
}

template <int DIM, int DIR, int ORDER, int VK, bool LES, class T, bool SHARE = false>
__global__ void __launch_bounds__(sweep_threads<DIR>(), DIR == 0 ? OUX_SWEEP_MINB_X : OUX_SWEEP_MINB_YZ)
k_sweep(StepArgs<T> A, int last) {
  extern __shared__ __align__(16) unsigned char smraw[];
  // coherent loads: measured as fast as the read-only path for y/z and faster for x
  constexpr int VB = vk_base(VK);
  constexpr bool HIGH = (VB == VK_C6 || VB == VK_C4 || VB == VK_ME4 || VB == VK_2D4);
  constexpr bool GR = sweep_uses_grads<DIM, VK>();
  sweep_tile<DIM, DIR, ORDER, VK, LES, T, default_rows<DIR>(), false, false, sweep_pf_mode<DIM, DIR, T>(), SHARE,
             GR, !HIGH || GR, sweep_tma<DIM, DIR, VK>()>(A, last, blockIdx.x, blockIdx.y, blockIdx.z, smraw,
                                                        threadIdx.x, sweep_threads<DIR>());
}

// The sweeps of sweep_tma configurations: k_sweep with the tile's tensor maps as a
// kernel parameter (`use` = 0: none; the tile is then filled by cp.async).
template <int DIM, int DIR, int ORDER, int VK, bool LES, class T, bool SHARE = false>
__global__ void __launch_bounds__(sweep_threads<DIR>(), DIR == 0 ? OUX_SWEEP_MINB_X : OUX_SWEEP_MINB_YZ)
k_sweep_tm(StepArgs<T> A, int last, const __grid_constant__ SweepMaps maps, int use) {
  extern __shared__ __align__(128) unsigned char smtile[];  // tensor copies land 128-byte aligned
  unsigned char* smraw = smtile;
  static_assert(sweep_tma<DIM, DIR, VK>(), "k_sweep_tm serves the TMA-staged sweeps");
  sweep_tile<DIM, DIR, ORDER, VK, LES, T, default_rows<DIR>(), false, false, sweep_pf_mode<DIM, DIR, T>(), SHARE,
             true, true, true>(A, last, blockIdx.x, blockIdx.y, blockIdx.z, smraw, threadIdx.x, sweep_threads<DIR>(),
                               use ? &maps : nullptr);
}

}  // namespace oux
