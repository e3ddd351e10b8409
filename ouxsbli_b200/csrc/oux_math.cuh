// Device-side face-flux arithmetic for the OUxSBLI time step.
//
// Every function here evaluates the same formula, in the same operation
// order, as the reference kernel it cites (paths relative to the OUxSBLI
// repository), so that an FP64 build compiled without FMA contraction
// (-fmad=false) reproduces the reference arithmetic bit for bit.  The
// mixed-precision build instantiates the same templates with float.
//
// Fortran intrinsics whose signed-zero behaviour the source leaves to the
// compiler are fixed as: SIGN(1,x) = copysign(1,x); MIN(a,b) = (b < a ? b : a);
// MAX(a,b) = (b > a ? b : a).
#pragma once
#include <cuda_runtime.h>
#include <math.h>

namespace oux {

struct PhysConst {
  double gamma, R, Pr, Prt, threshold;
  double gamma_1, over_gamma_1, R_over_gamma_1, Cp, Cp_over_Pr, sutherland;
  double gamma_over_gamma_1, tan10deg2;
  // mixed form only: FP32 pressure / temperature fields hold p - p_ref, T - T_ref
  double p_ref, T_ref;
};

template <class T> __device__ __forceinline__ T sgn1(T b) { return signbit(b) ? T(-1) : T(1); }
template <class T> __device__ __forceinline__ T fmin_f(T a, T b) { return (b < a) ? b : a; }
template <class T> __device__ __forceinline__ T fmax_f(T a, T b) { return (b > a) ? b : a; }

// ---- MUSCL reconstruction: src/calc_muscl.f90 --------------------------------
template <class T> __device__ __forceinline__ T minmod2(T x, T y) {  // :19-24
  T s = sgn1(x);
  return s * fmax_f(fmin_f(fabs(x), s * y), T(0));
}
template <class T> __device__ __forceinline__ T minmod3(T x, T y, T z) {  // :27-32
  T s = sgn1(x);
  return s * fmax_f(fmin_f(fmin_f(fabs(x), s * y), s * z), T(0));
}
template <class T> __device__ __forceinline__ T d33(T d1, T d2, T d3) {  // :35-41
  return minmod3(d1, T(2) * d2, T(2) * d3) - T(2) * minmod3(d2, T(2) * d1, T(2) * d3) +
         minmod3(d3, T(2) * d1, T(2) * d2);
}

template <class T> struct Coef {
  static constexpr double third = 1.0 / 3.0, two_third = 2.0 / 3.0, sixth = 1.0 / 6.0,
                          twelfth = 1.0 / 12.0, sixty = 1.0 / 60.0;
};

// MUSCL3rd (:44-88); tvd: 0 none, 1 minmod, 2 sensor-switched (hybrid)
template <class T>
__device__ __forceinline__ void muscl3(int tvd, T thr, T sensor, T a2, T a3, T d1, T d2, T d3,
                                       T& al, T& ar) {
  const T third = T(1.0 / 3.0);
  bool plain = (tvd == 0) || (tvd == 2 && sensor < thr);
  if (plain) {
    al = a2 + T(0.5) * (d1 + T(2) * d2) * third;
    ar = a3 - T(0.5) * (d3 + T(2) * d2) * third;
  } else {
    const T b = T((3.0 - 1.0 / 3.0) / (1.0 - 1.0 / 3.0));
    T t1 = minmod2(d1, b * d2), t2 = minmod2(d2, b * d1);
    al = a2 + T(0.5) * (t1 + T(2) * t2) * third;
    T t3 = minmod2(d3, b * d2), t4 = minmod2(d2, b * d3);
    ar = a3 - T(0.5) * (t3 + T(2) * t4) * third;
  }
}
// MUSCL4th (:91-139)
template <class T>
__device__ __forceinline__ void muscl4(int tvd, T thr, T sensor, T a2, T a3, T d1, T d2, T d3,
                                       T d4, T d5, T& al, T& ar) {
  const T sixth = T(1.0 / 6.0), twelfth = T(1.0 / 12.0);
  bool plain = (tvd == 0) || (tvd == 2 && sensor < thr);
  if (plain) {
    al = a2 + (T(-0.4) * d1 + T(2.2) * d2 + T(4.8) * d3 - T(0.6) * d4) * twelfth;
    ar = a3 - (T(-0.6) * d2 + T(4.8) * d3 + T(2.2) * d4 - T(0.4) * d5) * twelfth;
  } else {
    T dm = d3 - d33(d2, d3, d4) * sixth;
    T dlo = d2 - d33(d1, d2, d3) * sixth;
    T l1 = minmod2(dlo, T(4) * dm), r1 = minmod2(dm, T(4) * dlo);
    al = a2 + (l1 + T(2) * r1) * sixth;
    T dhi = d4 - d33(d3, d4, d5) * sixth;
    T l2 = minmod2(dm, T(4) * dhi), r2 = minmod2(dhi, T(4) * dm);
    ar = a3 - (r2 + T(2) * l2) * sixth;
  }
}
// delta4 / delta6 (:142-169) over the stencil a[0..2io+1] of one face
template <int ORDER, class T>
__device__ __forceinline__ void reconstruct(int tvd, T thr, T sensor, const T* a, T& al, T& ar) {
  if constexpr (ORDER == 2) {
    al = a[0]; ar = a[1];
  } else if constexpr (ORDER == 4) {
    T d1 = -a[0] + a[1], d2 = -a[1] + a[2], d3 = -a[2] + a[3];
    muscl3(tvd, thr, sensor, a[1], a[2], d1, d2, d3, al, ar);
  } else {
    T d1 = -a[0] + a[1], d2 = -a[1] + a[2], d3 = -a[2] + a[3], d4 = -a[3] + a[4], d5 = -a[4] + a[5];
    muscl4(tvd, thr, sensor, a[2], a[3], d1, d2, d3, d4, d5, al, ar);
  }
}
// pressure wiggle detector: 3D_solver/src/calc_hybrid.f90:75-81
template <class T> __device__ __forceinline__ T wiggle(T p1, T p2, T p3, T p4) {
  T phi1 = (-p1 + p2) * (-p2 + p3);
  T phi2 = (-p3 + p4) * (-p2 + p3);
  return T(0.5) * (T(1) - sgn1(fmin_f(phi1, phi2)));
}

// ---- KEEP split form: 3D_solver/src/calc_keep_3d.f90 ------------------------
// s[] holds 2io+2 stencil points; un = normal velocity; nd = normal axis.
// MX (mixed form): p and Tt are deviations from pr / tr; the momentum-flux
// pressure is formed from the deviations (its stencil weights sum to 1, so the
// constant cancels in the face difference), every other use adds the reference back.
template <int ORDER, class T, bool MX = false>
__device__ __forceinline__ void keep_flux(const T* rho, const T* u, const T* v, const T* w,
                                          const T* un, const T* pd, const T* Td, int nd, T Rg1,
                                          T F[5], T pr = T(0), T tr = T(0)) {
  const T n2 = nd == 0 ? T(1) : T(0), n3 = nd == 1 ? T(1) : T(0), n4 = nd == 2 ? T(1) : T(0);
  constexpr int NS = ORDER;
  T pf[NS], Tf[NS];
  const T* p = pd;
  const T* Tt = Td;
  if constexpr (MX) {
#pragma unroll
    for (int m = 0; m < NS; ++m) { pf[m] = pd[m] + pr; Tf[m] = Td[m] + tr; }
    p = pf;
    Tt = Tf;
  }
  if constexpr (ORDER == 2) {  // KEEP2 :1-15
    F[0] = T(0.25) * (rho[0] + rho[1]) * (un[0] + un[1]);
    F[1] = T(0.5) * (F[0] * (u[0] + u[1]) + (pd[0] + pd[1]) * n2);
    F[2] = T(0.5) * (F[0] * (v[0] + v[1]) + (pd[0] + pd[1]) * n3);
    F[3] = T(0.5) * (F[0] * (w[0] + w[1]) + (pd[0] + pd[1]) * n4);
    F[4] = F[0] * T(0.5) * (Tt[0] + Tt[1]) * Rg1;
    F[4] = F[4] + T(0.5) * (un[0] * p[1] + un[1] * p[0]);
    F[4] = F[4] + T(0.5) * F[0] * (u[0] * u[1] + v[0] * v[1] + w[0] * w[1]);
  } else if constexpr (ORDER == 4) {  // KEEP4 :18-56
    const T c24 = T(1.0 / 24.0), c48 = T(1.0 / 48.0), c12 = T(1.0 / 12.0), c712 = T(7.0 / 12.0);
    T A = (rho[1] + rho[2]) * (un[1] + un[2]);
    T B = (rho[1] + rho[3]) * (un[1] + un[3]);
    T Cc = (rho[0] + rho[2]) * (un[0] + un[2]);
    F[0] = T(1.0 / 3.0) * A - (B + Cc) * c24;
    A = T(1.0 / 6.0) * A;
    B = c48 * B;
    Cc = c48 * Cc;
    T AB = A - B, AC = A - Cc;
    T pres = -c12 * pd[0] + c712 * (pd[1] + pd[2]) - c12 * pd[3];
    F[1] = -Cc * u[0] + AB * u[1] + AC * u[2] - B * u[3] + pres * n2;
    F[2] = -Cc * v[0] + AB * v[1] + AC * v[2] - B * v[3] + pres * n3;
    F[3] = -Cc * w[0] + AB * w[1] + AC * w[2] - B * w[3] + pres * n4;
    T e = (-Cc * Tt[0] + AB * Tt[1] + AC * Tt[2] - B * Tt[3]) * Rg1;
    e = e + ((A * (u[1] * u[2] + v[1] * v[2] + w[1] * w[2])) -
             (B * (u[1] * u[3] + v[1] * v[3] + w[1] * w[3]) + Cc * (u[0] * u[2] + v[0] * v[2] + w[0] * w[2])));
    F[4] = e + (T(2.0 / 3.0) * (un[1] * p[2] + un[2] * p[1]) -
                c12 * (un[1] * p[3] + un[3] * p[1] + un[0] * p[2] + un[2] * p[0]));
  } else {  // KEEP6 :59-111
    const T c60 = T(1.0 / 60.0), c120 = T(1.0 / 120.0), c240 = T(1.0 / 240.0);
    T a1 = (rho[2] + rho[3]) * (un[2] + un[3]);
    T a2 = (rho[2] + rho[4]) * (un[2] + un[4]);
    T a3 = (rho[1] + rho[3]) * (un[1] + un[3]);
    T a4 = (rho[2] + rho[5]) * (un[2] + un[5]);
    T a5 = (rho[1] + rho[4]) * (un[1] + un[4]);
    T a6 = (rho[0] + rho[3]) * (un[0] + un[3]);
    F[0] = T(0.375) * a1 - T(0.075) * (a2 + a3) + (a4 + a5 + a6) * c120;
    a1 = T(0.1875) * a1;
    a2 = T(0.0375) * a2;
    a3 = T(0.0375) * a3;
    a4 = a4 * c240;
    a5 = a5 * c240;
    a6 = a6 * c240;
    T w35 = -a3 + a5, w124 = a1 - a2 + a4, w136 = a1 - a3 + a6, w25 = -a2 + a5;
    T pres = (pd[0] - T(8) * pd[1] + T(37) * (pd[2] + pd[3]) - T(8) * pd[4] + pd[5]) * c60;
    T m1 = a6 * u[0] + w35 * u[1] + w124 * u[2] + w136 * u[3] + w25 * u[4] + a4 * u[5];
    m1 = m1 + pres * n2;
    T m2 = a6 * v[0] + w35 * v[1] + w124 * v[2] + w136 * v[3] + w25 * v[4] + a4 * v[5];
    m2 = m2 + pres * n3;
    T m3 = a6 * w[0] + w35 * w[1] + w124 * w[2] + w136 * w[3] + w25 * w[4] + a4 * w[5];
    m3 = m3 + pres * n4;
    F[1] = m1; F[2] = m2; F[3] = m3;
    T e = (a6 * Tt[0] + w35 * Tt[1] + w124 * Tt[2] + w136 * Tt[3] + w25 * Tt[4] + a4 * Tt[5]) * Rg1;
    e = e + a1 * (u[2] * u[3] + v[2] * v[3] + w[2] * w[3]) -
        (a2 * (u[2] * u[4] + v[2] * v[4] + w[2] * w[4]) + a3 * (u[1] * u[3] + v[1] * v[3] + w[1] * w[3])) +
        (a4 * (u[2] * u[5] + v[2] * v[5] + w[2] * w[5]) + a5 * (u[1] * u[4] + v[1] * v[4] + w[1] * w[4]) +
         a6 * (u[0] * u[3] + v[0] * v[3] + w[0] * w[3]));
    F[4] = e + (T(0.75) * (un[2] * p[3] + un[3] * p[2]) -
                T(0.15) * (un[2] * p[4] + un[4] * p[2] + un[1] * p[3] + un[3] * p[1]) +
                (un[2] * p[5] + un[5] * p[2] + un[1] * p[4] + un[4] * p[1] + un[0] * p[3] + un[3] * p[0]) * c60);
  }
}

// ---- SLAU family: 3D_solver/src/calc_slau_3d.f90 -----------------------------
// MX: pd1, pd2 are pressure deviations from pr (see keep_flux)
template <class T, bool MX = false>
__device__ __forceinline__ void slau_flux(bool hr2, T r1, T r2, T u1, T u2, T v1, T v2, T w1, T w2,
                                          T un1, T un2, T pd1, T pd2, int nd, T HR, T gam, T g_g1,
                                          T F[5], T pr = T(0)) {
  const T n2 = nd == 0 ? T(1) : T(0), n3 = nd == 1 ? T(1) : T(0), n4 = nd == 2 ? T(1) : T(0);
  const T p1 = MX ? pd1 + pr : pd1, p2 = MX ? pd2 + pr : pd2;
  T or1 = T(1) / r1, or2 = T(1) / r2;
  // SLAU_common :1-36
  T cl = sqrt(gam * p1 * or1);
  T cr = sqrt(gam * p2 * or2);
  T c = T(0.5) * (cl + cr);
  T oc = T(1) / c;
  T Mp = un1 * oc, Mm = un2 * oc;
  T g = -fmax_f(fmin_f(Mp, T(0)), T(-1)) * fmin_f(fmax_f(Mm, T(0)), T(1));
  T gv = (T(1) - g) * (r1 * fabs(un1) + r2 * fabs(un2)) / (r1 + r2);
  T Vtp = gv + g * fabs(un1);
  T Vtm = gv + g * fabs(un2);
  T bp = (fabs(Mp) < T(1)) ? T(0.25) * (T(2) - Mp) * ((Mp + T(1)) * (Mp + T(1))) : T(0.5) * (T(1) + sgn1(Mp));
  T bm = (fabs(Mm) < T(1)) ? T(0.25) * (T(2) + Mm) * ((Mm - T(1)) * (Mm - T(1))) : T(0.5) * (T(1) + sgn1(-Mm));
  T dp = -pd1 + pd2;
  T k1 = T(0.5) * (u1 * u1 + v1 * v1 + w1 * w1);
  T k2 = T(0.5) * (u2 * u2 + v2 * v2 + w2 * w2);
  // bp + bm - 1 multiplies rho*c*|V| ~ 1/M: in the mixed form the subsonic branch
  // uses the identical factored polynomial 0.25 (Mp - Mm)(3 - Mp^2 - Mp Mm - Mm^2),
  // which has no cancellation in FP32
  T bsum1 = bp + bm - T(1);
  if constexpr (MX) {
    if (fabs(Mp) < T(1) && fabs(Mm) < T(1))
      bsum1 = T(0.25) * ((un1 - un2) * oc) * (T(3) - (Mp * Mp + Mp * Mm + Mm * Mm));
  }
  T mass, pres;
  if (!hr2) {  // SLAU1 :49-76
    T M = fmin_f(T(1), sqrt(k1 + k2) * oc);
    T x = (T(1) - M) * (T(1) - M);
    mass = T(0.25) * (r1 * (un1 + Vtp) + r2 * (un2 - Vtm) - x * dp * oc);
    pres = T(0.5) * (pd1 + pd2 + (bp - bm) * (-dp) + (T(1) - x) * bsum1 * (p1 + p2));
  } else {  // HRSLAU2 :79-104
    T V2 = sqrt(k1 + k2);
    T M = fmin_f(T(1), V2 * oc);
    T x = (T(1) - M) * (T(1) - M);
    mass = T(0.25) * (r1 * (un1 + Vtp) + r2 * (un2 - Vtm) - x * dp * oc);
    pres = T(0.5) * (pd1 + pd2 + (bp - bm) * (-dp) + HR * V2 * bsum1 * T(0.5) * (r1 + r2) * c);
  }
  T m1 = mass + fabs(mass), m2 = mass - fabs(mass);
  F[0] = m1 + m2;
  F[1] = m1 * u1 + m2 * u2 + pres * n2;
  F[2] = m1 * v1 + m2 * v2 + pres * n3;
  F[3] = m1 * w1 + m2 * w2 + pres * n4;
  // phi :39-46
  F[4] = m1 * ((p1 * g_g1 + r1 * k1) * or1) + m2 * ((p2 * g_g1 + r2 * k2) * or2);
}

// ---- Roe: 3D_solver/src/calc_roe_3d.f90 (normal velocity first) ---------------
// MX: pd1, pd2 are pressure deviations from pr; the central pressure term and the
// energy jump dQ5 use deviations, the enthalpies and the central energy flux full values
template <class T, bool MX = false>
__device__ __forceinline__ void roe_flux(T r1, T r2, T u1, T u2, T v1, T v2, T w1, T w2, T pd1, T pd2,
                                         T g1, T og1, T g_g1, T F[5], T pr = T(0)) {
  const T p1 = MX ? pd1 + pr : pd1, p2 = MX ? pd2 + pr : pd2;
  T k1 = T(0.5) * (u1 * u1 + v1 * v1 + w1 * w1);
  T k2 = T(0.5) * (u2 * u2 + v2 * v2 + w2 * w2);
  T e1 = p1 * og1 + r1 * k1;  // calc_Roe_common :53-77
  T e2 = p2 * og1 + r2 * k2;
  T ru1 = r1 * u1, ru2 = r2 * u2;
  T F1 = T(0.5) * (ru1 + ru2);
  T F2 = T(0.5) * (ru1 * u1 + ru2 * u2 + (pd1 + pd2));
  T F3 = T(0.5) * (ru1 * v1 + ru2 * v2);
  T F4 = T(0.5) * (ru1 * w1 + ru2 * w2);
  T F5 = T(0.5) * ((e1 + p1) * u1 + (e2 + p2) * u2);
  T q5;
  if constexpr (MX) q5 = -(pd1 * og1 + r1 * k1) + (pd2 * og1 + r2 * k2);
  else q5 = -e1 + e2;
  T q1 = -r1 + r2, q2 = -r1 * u1 + r2 * u2, q3 = -r1 * v1 + r2 * v2, q4 = -r1 * w1 + r2 * w2;
  T H1 = g_g1 * p1 / r1 + k1;  // calc_Roe_ave :37-50
  T H2 = g_g1 * p2 / r2 + k2;
  T sl = sqrt(r1), sr = sqrt(r2);
  T slr = T(1) / (sl + sr);
  T u = (sl * u1 + sr * u2) * slr, v = (sl * v1 + sr * v2) * slr, w = (sl * w1 + sr * w2) * slr;
  T H = (sl * H1 + sr * H2) * slr;
  T c = sqrt(g1 * (H - T(0.5) * (u * u + v * v + w * w)));
  T qq = T(0.5) * (u * u + v * v + w * w);  // calc_RARinv :1-34
  T oc = T(1) / c;
  T b2 = g1 * oc * oc;
  T b1 = qq * b2;
  T R1 = T(0.5) * ((b1 + u * oc) * q1 - (oc + b2 * u) * q2 - b2 * v * q3 - b2 * w * q4 + b2 * q5);
  T R2 = oc * (w * q1 - q4);
  T R3 = oc * (-v * q1 + q3);
  T R4 = (T(1) - b1) * q1 + b2 * (u * q2 + v * q3 + w * q4 - q5);
  T R5 = T(0.5) * ((b1 - u * oc) * q1 + (oc - b2 * u) * q2 - b2 * (v * q3 + w * q4 - q5));
  T l1 = fabs(u - c), l2 = fabs(u), l3 = fabs(u + c);
  T l2c = l2 * c, cu = c * u;
  F[0] = F1 - T(0.5) * (l1 * R1 + l2 * R4 + l3 * R5);
  F[1] = F2 - T(0.5) * (l1 * (u - c) * R1 + l2 * u * R4 + l3 * (u + c) * R5);
  F[2] = F3 - T(0.5) * (l1 * v * R1 + l2c * R3 + l2 * v * R4 + l3 * v * R5);
  F[3] = F4 - T(0.5) * (l1 * w * R1 - l2c * R2 + l2 * w * R4 + l3 * w * R5);
  F[4] = F5 - T(0.5) * (l1 * (H - cu) * R1 + l2 * (-w * c * R2 + v * c * R3 + qq * R4) + l3 * (H + cu) * R5);
}

// ---- viscous helpers ----------------------------------------------------------
// interp/diff of 3D_solver/src/calc_visc_cent.f90.fypp:2-21
template <int N, class T> __device__ __forceinline__ T v_interp(const T* a) {
  if constexpr (N == 4) return T(0.0625) * (-a[0] + T(9) * (a[1] + a[2]) - a[3]);
  else return T(0.00390625) * (T(3) * a[0] - T(25) * a[1] + T(150) * (a[2] + a[3]) - T(25) * a[4] + T(3) * a[5]);
}
template <int N, class T> __device__ __forceinline__ T v_diff(T d, const T* a) {
  if constexpr (N == 4) return (a[0] - T(27) * (a[1] - a[2]) - a[3]) * T(1.0 / 24.0) * d;
  else return (T(-0.0046875) * a[0] + T(0.065104167) * a[1] - T(1.171875) * (a[2] - a[3]) -
               T(0.065104167) * a[4] + T(0.0046875) * a[5]) * d;
}
// 3D_solver/src/calc_visc_me4_base.f90:4-8
template <class T> __device__ __forceinline__ T flux4(T a0, T a1, T a2) {
  return (-a0 + T(26) * a1 - a2) * T(1.0 / 24.0);
}
template <class T> __device__ __forceinline__ T i4(const T* a) {  // 4-point midpoint interpolation
  return T(0.0625) * (-a[0] + T(9) * (a[1] + a[2]) - a[3]);
}

}  // namespace oux
