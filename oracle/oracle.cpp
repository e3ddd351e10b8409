// CPU oracle for the OUxSBLI explicit time step -- TEST INFRASTRUCTURE ONLY.
//
// This file restates, in plain C++, the arithmetic of the reference's CUDA
// Fortran kernels for the periodic ("_in") hot path so that the GPU library can
// be checked against it.  It is never linked into, called by, or shipped with
// the product library; only tests/, __graft_entry__.smoke() and bench.py's
// cpu_baseline / --impl reference legs load it (as a checker / CPU baseline).
//
// Parity status: the reference is CUDA Fortran with no CPU build and cannot be
// compiled here (no Fortran compiler, no NVHPC).  This restatement is pinned by
// the reference's own known-answer tests (ETGV entropy/KE bounds, EVC
// convergence order, the ST shock tube against the exact Sod solution, the OS
// reflected oblique shock against the shock relations) re-run in tests/, not by
// golden vectors from the reference itself: "parity unpinned" against a run of
// the reference.
//
// Layout follows the reference exactly (Fortran column-major, 1-based indices
// in the accessors below): QJ(nx,nv,ny,nz) with nv = dim+2, x fastest, then the
// variable, then y, then z.  Ghost cells are stored (g = order/2 per side).
//
// Rounding conventions chosen where the Fortran source leaves them to the
// compiler:
//   * SIGN(1,x) follows copysign (a -0.0 argument gives -1).
//   * MIN(a,b) returns b only when b < a, else a.
//   * No FMA contraction (build with -ffp-contract=off); operations are
//     evaluated left to right as written in the Fortran expressions.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>

extern "C" {

// Config enums mirror ouxsbli_b200/csrc and include/oux.h.
enum { ORC_KEEP = 0, ORC_SLAU = 1, ORC_ROE = 2, ORC_HYBRID = 3 };
enum { ORC_EULER = 0, ORC_NS = 1, ORC_LES = 2 };
enum { ORC_CENTRAL = 0, ORC_ME4 = 1 };
enum { ORC_TVD_NONE = 0, ORC_TVD_TVD = 1, ORC_TVD_HYBRID = 2 };
enum { ORC_SLAU1 = 0, ORC_HRSLAU2 = 1 };

typedef struct orc_config {
  int dim;            // 2 or 3
  int nx, ny, nz;     // points incl. ghosts (nz = 1 for 2D)
  int order;          // 2, 4, 6 (convective)
  int scheme;         // ORC_KEEP ...
  int visc;           // ORC_EULER / ORC_NS / ORC_LES
  int visc_order;     // 2, 4, 6
  int visc_stencil;   // ORC_CENTRAL / ORC_ME4 (only with visc_order 6)
  int tvd;            // ORC_TVD_*
  int slau;           // ORC_SLAU1 / ORC_HRSLAU2
  int rk;             // 3 or 4
  int bc_x;           // 0 periodic; 1 non-periodic x (boundary flux kernels, one boundary cell a side)
  double gamma, R, Pr, Prt, threshold, dt;
  int bc_y;           // 0 periodic; 1 non-periodic y (2D, with bc_x = 1)
  int bkind[4];       // boundary-cell rule of the faces x lo, x hi, y lo, y hi:
                      // 0 zero gradient, 1 slip wall, 2 fixed values, 3 no-slip wall
  const double* bfix[4];  // fixed values of Q/J, nv x (ny for x faces, nx for y faces), variable-major
  int bc_z;           // 0 periodic; 1 non-periodic; z slab whose ghost planes at both ends (2), the
                      // upper end (3) or the lower end (4) are left to the halo exchange
  int ylast;          // 1: y faces applied after x faces (corners take their y rule)
  const signed char* bkinds[4];  // per-position rule of a face, or null
  double bpar[4][4];  // far-field state of a face: rho, tangential velocity, normal velocity, c
  int bkindz[2];      // 3D: rules of the faces z lo, z hi
  const double* bfix3[6];  // 3D: fixed values of the faces x lo .. z hi (pos j+ny k, i+nx k, i+nx j)
} orc_config;

}  // extern "C"

namespace {

struct Consts {
  double gamma, R, Pr, Prt, threshold, dt;
  double gamma_1, over_gamma_1, R_over_gamma_1, Cp, Cp_over_Pr, sutherland;
  double gamma_over_gamma_1, tan10deg2;
};

// src/mod_constant.f90.fypp:18-32
Consts make_consts(const orc_config& c) {
  Consts k;
  k.gamma = c.gamma; k.R = c.R; k.Pr = c.Pr; k.Prt = c.Prt;
  k.threshold = c.threshold; k.dt = c.dt;
  k.gamma_1 = c.gamma - 1.0;
  k.over_gamma_1 = 1.0 / (c.gamma - 1.0);
  k.R_over_gamma_1 = c.R / (c.gamma - 1.0);
  k.Cp = c.gamma * c.R / (c.gamma - 1.0);
  k.Cp_over_Pr = k.Cp / c.Pr;
  k.sutherland = 1.716e-5 * 384.2 * std::pow(273.2, -1.5);
  k.gamma_over_gamma_1 = c.gamma * k.over_gamma_1;
  double t = std::tan(10.0 * std::acos(-1.0) / 180.0);
  k.tan10deg2 = t * t;
  return k;
}

// ---- Fortran intrinsics with the conventions stated in the header ----------
inline double fsign1(double b) { return std::signbit(b) ? -1.0 : 1.0; }
inline double fmin2(double a, double b) { return (b < a) ? b : a; }
inline double fmax2(double a, double b) { return (b > a) ? b : a; }
inline double fmin3(double a, double b, double c) { return fmin2(fmin2(a, b), c); }

// ---- src/calc_muscl.f90 ---------------------------------------------------
// minmod2 :19-24, minmod3 :27-32
inline double minmod2(double x, double y) {
  double sgn = fsign1(x);
  return sgn * fmax2(fmin2(std::fabs(x), sgn * y), 0.0);
}
inline double minmod3(double x, double y, double z) {
  double sgn = fsign1(x);
  return sgn * fmax2(fmin3(std::fabs(x), sgn * y, sgn * z), 0.0);
}
// d33 :35-41
inline double d33(double d1, double d2, double d3) {
  return minmod3(d1, 2.0 * d2, 2.0 * d3) - 2.0 * minmod3(d2, 2.0 * d1, 2.0 * d3) +
         minmod3(d3, 2.0 * d1, 2.0 * d2);
}
const double one_third = 1.0 / 3.0, two_third = 2.0 / 3.0, one_sixth = 1.0 / 6.0,
             one_twelfth = 1.0 / 12.0, one_sixty = 1.0 / 60.0;
// MUSCL3rdnonTVD :44-51, MUSCL3rdMinmod :54-73, MUSCL3rdThreshold :76-88
void muscl3(int tvd, double thr, double sensor, double a2, double a3, double d1, double d2,
            double d3, double& al, double& ar) {
  bool nontvd = (tvd == ORC_TVD_NONE) || (tvd == ORC_TVD_HYBRID && sensor < thr);
  if (nontvd) {
    al = a2 + 0.5 * (d1 + 2.0 * d2) * one_third;
    ar = a3 - 0.5 * (d3 + 2.0 * d2) * one_third;
  } else {
    const double b = (3.0 - one_third) / (1.0 - one_third);
    double dt1 = minmod2(d1, b * d2);
    double dt2 = minmod2(d2, b * d1);
    al = a2 + 0.5 * (dt1 + 2.0 * dt2) * one_third;
    double dt3 = minmod2(d3, b * d2);
    double dt4 = minmod2(d2, b * d3);
    ar = a3 - 0.5 * (dt3 + 2.0 * dt4) * one_third;
  }
}
// MUSCL4thnonTVD :91-98, MUSCL4thTVD :101-122, MUSCL4thThreshold :125-139
void muscl4(int tvd, double thr, double sensor, double a2, double a3, double d1, double d2,
            double d3, double d4, double d5, double& al, double& ar) {
  bool nontvd = (tvd == ORC_TVD_NONE) || (tvd == ORC_TVD_HYBRID && sensor < thr);
  if (nontvd) {
    al = a2 + (-0.4 * d1 + 2.2 * d2 + 4.8 * d3 - 0.6 * d4) * one_twelfth;
    ar = a3 - (-0.6 * d2 + 4.8 * d3 + 2.2 * d4 - 0.4 * d5) * one_twelfth;
  } else {
    double delta2 = d3 - d33(d2, d3, d4) * one_sixth;
    {
      double delta1 = d2 - d33(d1, d2, d3) * one_sixth;
      double dl = minmod2(delta1, 4.0 * delta2);
      double dr = minmod2(delta2, 4.0 * delta1);
      al = a2 + (dl + 2.0 * dr) * one_sixth;
    }
    {
      double delta3 = d4 - d33(d3, d4, d5) * one_sixth;
      double dl = minmod2(delta2, 4.0 * delta3);
      double dr = minmod2(delta3, 4.0 * delta2);
      ar = a3 - (dr + 2.0 * dl) * one_sixth;
    }
  }
}
// delta4 :142-153 (4 points a[0..3]), delta6 :156-169 (6 points a[0..5])
void delta4(int tvd, double thr, double sensor, const double* a, double& al, double& ar) {
  double d1 = -a[0] + a[1], d2 = -a[1] + a[2], d3 = -a[2] + a[3];
  muscl3(tvd, thr, sensor, a[1], a[2], d1, d2, d3, al, ar);
}
void delta6(int tvd, double thr, double sensor, const double* a, double& al, double& ar) {
  double d1 = -a[0] + a[1], d2 = -a[1] + a[2], d3 = -a[2] + a[3], d4 = -a[3] + a[4],
         d5 = -a[4] + a[5];
  muscl4(tvd, thr, sensor, a[2], a[3], d1, d2, d3, d4, d5, al, ar);
}
// 3D_solver/src/calc_hybrid.f90:75-81
double wiggle(const double* p4) {
  double phi1 = (-p4[0] + p4[1]) * (-p4[1] + p4[2]);
  double phi2 = (-p4[2] + p4[3]) * (-p4[1] + p4[2]);
  return 0.5 * (1.0 - fsign1(fmin2(phi1, phi2)));
}

// ---- 3D_solver/src/calc_keep_3d.f90 (w = 0 reproduces the 2D twin) ---------
void keep_flux(int order, const double* rho, const double* u, const double* v, const double* w,
               const double* uu, const double* p, const double* T, int nd, const Consts& K,
               double F[5]) {
  const double one_24 = 1.0 / 24.0, one_48 = 1.0 / 48.0, one_60 = 1.0 / 60.0,
               one_120 = 1.0 / 120.0, one_240 = 1.0 / 240.0, seven_twelfth = 7.0 / 12.0;
  double N2 = nd == 0 ? 1.0 : 0.0, N3 = nd == 1 ? 1.0 : 0.0, N4 = nd == 2 ? 1.0 : 0.0;
  if (order == 2) {  // KEEP2 :1-15
    F[0] = 0.25 * (rho[0] + rho[1]) * (uu[0] + uu[1]);
    F[1] = 0.5 * (F[0] * (u[0] + u[1]) + (p[0] + p[1]) * N2);
    F[2] = 0.5 * (F[0] * (v[0] + v[1]) + (p[0] + p[1]) * N3);
    F[3] = 0.5 * (F[0] * (w[0] + w[1]) + (p[0] + p[1]) * N4);
    F[4] = F[0] * 0.5 * (T[0] + T[1]) * K.R_over_gamma_1;
    F[4] = F[4] + 0.5 * (uu[0] * p[1] + uu[1] * p[0]);
    F[4] = F[4] + 0.5 * F[0] * (u[0] * u[1] + v[0] * v[1] + w[0] * w[1]);
  } else if (order == 4) {  // KEEP4 :18-56
    double RV1 = (rho[1] + rho[2]) * (uu[1] + uu[2]);
    double RV2 = (rho[1] + rho[3]) * (uu[1] + uu[3]);
    double RV3 = (rho[0] + rho[2]) * (uu[0] + uu[2]);
    F[0] = one_third * RV1 - (RV2 + RV3) * one_24;
    RV1 = one_sixth * RV1;
    RV2 = one_48 * RV2;
    RV3 = one_48 * RV3;
    double RV1_RV2 = RV1 - RV2, RV1_RV3 = RV1 - RV3;
    double u1 = u[0], u2 = u[1], u3 = u[2], u4 = u[3];
    double v1 = v[0], v2 = v[1], v3 = v[2], v4 = v[3];
    double w1 = w[0], w2 = w[1], w3 = w[2], w4 = w[3];
    double pres = -one_twelfth * p[0] + seven_twelfth * (p[1] + p[2]) - one_twelfth * p[3];
    F[1] = -RV3 * u1 + RV1_RV2 * u2 + RV1_RV3 * u3 - RV2 * u4 + pres * N2;
    F[2] = -RV3 * v1 + RV1_RV2 * v2 + RV1_RV3 * v3 - RV2 * v4 + pres * N3;
    F[3] = -RV3 * w1 + RV1_RV2 * w2 + RV1_RV3 * w3 - RV2 * w4 + pres * N4;
    double ene = (-RV3 * T[0] + RV1_RV2 * T[1] + RV1_RV3 * T[2] - RV2 * T[3]) * K.R_over_gamma_1;
    ene = ene + ((RV1 * (u2 * u3 + v2 * v3 + w2 * w3)) -
                 (RV2 * (u2 * u4 + v2 * v4 + w2 * w4) + RV3 * (u1 * u3 + v1 * v3 + w1 * w3)));
    F[4] = ene + (two_third * (uu[1] * p[2] + uu[2] * p[1]) -
                  one_twelfth * (uu[1] * p[3] + uu[3] * p[1] + uu[0] * p[2] + uu[2] * p[0]));
  } else {  // KEEP6 :59-111
    double RV1 = (rho[2] + rho[3]) * (uu[2] + uu[3]);
    double RV2 = (rho[2] + rho[4]) * (uu[2] + uu[4]);
    double RV3 = (rho[1] + rho[3]) * (uu[1] + uu[3]);
    double RV4 = (rho[2] + rho[5]) * (uu[2] + uu[5]);
    double RV5 = (rho[1] + rho[4]) * (uu[1] + uu[4]);
    double RV6 = (rho[0] + rho[3]) * (uu[0] + uu[3]);
    F[0] = 0.375 * RV1 - 0.075 * (RV2 + RV3) + (RV4 + RV5 + RV6) * one_120;
    RV1 = 0.1875 * RV1;
    RV2 = 0.0375 * RV2;
    RV3 = 0.0375 * RV3;
    RV4 = RV4 * one_240;
    RV5 = RV5 * one_240;
    RV6 = RV6 * one_240;
    double RV3_RV5 = -RV3 + RV5;
    double RV1_RV2_RV4 = RV1 - RV2 + RV4;
    double RV1_RV3_RV6 = RV1 - RV3 + RV6;
    double RV2_RV5 = -RV2 + RV5;
    double pres = (p[0] - 8.0 * p[1] + 37.0 * (p[2] + p[3]) - 8.0 * p[4] + p[5]) * one_60;
    double ruu = RV6 * u[0] + RV3_RV5 * u[1] + RV1_RV2_RV4 * u[2] + RV1_RV3_RV6 * u[3] +
                 RV2_RV5 * u[4] + RV4 * u[5];
    ruu = ruu + pres * N2;
    double ruv = RV6 * v[0] + RV3_RV5 * v[1] + RV1_RV2_RV4 * v[2] + RV1_RV3_RV6 * v[3] +
                 RV2_RV5 * v[4] + RV4 * v[5];
    ruv = ruv + pres * N3;
    double ruw = RV6 * w[0] + RV3_RV5 * w[1] + RV1_RV2_RV4 * w[2] + RV1_RV3_RV6 * w[3] +
                 RV2_RV5 * w[4] + RV4 * w[5];
    ruw = ruw + pres * N4;
    F[1] = ruu; F[2] = ruv; F[3] = ruw;
    double ene = (RV6 * T[0] + RV3_RV5 * T[1] + RV1_RV2_RV4 * T[2] + RV1_RV3_RV6 * T[3] +
                  RV2_RV5 * T[4] + RV4 * T[5]) * K.R_over_gamma_1;
    ene = ene + RV1 * (u[2] * u[3] + v[2] * v[3] + w[2] * w[3]) -
          (RV2 * (u[2] * u[4] + v[2] * v[4] + w[2] * w[4]) +
           RV3 * (u[1] * u[3] + v[1] * v[3] + w[1] * w[3])) +
          (RV4 * (u[2] * u[5] + v[2] * v[5] + w[2] * w[5]) +
           RV5 * (u[1] * u[4] + v[1] * v[4] + w[1] * w[4]) +
           RV6 * (u[0] * u[3] + v[0] * v[3] + w[0] * w[3]));
    F[4] = ene + (0.75 * (uu[2] * p[3] + uu[3] * p[2]) -
                  0.15 * (uu[2] * p[4] + uu[4] * p[2] + uu[1] * p[3] + uu[3] * p[1]) +
                  (uu[2] * p[5] + uu[5] * p[2] + uu[1] * p[4] + uu[4] * p[1] + uu[0] * p[3] +
                   uu[3] * p[0]) * one_60);
  }
}

// ---- 3D_solver/src/calc_slau_3d.f90 -----------------------------------------
double phi_slau(double rho, double k, double p, double over_rho, const Consts& K) {
  return (p * K.gamma_over_gamma_1 + rho * k) * over_rho;  // :39-46
}
// SLAU_common :1-36, SLAU1 :49-76, HRSLAU2 :79-104.  nd selects Normal_x/y/z.
void slau_flux(int variant, double rho1, double rho2, double u1, double u2, double v1, double v2,
               double w1, double w2, double un1, double un2, double p1, double p2, int nd,
               double HR, const Consts& K, double F[5]) {
  double N2 = nd == 0 ? 1.0 : 0.0, N3 = nd == 1 ? 1.0 : 0.0, N4 = nd == 2 ? 1.0 : 0.0;
  double over_rho1 = 1.0 / rho1, over_rho2 = 1.0 / rho2;
  double cl = std::sqrt(K.gamma * p1 * over_rho1);
  double cr = std::sqrt(K.gamma * p2 * over_rho2);
  double c = 0.5 * (cl + cr);
  double over_c = 1.0 / c;
  double Mp = un1 * over_c, Mm = un2 * over_c;
  double g = -fmax2(fmin2(Mp, 0.0), -1.0) * fmin2(fmax2(Mm, 0.0), 1.0);
  double one_g_Vt = (1.0 - g) * (rho1 * std::fabs(un1) + rho2 * std::fabs(un2)) / (rho1 + rho2);
  double Vtp = one_g_Vt + g * std::fabs(un1);
  double Vtm = one_g_Vt + g * std::fabs(un2);
  double bp = (std::fabs(Mp) < 1.0) ? 0.25 * (2.0 - Mp) * ((Mp + 1.0) * (Mp + 1.0))
                                    : 0.5 * (1.0 + fsign1(Mp));
  double bm = (std::fabs(Mm) < 1.0) ? 0.25 * (2.0 + Mm) * ((Mm - 1.0) * (Mm - 1.0))
                                    : 0.5 * (1.0 + fsign1(-Mm));
  double dp = -p1 + p2;
  double k1 = 0.5 * (u1 * u1 + v1 * v1 + w1 * w1);
  double k2 = 0.5 * (u2 * u2 + v2 * v2 + w2 * w2);
  double mass, pres;
  if (variant == ORC_SLAU1) {
    double M = fmin2(1.0, std::sqrt(k1 + k2) * over_c);
    double x = (1.0 - M) * (1.0 - M);
    mass = 0.25 * (rho1 * (un1 + Vtp) + rho2 * (un2 - Vtm) - x * dp * over_c);
    pres = 0.5 * (p1 + p2 + (bp - bm) * (-dp) + (1.0 - x) * (bp + bm - 1.0) * (p1 + p2));
  } else {
    double Vec2 = std::sqrt(k1 + k2);
    double M = fmin2(1.0, Vec2 * over_c);
    double x = (1.0 - M) * (1.0 - M);
    mass = 0.25 * (rho1 * (un1 + Vtp) + rho2 * (un2 - Vtm) - x * dp * over_c);
    pres = 0.5 * (p1 + p2 + (bp - bm) * (-dp) + HR * Vec2 * (bp + bm - 1.0) * 0.5 * (rho1 + rho2) * c);
  }
  double mass1 = mass + std::fabs(mass), mass2 = mass - std::fabs(mass);
  F[0] = mass1 + mass2;
  F[1] = mass1 * u1 + mass2 * u2 + pres * N2;
  F[2] = mass1 * v1 + mass2 * v2 + pres * N3;
  F[3] = mass1 * w1 + mass2 * w2 + pres * N4;
  F[4] = mass1 * phi_slau(rho1, k1, p1, over_rho1, K) + mass2 * phi_slau(rho2, k2, p2, over_rho2, K);
}

// ---- 3D_solver/src/calc_roe_3d.f90 (rotated variables, returns F in (n,t1,t2)) ----
void roe_flux(double rho1, double rho2, double u1, double u2, double v1, double v2, double w1,
              double w2, double p1, double p2, const Consts& K, double F[5]) {
  double k1 = 0.5 * (u1 * u1 + v1 * v1 + w1 * w1);
  double k2 = 0.5 * (u2 * u2 + v2 * v2 + w2 * w2);
  // calc_Roe_common :53-77
  double e1 = p1 * K.over_gamma_1 + rho1 * k1;
  double e2 = p2 * K.over_gamma_1 + rho2 * k2;
  double rhou1 = rho1 * u1, rhou2 = rho2 * u2;
  double F1 = 0.5 * (rhou1 + rhou2);
  double F2 = 0.5 * (rhou1 * u1 + rhou2 * u2 + (p1 + p2));
  double F3 = 0.5 * (rhou1 * v1 + rhou2 * v2);
  double F4 = 0.5 * (rhou1 * w1 + rhou2 * w2);
  double F5 = 0.5 * ((e1 + p1) * u1 + (e2 + p2) * u2);
  double dQ1 = -rho1 + rho2, dQ2 = -rho1 * u1 + rho2 * u2, dQ3 = -rho1 * v1 + rho2 * v2,
         dQ4 = -rho1 * w1 + rho2 * w2, dQ5 = -e1 + e2;
  // calc_Roe_ave :37-50
  double H1 = K.gamma_over_gamma_1 * p1 / rho1 + k1;
  double H2 = K.gamma_over_gamma_1 * p2 / rho2 + k2;
  double rl = std::sqrt(rho1), rr = std::sqrt(rho2);
  double rlr = 1.0 / (rl + rr);
  double u = (rl * u1 + rr * u2) * rlr;
  double v = (rl * v1 + rr * v2) * rlr;
  double w = (rl * w1 + rr * w2) * rlr;
  double H = (rl * H1 + rr * H2) * rlr;
  double c = std::sqrt(K.gamma_1 * (H - 0.5 * (u * u + v * v + w * w)));
  // calc_RARinv :1-34
  double q2 = 0.5 * (u * u + v * v + w * w);
  double oc = 1.0 / c;
  double b2 = K.gamma_1 * oc * oc;
  double b1 = q2 * b2;
  double R1 = 0.5 * ((b1 + u * oc) * dQ1 - (oc + b2 * u) * dQ2 - b2 * v * dQ3 - b2 * w * dQ4 + b2 * dQ5);
  double R2 = oc * (w * dQ1 - dQ4);
  double R3 = oc * (-v * dQ1 + dQ3);
  double R4 = (1.0 - b1) * dQ1 + b2 * (u * dQ2 + v * dQ3 + w * dQ4 - dQ5);
  double R5 = 0.5 * ((b1 - u * oc) * dQ1 + (oc - b2 * u) * dQ2 - b2 * (v * dQ3 + w * dQ4 - dQ5));
  double a1 = std::fabs(u - c), a2 = std::fabs(u), a3 = std::fabs(u + c);
  double a2c = a2 * c, cu = c * u;
  F1 = F1 - 0.5 * (a1 * R1 + a2 * R4 + a3 * R5);
  F2 = F2 - 0.5 * (a1 * (u - c) * R1 + a2 * u * R4 + a3 * (u + c) * R5);
  F3 = F3 - 0.5 * (a1 * v * R1 + a2c * R3 + a2 * v * R4 + a3 * v * R5);
  F4 = F4 - 0.5 * (a1 * w * R1 - a2c * R2 + a2 * w * R4 + a3 * w * R5);
  F5 = F5 - 0.5 * (a1 * (H - cu) * R1 + a2 * (-w * c * R2 + v * c * R3 + q2 * R4) + a3 * (H + cu) * R5);
  F[0] = F1; F[1] = F2; F[2] = F3; F[3] = F4; F[4] = F5;
}

// ---- Solver state in the reference layout -----------------------------------
struct Grid {
  int dim, nx, ny, nz, nv;
  std::vector<double> xix, etay, zetaz;   // 1/dx (n-1)
  std::vector<double> jac;                // (nx,ny)
  std::vector<double> dtdxdy, dtdydz, dtdzdx;  // 3D metrics
  std::vector<double> dtdx, dtdy;              // 2D metrics
};

struct Work {
  std::vector<double> Q, T, mu, mut, qc2, sensor, E, F, G;
};

struct Ctx {
  orc_config c;
  Consts K;
  Grid g;
  Work w;
  int nx, ny, nz, nv;
  // accessors (1-based)
  inline size_t qidx(int i, int l, int j, int k) const {
    return (((size_t)(k - 1) * ny + (j - 1)) * nv + (l - 1)) * nx + (i - 1);
  }
  inline size_t sidx(int i, int j, int k) const {
    return ((size_t)(k - 1) * ny + (j - 1)) * nx + (i - 1);
  }
  // E(5,nx-1,ny-2,nz-2) etc.; for 2D, nz-2 -> 1 and G unused
  inline size_t eidx(int l, int i, int j, int k) const {
    int kk = (nz >= 3) ? (nz - 2) : 1;
    (void)kk;
    return (((size_t)(k - 1) * (ny - 2) + (j - 1)) * (nx - 1) + (i - 1)) * 5 + (l - 1);
  }
  inline size_t fidx(int l, int i, int j, int k) const {
    return (((size_t)(k - 1) * (ny - 1) + (j - 1)) * (nx - 2) + (i - 1)) * 5 + (l - 1);
  }
  inline size_t gidx(int l, int i, int j, int k) const {
    return (((size_t)(k - 1) * (ny - 2) + (j - 1)) * (nx - 2) + (i - 1)) * 5 + (l - 1);
  }
};

// ---- src/set_coordinate.f90 set_Jacobian_xy3 :99-117 / xy2 :80-96 ; preprocess metrics ----
void setup_grid(Ctx& C, const double* dx, const double* dy, const double* dz) {
  Grid& g = C.g;
  int nx = C.nx, ny = C.ny, nz = C.nz;
  g.xix.resize(nx - 1); g.etay.resize(ny - 1);
  for (int i = 0; i < nx - 1; ++i) g.xix[i] = 1.0 / dx[i];
  for (int j = 0; j < ny - 1; ++j) g.etay[j] = 1.0 / dy[j];
  g.jac.assign((size_t)nx * ny, 0.0);
  auto J = [&](int i, int j) -> double& { return g.jac[(size_t)(j - 1) * nx + (i - 1)]; };
  if (C.c.dim == 3) {
    g.zetaz.resize(nz - 1);
    for (int k = 0; k < nz - 1; ++k) g.zetaz[k] = 1.0 / dz[k];
    for (int j = 2; j <= ny - 1; ++j)
      for (int i = 2; i <= nx - 1; ++i)
        J(i, j) = 8.0 / ((dx[i - 2] + dx[i - 1]) * (dy[j - 2] + dy[j - 1]) * 2.0 * dz[0]);
  } else {
    for (int j = 2; j <= ny - 1; ++j)
      for (int i = 2; i <= nx - 1; ++i)
        J(i, j) = 4.0 / ((dx[i - 2] + dx[i - 1]) * (dy[j - 2] + dy[j - 1]));
  }
  for (int i = 1; i <= nx; ++i) { J(i, 1) = J(i, 2); J(i, ny) = J(i, ny - 1); }
  for (int j = 1; j <= ny; ++j) { J(1, j) = J(2, j); J(nx, j) = J(nx - 1, j); }
  double dt = C.c.dt;
  if (C.c.dim == 3) {  // 3D_solver/src/preprocess.f90.fypp:76-87
    g.dtdxdy.resize((size_t)(nx - 2) * (ny - 2));
    g.dtdydz.resize((size_t)(ny - 2) * (nz - 2));
    g.dtdzdx.resize((size_t)(nx - 2) * (nz - 2));
    for (int j = 1; j <= ny - 2; ++j)
      for (int i = 1; i <= nx - 2; ++i)
        g.dtdxdy[(size_t)(j - 1) * (nx - 2) + (i - 1)] =
            0.25 * dt * (dx[i - 1] + dx[i]) * (dy[j - 1] + dy[j]);
    for (int k = 1; k <= nz - 2; ++k)
      for (int j = 1; j <= ny - 2; ++j)
        g.dtdydz[(size_t)(k - 1) * (ny - 2) + (j - 1)] =
            0.25 * dt * (dy[j - 1] + dy[j]) * (dz[k - 1] + dz[k]);
    for (int k = 1; k <= nz - 2; ++k)
      for (int i = 1; i <= nx - 2; ++i)
        g.dtdzdx[(size_t)(k - 1) * (nx - 2) + (i - 1)] =
            0.25 * dt * (dz[k - 1] + dz[k]) * (dx[i - 1] + dx[i]);
  } else {  // 2D_solver/src/preprocess.f90.fypp:96-101
    g.dtdx.resize(nx - 2); g.dtdy.resize(ny - 2);
    for (int i = 1; i <= nx - 2; ++i) g.dtdx[i - 1] = 0.5 * dt * (dx[i - 1] + dx[i]);
    for (int j = 1; j <= ny - 2; ++j) g.dtdy[j - 1] = 0.5 * dt * (dy[j - 1] + dy[j]);
  }
}

// ---- src/calc_physical_quantities.f90:7-116 -----------------------------------
void quantities(Ctx& C, const double* QJ) {
  int nx = C.nx, ny = C.ny, nz = C.nz;
  const Consts& K = C.K;
  bool visc = C.c.visc != ORC_EULER;
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) {
        double Jv = C.g.jac[(size_t)(j - 1) * nx + (i - 1)];
        double over_Q1 = 1.0 / QJ[C.qidx(i, 1, j, k)];
        double rho = Jv * QJ[C.qidx(i, 1, j, k)];
        double u = QJ[C.qidx(i, 2, j, k)] * over_Q1;
        double v = QJ[C.qidx(i, 3, j, k)] * over_Q1;
        double p, w = 0.0;
        if (C.c.dim == 3) {
          w = QJ[C.qidx(i, 4, j, k)] * over_Q1;
          p = K.gamma_1 * (Jv * QJ[C.qidx(i, 5, j, k)] - 0.5 * rho * (u * u + v * v + w * w));
        } else {
          p = K.gamma_1 * (Jv * QJ[C.qidx(i, 4, j, k)] - 0.5 * rho * (u * u + v * v));
        }
        C.w.Q[C.qidx(i, 1, j, k)] = rho;
        C.w.Q[C.qidx(i, 2, j, k)] = u;
        C.w.Q[C.qidx(i, 3, j, k)] = v;
        if (C.c.dim == 3) {
          C.w.Q[C.qidx(i, 4, j, k)] = w;
          C.w.Q[C.qidx(i, 5, j, k)] = p;
        } else {
          C.w.Q[C.qidx(i, 4, j, k)] = p;
        }
        double temp = p / (K.R * rho);
        C.w.T[C.sidx(i, j, k)] = temp;
        if (visc) C.w.mu[C.sidx(i, j, k)] = K.sutherland / (temp + 111.0) * (temp * std::sqrt(temp));
      }
}

// primitive accessors: rho,u,v,w,p (w=0 and p at index 4 in 2D)
struct Prim {
  const Ctx& C;
  double rho(int i, int j, int k) const { return C.w.Q[C.qidx(i, 1, j, k)]; }
  double u(int i, int j, int k) const { return C.w.Q[C.qidx(i, 2, j, k)]; }
  double v(int i, int j, int k) const { return C.w.Q[C.qidx(i, 3, j, k)]; }
  double w(int i, int j, int k) const { return C.c.dim == 3 ? C.w.Q[C.qidx(i, 4, j, k)] : 0.0; }
  double p(int i, int j, int k) const { return C.w.Q[C.qidx(i, C.nv, j, k)]; }
  double T(int i, int j, int k) const { return C.w.T[C.sidx(i, j, k)]; }
  double mu(int i, int j, int k) const { return C.w.mu[C.sidx(i, j, k)]; }
  double mut(int i, int j, int k) const { return C.w.mut[C.sidx(i, j, k)]; }
  double qc2(int i, int j, int k) const { return C.w.qc2[C.sidx(i, j, k)]; }
  double vel(int comp, int i, int j, int k) const {
    return comp == 0 ? u(i, j, k) : comp == 1 ? v(i, j, k) : w(i, j, k);
  }
};

// ---- 3D_solver/src/calc_hybrid.f90:11-72 ; 2D_solver/src/calc_hybrid.f90:11-55 ----
void ducros(Ctx& C) {
  int nx = C.nx, ny = C.ny, nz = C.nz;
  Prim P{C};
  std::vector<double>& fd = C.w.sensor;
  const double eps = 1.0e-12;
  if (C.c.dim == 3) {
#pragma omp parallel for schedule(static)
    for (int k = 2; k <= nz - 1; ++k)
      for (int j = 2; j <= ny - 1; ++j)
        for (int i = 2; i <= nx - 1; ++i) {
          double dx_tmp = 0.25 * (C.g.xix[i - 2] + C.g.xix[i - 1]);
          double dy_tmp = 0.25 * (C.g.etay[j - 2] + C.g.etay[j - 1]);
          double dz_tmp = 0.25 * (C.g.zetaz[k - 2] + C.g.zetaz[k - 1]);
          double dudx = (-P.u(i - 1, j, k) + P.u(i + 1, j, k)) * dx_tmp;
          double dvdx = (-P.v(i - 1, j, k) + P.v(i + 1, j, k)) * dx_tmp;
          double dwdx = (-P.w(i - 1, j, k) + P.w(i + 1, j, k)) * dx_tmp;
          double dudy = (-P.u(i, j - 1, k) + P.u(i, j + 1, k)) * dy_tmp;
          double dvdy = (-P.v(i, j - 1, k) + P.v(i, j + 1, k)) * dy_tmp;
          double dwdy = (-P.w(i, j - 1, k) + P.w(i, j + 1, k)) * dy_tmp;
          double dudz = (-P.u(i, j, k - 1) + P.u(i, j, k + 1)) * dz_tmp;
          double dvdz = (-P.v(i, j, k - 1) + P.v(i, j, k + 1)) * dz_tmp;
          double dwdz = (-P.w(i, j, k - 1) + P.w(i, j, k + 1)) * dz_tmp;
          double div = dudx + dvdy + dwdz;
          double r1 = dwdy - dvdz, r2 = dudz - dwdx, r3 = dvdx - dudy;
          double f = (div * div) / (div * div + (r1 * r1 + r2 * r2 + r3 * r3) + eps);
          fd[C.sidx(i, j, k)] = fmin2(1.0, f);
        }
    // boundary copies (same cell-by-cell assignments as the kernel's tail)
    for (int k = 2; k <= nz - 1; ++k)
      for (int j = 2; j <= ny - 1; ++j)
        for (int i = 2; i <= nx - 1; ++i) {
          double f = fd[C.sidx(i, j, k)];
          if (i == 2) fd[C.sidx(1, j, k)] = f; else if (i == nx - 1) fd[C.sidx(nx, j, k)] = f;
          if (j == 2) fd[C.sidx(i, 1, k)] = f; else if (j == ny - 1) fd[C.sidx(i, ny, k)] = f;
          if (k == 2) fd[C.sidx(i, j, 1)] = f; else if (k == nz - 1) fd[C.sidx(i, j, nz)] = f;
        }
  } else {
    for (int j = 2; j <= ny - 1; ++j)
      for (int i = 2; i <= nx - 1; ++i) {
        double dx_tmp = 0.25 * (C.g.xix[i - 2] + C.g.xix[i - 1]);
        double dy_tmp = 0.25 * (C.g.etay[j - 2] + C.g.etay[j - 1]);
        double dudx = (-P.u(i - 1, j, 1) + P.u(i + 1, j, 1)) * dx_tmp;
        double dvdx = (-P.v(i - 1, j, 1) + P.v(i + 1, j, 1)) * dx_tmp;
        double dudy = (-P.u(i, j - 1, 1) + P.u(i, j + 1, 1)) * dy_tmp;
        double dvdy = (-P.v(i, j - 1, 1) + P.v(i, j + 1, 1)) * dy_tmp;
        double div = dudx + dvdy;
        double rot = dvdx - dudy;
        double f = (div * div) / (div * div + rot * rot + eps);
        fd[C.sidx(i, j, 1)] = fmin2(1.0, f);
      }
    for (int j = 2; j <= ny - 1; ++j)
      for (int i = 2; i <= nx - 1; ++i) {
        double f = fd[C.sidx(i, j, 1)];
        if (i == 2) fd[C.sidx(1, j, 1)] = f; else if (i == nx - 1) fd[C.sidx(nx, j, 1)] = f;
        if (j == 2) fd[C.sidx(i, 1, 1)] = f; else if (j == ny - 1) fd[C.sidx(i, ny, 1)] = f;
      }
  }
}

// ---- convective face flux (calc_{keep,slau,hybrid,roe}_kernel_internal) ----------
// dir: 0 x, 1 y, 2 z.  Face between cells c and c+1 along dir; (i,j,k) is cell c.
// ord: the stencil order of this face -- the configured order for the interior
// kernels; lower next to a non-periodic boundary (2D_solver/src/calc_slau_kernel,
// calc_keep_kernel, calc_hybrid_kernel .f90.fypp: 6 -> 4 -> 2 / first order).
void conv_face(const Ctx& C, int dir, int i, int j, int k, double F[5], int ord) {
  Prim P{C};
  const Consts& K = C.K;
  int io = ord / 2 - 1;
  int n = 2 * io + 2;
  double rho[6], u[6], v[6], w[6], p[6], T[6];
  for (int m = 0; m < n; ++m) {
    int off = m - io;
    int ii = i + (dir == 0 ? off : 0), jj = j + (dir == 1 ? off : 0), kk = k + (dir == 2 ? off : 0);
    rho[m] = P.rho(ii, jj, kk); u[m] = P.u(ii, jj, kk); v[m] = P.v(ii, jj, kk);
    w[m] = P.w(ii, jj, kk); p[m] = P.p(ii, jj, kk); T[m] = P.T(ii, jj, kk);
  }
  const double* un = dir == 0 ? u : dir == 1 ? v : w;
  int scheme = C.c.scheme;
  if (scheme == ORC_KEEP) { keep_flux(ord, rho, u, v, w, un, p, T, dir, K, F); return; }
  double s0 = C.w.sensor[C.sidx(i, j, k)];
  double s1 = C.w.sensor[C.sidx(i + (dir == 0), j + (dir == 1), k + (dir == 2))];
  double fd = 0.5 * (s0 + s1);
  if (scheme == ORC_HYBRID && fd <= K.threshold) {
    keep_flux(ord, rho, u, v, w, un, p, T, dir, K, F);
    return;
  }
  double L[5], Rr[5];
  double* arr[5] = {rho, u, v, w, p};
  for (int q = 0; q < 5; ++q) {
    if (ord == 2) { L[q] = arr[q][0]; Rr[q] = arr[q][1]; }
    else if (ord == 4) delta4(C.c.tvd, K.threshold, fd, arr[q], L[q], Rr[q]);
    else delta6(C.c.tvd, K.threshold, fd, arr[q], L[q], Rr[q]);
  }
  if (scheme == ORC_SLAU) {
    double HR;
    if (ord == 2) HR = 1.0;
    else HR = wiggle(p + (ord == 6 ? 1 : 0));  // p(2:5) for 6th, p(1:4) for 4th
    double un1 = dir == 0 ? L[1] : dir == 1 ? L[2] : L[3];
    double un2 = dir == 0 ? Rr[1] : dir == 1 ? Rr[2] : Rr[3];
    slau_flux(C.c.slau, L[0], Rr[0], L[1], Rr[1], L[2], Rr[2], L[3], Rr[3], un1, un2, L[4], Rr[4],
              dir, HR, K, F);
  } else if (scheme == ORC_HYBRID) {
    double un1 = dir == 0 ? L[1] : dir == 1 ? L[2] : L[3];
    double un2 = dir == 0 ? Rr[1] : dir == 1 ? Rr[2] : Rr[3];
    slau_flux(C.c.slau, L[0], Rr[0], L[1], Rr[1], L[2], Rr[2], L[3], Rr[3], un1, un2, L[4], Rr[4],
              dir, 1.0, K, F);
  } else {  // Roe: rotate (u,v,w) so the normal comes first, rotate the result back
    double Fr[5];
    if (dir == 0) {
      roe_flux(L[0], Rr[0], L[1], Rr[1], L[2], Rr[2], L[3], Rr[3], L[4], Rr[4], K, Fr);
      F[0] = Fr[0]; F[1] = Fr[1]; F[2] = Fr[2]; F[3] = Fr[3]; F[4] = Fr[4];
    } else if (dir == 1) {  // calc_roe_y_in: (v,w,u) -> F(1),F(3),F(4),F(2),F(5)
      roe_flux(L[0], Rr[0], L[2], Rr[2], L[3], Rr[3], L[1], Rr[1], L[4], Rr[4], K, Fr);
      F[0] = Fr[0]; F[2] = Fr[1]; F[3] = Fr[2]; F[1] = Fr[3]; F[4] = Fr[4];
    } else {  // calc_roe_z_in: (w,u,v) -> G(1),G(4),G(2),G(3),G(5)
      roe_flux(L[0], Rr[0], L[3], Rr[3], L[1], Rr[1], L[2], Rr[2], L[4], Rr[4], K, Fr);
      F[0] = Fr[0]; F[3] = Fr[1]; F[1] = Fr[2]; F[2] = Fr[3]; F[4] = Fr[4];
    }
  }
}

void calc_conv(Ctx& C) {
  int nx = C.nx, ny = C.ny, nz = C.nz;
  int io = C.c.order / 2 - 1;
  double F[5];
  int kz0 = C.c.dim == 3 ? 2 : 1, kz1 = C.c.dim == 3 ? nz - 1 : 1;
  // x faces: i in io+1..nx-(io+1) (interior kernels) or, with a non-periodic x
  // (bc_x = 1), every face 1..nx-1 with the order lowered next to the boundary;
  // j 2..ny-1, k 2..nz-1
  const int ord = C.c.order;
  const int i0 = C.c.bc_x ? 1 : io + 1, i1 = C.c.bc_x ? nx - 1 : nx - (io + 1);
#pragma omp parallel for schedule(static) private(F)
  for (int k = kz0; k <= kz1; ++k)
    for (int j = 2; j <= ny - 1; ++j)
      for (int i = i0; i <= i1; ++i) {
        int o = ord;
        if (C.c.bc_x) o = (ord == 6 && 3 <= i && i <= nx - 3) ? 6 : (ord >= 4 && 2 <= i && i <= nx - 2) ? 4 : 2;
        conv_face(C, 0, i, j, k, F, o);
        if (C.c.dim == 2) F[3] = F[4];  // 2D variables: rho, rho u, rho v, E
        for (int l = 0; l < C.nv; ++l) C.w.E[C.eidx(l + 1, i, j - 1, C.c.dim == 3 ? k - 1 : 1)] = F[l];
      }
  // y faces: j in io+1..ny-(io+1), or every face 1..ny-1 with a non-periodic y
  // (calc_*_y, 2D_solver/src/calc_slau_kernel.f90.fypp:116-204); i 2..nx-1
  const int j0 = C.c.bc_y ? 1 : io + 1, j1 = C.c.bc_y ? ny - 1 : ny - (io + 1);
#pragma omp parallel for schedule(static) private(F)
  for (int k = kz0; k <= kz1; ++k)
    for (int j = j0; j <= j1; ++j)
      for (int i = 2; i <= nx - 1; ++i) {
        int o = ord;
        if (C.c.bc_y) o = (ord == 6 && 3 <= j && j <= ny - 3) ? 6 : (ord >= 4 && 2 <= j && j <= ny - 2) ? 4 : 2;
        conv_face(C, 1, i, j, k, F, o);
        if (C.c.dim == 2) F[3] = F[4];
        for (int l = 0; l < C.nv; ++l) C.w.F[C.fidx(l + 1, i - 1, j, C.c.dim == 3 ? k - 1 : 1)] = F[l];
      }
  // z faces: k in io+1..nz-(io+1), or every face 1..nz-1 with a non-periodic z (the
  // 3D boundary kernels calc_*_z, 3D_solver/src/calc_slau_kernel.f90.fypp)
  const bool zb = C.c.dim == 3 && C.c.bc_z == 1;
  const int k0 = zb ? 1 : io + 1, k1 = zb ? nz - 1 : nz - (io + 1);
  if (C.c.dim == 3)
#pragma omp parallel for schedule(static) private(F)
    for (int k = k0; k <= k1; ++k)
      for (int j = 2; j <= ny - 1; ++j)
        for (int i = 2; i <= nx - 1; ++i) {
          int o = ord;
          if (zb) o = (ord == 6 && 3 <= k && k <= nz - 3) ? 6 : (ord >= 4 && 2 <= k && k <= nz - 2) ? 4 : 2;
          conv_face(C, 2, i, j, k, F, o);
          for (int l = 0; l < 5; ++l) C.w.G[C.gidx(l + 1, i - 1, j - 1, k)] = F[l];
        }
}

// ---- 3D_solver/src/calc_les.f90 -------------------------------------------------
double test_filter(const double x[3][3][3]) {  // :74-80 ; x[k][j][i]
  return x[1][1][1] + 0.25 * (x[1][1][0] - 2.0 * x[1][1][1] + x[1][1][2] + x[1][0][1] -
                              2.0 * x[1][1][1] + x[1][2][1] + x[0][1][1] - 2.0 * x[1][1][1] +
                              x[2][1][1]);
}
void calc_differential(const double u[3][3][3], const double v[3][3][3], const double w[3][3][3],
                       double dx, double dy, double dz, double d[9]) {  // :11-27
  d[0] = 0.5 * (-u[1][1][0] + u[1][1][2]) * dx;  // dudx
  d[1] = 0.5 * (-u[1][0][1] + u[1][2][1]) * dy;  // dudy
  d[2] = 0.5 * (-u[0][1][1] + u[2][1][1]) * dz;  // dudz
  d[3] = 0.5 * (-v[1][1][0] + v[1][1][2]) * dx;
  d[4] = 0.5 * (-v[1][0][1] + v[1][2][1]) * dy;
  d[5] = 0.5 * (-v[0][1][1] + v[2][1][1]) * dz;
  d[6] = 0.5 * (-w[1][1][0] + w[1][1][2]) * dx;
  d[7] = 0.5 * (-w[1][0][1] + w[1][2][1]) * dy;
  d[8] = 0.5 * (-w[0][1][1] + w[2][1][1]) * dz;
}
double sms(const double u[3][3][3], const double v[3][3][3], const double w[3][3][3],
           const double ut[3][3][3], const double vt[3][3][3], const double wt[3][3][3], double dx,
           double dy, double dz, double qc2, const Consts& K) {  // :30-71
  const double Cm = 0.06, alpha = 0.5;
  double a[9], h[9];
  calc_differential(u, v, w, dx, dy, dz, a);
  calc_differential(ut, vt, wt, dx, dy, dz, h);
  double dudx = a[0], dudy = a[1], dudz = a[2], dvdx = a[3], dvdy = a[4], dvdz = a[5],
         dwdx = a[6], dwdy = a[7], dwdz = a[8];
  double vor1 = dwdy - dvdz, vor2c = dudz - dwdx, vor3 = dvdx - dudy;
  double vh1 = h[7] - h[5], vh2 = h[2] - h[6], vh3 = h[3] - h[1];
  double vd1 = vor1 - vh1, vd2 = vor2c - vh2, vd3 = vor3 - vh3;
  double vor2 = vor1 * vor1 + vor2c * vor2c + vor3 * vor3;
  double vorh2 = vh1 * vh1 + vh2 * vh2 + vh3 * vh3;
  double vd2s = vd1 * vd1 + vd2 * vd2 + vd3 * vd3;
  double svor2 = 2.0 * std::sqrt(vor2) * std::sqrt(vorh2) + vorh2 + vor2 - vd2s;
  double tan2;
  if (std::fabs(svor2) < 1.0e-30) tan2 = 0.0;
  else tan2 = (2.0 * std::sqrt(vorh2) * std::sqrt(vor2) - vorh2 - vor2 + vd2s) / svor2;
  double rtheta = tan2 / K.tan10deg2;
  double ftheta = fmin2(1.0, rtheta * rtheta);
  double S2 = 2.0 * (dudx * dudx + dvdy * dvdy + dwdz * dwdz) +
              ((dvdx + dudy) * (dvdx + dudy) + (dwdy + dvdz) * (dwdy + dvdz) +
               (dudz + dwdx) * (dudz + dwdx));
  double mn = fmin3(dx, dy, dz);
  double a1 = mn / dx, a2 = mn / dy;
  double la1 = std::log(a1), la2 = std::log(a2);
  double delta = std::cosh(std::sqrt(4.0 * (la1 * la1 - la1 * la2 + la2 * la2) / 27.0)) *
                 std::pow(dx * dy * dz, -1.0 / 3.0);
  return ftheta * Cm * std::pow(S2, 0.5 * alpha) * std::pow(qc2, 0.5 * (1.0 - alpha)) *
         std::pow(delta, 1.0 + alpha);
}
void calc_mut(Ctx& C) {  // :96-125 plus set_bc_mut_common (set_bc_common.f90:296-335)
  int nx = C.nx, ny = C.ny, nz = C.nz;
  Prim P{C};
  std::fill(C.w.mut.begin(), C.w.mut.end(), 0.0);
  std::fill(C.w.qc2.begin(), C.w.qc2.end(), 0.0);
#pragma omp parallel for schedule(static)
  for (int k = 2; k <= nz - 1; ++k)
    for (int j = 2; j <= ny - 1; ++j)
      for (int i = 2; i <= nx - 1; ++i) {
        double u3[3][3][3], v3[3][3][3], w3[3][3][3], ut[3][3][3], vt[3][3][3], wt[3][3][3];
        for (int c = 0; c < 3; ++c)
          for (int b = 0; b < 3; ++b)
            for (int a = 0; a < 3; ++a) {
              u3[c][b][a] = P.u(i - 1 + a, j - 1 + b, k - 1 + c);
              v3[c][b][a] = P.v(i - 1 + a, j - 1 + b, k - 1 + c);
              w3[c][b][a] = P.w(i - 1 + a, j - 1 + b, k - 1 + c);
            }
        if (3 <= i && i <= nx - 2 && 3 <= j && j <= ny - 2 && 3 <= k && k <= nz - 2) {
          for (int c = 0; c < 3; ++c)
            for (int b = 0; b < 3; ++b)
              for (int a = 0; a < 3; ++a) {
                double xs[3][3][3], ys[3][3][3], zs[3][3][3];
                for (int cc = 0; cc < 3; ++cc)
                  for (int bb = 0; bb < 3; ++bb)
                    for (int aa = 0; aa < 3; ++aa) {
                      int ii = i - 2 + a + aa, jj = j - 2 + b + bb, kk = k - 2 + c + cc;
                      xs[cc][bb][aa] = P.u(ii, jj, kk);
                      ys[cc][bb][aa] = P.v(ii, jj, kk);
                      zs[cc][bb][aa] = P.w(ii, jj, kk);
                    }
                ut[c][b][a] = test_filter(xs);
                vt[c][b][a] = test_filter(ys);
                wt[c][b][a] = test_filter(zs);
              }
        } else {
          std::memcpy(ut, u3, sizeof(u3)); std::memcpy(vt, v3, sizeof(v3));
          std::memcpy(wt, w3, sizeof(w3));
        }
        double du = u3[1][1][1] - ut[1][1][1], dv = v3[1][1][1] - vt[1][1][1],
               dw = w3[1][1][1] - wt[1][1][1];
        double q = 0.5 * (du * du + dv * dv + dw * dw);
        C.w.qc2[C.sidx(i, j, k)] = q;
        C.w.mut[C.sidx(i, j, k)] = P.rho(i, j, k) * sms(u3, v3, w3, ut, vt, wt, C.g.xix[i - 1],
                                                        C.g.etay[j - 1], C.g.zetaz[k - 1], q, C.K);
      }
  std::vector<double>* arrs[2] = {&C.w.mut, &C.w.qc2};
  const bool walls = C.c.bc_x || C.c.bc_y || C.c.bc_z == 1;
  if (walls) {
    // a non-periodic face takes its neighbour's value, 0 on a no-slip wall (set_bc_mut
    // of 3D_solver/TBL/set.f90 and SBLI/set.f90: wall 0, top and outlet copies); a
    // periodic one its image at distance n-2 as set_bc_mut_common does; x faces for
    // the interior rows, then y faces, then z faces over everything before them
    const bool per[3] = {!C.c.bc_x, !C.c.bc_y, C.c.bc_z == 0};
    const int n[3] = {nx, ny, nz};
    auto kind = [&](int f) { return f < 4 ? C.c.bkind[f] : C.c.bkindz[f - 4]; };
    for (auto* ap : arrs) {
      std::vector<double>& a = *ap;
      for (int ax = 0; ax < 3; ++ax)
        for (int side = 0; side < 2; ++side) {
          const int c = side ? n[ax] : 1;
          const int s = per[ax] ? (side ? 2 : n[ax] - 1) : (side ? n[ax] - 1 : 2);
          const bool zero = !per[ax] && kind(2 * ax + side) == 3;
          // the other two axes: interior cells for x, all cells of the earlier axes after
          const int o1 = (ax + 1) % 3, o2 = (ax + 2) % 3;
          for (int q2 = 1; q2 <= n[o2]; ++q2)
            for (int q1 = 1; q1 <= n[o1]; ++q1) {
              // x: rows j, k interior; y: i all, k interior; z: everything
              int idx[3];
              idx[ax] = c; idx[o1] = q1; idx[o2] = q2;
              bool in = true;
              if (ax == 0) in = idx[1] >= 2 && idx[1] <= ny - 1 && idx[2] >= 2 && idx[2] <= nz - 1;
              if (ax == 1) in = idx[2] >= 2 && idx[2] <= nz - 1;
              if (!in) continue;
              int sidx[3] = {idx[0], idx[1], idx[2]};
              sidx[ax] = s;
              a[C.sidx(idx[0], idx[1], idx[2])] = zero ? 0.0 : a[C.sidx(sidx[0], sidx[1], sidx[2])];
            }
        }
    }
    return;
  }
  for (auto* ap : arrs) {
    std::vector<double>& a = *ap;
    for (int k = 2; k <= nz - 1; ++k)
      for (int j = 2; j <= ny - 1; ++j) {
        a[C.sidx(1, j, k)] = a[C.sidx(nx - 1, j, k)];
        a[C.sidx(nx, j, k)] = a[C.sidx(2, j, k)];
      }
    for (int k = 2; k <= nz - 1; ++k)
      for (int i = 2; i <= nx - 1; ++i) {
        a[C.sidx(i, 1, k)] = a[C.sidx(i, ny - 1, k)];
        a[C.sidx(i, ny, k)] = a[C.sidx(i, 2, k)];
      }
    for (int k = 2; k <= nz - 1; ++k) {
      a[C.sidx(1, 1, k)] = a[C.sidx(nx - 1, ny - 1, k)];
      a[C.sidx(nx, 1, k)] = a[C.sidx(2, ny - 1, k)];
      a[C.sidx(1, ny, k)] = a[C.sidx(nx - 1, 2, k)];
      a[C.sidx(nx, ny, k)] = a[C.sidx(2, 2, k)];
    }
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) {
        a[C.sidx(i, j, 1)] = a[C.sidx(i, j, nz - 1)];
        a[C.sidx(i, j, nz)] = a[C.sidx(i, j, 2)];
      }
  }
}

// ---- viscous fluxes ------------------------------------------------------------
// 3D_solver/src/calc_visc_cent.f90.fypp:2-21
double interpN(int N, const double* a) {
  if (N == 4) return 0.0625 * (-a[0] + 9.0 * (a[1] + a[2]) - a[3]);
  return 0.00390625 * (3.0 * a[0] - 25.0 * a[1] + 150.0 * (a[2] + a[3]) - 25.0 * a[4] + 3.0 * a[5]);
}
double diffN(int N, double d, const double* a) {
  if (N == 4) return (a[0] - 27.0 * (a[1] - a[2]) - a[3]) * (1.0 / 24.0) * d;
  return (-0.0046875 * a[0] + 0.065104167 * a[1] - 1.171875 * (a[2] - a[3]) - 0.065104167 * a[4] +
          0.0046875 * a[5]) * d;
}
// calc_visc_cent.f90.fypp:23-91 (N = 4 or 6)
void tau_straight_c(int N, bool les, const double* mu, const double* mut, const double* u,
                    const double* vy, const double* wz, double d, double& t11, double& ut11) {
  double mui = interpN(N, mu), vyi = interpN(N, vy), wzi = interpN(N, wz), ux = diffN(N, d, u);
  t11 = two_third * mui * (2.0 * ux - vyi - wzi);
  ut11 = interpN(N, u) * t11;
  if (les) {
    mui = 0.5 * (mui + interpN(N, mut));
    t11 = two_third * mui * (2.0 * ux - vyi - wzi);
  }
}
void tau_cross_c(int N, bool les, const double* mu, const double* mut, const double* v,
                 const double* uy, double d, double& t12, double& vt12) {
  double mui = interpN(N, mu), uyi = interpN(N, uy), vx = diffN(N, d, v);
  t12 = mui * (uyi + vx);
  vt12 = interpN(N, v) * t12;
  if (les) {
    mui = 0.5 * (mui + interpN(N, mut));
    t12 = mui * (uyi + vx);
  }
}
// 3D_solver/src/calc_visc_me4_base.f90:4-111 (mu3 are face-interpolated values)
double flux4(const double* a) { return (-a[0] + 26.0 * a[1] - a[2]) * (1.0 / 24.0); }
void tau_straight_me4(bool les, const double* mu, const double* mut, const double* u,
                      const double* vy, const double* wz, double d, double& t11, double& ut11) {
  const double one_24 = 1.0 / 24.0;
  if (!les) {
    double t[3];
    for (int m = 0; m < 3; ++m)
      t[m] = two_third * mu[m] *
             ((2.25 * (-u[m + 1] + u[m + 2]) - (-u[m] + u[m + 3]) * one_twelfth) * d -
              0.0625 * (-vy[m] + 9.0 * (vy[m + 1] + vy[m + 2]) - vy[m + 3]) -
              0.0625 * (-wz[m] + 9.0 * (wz[m + 1] + wz[m + 2]) - wz[m + 3]));
    t11 = (-t[0] + 26.0 * t[1] - t[2]) * one_24;
    for (int m = 0; m < 3; ++m) t[m] = 0.0625 * (-u[m] + 9.0 * (u[m + 1] + u[m + 2]) - u[m + 3]) * t[m];
    ut11 = (-t[0] + 26.0 * t[1] - t[2]) * one_24;
  } else {
    double t1[3], t2[3];
    for (int m = 0; m < 3; ++m) {
      t1[m] = (2.25 * (-u[m + 1] + u[m + 2]) - (-u[m] + u[m + 3]) * one_twelfth) * d;
      t1[m] = t1[m] - 0.0625 * (-vy[m] + 9.0 * (vy[m + 1] + vy[m + 2]) - vy[m + 3]);
      t1[m] = t1[m] - 0.0625 * (-wz[m] + 9.0 * (wz[m + 1] + wz[m + 2]) - wz[m + 3]);
    }
    for (int m = 0; m < 3; ++m) t2[m] = two_third * mu[m] * t1[m];
    for (int m = 0; m < 3; ++m) t2[m] = 0.0625 * (-u[m] + 9.0 * (u[m + 1] + u[m + 2]) - u[m + 3]) * t2[m];
    ut11 = (-t2[0] + 26.0 * t2[1] - t2[2]) * one_24;
    for (int m = 0; m < 3; ++m) t2[m] = two_third * (mu[m] + mut[m]) * t1[m];
    t11 = (-t2[0] + 26.0 * t2[1] - t2[2]) * one_24;
  }
}
void tau_cross_me4(bool les, const double* mu, const double* mut, const double* v,
                   const double* uy, double d, double& t12, double& vt12) {
  const double one_24 = 1.0 / 24.0;
  if (!les) {
    double t[3];
    for (int m = 0; m < 3; ++m)
      t[m] = mu[m] * ((1.125 * (-v[m + 1] + v[m + 2]) - (-v[m] + v[m + 3]) * one_24) * d +
                      0.0625 * (-uy[m] + 9.0 * (uy[m + 1] + uy[m + 2]) - uy[m + 3]));
    t12 = (-t[0] + 26.0 * t[1] - t[2]) * one_24;
    for (int m = 0; m < 3; ++m) t[m] = 0.0625 * (-v[m] + 9.0 * (v[m + 1] + v[m + 2]) - v[m + 3]) * t[m];
    vt12 = (-t[0] + 26.0 * t[1] - t[2]) * one_24;
  } else {
    double t1[3], t2[3];
    for (int m = 0; m < 3; ++m) {
      t1[m] = (1.125 * (-v[m + 1] + v[m + 2]) - (-v[m] + v[m + 3]) * one_24) * d;
      t1[m] = t1[m] + 0.0625 * (-uy[m] + 9.0 * (uy[m + 1] + uy[m + 2]) - uy[m + 3]);
    }
    for (int m = 0; m < 3; ++m) t2[m] = mu[m] * t1[m];
    for (int m = 0; m < 3; ++m) t2[m] = 0.0625 * (-v[m] + 9.0 * (v[m + 1] + v[m + 2]) - v[m + 3]) * t2[m];
    vt12 = (-t2[0] + 26.0 * t2[1] - t2[2]) * one_24;
    for (int m = 0; m < 3; ++m) t2[m] = (mu[m] + mut[m]) * t1[m];
    t12 = (-t2[0] + 26.0 * t2[1] - t2[2]) * one_24;
  }
}

// Node derivative of velocity component `comp` along `ddir` at cell (i,j,k):
// load_smem_visc_cent.f90.fypp:51-70 (6th, VISC 6) and the 4th-order form
// used by VISC 4 and ME4 (load_smem_visc_me4_base.f90:120-127).
double node_deriv(const Ctx& C, int comp, int ddir, int i, int j, int k, bool sixth) {
  Prim P{C};
  auto q = [&](int off) {
    return P.vel(comp, i + (ddir == 0 ? off : 0), j + (ddir == 1 ? off : 0), k + (ddir == 2 ? off : 0));
  };
  double inv = ddir == 0 ? C.g.xix[i - 1] : ddir == 1 ? C.g.etay[j - 1] : C.g.zetaz[k - 1];
  if (sixth)
    return (one_sixty * (-q(-3) + q(3)) + 0.15 * (q(-2) - q(2)) + 0.75 * (-q(-1) + q(1))) * inv;
  return (two_third * (-q(-1) + q(1)) - one_twelfth * (-q(-2) + q(2))) * inv;
}

// High-order viscous face flux (Central-4/6 or ME4) for the face c+1/2 along dir.
// calc_visc_high_internal.f90.fypp:43-600.  Returns the 4 subtracted terms.
void visc_face_high(const Ctx& C, int dir, int i, int j, int k, double out[4]) {
  Prim P{C};
  const Consts& K = C.K;
  bool les = C.c.visc == ORC_LES;
  bool me4 = (C.c.visc_order == 6 && C.c.visc_stencil == ORC_ME4);
  int N = C.c.visc_order;  // 4 or 6
  bool sixth = (N == 6 && !me4);
  int lo = (N == 4) ? -1 : -2;  // stencil cell offsets lo..lo+len-1
  int len = (N == 4) ? 4 : 6;
  // the three velocity components in the rotated order (normal, t1, t2)
  int cn = dir, ca = dir == 0 ? 1 : 0, cb = dir == 2 ? 1 : 2;
  auto at = [&](int off, int& ii, int& jj, int& kk) {
    ii = i + (dir == 0 ? off : 0); jj = j + (dir == 1 ? off : 0); kk = k + (dir == 2 ? off : 0);
  };
  double un[6], ua[6], ub[6], dna[6], dnb[6], dan[6], dbn[6], Ts[6], mus[6], muts[6], H[6];
  double uvw[3][6];
  // derivative arrays: for Ev: u, vy, wz (straight), v & uy (cross), w & uz (cross)
  //   straight uses normal velocity + tangential derivatives of tangential components
  //   cross (t1): tangential velocity v, derivative of normal velocity along t1 (uy)
  int da = ca, db = cb;  // cross terms: derivative of the normal velocity along each tangent
  for (int m = 0; m < len; ++m) {
    int ii, jj, kk;
    at(lo + m, ii, jj, kk);
    un[m] = P.vel(cn, ii, jj, kk);
    ua[m] = P.vel(ca, ii, jj, kk);
    ub[m] = P.vel(cb, ii, jj, kk);
    // straight stress uses the cyclic pair: Ev (vy, wz), Fv (wz, ux), Gv (ux, vy)
    dna[m] = node_deriv(C, (dir + 1) % 3, (dir + 1) % 3, ii, jj, kk, sixth);
    dnb[m] = node_deriv(C, (dir + 2) % 3, (dir + 2) % 3, ii, jj, kk, sixth);
    uvw[0][m] = P.u(ii, jj, kk); uvw[1][m] = P.v(ii, jj, kk); uvw[2][m] = P.w(ii, jj, kk);
    dan[m] = node_deriv(C, cn, da, ii, jj, kk, sixth);  // e.g. uy
    dbn[m] = node_deriv(C, cn, db, ii, jj, kk, sixth);  // e.g. uz
    Ts[m] = P.T(ii, jj, kk);
    mus[m] = P.mu(ii, jj, kk);
    muts[m] = les ? P.mut(ii, jj, kk) : 0.0;
  }
  double inv = dir == 0 ? C.g.xix[i - 1] : dir == 1 ? C.g.etay[j - 1] : C.g.zetaz[k - 1];
  double tnn, tna, tnb, utnn, vtna, wtnb, kT, Hsgs = 0.0;
  // For 2D there is no second tangential direction: treated like the 3D kernel
  // with w = 0 is NOT the reference (2D uses its own kernels); 2D is handled elsewhere.
  if (!me4) {
    kT = K.Cp_over_Pr * interpN(N, mus) * diffN(N, inv, Ts);
    tau_straight_c(N, les, mus, muts, un, dna, dnb, inv, tnn, utnn);
    tau_cross_c(N, les, mus, muts, ua, dan, inv, tna, vtna);
    tau_cross_c(N, les, mus, muts, ub, dbn, inv, tnb, wtnb);
    if (les) {
      for (int m = 0; m < len; ++m) {
        int ii, jj, kk;
        at(lo + m, ii, jj, kk);
        H[m] = K.Cp * Ts[m] + 0.5 * (uvw[0][m] * uvw[0][m] + uvw[1][m] * uvw[1][m] + uvw[2][m] * uvw[2][m]) +
               P.qc2(ii, jj, kk);
      }
      Hsgs = -interpN(N, muts) * diffN(N, inv, H) / K.Prt;
    }
  } else {
    // mu3 at faces c-1/2, c+1/2, c+3/2 from mu(c-2..c+3)
    double mu3[3], mut3[3], kT3[3];
    for (int m = 0; m < 3; ++m) {
      mu3[m] = 0.0625 * (9.0 * (mus[m + 1] + mus[m + 2]) - (mus[m] + mus[m + 3]));
      mut3[m] = les ? 0.0625 * (9.0 * (muts[m + 1] + muts[m + 2]) - (muts[m] + muts[m + 3])) : 0.0;
    }
    for (int m = 0; m < 3; ++m)
      kT3[m] = K.Cp_over_Pr * mu3[m] *
               (1.125 * (-Ts[m + 1] + Ts[m + 2]) - (-Ts[m] + Ts[m + 3]) * (1.0 / 24.0)) * inv;
    kT = flux4(kT3);
    tau_straight_me4(les, mu3, mut3, un, dna, dnb, inv, tnn, utnn);
    tau_cross_me4(les, mu3, mut3, ua, dan, inv, tna, vtna);
    tau_cross_me4(les, mu3, mut3, ub, dbn, inv, tnb, wtnb);
    if (les) {
      double H4[4];
      for (int m = 0; m < 4; ++m) {
        int ii, jj, kk;
        at(-1 + m, ii, jj, kk);
        int s = m + 1;  // index into the 6-point arrays (offset -2)
        H4[m] = K.Cp * Ts[s] + 0.5 * (uvw[0][s] * uvw[0][s] + uvw[1][s] * uvw[1][s] + uvw[2][s] * uvw[2][s]) +
                P.qc2(ii, jj, kk);
      }
      Hsgs = -flux4(mut3) * (1.125 * (-H4[1] + H4[2]) - (-H4[0] + H4[3]) * (1.0 / 24.0)) * inv / K.Prt;
    }
  }
  // subtract order: normal-momentum (tnn), t1 (tna), t2 (tnb) mapped back to x,y,z
  double t[3];
  t[cn] = tnn; t[ca] = tna; t[cb] = tnb;
  out[0] = t[0]; out[1] = t[1]; out[2] = t[2];
  // energy: u*t + v*t + w*t in x,y,z order (utxx + vtxy + wtxz etc.)
  double work[3];
  work[cn] = utnn; work[ca] = vtna; work[cb] = wtnb;
  double e = work[0] + work[1] + work[2] + kT;
  if (les) e = e + Hsgs;
  out[3] = e;
}

// Gaitonde-Visbal 2nd order (3D_solver/src/calc_visc2.f90.fypp:17-418)
void visc_face_gv2(const Ctx& C, int dir, int i, int j, int k, double out[4]) {
  Prim P{C};
  const Consts& K = C.K;
  bool les = C.c.visc == ORC_LES;
  int i2 = i + (dir == 0), j2 = j + (dir == 1), k2 = k + (dir == 2);
  double inv = dir == 0 ? C.g.xix[i - 1] : dir == 1 ? C.g.etay[j - 1] : C.g.zetaz[k - 1];
  double md = 0.5 * (P.mu(i, j, k) + P.mu(i2, j2, k2)) * inv;
  double vw = K.Cp_over_Pr * md * (-P.T(i, j, k) + P.T(i2, j2, k2));
  double dn[3], sg[3] = {0.0, 0.0, 0.0}, Hsgs = 0.0;
  for (int c = 0; c < 3; ++c) dn[c] = md * (-P.vel(c, i, j, k) + P.vel(c, i2, j2, k2));
  if (les) {
    double msd = 0.5 * (P.mut(i, j, k) + P.mut(i2, j2, k2)) * inv;
    auto Hf = [&](int a, int b, int c) {
      return K.Cp * P.T(a, b, c) +
             0.5 * (P.u(a, b, c) * P.u(a, b, c) + P.v(a, b, c) * P.v(a, b, c) +
                    P.w(a, b, c) * P.w(a, b, c)) + P.qc2(a, b, c);
    };
    double H1 = Hf(i, j, k), H2 = Hf(i2, j2, k2);
    Hsgs = -msd * (-H1 + H2) / K.Prt;
    for (int c = 0; c < 3; ++c) sg[c] = msd * (-P.vel(c, i, j, k) + P.vel(c, i2, j2, k2));
  }
  // derivative of velocity component c along the tangential axis t, with
  // mu (or mut) averaged over the four cells around the face edge
  auto cross = [&](bool sgs, int c, int t) {
    int ti = t == 0, tj = t == 1, tk = t == 2;
    auto m = [&](int a, int b, int cc) { return sgs ? P.mut(a, b, cc) : P.mu(a, b, cc); };
    double m1 = 0.0625 * (m(i - ti, j - tj, k - tk) + m(i, j, k) + m(i2 - ti, j2 - tj, k2 - tk) + m(i2, j2, k2));
    double m2 = 0.0625 * (m(i, j, k) + m(i + ti, j + tj, k + tk) + m(i2, j2, k2) + m(i2 + ti, j2 + tj, k2 + tk));
    double dtv = t == 0 ? C.g.xix[i - 1] : t == 1 ? C.g.etay[j - 1] : C.g.zetaz[k - 1];
    return (m1 * (-P.vel(c, i - ti, j - tj, k - tk) - P.vel(c, i2 - ti, j2 - tj, k2 - tk)) +
            (m1 - m2) * (P.vel(c, i, j, k) + P.vel(c, i2, j2, k2)) +
            m2 * (P.vel(c, i + ti, j + tj, k + tk) + P.vel(c, i2 + ti, j2 + tj, k2 + tk))) * dtv;
  };
  double uS = P.u(i, j, k) + P.u(i2, j2, k2), vS = P.v(i, j, k) + P.v(i2, j2, k2),
         wS = P.w(i, j, k) + P.w(i2, j2, k2);
  double s1, s2, s3;
  if (dir == 0) {
    double txx = two_third * (2.0 * dn[0] - cross(false, 1, 1) - cross(false, 2, 2));
    double txy = cross(false, 0, 1) + dn[1];
    double txz = dn[2] + cross(false, 0, 2);
    vw = vw + 0.5 * (uS * txx + vS * txy + wS * txz);
    if (les) {
      txx = txx + two_third * (2.0 * sg[0] - cross(true, 1, 1) - cross(true, 2, 2));
      txy = txy + cross(true, 0, 1) + sg[1];
      txz = txz + sg[2] + cross(true, 0, 2);
    }
    s1 = txx; s2 = txy; s3 = txz;
  } else if (dir == 1) {
    double tyx = dn[0] + cross(false, 1, 0);
    double tyy = two_third * (2.0 * dn[1] - cross(false, 2, 2) - cross(false, 0, 0));
    double tyz = cross(false, 1, 2) + dn[2];
    vw = vw + 0.5 * (uS * tyx + vS * tyy + wS * tyz);
    if (les) {
      tyx = tyx + sg[0] + cross(true, 1, 0);
      tyy = tyy + two_third * (2.0 * sg[1] - cross(true, 2, 2) - cross(true, 0, 0));
      tyz = tyz + cross(true, 1, 2) + sg[2];
    }
    s1 = tyx; s2 = tyy; s3 = tyz;
  } else {
    double tzx = cross(false, 2, 0) + dn[0];
    double tzy = dn[1] + cross(false, 2, 1);
    double tzz = two_third * (2.0 * dn[2] - cross(false, 0, 0) - cross(false, 1, 1));
    vw = vw + 0.5 * (uS * tzx + vS * tzy + wS * tzz);
    if (les) {
      tzx = tzx + cross(true, 2, 0) + sg[0];
      tzy = tzy + sg[1] + cross(true, 2, 1);
      tzz = tzz + two_third * (2.0 * sg[2] - cross(true, 0, 0) - cross(true, 1, 1));
    }
    s1 = tzx; s2 = tzy; s3 = tzz;
  }
  out[0] = s1; out[1] = s2; out[2] = s3;
  out[3] = les ? (vw + Hsgs) : vw;
}

// 2nd-order fallback of the high-order viscous kernels outside their guard, written
// per direction as the reference writes it (LES: the SGS stresses added after the
// work terms, and the SGS enthalpy flux):
// calc_Ev (3D_solver/src/calc_visc_high.f90.fypp:194-260), calc_Fv (:432-497),
// calc_Gv (:674-739).  Returns the 4 subtracted terms like visc_face_high.
void visc_face_fb3(const Ctx& C, int dir, int i, int j, int k, double out[4]) {
  Prim P{C};
  const Consts& K = C.K;
  const double dxi = C.g.xix[i - 1], dyj = C.g.etay[j - 1], dzk = C.g.zetaz[k - 1];
  // 0.25 (m1 (-a(-) + a(0) - a2(-) + a2(0)) + m2 (-a(0) + a(+) - a2(0) + a2(+))) d, the
  // tangential derivative of field `a` (a2: the face's second cell) along `t`
  auto tder = [&](int comp, int t, int i2, int j2, int k2, double m1, double m2, double d) {
    int di = t == 0, dj = t == 1, dk = t == 2;
    auto a = [&](int ii, int jj, int kk) { return P.vel(comp, ii, jj, kk); };
    return 0.25 * (m1 * (-a(i - di, j - dj, k - dk) + a(i, j, k) - a(i2 - di, j2 - dj, k2 - dk) + a(i2, j2, k2)) +
                   m2 * (-a(i, j, k) + a(i + di, j + dj, k + dk) - a(i2, j2, k2) + a(i2 + di, j2 + dj, k2 + dk))) *
           d;
  };
  auto mavg = [&](int t, int i2, int j2, int k2, double& m1, double& m2) {
    int di = t == 0, dj = t == 1, dk = t == 2;
    m1 = 0.25 * (P.mu(i - di, j - dj, k - dk) + P.mu(i, j, k) + P.mu(i2 - di, j2 - dj, k2 - dk) + P.mu(i2, j2, k2));
    m2 = 0.25 * (P.mu(i, j, k) + P.mu(i + di, j + dj, k + dk) + P.mu(i2, j2, k2) + P.mu(i2 + di, j2 + dj, k2 + dk));
  };
  auto mavg_sgs = [&](int t, int i2, int j2, int k2, double& m1, double& m2) {
    int di = t == 0, dj = t == 1, dk = t == 2;
    m1 = 0.25 * (P.mut(i - di, j - dj, k - dk) + P.mut(i, j, k) + P.mut(i2 - di, j2 - dj, k2 - dk) + P.mut(i2, j2, k2));
    m2 = 0.25 * (P.mut(i, j, k) + P.mut(i + di, j + dj, k + dk) + P.mut(i2, j2, k2) + P.mut(i2 + di, j2 + dj, k2 + dk));
  };
  const bool les = C.c.visc == ORC_LES;
  auto Hs = [&](int ii, int jj, int kk) {
    double u = P.u(ii, jj, kk), v = P.v(ii, jj, kk), w = P.w(ii, jj, kk);
    return K.Cp * P.T(ii, jj, kk) + 0.5 * (u * u + v * v + w * w) + P.qc2(ii, jj, kk);
  };
  if (dir == 0) {
    const int i2 = i + 1;
    double mx = 0.5 * (P.mu(i, j, k) + P.mu(i2, j, k));
    double kTx = K.Cp_over_Pr * mx * (-P.T(i, j, k) + P.T(i2, j, k)) * dxi;
    double m1, m2;
    mavg(1, i2, j, k, m1, m2);
    double muy = tder(0, 1, i2, j, k, m1, m2, dyj), mvy = tder(1, 1, i2, j, k, m1, m2, dyj);
    mavg(2, i2, j, k, m1, m2);
    double muz = tder(0, 2, i2, j, k, m1, m2, dzk), mwz = tder(2, 2, i2, j, k, m1, m2, dzk);
    double mux = mx * (-P.u(i, j, k) + P.u(i2, j, k)) * dxi;
    double mvx = mx * (-P.v(i, j, k) + P.v(i2, j, k)) * dxi;
    double mwx = mx * (-P.w(i, j, k) + P.w(i2, j, k)) * dxi;
    double txx = two_third * (2.0 * mux - mvy - mwz);
    double txy = muy + mvx;
    double txz = mwx + muz;
    double utxx = 0.5 * (P.u(i, j, k) + P.u(i2, j, k)) * txx;
    double vtxy = 0.5 * (P.v(i, j, k) + P.v(i2, j, k)) * txy;
    double wtxz = 0.5 * (P.w(i, j, k) + P.w(i2, j, k)) * txz;
    double Hsgs = 0.0;
    if (les) {
      double mxsgs = 0.5 * (P.mut(i, j, k) + P.mut(i2, j, k));
      mavg_sgs(1, i2, j, k, m1, m2);
      double muysgs = tder(0, 1, i2, j, k, m1, m2, dyj), mvysgs = tder(1, 1, i2, j, k, m1, m2, dyj);
      mavg_sgs(2, i2, j, k, m1, m2);
      double muzsgs = tder(0, 2, i2, j, k, m1, m2, dzk), mwzsgs = tder(2, 2, i2, j, k, m1, m2, dzk);
      double muxsgs = mxsgs * (-P.u(i, j, k) + P.u(i2, j, k)) * dxi;
      double mvxsgs = mxsgs * (-P.v(i, j, k) + P.v(i2, j, k)) * dxi;
      double mwxsgs = mxsgs * (-P.w(i, j, k) + P.w(i2, j, k)) * dxi;
      txx = txx + two_third * (2.0 * muxsgs - mvysgs - mwzsgs);
      txy = txy + muysgs + mvxsgs;
      txz = txz + mwxsgs + muzsgs;
      Hsgs = -mxsgs * (-Hs(i, j, k) + Hs(i2, j, k)) * dxi / K.Prt;
    }
    out[0] = txx; out[1] = txy; out[2] = txz; out[3] = utxx + vtxy + wtxz + kTx;
    if (les) out[3] = out[3] + Hsgs;
  } else if (dir == 1) {
    const int j2 = j + 1;
    double my = 0.5 * (P.mu(i, j, k) + P.mu(i, j2, k));
    double kTy = K.Cp_over_Pr * my * (-P.T(i, j, k) + P.T(i, j2, k)) * dyj;
    double m1, m2;
    mavg(0, i, j2, k, m1, m2);
    double mux = tder(0, 0, i, j2, k, m1, m2, dxi), mvx = tder(1, 0, i, j2, k, m1, m2, dxi);
    mavg(2, i, j2, k, m1, m2);
    double mvz = tder(1, 2, i, j2, k, m1, m2, dzk), mwz = tder(2, 2, i, j2, k, m1, m2, dzk);
    double muy = my * (-P.u(i, j, k) + P.u(i, j2, k)) * dyj;
    double mvy = my * (-P.v(i, j, k) + P.v(i, j2, k)) * dyj;
    double mwy = my * (-P.w(i, j, k) + P.w(i, j2, k)) * dyj;
    double tyx = muy + mvx;
    double tyy = two_third * (2.0 * mvy - mwz - mux);
    double tyz = mvz + mwy;
    double utyx = 0.5 * (P.u(i, j, k) + P.u(i, j2, k)) * tyx;
    double vtyy = 0.5 * (P.v(i, j, k) + P.v(i, j2, k)) * tyy;
    double wtyz = 0.5 * (P.w(i, j, k) + P.w(i, j2, k)) * tyz;
    double Hsgs = 0.0;
    if (les) {
      double mysgs = 0.5 * (P.mut(i, j, k) + P.mut(i, j2, k));
      mavg_sgs(0, i, j2, k, m1, m2);
      double muxsgs = tder(0, 0, i, j2, k, m1, m2, dxi), mvxsgs = tder(1, 0, i, j2, k, m1, m2, dxi);
      mavg_sgs(2, i, j2, k, m1, m2);
      double mvzsgs = tder(1, 2, i, j2, k, m1, m2, dzk), mwzsgs = tder(2, 2, i, j2, k, m1, m2, dzk);
      double muysgs = mysgs * (-P.u(i, j, k) + P.u(i, j2, k)) * dyj;
      double mvysgs = mysgs * (-P.v(i, j, k) + P.v(i, j2, k)) * dyj;
      double mwysgs = mysgs * (-P.w(i, j, k) + P.w(i, j2, k)) * dyj;
      tyx = tyx + muysgs + mvxsgs;
      tyy = tyy + two_third * (2.0 * mvysgs - mwzsgs - muxsgs);
      tyz = tyz + mvzsgs + mwysgs;
      Hsgs = -mysgs * (-Hs(i, j, k) + Hs(i, j2, k)) * dyj / K.Prt;
    }
    out[0] = tyx; out[1] = tyy; out[2] = tyz; out[3] = utyx + vtyy + wtyz + kTy;
    if (les) out[3] = out[3] + Hsgs;
  } else {
    const int k2 = k + 1;
    double m1, m2;
    mavg(0, i, j, k2, m1, m2);
    double mux = tder(0, 0, i, j, k2, m1, m2, dxi), mwx = tder(2, 0, i, j, k2, m1, m2, dxi);
    mavg(1, i, j, k2, m1, m2);
    double mvy = tder(1, 1, i, j, k2, m1, m2, dyj), mwy = tder(2, 1, i, j, k2, m1, m2, dyj);
    double mz = 0.5 * (P.mu(i, j, k) + P.mu(i, j, k2));
    double kTz = K.Cp_over_Pr * mz * (-P.T(i, j, k) + P.T(i, j, k2)) * dzk;
    double muz = mz * (-P.u(i, j, k) + P.u(i, j, k2)) * dzk;
    double mvz = mz * (-P.v(i, j, k) + P.v(i, j, k2)) * dzk;
    double mwz = mz * (-P.w(i, j, k) + P.w(i, j, k2)) * dzk;
    double tzx = mwx + muz;
    double tzy = mvz + mwy;
    double tzz = two_third * (2.0 * mwz - mux - mvy);
    double utzx = 0.5 * (P.u(i, j, k) + P.u(i, j, k2)) * tzx;
    double vtzy = 0.5 * (P.v(i, j, k) + P.v(i, j, k2)) * tzy;
    double wtzz = 0.5 * (P.w(i, j, k) + P.w(i, j, k2)) * tzz;
    double Hsgs = 0.0;
    if (les) {
      mavg_sgs(0, i, j, k2, m1, m2);
      double muxsgs = tder(0, 0, i, j, k2, m1, m2, dxi), mwxsgs = tder(2, 0, i, j, k2, m1, m2, dxi);
      mavg_sgs(1, i, j, k2, m1, m2);
      double mvysgs = tder(1, 1, i, j, k2, m1, m2, dyj), mwysgs = tder(2, 1, i, j, k2, m1, m2, dyj);
      double mzsgs = 0.5 * (P.mut(i, j, k) + P.mut(i, j, k2));
      double muzsgs = mzsgs * (-P.u(i, j, k) + P.u(i, j, k2)) * dzk;
      double mvzsgs = mzsgs * (-P.v(i, j, k) + P.v(i, j, k2)) * dzk;
      double mwzsgs = mzsgs * (-P.w(i, j, k) + P.w(i, j, k2)) * dzk;
      tzx = tzx + mwxsgs + muzsgs;
      tzy = tzy + mvzsgs + mwysgs;
      tzz = tzz + two_third * (2.0 * mwzsgs - muxsgs - mvysgs);
      Hsgs = -mzsgs * (-Hs(i, j, k) + Hs(i, j, k2)) * dzk / K.Prt;
    }
    out[0] = tzx; out[1] = tzy; out[2] = tzz; out[3] = utzx + vtzy + wtzz + kTz;
    if (les) out[3] = out[3] + Hsgs;
  }
}

void calc_visc3(Ctx& C) {
  int nx = C.nx, ny = C.ny, nz = C.nz;
  double o[4];
  int vo = C.c.visc_order;
  auto apply = [&](double* f, const double o4[4]) {
    f[1] = f[1] - o4[0]; f[2] = f[2] - o4[1]; f[3] = f[3] - o4[2]; f[4] = f[4] - o4[3];
  };
  if (vo == 2) {
#pragma omp parallel for schedule(static) private(o)
    for (int k = 2; k <= nz - 1; ++k)
      for (int j = 2; j <= ny - 1; ++j)
        for (int i = 1; i <= nx - 1; ++i) { visc_face_gv2(C, 0, i, j, k, o); apply(&C.w.E[C.eidx(1, i, j - 1, k - 1)], o); }
#pragma omp parallel for schedule(static) private(o)
    for (int k = 2; k <= nz - 1; ++k)
      for (int j = 1; j <= ny - 1; ++j)
        for (int i = 2; i <= nx - 1; ++i) { visc_face_gv2(C, 1, i, j, k, o); apply(&C.w.F[C.fidx(1, i - 1, j, k - 1)], o); }
#pragma omp parallel for schedule(static) private(o)
    for (int k = 1; k <= nz - 1; ++k)
      for (int j = 2; j <= ny - 1; ++j)
        for (int i = 2; i <= nx - 1; ++i) { visc_face_gv2(C, 2, i, j, k, o); apply(&C.w.G[C.gidx(1, i - 1, j - 1, k)], o); }
    return;
  }
  bool me4 = (vo == 6 && C.c.visc_stencil == ORC_ME4);
  // interior guards: calc_visc_high_internal.f90.fypp (Ev :114/139/169, Fv :350/376/406, Gv :592/618/648)
  int a0, a1, b0, b1;  // normal-direction face range and transverse cell range
  if (vo == 4) { a0 = 2; a1 = 2; b0 = 3; b1 = 2; }
  else if (me4) { a0 = 3; a1 = 3; b0 = 3; b1 = 2; }
  else { a0 = 3; a1 = 3; b0 = 4; b1 = 3; }
  const bool walls = C.c.bc_x || C.c.bc_y || C.c.bc_z == 1 || C.c.bc_z == 3 || C.c.bc_z == 4;
  if (walls) {
    // every face of the kernels' launch ranges, the guard choosing the stencil
    // (calc_visc_high.f90.fypp: Ev i 1..nx-1, j 2..ny-1, k 2..nz-1, and alike)
    auto face = [&](int dir, int i, int j, int k, double o4[4]) {
      const int c[3] = {i, j, k}, n[3] = {nx, ny, nz};
      bool in = true;
      for (int a = 0; a < 3; ++a)
        in = in && (a == dir ? (a0 <= c[a] && c[a] <= n[a] - a1) : (b0 <= c[a] && c[a] <= n[a] - b1));
      if (in) visc_face_high(C, dir, i, j, k, o4);
      else visc_face_fb3(C, dir, i, j, k, o4);
    };
#pragma omp parallel for schedule(static) private(o)
    for (int k = 2; k <= nz - 1; ++k)
      for (int j = 2; j <= ny - 1; ++j)
        for (int i = 1; i <= nx - 1; ++i) { face(0, i, j, k, o); apply(&C.w.E[C.eidx(1, i, j - 1, k - 1)], o); }
#pragma omp parallel for schedule(static) private(o)
    for (int k = 2; k <= nz - 1; ++k)
      for (int j = 1; j <= ny - 1; ++j)
        for (int i = 2; i <= nx - 1; ++i) { face(1, i, j, k, o); apply(&C.w.F[C.fidx(1, i - 1, j, k - 1)], o); }
#pragma omp parallel for schedule(static) private(o)
    for (int k = 1; k <= nz - 1; ++k)
      for (int j = 2; j <= ny - 1; ++j)
        for (int i = 2; i <= nx - 1; ++i) { face(2, i, j, k, o); apply(&C.w.G[C.gidx(1, i - 1, j - 1, k)], o); }
    return;
  }
#pragma omp parallel for schedule(static) private(o)
  for (int k = b0; k <= nz - b1; ++k)
    for (int j = b0; j <= ny - b1; ++j)
      for (int i = a0; i <= nx - a1; ++i) { visc_face_high(C, 0, i, j, k, o); apply(&C.w.E[C.eidx(1, i, j - 1, k - 1)], o); }
#pragma omp parallel for schedule(static) private(o)
  for (int k = b0; k <= nz - b1; ++k)
    for (int j = a0; j <= ny - a1; ++j)
      for (int i = b0; i <= nx - b1; ++i) { visc_face_high(C, 1, i, j, k, o); apply(&C.w.F[C.fidx(1, i - 1, j, k - 1)], o); }
#pragma omp parallel for schedule(static) private(o)
  for (int k = a0; k <= nz - a1; ++k)
    for (int j = b0; j <= ny - b1; ++j)
      for (int i = b0; i <= nx - b1; ++i) { visc_face_high(C, 2, i, j, k, o); apply(&C.w.G[C.gidx(1, i - 1, j - 1, k)], o); }
}

// 2D viscous: 2D_solver/src/calc_visc4.f90.fypp (ME4-form, 4th order) and calc_visc2.f90.fypp
void calc_visc2d(Ctx& C) {
  int nx = C.nx, ny = C.ny;
  Prim P{C};
  const Consts& K = C.K;
  const double one_24 = 1.0 / 24.0;
  if (C.c.visc_order == 4) {
    auto d4 = [&](int comp, int ddir, int i, int j) {
      return node_deriv(C, comp, ddir, i, j, 1, false);
    };
    // calc_Ev4 (2D_solver/src/calc_visc4.f90.fypp:36-82): 4th order inside the
    // guard, 2nd-order fallback on the remaining faces
    for (int j = 2; j <= ny - 1; ++j)
      for (int i = 1; i <= nx - 1; ++i) {
        double txx, utxx, txy, vtxy, kT;
        if (3 <= i && i <= nx - 3 && 3 <= j && j <= ny - 2) {
          double mus[6], Ts[6], u[6], v[6], vy[6], uy[6], mu3[3], kT3[3];
          for (int m = 0; m < 6; ++m) {
            mus[m] = P.mu(i - 2 + m, j, 1); Ts[m] = P.T(i - 2 + m, j, 1);
            u[m] = P.u(i - 2 + m, j, 1); v[m] = P.v(i - 2 + m, j, 1);
            vy[m] = d4(1, 1, i - 2 + m, j); uy[m] = d4(0, 1, i - 2 + m, j);
          }
          for (int m = 0; m < 3; ++m) mu3[m] = 0.0625 * (9.0 * (mus[m + 1] + mus[m + 2]) - (mus[m] + mus[m + 3]));
          for (int m = 0; m < 3; ++m)
            kT3[m] = K.Cp_over_Pr * mu3[m] * (1.125 * (-Ts[m + 1] + Ts[m + 2]) - (-Ts[m] + Ts[m + 3]) * one_24) * C.g.xix[i - 1];
          kT = flux4(kT3);
          double t[3];
          for (int m = 0; m < 3; ++m)
            t[m] = two_third * mu3[m] * ((2.25 * (-u[m + 1] + u[m + 2]) - (-u[m] + u[m + 3]) * one_twelfth) * C.g.xix[i - 1] -
                                        0.0625 * (-vy[m] + 9.0 * (vy[m + 1] + vy[m + 2]) - vy[m + 3]));
          txx = (-t[0] + 26.0 * t[1] - t[2]) * one_24;
          for (int m = 0; m < 3; ++m) t[m] = 0.0625 * (-u[m] + 9.0 * (u[m + 1] + u[m + 2]) - u[m + 3]) * t[m];
          utxx = (-t[0] + 26.0 * t[1] - t[2]) * one_24;
          tau_cross_me4(false, mu3, mu3, v, uy, C.g.xix[i - 1], txy, vtxy);
        } else {
          double dxi = C.g.xix[i - 1], dyj = C.g.etay[j - 1];
          double mx = 0.5 * (P.mu(i, j, 1) + P.mu(i + 1, j, 1));
          kT = K.Cp_over_Pr * mx * (-P.T(i, j, 1) + P.T(i + 1, j, 1)) * dxi;
          double my1 = 0.25 * (P.mu(i, j - 1, 1) + P.mu(i, j, 1) + P.mu(i + 1, j - 1, 1) + P.mu(i + 1, j, 1));
          double my2 = 0.25 * (P.mu(i, j, 1) + P.mu(i, j + 1, 1) + P.mu(i + 1, j, 1) + P.mu(i + 1, j + 1, 1));
          double muy = 0.25 * (my1 * (-P.u(i, j - 1, 1) + P.u(i, j, 1) - P.u(i + 1, j - 1, 1) + P.u(i + 1, j, 1)) +
                               my2 * (-P.u(i, j, 1) + P.u(i, j + 1, 1) - P.u(i + 1, j, 1) + P.u(i + 1, j + 1, 1))) * dyj;
          double mvy = 0.25 * (my1 * (-P.v(i, j - 1, 1) + P.v(i, j, 1) - P.v(i + 1, j - 1, 1) + P.v(i + 1, j, 1)) +
                               my2 * (-P.v(i, j, 1) + P.v(i, j + 1, 1) - P.v(i + 1, j, 1) + P.v(i + 1, j + 1, 1))) * dyj;
          double mux = mx * (-P.u(i, j, 1) + P.u(i + 1, j, 1)) * dxi;
          double mvx = mx * (-P.v(i, j, 1) + P.v(i + 1, j, 1)) * dxi;
          txx = two_third * (2.0 * mux - mvy);
          txy = muy + mvx;
          utxx = 0.5 * (P.u(i, j, 1) + P.u(i + 1, j, 1)) * txx;
          vtxy = 0.5 * (P.v(i, j, 1) + P.v(i + 1, j, 1)) * txy;
        }
        double* e = &C.w.E[C.eidx(1, i, j - 1, 1)];
        e[1] = e[1] - txx; e[2] = e[2] - txy; e[3] = e[3] - (utxx + vtxy + kT);
      }
    // calc_Fv4 (2D_solver/src/calc_visc4.f90.fypp:104-152)
    for (int j = 1; j <= ny - 1; ++j)
      for (int i = 2; i <= nx - 1; ++i) {
        double tyy, vtyy, tyx, utyx, kT;
        if (3 <= i && i <= nx - 2 && 3 <= j && j <= ny - 3) {
          double mus[6], Ts[6], u[6], v[6], ux[6], vx[6], mu3[3], kT3[3];
          for (int m = 0; m < 6; ++m) {
            mus[m] = P.mu(i, j - 2 + m, 1); Ts[m] = P.T(i, j - 2 + m, 1);
            u[m] = P.u(i, j - 2 + m, 1); v[m] = P.v(i, j - 2 + m, 1);
            ux[m] = d4(0, 0, i, j - 2 + m); vx[m] = d4(1, 0, i, j - 2 + m);
          }
          for (int m = 0; m < 3; ++m) mu3[m] = 0.0625 * (9.0 * (mus[m + 1] + mus[m + 2]) - (mus[m] + mus[m + 3]));
          for (int m = 0; m < 3; ++m)
            kT3[m] = K.Cp_over_Pr * mu3[m] * (1.125 * (-Ts[m + 1] + Ts[m + 2]) - (-Ts[m] + Ts[m + 3]) * one_24) * C.g.etay[j - 1];
          kT = flux4(kT3);
          double t[3];
          for (int m = 0; m < 3; ++m)
            t[m] = two_third * mu3[m] * ((2.25 * (-v[m + 1] + v[m + 2]) - (-v[m] + v[m + 3]) * one_twelfth) * C.g.etay[j - 1] -
                                        0.0625 * (-ux[m] + 9.0 * (ux[m + 1] + ux[m + 2]) - ux[m + 3]));
          tyy = (-t[0] + 26.0 * t[1] - t[2]) * one_24;
          for (int m = 0; m < 3; ++m) t[m] = 0.0625 * (-v[m] + 9.0 * (v[m + 1] + v[m + 2]) - v[m + 3]) * t[m];
          vtyy = (-t[0] + 26.0 * t[1] - t[2]) * one_24;
          tau_cross_me4(false, mu3, mu3, u, vx, C.g.etay[j - 1], tyx, utyx);
        } else {
          double dxi = C.g.xix[i - 1], dyj = C.g.etay[j - 1];
          double my = 0.5 * (P.mu(i, j, 1) + P.mu(i, j + 1, 1));
          double mx1 = 0.25 * (P.mu(i - 1, j, 1) + P.mu(i, j, 1) + P.mu(i - 1, j + 1, 1) + P.mu(i, j + 1, 1));
          double mx2 = 0.25 * (P.mu(i, j, 1) + P.mu(i + 1, j, 1) + P.mu(i, j + 1, 1) + P.mu(i + 1, j + 1, 1));
          double mux = 0.25 * (mx1 * (-P.u(i - 1, j, 1) + P.u(i, j, 1) - P.u(i - 1, j + 1, 1) + P.u(i, j + 1, 1)) +
                               mx2 * (-P.u(i, j, 1) + P.u(i + 1, j, 1) - P.u(i, j + 1, 1) + P.u(i + 1, j + 1, 1))) * dxi;
          double mvx = 0.25 * (mx1 * (-P.v(i - 1, j, 1) + P.v(i, j, 1) - P.v(i - 1, j + 1, 1) + P.v(i, j + 1, 1)) +
                               mx2 * (-P.v(i, j, 1) + P.v(i + 1, j, 1) - P.v(i, j + 1, 1) + P.v(i + 1, j + 1, 1))) * dxi;
          kT = K.Cp_over_Pr * my * (-P.T(i, j, 1) + P.T(i, j + 1, 1)) * dyj;
          double muy = my * (-P.u(i, j, 1) + P.u(i, j + 1, 1)) * dyj;
          double mvy = my * (-P.v(i, j, 1) + P.v(i, j + 1, 1)) * dyj;
          tyx = muy + mvx;
          tyy = two_third * (2.0 * mvy - mux);
          utyx = 0.5 * (P.u(i, j, 1) + P.u(i, j + 1, 1)) * tyx;
          vtyy = 0.5 * (P.v(i, j, 1) + P.v(i, j + 1, 1)) * tyy;
        }
        double* f = &C.w.F[C.fidx(1, i - 1, j, 1)];
        f[1] = f[1] - tyx; f[2] = f[2] - tyy; f[3] = f[3] - (utyx + vtyy + kT);
      }
  } else {
    // 2D Gaitonde-Visbal (2D_solver/src/calc_visc2.f90.fypp)
    for (int j = 2; j <= ny - 1; ++j)
      for (int i = 1; i <= nx - 1; ++i) {
        double mudx = 0.5 * (P.mu(i, j, 1) + P.mu(i + 1, j, 1)) * C.g.xix[i - 1];
        double vw = K.Cp_over_Pr * mudx * (-P.T(i, j, 1) + P.T(i + 1, j, 1));
        double mux = mudx * (-P.u(i, j, 1) + P.u(i + 1, j, 1));
        double mvx = mudx * (-P.v(i, j, 1) + P.v(i + 1, j, 1));
        double my1 = 0.0625 * (P.mu(i, j - 1, 1) + P.mu(i, j, 1) + P.mu(i + 1, j - 1, 1) + P.mu(i + 1, j, 1));
        double my2 = 0.0625 * (P.mu(i, j, 1) + P.mu(i, j + 1, 1) + P.mu(i + 1, j, 1) + P.mu(i + 1, j + 1, 1));
        double muy = (my1 * (-P.u(i, j - 1, 1) - P.u(i + 1, j - 1, 1)) + (my1 - my2) * (P.u(i, j, 1) + P.u(i + 1, j, 1)) +
                      my2 * (P.u(i, j + 1, 1) + P.u(i + 1, j + 1, 1))) * C.g.etay[j - 1];
        double mvy = (my1 * (-P.v(i, j - 1, 1) - P.v(i + 1, j - 1, 1)) + (my1 - my2) * (P.v(i, j, 1) + P.v(i + 1, j, 1)) +
                      my2 * (P.v(i, j + 1, 1) + P.v(i + 1, j + 1, 1))) * C.g.etay[j - 1];
        double txx = two_third * (2.0 * mux - mvy);
        double txy = muy + mvx;
        vw = vw + 0.5 * ((P.u(i, j, 1) + P.u(i + 1, j, 1)) * txx + (P.v(i, j, 1) + P.v(i + 1, j, 1)) * txy);
        double* e = &C.w.E[C.eidx(1, i, j - 1, 1)];
        e[1] = e[1] - txx; e[2] = e[2] - txy; e[3] = e[3] - vw;
      }
    for (int j = 1; j <= ny - 1; ++j)
      for (int i = 2; i <= nx - 1; ++i) {
        double mudy = 0.5 * (P.mu(i, j, 1) + P.mu(i, j + 1, 1)) * C.g.etay[j - 1];
        double vw = K.Cp_over_Pr * mudy * (-P.T(i, j, 1) + P.T(i, j + 1, 1));
        double muy = mudy * (-P.u(i, j, 1) + P.u(i, j + 1, 1));
        double mvy = mudy * (-P.v(i, j, 1) + P.v(i, j + 1, 1));
        double mx1 = 0.0625 * (P.mu(i - 1, j, 1) + P.mu(i, j, 1) + P.mu(i - 1, j + 1, 1) + P.mu(i, j + 1, 1));
        double mx2 = 0.0625 * (P.mu(i, j, 1) + P.mu(i + 1, j, 1) + P.mu(i, j + 1, 1) + P.mu(i + 1, j + 1, 1));
        double mux = (mx1 * (-P.u(i - 1, j, 1) - P.u(i - 1, j + 1, 1)) + (mx1 - mx2) * (P.u(i, j, 1) + P.u(i, j + 1, 1)) +
                      mx2 * (P.u(i + 1, j, 1) + P.u(i + 1, j + 1, 1))) * C.g.xix[i - 1];
        double mvx = (mx1 * (-P.v(i - 1, j, 1) - P.v(i - 1, j + 1, 1)) + (mx1 - mx2) * (P.v(i, j, 1) + P.v(i, j + 1, 1)) +
                      mx2 * (P.v(i + 1, j, 1) + P.v(i + 1, j + 1, 1))) * C.g.xix[i - 1];
        double tyx = muy + mvx;
        double tyy = two_third * (2.0 * mvy - mux);
        vw = vw + 0.5 * ((P.u(i, j, 1) + P.u(i, j + 1, 1)) * tyx + (P.v(i, j, 1) + P.v(i, j + 1, 1)) * tyy);
        double* f = &C.w.F[C.fidx(1, i - 1, j, 1)];
        f[1] = f[1] - tyx; f[2] = f[2] - tyy; f[3] = f[3] - vw;
      }
  }
}

void calc_efg(Ctx& C, const double* QJ) {
  quantities(C, QJ);
  if (C.c.scheme != ORC_KEEP) ducros(C);
  calc_conv(C);
  if (C.c.visc == ORC_EULER) return;
  if (C.c.dim == 3) {
    if (C.c.visc == ORC_LES) calc_mut(C);
    calc_visc3(C);
  } else {
    calc_visc2d(C);
  }
}

// R for cell (i+1,j+1,k+1), coef-scaled metrics: 3D_solver/src/calc_steps.f90:8-38
void calc_R3(const Ctx& C, int i, int j, int k, double cxy, double cyz, double czx, double R[5]) {
  for (int l = 1; l <= 5; ++l) R[l - 1] = cyz * (-C.w.E[C.eidx(l, i, j, k)] + C.w.E[C.eidx(l, i + 1, j, k)]);
  for (int l = 1; l <= 5; ++l) R[l - 1] = R[l - 1] + czx * (-C.w.F[C.fidx(l, i, j, k)] + C.w.F[C.fidx(l, i, j + 1, k)]);
  for (int l = 1; l <= 5; ++l) R[l - 1] = R[l - 1] + cxy * (-C.w.G[C.gidx(l, i, j, k)] + C.w.G[C.gidx(l, i, j, k + 1)]);
}
// 2D_solver/src/calc_steps.f90:8-28 (4 variables; E/F stored with a 5-slot stride here)
void calc_R2(const Ctx& C, int i, int j, double cdx, double cdy, double R[4]) {
  for (int l = 1; l <= 4; ++l) R[l - 1] = cdy * (-C.w.E[C.eidx(l, i, j, 1)] + C.w.E[C.eidx(l, i + 1, j, 1)]);
  for (int l = 1; l <= 4; ++l) R[l - 1] = R[l - 1] + cdx * (-C.w.F[C.fidx(l, i, j, 1)] + C.w.F[C.fidx(l, i, j + 1, 1)]);
}

// Compute R over the (nx-2)x(ny-2)[x(nz-2)] update region with coef scaling.
// mode: how to combine; see the stage kernels in calc_steps.f90.
void residual(Ctx& C, double coef, std::vector<double>& Rout) {
  int nx = C.nx, ny = C.ny, nz = C.nz, nv = C.nv;
  if (C.c.dim == 3) {
    Rout.assign((size_t)(nx - 2) * nv * (ny - 2) * (nz - 2), 0.0);
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= nz - 2; ++k)
      for (int j = 1; j <= ny - 2; ++j)
        for (int i = 1; i <= nx - 2; ++i) {
          double cxy = coef * C.g.dtdxdy[(size_t)(j - 1) * (nx - 2) + (i - 1)];
          double cyz = coef * C.g.dtdydz[(size_t)(k - 1) * (ny - 2) + (j - 1)];
          double czx = coef * C.g.dtdzdx[(size_t)(k - 1) * (nx - 2) + (i - 1)];
          double R[5];
          calc_R3(C, i, j, k, cxy, cyz, czx, R);
          for (int l = 0; l < 5; ++l)
            Rout[(((size_t)(k - 1) * (ny - 2) + (j - 1)) * nv + l) * (nx - 2) + (i - 1)] = R[l];
        }
  } else {
    Rout.assign((size_t)(nx - 2) * nv * (ny - 2), 0.0);
    for (int j = 1; j <= ny - 2; ++j)
      for (int i = 1; i <= nx - 2; ++i) {
        double cdx = coef * C.g.dtdx[i - 1];
        double cdy = coef * C.g.dtdy[j - 1];
        double R[4];
        calc_R2(C, i, j, cdx, cdy, R);
        for (int l = 0; l < 4; ++l) Rout[((size_t)(j - 1) * nv + l) * (nx - 2) + (i - 1)] = R[l];
      }
  }
}

// ---- ghost / boundary-cell fill ----------------------------------------------------
// Periodic directions: set_bc_common.f90 set_bc_cyclic{2,4,6} (3D :101-273, 2D :74-210).
// Non-periodic directions (bc_x / bc_y = 1): one boundary cell a side, set from the
// adjacent interior cell by the face's rule -- what a case's set_bc does
// (2D_solver/OS/set.f90:50-90: y rows first for every column, then x columns for every
// row; 2D_solver/ST/set.f90: zero-gradient x).  Rules: 0 copy, 1 copy with the normal
// momentum negated, 2 the given values, 3 no-slip wall (the neighbour's density and
// pressure, zero momentum).
// pos: 1-based j (x faces) / i (y faces); (bi, bj), (ni, nj): 1-based boundary cell and
// neighbour, for the Jacobian of the far-field rule
void bc_rule(const Ctx& C, int f, int pos, double* v, int bi, int bj, int ni, int nj) {
  int kind = C.c.bkinds[f] ? (int)C.c.bkinds[f][pos - 1] : C.c.bkind[f];
  if (kind == 1) {
    int n = f < 2 ? 1 : 2;
    v[n] = -v[n];
  } else if (kind == 2) {
    int len = f < 2 ? C.ny : C.nx;
    for (int l = 0; l < C.nv; ++l) v[l] = C.c.bfix[f][(size_t)l * len + (pos - 1)];
  } else if (kind == 3) {  // no-slip wall: 2D_solver/ST/set.f90, 2D_solver/BL0/set.f90 wall rows
    double p_wall = C.K.gamma_1 * (v[3] - 0.5 * (v[1] * v[1] + v[2] * v[2]) / v[0]);
    v[1] = 0.0;
    v[2] = 0.0;
    v[3] = p_wall * C.K.over_gamma_1;
  } else if (kind == 4) {  // far field: Riemann invariants, the top row of 2D_solver/BL0/set.f90
    const double* P = C.c.bpar[f];
    const int n = f < 2 ? 1 : 2, t = 3 - n;
    const double Jn = C.g.jac[(size_t)(nj - 1) * C.nx + (ni - 1)];
    const double Jt = 1.0 / C.g.jac[(size_t)(bj - 1) * C.nx + (bi - 1)];
    const double pin = C.K.gamma_1 * (v[3] - 0.5 * (v[1] * v[1] + v[2] * v[2]) / v[0]) * Jn;
    const double rhoin = v[0] * Jn;
    const double cin = std::sqrt(C.K.gamma * pin / rhoin);
    const double vin = v[n] / v[0];
    const double Rp = vin + 2.0 * cin * C.K.over_gamma_1;
    const double Rm = P[2] - 2.0 * P[3] * C.K.over_gamma_1;
    const double vb = 0.5 * (Rp + Rm);
    const double cb = 0.25 * C.K.gamma_1 * (Rp - Rm);
    const double rhob = std::pow(cb * (1.0 / P[3]), 2.0 * C.K.over_gamma_1) * P[0];
    const double pb = (rhob * (cb * cb)) * (1.0 / C.K.gamma);
    v[0] = rhob * Jt;
    v[t] = rhob * P[1] * Jt;
    v[n] = rhob * vb * Jt;
    v[3] = (pb * C.K.over_gamma_1 + 0.5 * rhob * (P[1] * P[1] + vb * vb)) * Jt;
  } else if (kind == 5) {  // Neumann: 3D_solver/src/set_bc_tbl_sbli.f90:6-36 without w
    const double Jn = C.g.jac[(size_t)(nj - 1) * C.nx + (ni - 1)];
    const double Jt = 1.0 / C.g.jac[(size_t)(bj - 1) * C.nx + (bi - 1)];
    const double over_QJ1 = 1.0 / v[0];
    const double rhob = v[0] * Jn, ub = v[1] * over_QJ1, vb = v[2] * over_QJ1;
    const double pb = C.K.gamma_1 * (v[3] * Jn - 0.5 * rhob * (ub * ub + vb * vb));
    v[0] = rhob * Jt;
    v[1] = rhob * ub * Jt;
    v[2] = rhob * vb * Jt;
    v[3] = (pb * C.K.over_gamma_1 + 0.5 * rhob * (ub * ub + vb * vb)) * Jt;
  }
}

// 3D with non-periodic directions (order 2, one boundary cell a side): the x, y and
// z faces' rules in that order (3D_solver/STZ/set.f90 set_bc), each applied to the
// value the previous ones left beside it.
void fill_ghosts_3d_bnd(const Ctx& C, double* Q) {
  const int n[3] = {C.nx, C.ny, C.nz}, g = C.c.order / 2, nv = C.nv;
  const int bz = C.c.bc_z;
  const bool per[3] = {!C.c.bc_x, !C.c.bc_y, bz == 0};
  const bool blo[3] = {(bool)C.c.bc_x, (bool)C.c.bc_y, bz == 1 || bz == 3};
  const bool bhi[3] = {(bool)C.c.bc_x, (bool)C.c.bc_y, bz == 1 || bz == 4};
  const bool halo_lo = bz == 2 || bz == 4, halo_hi = bz == 2 || bz == 3;
#pragma omp parallel for schedule(static)
  for (int k = 0; k < n[2]; ++k)
    for (int j = 0; j < n[1]; ++j)
      for (int i = 0; i < n[0]; ++i) {
        if ((halo_lo && k < g) || (halo_hi && k >= n[2] - g)) continue;
        const int c[3] = {i, j, k};
        int src[3], cur[3];
        bool bnd[3], inside = true;
        for (int a = 0; a < 3; ++a) {
          src[a] = c[a];
          bnd[a] = false;
          if (per[a]) {
            if (c[a] < g || c[a] >= n[a] - g) {
              src[a] = (c[a] - g + (n[a] - 2 * g)) % (n[a] - 2 * g) + g;
              inside = false;
            }
          } else if ((c[a] == 0 && blo[a]) || (c[a] == n[a] - 1 && bhi[a])) {
            bnd[a] = true;
            src[a] = c[a] == 0 ? 1 : n[a] - 2;
            inside = false;
          }
          cur[a] = src[a];
        }
        if (inside) continue;
        double v[5];
        for (int l = 0; l < nv; ++l) v[l] = Q[C.qidx(src[0] + 1, l + 1, src[1] + 1, src[2] + 1)];
        for (int a = 0; a < 3; ++a) {
          if (!bnd[a]) continue;
          cur[a] = c[a];
          const int f = 2 * a + (c[a] == 0 ? 0 : 1);
          const int kind = f < 4 ? C.c.bkind[f] : C.c.bkindz[f - 4];
          if (kind == 1) {
            v[1 + a] = -v[1 + a];
          } else if (kind == 2) {
            const size_t pos = a == 0 ? cur[1] + (size_t)n[1] * cur[2]
                                      : (a == 1 ? cur[0] + (size_t)n[0] * cur[2] : cur[0] + (size_t)n[0] * cur[1]);
            const size_t len = a == 0 ? (size_t)n[1] * n[2] : (a == 1 ? (size_t)n[0] * n[2] : (size_t)n[0] * n[1]);
            for (int l = 0; l < nv; ++l) v[l] = C.c.bfix3[f][l * len + pos];
          } else if (kind == 3) {
            double p_wall = C.K.gamma_1 * (v[4] - 0.5 * (v[1] * v[1] + v[2] * v[2] + v[3] * v[3]) / v[0]);
            v[1] = 0.0;
            v[2] = 0.0;
            v[3] = 0.0;
            v[4] = p_wall * C.K.over_gamma_1;
          } else if (kind == 4 || kind == 5) {
            // Jacobian(i, j) of the boundary cell and of the cell its value came from
            const int bi = cur[0], bj = cur[1];
            const int ni = a == 0 ? src[0] : cur[0], nj = a == 1 ? src[1] : cur[1];
            const double Jn = C.g.jac[(size_t)nj * C.nx + ni];
            const double Jt = 1.0 / C.g.jac[(size_t)bj * C.nx + bi];
            if (kind == 4) {
              // 3D_solver/src/set_bc_tbl_sbli.f90:38-76 (set_bc_Riemann_tbl_top_down) on y
              // high; on x high the same along x with v the far field's tangential velocity
              const double* P = C.c.bpar[f];
              const int nn = 1 + a, t1 = a == 0 ? 2 : 1, t2 = 3;
              double pin = C.K.gamma_1 * (v[4] - 0.5 * (v[1] * v[1] + v[2] * v[2] + v[3] * v[3]) / v[0]) * Jn;
              double rhoin = v[0] * Jn;
              double cin = std::sqrt(C.K.gamma * pin / rhoin);
              double vin = v[nn] / v[0];
              double Rp = vin + 2.0 * cin * C.K.over_gamma_1;
              double Rm = P[2] - 2.0 * P[3] * C.K.over_gamma_1;
              double vb = 0.5 * (Rp + Rm);
              double cb = 0.25 * C.K.gamma_1 * (Rp - Rm);
              double rhob = std::pow(cb * (1.0 / P[3]), 2.0 * C.K.over_gamma_1) * P[0];
              double pb = (rhob * (cb * cb)) * (1.0 / C.K.gamma);
              v[0] = rhob * Jt;
              v[t1] = rhob * P[1] * Jt;
              v[nn] = rhob * vb * Jt;
              v[t2] = 0.0;
              v[4] = (pb * C.K.over_gamma_1 + 0.5 * rhob * (P[1] * P[1] + vb * vb)) * Jt;
            } else {
              // 3D_solver/src/set_bc_tbl_sbli.f90:6-36 (set_bc_Neumann_tbl_top_down)
              double over_QJ1 = 1.0 / v[0];
              double rhob = v[0] * Jn;
              double ub = v[1] * over_QJ1, vb = v[2] * over_QJ1, wb = v[3] * over_QJ1;
              double pb = C.K.gamma_1 * (v[4] * Jn - 0.5 * rhob * (ub * ub + vb * vb + wb * wb));
              v[0] = rhob * Jt;
              v[1] = rhob * ub * Jt;
              v[2] = rhob * vb * Jt;
              v[3] = rhob * wb * Jt;
              v[4] = (pb * C.K.over_gamma_1 + 0.5 * rhob * (ub * ub + vb * vb + wb * wb)) * Jt;
            }
          }
        }
        for (int l = 0; l < nv; ++l) Q[C.qidx(i + 1, l + 1, j + 1, k + 1)] = v[l];
      }
}

void fill_ghosts(const Ctx& C, double* Q) {
  if (C.c.dim == 3 && (C.c.bc_x || C.c.bc_y || C.c.bc_z == 1 || C.c.bc_z == 3 || C.c.bc_z == 4)) {
    fill_ghosts_3d_bnd(C, Q);
    return;
  }
  int nx = C.nx, ny = C.ny, nz = C.nz, nv = C.nv, g = C.c.order / 2;
  int gx = C.c.bc_x ? 1 : g, gy = C.c.bc_y ? 1 : g;
  int Nx = nx - 2 * gx, Ny = ny - 2 * gy, Nz = nz - 2 * g;
  auto wrap = [](int i, int g, int N) {  // 1-based padded index -> 1-based interior image
    int t = i - g - 1;
    t = ((t % N) + N) % N;
    return t + g + 1;
  };
  // every value comes from interior cells only, so the cells can be set in place in
  // any order
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) {
        // z slab (COMMZ, calc_para.f90:343-384): z ghost planes come from the neighbours
        if (C.c.dim == 3 && C.c.bc_z == 2 && (k <= g || k > nz - g)) continue;
        bool xb = C.c.bc_x && (i == 1 || i == nx), yb = C.c.bc_y && (j == 1 || j == ny);
        int kk = C.c.dim == 3 ? wrap(k, g, Nz) : 1;
        double v[5];
        if (!xb && !yb) {
          int ii = wrap(i, gx, Nx), jj = wrap(j, gy, Ny);
          if (ii == i && jj == j && kk == k) continue;
          for (int l = 1; l <= nv; ++l) Q[C.qidx(i, l, j, k)] = Q[C.qidx(ii, l, jj, kk)];
          continue;
        } else if (xb && yb) {  // corner: the rule applied last, to the other one's boundary value
          int in = i == 1 ? 2 : nx - 1, jn = j == 1 ? 2 : ny - 1;
          for (int l = 1; l <= nv; ++l) v[l - 1] = Q[C.qidx(in, l, jn, kk)];
          if (!C.c.ylast) {
            bc_rule(C, j == 1 ? 2 : 3, in, v, in, j, in, jn);
            bc_rule(C, i == 1 ? 0 : 1, j, v, i, j, in, j);
          } else {
            bc_rule(C, i == 1 ? 0 : 1, jn, v, i, jn, in, jn);
            bc_rule(C, j == 1 ? 2 : 3, i, v, i, j, i, jn);
          }
        } else if (xb) {
          int in = i == 1 ? 2 : nx - 1;
          int jj = C.c.bc_y ? j : wrap(j, gy, Ny);
          for (int l = 1; l <= nv; ++l) v[l - 1] = Q[C.qidx(in, l, jj, kk)];
          bc_rule(C, i == 1 ? 0 : 1, j, v, i, jj, in, jj);
        } else {
          int jn = j == 1 ? 2 : ny - 1;
          int ii = C.c.bc_x ? i : wrap(i, gx, Nx);
          for (int l = 1; l <= nv; ++l) v[l - 1] = Q[C.qidx(ii, l, jn, kk)];
          bc_rule(C, j == 1 ? 2 : 3, i, v, ii, j, ii, jn);
        }
        for (int l = 1; l <= nv; ++l) Q[C.qidx(i, l, j, k)] = v[l - 1];
      }
}

struct Solver {
  Ctx C;
  std::vector<double> QJ2, Rs, R;
};

void init_ctx(Ctx& C, const orc_config* cfg, const double* dx, const double* dy, const double* dz) {
  C.c = *cfg;
  C.K = make_consts(*cfg);
  C.nx = cfg->nx; C.ny = cfg->ny; C.nz = cfg->dim == 3 ? cfg->nz : 1;
  C.nv = cfg->dim + 2;
  size_t npts = (size_t)C.nx * C.ny * C.nz;
  C.w.Q.assign(npts * C.nv, 0.0);
  C.w.T.assign(npts, 0.0);
  C.w.mu.assign(npts, 0.0);
  C.w.mut.assign(npts, 0.0);
  C.w.qc2.assign(npts, 0.0);
  C.w.sensor.assign(npts, 0.0);
  int nzf = cfg->dim == 3 ? C.nz - 2 : 1;
  C.w.E.assign((size_t)5 * (C.nx - 1) * (C.ny - 2) * nzf, 0.0);
  C.w.F.assign((size_t)5 * (C.nx - 2) * (C.ny - 1) * nzf, 0.0);
  if (cfg->dim == 3) C.w.G.assign((size_t)5 * (C.nx - 2) * (C.ny - 2) * (C.nz - 1), 0.0);
  setup_grid(C, dx, dy, dz);
}

// Update cells 2..n-1 (1-based) in each direction, as the step kernels do.
template <class Fn>
void for_update(const Ctx& C, Fn fn) {
  int nx = C.nx, ny = C.ny, nz = C.nz;
  if (C.c.dim == 3) {
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= nz - 2; ++k)
      for (int j = 1; j <= ny - 2; ++j)
        for (int i = 1; i <= nx - 2; ++i) fn(i, j, k);
  } else {
    for (int j = 1; j <= ny - 2; ++j)
      for (int i = 1; i <= nx - 2; ++i) fn(i, j, 1);
  }
}
inline size_t ridx(const Ctx& C, int i, int l, int j, int k) {
  return (((size_t)(k - 1) * (C.ny - 2) + (j - 1)) * C.nv + l) * (C.nx - 2) + (i - 1);
}
inline size_t qup(const Ctx& C, int i, int l, int j, int k) {  // cell (i+1, j+1, k+1)
  return C.qidx(i + 1, l + 1, j + 1, C.c.dim == 3 ? k + 1 : 1);
}

// Stage st of one time step: 3D_solver/src/calc_time_dev.f90.fypp:81-101 (RK3),
// :264-287 (RK4).  QJ holds Q^n (the last stage writes Q^{n+1} into it), QJ2 the
// stage state and Rs the RK4 accumulator, all kept by the caller between stages.
void one_stage(Ctx& C, std::vector<double>& R, double* QJ, double* QJ2, double* Rs, int st) {
  int nv = C.nv;
  if (C.c.rk == 3) {
    if (st == 0) {
      calc_efg(C, QJ);
      residual(C, 1.0, R);
      for_update(C, [&](int i, int j, int k) {
        for (int l = 0; l < nv; ++l) QJ2[qup(C, i, l, j, k)] = QJ[qup(C, i, l, j, k)] - R[ridx(C, i, l, j, k)];
      });
      fill_ghosts(C, QJ2);
    } else if (st == 1) {
      calc_efg(C, QJ2);
      residual(C, 0.25, R);
      for_update(C, [&](int i, int j, int k) {
        for (int l = 0; l < nv; ++l) {
          size_t q = qup(C, i, l, j, k);
          QJ2[q] = (0.75 * QJ[q] + 0.25 * QJ2[q] - R[ridx(C, i, l, j, k)]) * 1.0;
        }
      });
      fill_ghosts(C, QJ2);
    } else {
      calc_efg(C, QJ2);
      residual(C, 2.0, R);
      for_update(C, [&](int i, int j, int k) {
        for (int l = 0; l < nv; ++l) {
          size_t q = qup(C, i, l, j, k);
          QJ[q] = (2.0 * QJ2[q] + 1.0 * QJ[q] - R[ridx(C, i, l, j, k)]) * one_third;
        }
      });
      fill_ghosts(C, QJ);
    }
  } else {
    const double c1[3] = {0.5, 0.5, 1.0}, c2[3] = {1.0, 2.0, 2.0};
    if (st < 3) {
      calc_efg(C, st == 0 ? QJ : QJ2);
      residual(C, 1.0, R);
      for_update(C, [&](int i, int j, int k) {
        for (int l = 0; l < nv; ++l) {
          size_t q = qup(C, i, l, j, k), r = ridx(C, i, l, j, k);
          QJ2[q] = QJ[q] - c1[st] * R[r];
          Rs[r] = Rs[r] + c2[st] * R[r];
        }
      });
      fill_ghosts(C, QJ2);
    } else {
      calc_efg(C, QJ2);
      residual(C, 1.0, R);
      for_update(C, [&](int i, int j, int k) {
        for (int l = 0; l < nv; ++l) {
          size_t q = qup(C, i, l, j, k), r = ridx(C, i, l, j, k);
          double Rl = Rs[r] + R[r];
          QJ[q] = QJ[q] - Rl * one_sixth;
          Rs[r] = 0.0;
        }
      });
      fill_ghosts(C, QJ);
    }
  }
}

void one_step(Solver& S, double* QJ) {
  const int nst = S.C.c.rk == 3 ? 3 : 4;
  for (int st = 0; st < nst; ++st) one_stage(S.C, S.R, QJ, S.QJ2.data(), S.Rs.data(), st);
}

}  // namespace

extern "C" {

// Advance QJ (reference layout, Q/J incl. ghosts) by nsteps time steps.
int orc_step(const orc_config* cfg, const double* dx, const double* dy, const double* dz,
             double* QJ, int nsteps) {
  Solver S;
  init_ctx(S.C, cfg, dx, dy, dz);
  S.QJ2.assign(QJ, QJ + S.C.w.Q.size());
  S.Rs.assign((size_t)(S.C.nx - 2) * S.C.nv * (S.C.ny - 2) * (cfg->dim == 3 ? S.C.nz - 2 : 1), 0.0);
  for (int n = 0; n < nsteps; ++n) one_step(S, QJ);
  return 0;
}

// One RK stage on caller-kept arrays (a z slab's stepping between halo exchanges):
// QJ = Q^n (Q^{n+1} after the last stage), QJ2 = the stage state (same layout),
// Rs = the RK4 accumulator ((nx-2, nv, ny-2, nz-2), zero at the start of a step).
int orc_stage(const orc_config* cfg, const double* dx, const double* dy, const double* dz, double* QJ,
              double* QJ2, double* Rs, int stage) {
  Ctx C;
  init_ctx(C, cfg, dx, dy, dz);
  std::vector<double> R;
  one_stage(C, R, QJ, QJ2, Rs, stage);
  return 0;
}

// The stage residual R = dt*S*(flux differences) for the state QJ (coef = 1),
// over the (nx-2, nv, ny-2[, nz-2]) update region, as calc_R produces it.
int orc_rhs(const orc_config* cfg, const double* dx, const double* dy, const double* dz,
            const double* QJ, double* R_out) {
  Solver S;
  init_ctx(S.C, cfg, dx, dy, dz);
  calc_efg(S.C, QJ);
  residual(S.C, 1.0, S.R);
  std::memcpy(R_out, S.R.data(), S.R.size() * sizeof(double));
  return 0;
}

// Primitive/aux fields of calc_EFG for QJ: fields out (nx,ny,nz) each:
// rho,u,v,w,p,T,mu,sensor,mut,qc2 (10 arrays back to back).
int orc_fields(const orc_config* cfg, const double* dx, const double* dy, const double* dz,
               const double* QJ, double* out) {
  Solver S;
  init_ctx(S.C, cfg, dx, dy, dz);
  calc_efg(S.C, QJ);
  Ctx& C = S.C;
  size_t n = (size_t)C.nx * C.ny * C.nz;
  Prim P{C};
  for (int k = 1; k <= C.nz; ++k)
    for (int j = 1; j <= C.ny; ++j)
      for (int i = 1; i <= C.nx; ++i) {
        size_t s = C.sidx(i, j, k);
        out[0 * n + s] = P.rho(i, j, k); out[1 * n + s] = P.u(i, j, k);
        out[2 * n + s] = P.v(i, j, k); out[3 * n + s] = P.w(i, j, k);
        out[4 * n + s] = P.p(i, j, k); out[5 * n + s] = C.w.T[s];
        out[6 * n + s] = C.w.mu[s]; out[7 * n + s] = C.w.sensor[s];
        out[8 * n + s] = C.w.mut[s]; out[9 * n + s] = C.w.qc2[s];
      }
  return 0;
}

// The Jacobian J(nx,ny) the reference builds from the spacings.
int orc_jacobian(const orc_config* cfg, const double* dx, const double* dy, const double* dz,
                 double* J_out) {
  Ctx C;
  C.c = *cfg; C.nx = cfg->nx; C.ny = cfg->ny; C.nz = cfg->dim == 3 ? cfg->nz : 1;
  C.nv = cfg->dim + 2;
  setup_grid(C, dx, dy, dz);
  std::memcpy(J_out, C.g.jac.data(), C.g.jac.size() * sizeof(double));
  return 0;
}

// Ghost / boundary-cell fill of QJ (the grid's spacings give the Jacobian the
// far-field rule reads).
int orc_fill_ghosts(const orc_config* cfg, const double* dx, const double* dy, const double* dz, double* QJ) {
  Ctx C;
  init_ctx(C, cfg, dx, dy, dz);
  fill_ghosts(C, QJ);
  return 0;
}

// Diagnostics in the reference's form (src/print.f90:42-122): float32 fields,
// running sum rounded to float32 each term; out[0]=ke, out[1]=entropy.
// rho/p (n), vel (3n) are the float32 arrays of make_1d_for_print.
int orc_diag_f32(int nx, int ny, int nz, int order, double gamma, const float* rho_flat,
                 const float* p_flat, const float* vel_flat, double* out) {
  int off = order / 2;
  float ent = 0.0f, ke = 0.0f;
  for (int k = 1 + off; k <= nz - off; ++k)
    for (int j = 1 + off; j <= ny - off; ++j)
      for (int i = 1 + off; i <= nx - off; ++i) {
        size_t l = (size_t)(i - 1) + (size_t)(j - 1) * nx + (size_t)(k - 1) * nx * ny;
        size_t m = 3 * l;
        ent = (float)((double)ent + (double)rho_flat[l] *
                                        std::log((double)p_flat[l] * std::pow((double)rho_flat[l], -gamma)));
        ke = (float)((double)ke + 0.5 * (double)rho_flat[l] *
                                      ((double)vel_flat[m] * vel_flat[m] + (double)vel_flat[m + 1] * vel_flat[m + 1] +
                                       (double)vel_flat[m + 2] * vel_flat[m + 2]));
      }
  double cnt = (double)((long long)(nx - order) * (ny - order) * (nz - order));
  out[0] = (double)(float)((double)ke / cnt);
  out[1] = (double)(float)((double)ent / cnt);
  return 0;
}

}  // extern "C"
