// ice_physics.cuh -- device arithmetic of ICE's dispersed-phase step: closures,
// limiters, MUSCL reconstruction, Riemann solvers, shock sensor, drag, heat,
// evaporation and the cell source.
//
// Every function keeps the reference's operation order (a Fortran chain of * / + -
// evaluates left to right) and the library is compiled with --fmad=false, so the
// plain form (R = double) rounds exactly as the unfused Fortran source does.
// Constants the reference writes as default-real (single precision) literals are
// promoted from float as gfortran promotes them (1e-25 in the closures, 1e-20 in
// drag and tau, 1e+5 in compute_dt).
//
// R is the arithmetic type of reconstruction, Riemann fluxes and sources: double in
// the plain form, float in the FP32-flux form (the RK accumulation, dt and norms stay
// double in both, in ice_gpu.cu).
//
// References (file:line in the ICE sources):
//   closures      physics/Lib_Model_MK.f90:11-184, Lib_Model_IG.f90:11-202, Lib_Model_AG.f90:11-296
//   limiters      numerics/space/Lib_Limiters.f90:314-493
//   reconstruct   numerics/space/Lib_Reconstruction.f90:17-99
//   Riemann       numerics/fluxes/riemann/Lib_Riemann.f90:61-241
//   sensor        numerics/space/Lib_Shock_Detector.f90:17-42
//   drag / heat   physics/Lib_Drag.f90:83-324, physics/Lib_Heat.f90:68-160
//   evaporation   physics/Lib_Evaporation.f90:129-261, 287-545, 738-745
//   source        physics/Mod_Sources.f90:230-274, 465-622
#pragma once
#include <cstdint>
#include <cmath>
#include "../../include/ice_gpu.h"
#include "../../include/ice_math.h"

namespace ice {

constexpr int MK = ICE_CLOSURE_MK, IG = ICE_CLOSURE_IG, AG = ICE_CLOSURE_AG;

template <int CL> struct NC;
template <> struct NC<MK> { static constexpr int v = 6; };
template <> struct NC<IG> { static constexpr int v = 7; };
template <> struct NC<AG> { static constexpr int v = 12; };

constexpr double kPi = 3.14159265358979323846;
constexpr double kSigmaSB = 5.670374419e-8;
constexpr double kRhoEmpty = 1e-6;
constexpr double kThetaCap = 1.0;
constexpr double kRu = 8314.46;
constexpr double kPatm = 101325.0;
constexpr double kXsCap = 1e-12;

// Material constants of one family on the constant-property path, in device-friendly form.
struct Mat {
  double rho, cp, lv, emiss;
  int evap, intf;
  double ep[ICE_GPU_NEP];
};
enum { EP_MV = 0, EP_LV, EP_CPV, EP_LE, EP_YINF, EP_LVMVRU, EP_INVTB, EP_ALPHAE };

template <typename R> __device__ __forceinline__ R epsv() { return (R)(double)1e-25f; }

__device__ __forceinline__ bool not_finite(double x) {
  return ((__double_as_longlong(x) >> 52) & 0x7FF) == 0x7FF;
}
__device__ __forceinline__ bool not_finite(float x) { return !isfinite(x); }

template <typename R> __device__ __forceinline__ R mn(R a, R b) { return b < a ? b : a; }
template <typename R> __device__ __forceinline__ R mx(R a, R b) { return b > a ? b : a; }

// Transcendentals: the deterministic functions of ice_math.h in the plain form (the same bits as
// the host restatement); the fast single-precision intrinsics in the FP32-flux form (whose budget
// is 1e-4 relative L1).
__device__ __forceinline__ double ex(double x) { return ice_exp(x); }
__device__ __forceinline__ double lg(double x) { return ice_log(x); }
__device__ __forceinline__ double lg10(double x) { return ice_log10(x); }
__device__ __forceinline__ double pw(double x, double y) { return ice_pow(x, y); }
__device__ __forceinline__ double th(double x) { return ice_tanh(x); }
__device__ __forceinline__ float ex(float x) { return __expf(x); }
__device__ __forceinline__ float lg(float x) { return __logf(x); }
__device__ __forceinline__ float lg10(float x) { return __log10f(x); }
__device__ __forceinline__ float pw(float x, float y) { return __powf(x, y); }
__device__ __forceinline__ float th(float x) { return tanhf(x); }
// convergence tolerances of the iterative closures: the reference's in FP64; in FP32 the
// iterations stop at single-precision resolution instead of running to their caps
// The Langmuir-Knudsen iteration's relative tolerance: the reference's 1e-12 in FP64; in the FP32-flux
// form 1e-5 (about 80 units in the last place): 1e-6 lies within the rounding noise of the single-
// precision iterates, which then often ran to the 30-iteration cap.
template <typename R> __device__ __forceinline__ R tol_picard() { return sizeof(R) == 8 ? (R)1.e-12 : (R)1.e-5f; }
template <typename R> __device__ __forceinline__ R tol_newton() { return sizeof(R) == 8 ? (R)1.0e-13 : (R)1.0e-6f; }

// Limiters the kernels specialise at compile time; any other runs through the run-time switch.
constexpr int LIM_ANY = -1;

// gfortran NORM2 of three values (scaled sum of squares), Mod_dt.f90:269, Mod_Sources.f90:35
template <typename R> __device__ __forceinline__ R norm2_3(R a, R b, R c) {
  R v[3] = {a, b, c};
  R scale = (R)0, s = (R)1;
#pragma unroll
  for (int m = 0; m < 3; ++m) {
    if (v[m] != (R)0) {
      R ax = fabs(v[m]);
      if (scale < ax) { R q = scale / ax; s = (R)1 + s * q * q; scale = ax; }
      else            { R q = ax / scale; s = s + q * q; }
    }
  }
  return sqrt(s) * scale;
}

// ------------------------------------------------------------------ closures
template <int CL, typename R> __device__ __forceinline__ void prim2cons(const R* p, R* c, R cp) {
  R n2 = p[1]*p[1] + p[2]*p[2] + p[3]*p[3];
  c[0] = p[0];
  c[1] = p[0]*p[1]; c[2] = p[0]*p[2]; c[3] = p[0]*p[3];
  if constexpr (CL == MK) {
    c[4] = p[0]*cp*p[4] + (R)0.5*p[0]*n2;
    c[5] = p[5];
  } else if constexpr (CL == IG) {
    c[4] = p[0]*n2 + (R)3*p[4];
    c[5] = p[0]*cp*p[5] + (R)0.5*c[4];
    c[6] = p[6];
  } else {
    c[4] = p[0]*p[1]*p[1] + p[4];
    c[5] = p[0]*p[1]*p[2] + p[5];
    c[6] = p[0]*p[1]*p[3] + p[6];
    c[7] = p[0]*p[2]*p[2] + p[7];
    c[8] = p[0]*p[2]*p[3] + p[8];
    c[9] = p[0]*p[3]*p[3] + p[9];
    c[10] = p[0]*cp*p[10] + (R)0.5*(c[4] + c[7] + c[9]);
    c[11] = p[11];
  }
}

// cons -> prim with the reference's floors (Lib_Model_*: cons_2_prim_*). FAST (the FP32-flux form):
// the velocities multiply by one reciprocal of the density instead of three divisions.
template <int CL, bool FAST = false> __device__ __forceinline__ void cons2prim(const double* c, double* p, double cp) {
  const double eps = epsv<double>();
  p[0] = c[0];
  if constexpr (FAST) {
    const double inv = 1.0 / (p[0] + eps);
    p[1] = c[1] * inv; p[2] = c[2] * inv; p[3] = c[3] * inv;
  } else {
    p[1] = c[1] / (p[0] + eps); p[2] = c[2] / (p[0] + eps); p[3] = c[3] / (p[0] + eps);
  }
  double n2 = p[1]*p[1] + p[2]*p[2] + p[3]*p[3];
  if constexpr (CL == MK) {
    p[4] = (c[4] - 0.5*p[0]*n2) / (cp*p[0] + eps);
    p[5] = c[5];
    if (p[0] < eps) {
#pragma unroll
      for (int v = 0; v < 6; ++v) p[v] = eps;
    }
    if (p[4] < eps) p[4] = eps;
    if (p[5] < eps) p[5] = eps;
  } else if constexpr (CL == IG) {
    p[4] = 1.0/3.0 * (c[4] - p[0]*n2);
    if (p[0] <= kRhoEmpty && p[4] > p[0]*kThetaCap) p[4] = p[0]*kThetaCap;
    p[5] = (c[5] - 0.5*c[4]) / (cp*p[0] + eps);
    p[6] = c[6];
    if (p[0] < eps) {
#pragma unroll
      for (int v = 0; v < 7; ++v) p[v] = eps;
    }
    if (p[4] < eps) p[4] = eps;
    if (p[5] < eps) p[5] = eps;
    if (p[6] < eps) p[6] = eps;
  } else {
    p[4] = c[4] - p[0]*p[1]*p[1];
    p[5] = c[5] - p[0]*p[1]*p[2];
    p[6] = c[6] - p[0]*p[1]*p[3];
    p[7] = c[7] - p[0]*p[2]*p[2];
    p[8] = c[8] - p[0]*p[2]*p[3];
    p[9] = c[9] - p[0]*p[3]*p[3];
    p[10] = (c[10] - 0.5*(c[4] + c[7] + c[9])) / (cp*p[0] + eps);
    p[11] = c[11];
    if (p[0] <= kRhoEmpty && p[4] + p[7] + p[9] > 3.0*p[0]*kThetaCap) {
      double f = 3.0*p[0]*kThetaCap / (p[4] + p[7] + p[9]);
#pragma unroll
      for (int v = 4; v < 10; ++v) p[v] = p[v] * f;
    }
    if (p[0] < eps) {
#pragma unroll
      for (int v = 0; v < 12; ++v) p[v] = eps;
      p[5] = 0.0; p[6] = 0.0; p[8] = 0.0;
    }
    if (p[4] < eps) p[4] = eps;
    if (fabs(p[5]) < eps) p[5] = 0.0;
    if (fabs(p[6]) < eps) p[6] = 0.0;
    if (p[7] < eps) p[7] = eps;
    if (fabs(p[8]) < eps) p[8] = 0.0;
    if (p[9] < eps) p[9] = eps;
    if (p[10] < eps) p[10] = eps;
    if (p[11] < eps) p[11] = eps;
  }
}

// The chosen form's realizability correction of an occupied AG cell (FP64, after cons -> prim and
// its floors, which keep the density and the diagonal of the covariance positive). Single-precision
// fluxes can carry the covariance P of a nearly singular cell across the positive-definite bound by a
// rounding; the correction takes such a cell back inside. Sylvester's test (P11 > 0 by the floors,
// then the 2 x 2 leading minor and the determinant) passes for a positive definite P at the cost of a
// few products. Otherwise, with D the diagonal of P, the correlation C = D^-1/2 P D^-1/2 = I + O has
// a unit diagonal, and scaling every off-diagonal of P by s scales O by s: the eigenvalues of C become
// 1 + s mu_i. With mu the smallest eigenvalue of O (the trace-free 3 x 3 case of the closed-form
// symmetric eigenvalues, 2 q cos(theta + 2 pi / 3)), a cell whose smallest correlation eigenvalue
// 1 + mu lies in [-kRealizeBand, 0) has its off-diagonals scaled by s = (1 - kRealizeMargin) / -mu,
// so that it becomes kRealizeMargin; the diagonal, hence the trace and the energy, is kept. A larger
// violation is the scheme's own (the reference's FP64 path produces them too, for instance in the
// first steps of a cloud, and keeps them: its floors are all it applies, Lib_Model_AG.f90:81-90), and
// so are cells at or below rho_empty, which keep the reference's dispersion cap: both are left as the
// reference leaves them. Returns true when it changed the state. The plain form never calls it.
constexpr double kRealizeMargin = 1e-6;
constexpr double kRealizeBand = 1e-4;
template <int CL> __device__ __forceinline__ bool realize(double* p) {
  if constexpr (CL != AG) {
    return false;
  } else {
    if (!(p[0] > kRhoEmpty)) return false;
    const double m2 = p[4]*p[7] - p[5]*p[5];
    const double det = p[4]*(p[7]*p[9] - p[8]*p[8]) - p[5]*(p[5]*p[9] - p[8]*p[6]) + p[6]*(p[5]*p[8] - p[7]*p[6]);
    if (m2 > 0.0 && det > 0.0) return false;
    const double c12 = p[5] / sqrt(p[4]*p[7]), c13 = p[6] / sqrt(p[4]*p[9]), c23 = p[8] / sqrt(p[7]*p[9]);
    const double q2 = (c12*c12 + c13*c13 + c23*c23) / 3.0;
    if (!(q2 > 0.0)) return false;
    const double q = sqrt(q2);
    double r = (c12*c13*c23) / (q2*q);
    r = fmin(1.0, fmax(-1.0, r));
    const double mu = 2.0*q*cos(acos(r) / 3.0 + 2.0943951023931957);
    if (!(1.0 + mu < 0.0 && 1.0 + mu >= -kRealizeBand)) return false;
    const double sc = (1.0 - kRealizeMargin) / -mu;
    p[5] = p[5]*sc; p[6] = p[6]*sc; p[8] = p[8]*sc;
    return true;
  }
}

template <int CL, typename R> __device__ __forceinline__ bool check_prim(const R* p) {
  constexpr int nc = NC<CL>::v;
  bool bad = false;
#pragma unroll
  for (int v = 0; v < nc; ++v) bad |= not_finite(p[v]);
  if (bad || p[0] < (R)0) return false;
  if constexpr (CL == IG) { if (p[4] < (R)0) return false; }
  if constexpr (CL == AG) { if (p[4] < (R)0 || p[7] < (R)0 || p[9] < (R)0) return false; }
  return true;
}

template <int CL, typename R> __device__ __forceinline__ R wavespeed(const R* p, const R* n) {
  if constexpr (CL == MK) {
    return (R)0;
  } else if constexpr (CL == IG) {
    R pr = (p[4] + p[4] + p[4]) / (R)3;
    return sqrt((R)3*pr / (p[0] + epsv<R>()));
  } else {
    R pnn = n[0]*(p[4]*n[0] + p[5]*n[1] + p[6]*n[2]) +
            n[1]*(p[5]*n[0] + p[7]*n[1] + p[8]*n[2]) +
            n[2]*(p[6]*n[0] + p[8]*n[1] + p[9]*n[2]);
    return sqrt((R)3*fmax(pnn, (R)0) / (p[0] + epsv<R>()));
  }
}

template <int CL, typename R> __device__ __forceinline__ void flux_make(const R* p, const R* n, R* f, R cp) {
  R n2 = p[1]*p[1] + p[2]*p[2] + p[3]*p[3];
  R un = p[1]*n[0] + p[2]*n[1] + p[3]*n[2];
  f[0] = p[0]*un;
  if constexpr (CL == MK) {
    f[1] = f[0]*p[1]; f[2] = f[0]*p[2]; f[3] = f[0]*p[3];
    f[4] = f[0]*((R)0.5*n2 + cp*p[4]);
    f[5] = p[5]*un;
  } else if constexpr (CL == IG) {
    f[1] = f[0]*p[1] + p[4]*n[0];
    f[2] = f[0]*p[2] + p[4]*n[1];
    f[3] = f[0]*p[3] + p[4]*n[2];
    f[4] = f[0]*n2 + (R)5*p[4]*un;
    f[5] = f[0]*((R)0.5*n2 + cp*p[5]) + (R)2.5*p[4]*un;
    f[6] = p[6]*un;
  } else {
    R p1n = p[4]*n[0] + p[5]*n[1] + p[6]*n[2];
    R p2n = p[5]*n[0] + p[7]*n[1] + p[8]*n[2];
    R p3n = p[6]*n[0] + p[8]*n[1] + p[9]*n[2];
    f[1] = f[0]*p[1] + p1n;
    f[2] = f[0]*p[2] + p2n;
    f[3] = f[0]*p[3] + p3n;
    f[4] = f[0]*p[1]*p[1] + un*p[4] + p[1]*p1n + p[1]*p1n;
    f[5] = f[0]*p[1]*p[2] + un*p[5] + p[1]*p2n + p[2]*p1n;
    f[6] = f[0]*p[1]*p[3] + un*p[6] + p[1]*p3n + p[3]*p1n;
    f[7] = f[0]*p[2]*p[2] + un*p[7] + p[2]*p2n + p[2]*p2n;
    f[8] = f[0]*p[2]*p[3] + un*p[8] + p[2]*p3n + p[3]*p2n;
    f[9] = f[0]*p[3]*p[3] + un*p[9] + p[3]*p3n + p[3]*p3n;
    f[10] = f[0]*((R)0.5*n2 + (R)0.5*(p[4] + p[7] + p[9])/(p[0] + epsv<R>()) + cp*p[10])
          + p[1]*p1n + p[2]*p2n + p[3]*p3n;
    f[11] = p[11]*un;
  }
}

// The pressure part P of a flux, f = un*c + P (zero for MK), as the FP32-flux form splits it.
// Derived from flux_make and prim2cons: IG P_i = p n_i, P_4 = 2 p un, P_5 = p un; AG P_i = (P n)_i,
// P_ij = u_i (P n)_j + u_j (P n)_i, P_10 = u.(P n) - tr(P) un eps / 2(rho + eps).
template <int CL, typename R> __device__ __forceinline__ void press_part(const R* p, const R* n, R un, R* P) {
  constexpr int nc = NC<CL>::v;
#pragma unroll
  for (int v = 0; v < nc; ++v) P[v] = (R)0;
  if constexpr (CL == IG) {
    P[1] = p[4]*n[0]; P[2] = p[4]*n[1]; P[3] = p[4]*n[2];
    P[4] = (R)2*p[4]*un; P[5] = p[4]*un;
  } else if constexpr (CL == AG) {
    R p1n = p[4]*n[0] + p[5]*n[1] + p[6]*n[2];
    R p2n = p[5]*n[0] + p[7]*n[1] + p[8]*n[2];
    R p3n = p[6]*n[0] + p[8]*n[1] + p[9]*n[2];
    P[1] = p1n; P[2] = p2n; P[3] = p3n;
    P[4] = (R)2*p[1]*p1n; P[5] = p[1]*p2n + p[2]*p1n; P[6] = p[1]*p3n + p[3]*p1n;
    P[7] = (R)2*p[2]*p2n; P[8] = p[2]*p3n + p[3]*p2n; P[9] = (R)2*p[3]*p3n;
    P[10] = p[1]*p1n + p[2]*p2n + p[3]*p3n
          - (R)0.5*(p[4] + p[7] + p[9])*un*(epsv<R>()/(p[0] + epsv<R>()));
  }
}

// H P H, H = I - 2 n n^T (Lib_Model_AG.f90:181-200)
__device__ __forceinline__ void mirror_tensor(const double* p, const double* n, double* pm) {
  double t0 = p[0]*n[0] + p[1]*n[1] + p[2]*n[2];
  double t1 = p[1]*n[0] + p[3]*n[1] + p[4]*n[2];
  double t2 = p[2]*n[0] + p[4]*n[1] + p[5]*n[2];
  double s = n[0]*t0 + n[1]*t1 + n[2]*t2;
  pm[0] = p[0] - 4.0*n[0]*t0 + 4.0*s*n[0]*n[0];
  pm[1] = p[1] - 2.0*(n[0]*t1 + t0*n[1]) + 4.0*s*n[0]*n[1];
  pm[2] = p[2] - 2.0*(n[0]*t2 + t0*n[2]) + 4.0*s*n[0]*n[2];
  pm[3] = p[3] - 4.0*n[1]*t1 + 4.0*s*n[1]*n[1];
  pm[4] = p[4] - 2.0*(n[1]*t2 + t1*n[2]) + 4.0*s*n[1]*n[2];
  pm[5] = p[5] - 4.0*n[2]*t2 + 4.0*s*n[2]*n[2];
}

// ------------------------------------------------------------------ limiters
// The slope ratio y / (x + 1e-30). In single precision it is clamped to |r| <= 1e15: a zero slope
// beside a steep one (number densities reach 1e19 m^-4) would overflow to infinity and every
// limiter would return inf/inf; all of them have reached their limit value long before 1e15
// (and cy r > 2 there), so the clamp changes no limited slope.
template <typename R> __device__ __forceinline__ R slope_ratio(R y, R x) {
  R ru = y / (x + (R)1e-30);
  if constexpr (sizeof(R) == 4) ru = fmaxf(fminf(ru, 1e15f), -1e15f);
  return ru;
}

// Single-precision reciprocal by the hardware approximation (relative error about 2^-23): the
// FP32-flux form's divisions by lengths and by the limiter's harmonic sum.
__device__ __forceinline__ float rcp_fast(float x) { return __fdividef(1.0f, x); }

// The FP32-flux form's van Leer and minmod: the same limited slope phi(r) x, r = y / x, written
// without the ratio. Van Leer: for x, y of one sign phi x = 2xy / (x + y), capped as the reference
// caps phi by cx and cy r, i.e. |.| <= cx |x| and <= cy |y|; zero otherwise. Minmod: the smaller of
// x and y in magnitude when they share a sign, else zero. One reciprocal (van Leer) or none
// (minmod) in place of two divisions, and no product x y that could overflow single precision.
__device__ __forceinline__ float vanleer_f(float x, float y, float cx, float cy) {
  const float a = fabsf(x), b = fabsf(y);
  if (!((x > 0.f && y > 0.f) || (x < 0.f && y < 0.f))) return 0.f;
  float h = 2.f * a * (b * rcp_fast(a + b));
  h = fminf(h, fminf(cx * a, cy * b));
  return x > 0.f ? h : -h;
}
__device__ __forceinline__ float minmod_f(float x, float y) {
  if (!((x > 0.f && y > 0.f) || (x < 0.f && y < 0.f))) return 0.f;
  return fabsf(x) < fabsf(y) ? x : y;
}

template <int LIM, typename R> __device__ __forceinline__ R limiter(int lim, R x, R y, R cx, R cy) {
  if constexpr (sizeof(R) == 4 && LIM == ICE_LIM_VANLEER) return vanleer_f(x, y, cx, cy);
  if constexpr (sizeof(R) == 4 && LIM == ICE_LIM_MINMOD) return minmod_f(x, y);
  if constexpr (LIM == ICE_LIM_VANLEER) {
    R ru = slope_ratio(y, x);
    R phi = (ru + fabs(ru)) / ((R)1 + fabs(ru));
    if (ru > (R)0) phi = mn(mn(phi, cx), cy*ru);
    return phi * x;
  } else if constexpr (LIM == ICE_LIM_MINMOD) {
    R ru = slope_ratio(y, x);
    R phi = mx((R)0, mn((R)1, ru));
    return phi * x;
  }
  if (lim == ICE_LIM_IORD) return (R)0;
  R ru = slope_ratio(y, x), phi;
  switch (lim) {
    case ICE_LIM_MINMOD: phi = mx((R)0, mn((R)1, ru)); return phi * x;
    case ICE_LIM_VANALBADA: phi = (ru*ru + ru) / (ru*ru + (R)1); break;
    case ICE_LIM_VANLEER: phi = (ru + fabs(ru)) / ((R)1 + fabs(ru)); break;
    case ICE_LIM_OSPRE: phi = ((R)1.5*(ru*ru + ru)) / (ru*ru + ru + (R)1); break;
    case ICE_LIM_UMIST: phi = mx((R)0, mn(mn(mn((R)2*ru, (R)0.25 + (R)0.75*ru), (R)0.75 + (R)0.25*ru), (R)2)); break;
    case ICE_LIM_OSHER: phi = mx((R)0, mn(ru, (R)1.5)); break;
    case ICE_LIM_SWEBY: phi = mx(mx((R)0, mn((R)1.5*ru, (R)1)), mn(ru, (R)1.5)); break;
    case ICE_LIM_MC: phi = mx((R)0, mn(mn((R)2*ru, (R)0.5*((R)1 + ru)), (R)2)); break;
    case ICE_LIM_KOREN: phi = mx((R)0, mn((R)2*ru, mn(((R)1 + (R)2*ru)/(R)3, (R)2))); break;
    case ICE_LIM_SUPERBEE: phi = mx(mx((R)0, mn((R)2*ru, (R)1)), mn(ru, (R)2)); break;
    default: return (R)0;
  }
  if (ru > (R)0) phi = mn(mn(phi, cx), cy*ru);
  return phi * x;
}

// The four cells of a stencil: a source of values q(s, v), s = 0..3 (prev, local, next, next2).
// state_reconstruction + slope_bounds; returns true when the first-order fallback is itself
// unphysical (report_stencil).
template <int CL, int LIM, typename R, typename Q>
__device__ __forceinline__ bool reconstruct(int lim, const Q& q, R dl0, R dl1, R dl2, R dll, R dlr,
                                            R* pl, R* pr, R beta) {
  constexpr int nc = NC<CL>::v;
  R cxl, cyl, cxr, cyr, limval = beta;
  if (dll > (R)0) { cxl = dl1/dll; cyl = dl0/dll; } else { cxl = (R)2; cyl = (R)2; }
  if (dlr > (R)0) { cxr = dl2/dlr; cyr = dl1/dlr; } else { cxr = (R)2; cyr = (R)2; }
  const R re = (R)kRhoEmpty;
  R r0 = q(0, 0), r1 = q(1, 0), r2 = q(2, 0), r3 = q(3, 0);
  bool first_l = r0 <= re || r1 <= re || r2 <= re;
  bool first_r = r1 <= re || r2 <= re || r3 <= re;
  if (first_l) {
#pragma unroll
    for (int v = 0; v < nc; ++v) pl[v] = q(1, v);
  }
  if (first_r) {
#pragma unroll
    for (int v = 0; v < nc; ++v) pr[v] = q(2, v);
  }
  bool st_l = first_l, st_r = first_r;
  // FP32-flux form: the three lengths' reciprocals once per face in place of a division per variable
  R i0 = (R)1, i1 = (R)1, i2 = (R)1;
  if constexpr (sizeof(R) == 4) { i0 = rcp_fast(dl0); i1 = rcp_fast(dl1); i2 = rcp_fast(dl2); }
  // the weight halves each pass: from any weight <= 1 it is below 1e-18 within 61 passes; the
  // cap only guards a non-finite weight, for which the reference would not end
  for (int pass = 0; (!st_l || !st_r) && pass < 256; ++pass) {
    if (pass == 255) limval = (R)0;
#pragma unroll
    for (int v = 0; v < nc; ++v) {
      R a1 = q(1, v), a2 = q(2, v);
      R slope1 = sizeof(R) == 4 ? (a2 - a1) * i1 : (a2 - a1) / dl1;
      if (!first_l) {
        R slope0 = sizeof(R) == 4 ? (a1 - q(0, v)) * i0 : (a1 - q(0, v)) / dl0;
        R sl = limiter<LIM>(lim, slope1, slope0, cxl, cyl) * limval;
        pl[v] = a1 + sl*dll;
      }
      if (!first_r) {
        R slope2 = sizeof(R) == 4 ? (q(3, v) - a2) * i2 : (q(3, v) - a2) / dl2;
        R sr = limiter<LIM>(lim, slope2, slope1, cxr, cyr) * limval;
        pr[v] = a2 - sr*dlr;
      }
    }
    if (!first_l) st_l = check_prim<CL>(pl);
    if (!first_r) st_r = check_prim<CL>(pr);
    limval = (R)0.5*limval;
    if (limval < (R)1e-18 && !(st_l && st_r)) {
#pragma unroll
      for (int v = 0; v < nc; ++v) { pl[v] = q(1, v); pr[v] = q(2, v); }
      if (!(check_prim<CL>(pl) && check_prim<CL>(pr))) return true;
      break;
    }
  }
  return false;
}

// ------------------------------------------------------------------ Riemann
// The plain form evaluates the reference's formulas in its order. The FP32-flux form evaluates
// Rusanov and the HLLE mixed state in the upwind-split form sum_s ((un_s - S_s) c_s + P_s), which
// is the same expression regrouped: the mass flux it gives from a state is zero exactly when that
// state's weight (un_s - S_s) is, and its other fluxes stay in proportion. Unsplit, a full cell
// moving away from an empty neighbour leaves f - A c = one single-precision rounding of its
// momentum flux with no mass flux beside it, and the neighbour's velocity becomes that residual
// over its near-zero density.
template <typename R> __device__ __forceinline__ void saurel(const R* p1, const R* p4, const R* n, R* f, R cp) {
  R vn1 = p1[1]*n[0] + p1[2]*n[1] + p1[3]*n[2];
  R vn4 = p4[1]*n[0] + p4[2]*n[1] + p4[3]*n[2];
  R vn = (R)0.5*(vn1 + vn4);
  if (vn > (R)0 || vn < (R)0) {
    const R* p = vn > (R)0 ? p1 : p4;
    R vs = vn > (R)0 ? vn1 : vn4;
    R ut = (p[1] - vs*n[0]), vt = (p[2] - vs*n[1]), wt = (p[3] - vs*n[2]);
    R uu = vs*n[0] + ut, vv = vs*n[1] + vt, ww = vs*n[2] + wt;
    f[0] = p[0]*vn;
    f[1] = uu*f[0]; f[2] = vv*f[0]; f[3] = ww*f[0];
    f[4] = f[0]*((R)0.5*(uu*uu + vv*vv + ww*ww) + cp*p[4]);
    f[5] = p[5]*vn;
  } else {
#pragma unroll
    for (int v = 0; v < 6; ++v) f[v] = (R)0;
  }
}

// The FP32-flux form's Rusanov flux with the two states of the face side by side in float2 pairs
// (x: the left state, y: the right), so that one packed FFMA2 / FMUL2 / FADD2 does the work of the two
// sides: the normal speeds, the closure's conservative variables, the pressure parts and the
// normal pressure of the signal speeds. The same operations per side as rusanov's FP32 branch.
__device__ __forceinline__ float2 sp2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

template <int CL> __device__ __forceinline__ void rusanov_pair(const float* p1, const float* p4, const float* n,
                                                               float* f, float cp) {
  constexpr int nc = NC<CL>::v;
  float2 P[nc], C[nc], Q[nc];
#pragma unroll
  for (int v = 0; v < nc; ++v) P[v] = make_float2(p1[v], p4[v]);
  const float2 n0 = sp2(n[0]), n1 = sp2(n[1]), n2 = sp2(n[2]);
  const float2 un = fma2(P[3], n2, fma2(P[2], n1, mul2(P[1], n0)));
  const float2 n2v = fma2(P[3], P[3], fma2(P[2], P[2], mul2(P[1], P[1])));
  // conservative variables (prim2cons)
  C[0] = P[0];
  C[1] = mul2(P[0], P[1]); C[2] = mul2(P[0], P[2]); C[3] = mul2(P[0], P[3]);
  float2 s = sp2(0.f);            // signal speeds
#pragma unroll
  for (int v = 0; v < nc; ++v) Q[v] = sp2(0.f);
  const float eps = epsv<float>();
  if constexpr (CL == MK) {
    C[4] = fma2(mul2(P[0], sp2(cp)), P[4], mul2(mul2(sp2(0.5f), P[0]), n2v));
    C[5] = P[5];
  } else if constexpr (CL == IG) {
    C[4] = fma2(P[0], n2v, mul2(sp2(3.f), P[4]));
    C[5] = fma2(mul2(P[0], sp2(cp)), P[5], mul2(sp2(0.5f), C[4]));
    C[6] = P[6];
    Q[1] = mul2(P[4], n0); Q[2] = mul2(P[4], n1); Q[3] = mul2(P[4], n2);
    Q[4] = mul2(mul2(sp2(2.f), P[4]), un); Q[5] = mul2(P[4], un);
    const float2 pr = mul2(add2(add2(P[4], P[4]), P[4]), sp2(1.f / 3.f));
    s = make_float2(sqrtf(3.f*pr.x / (P[0].x + eps)), sqrtf(3.f*pr.y / (P[0].y + eps)));
  } else {
    const float2 m0 = mul2(P[0], P[1]), m1 = mul2(P[0], P[2]), m2 = mul2(P[0], P[3]);
    C[4] = fma2(m0, P[1], P[4]); C[5] = fma2(m0, P[2], P[5]); C[6] = fma2(m0, P[3], P[6]);
    C[7] = fma2(m1, P[2], P[7]); C[8] = fma2(m1, P[3], P[8]); C[9] = fma2(m2, P[3], P[9]);
    C[10] = fma2(mul2(P[0], sp2(cp)), P[10], mul2(sp2(0.5f), add2(add2(C[4], C[7]), C[9])));
    C[11] = P[11];
    const float2 p1n = fma2(P[6], n2, fma2(P[5], n1, mul2(P[4], n0)));
    const float2 p2n = fma2(P[8], n2, fma2(P[7], n1, mul2(P[5], n0)));
    const float2 p3n = fma2(P[9], n2, fma2(P[8], n1, mul2(P[6], n0)));
    Q[1] = p1n; Q[2] = p2n; Q[3] = p3n;
    Q[4] = mul2(mul2(sp2(2.f), P[1]), p1n); Q[5] = fma2(P[1], p2n, mul2(P[2], p1n)); Q[6] = fma2(P[1], p3n, mul2(P[3], p1n));
    Q[7] = mul2(mul2(sp2(2.f), P[2]), p2n); Q[8] = fma2(P[2], p3n, mul2(P[3], p2n)); Q[9] = mul2(mul2(sp2(2.f), P[3]), p3n);
    const float2 tr = add2(add2(P[4], P[7]), P[9]);
    const float2 e = make_float2(eps / (P[0].x + eps), eps / (P[0].y + eps));
    Q[10] = fma2(P[1], p1n, fma2(P[2], p2n, mul2(P[3], p3n)));
    Q[10] = add2(Q[10], mul2(mul2(mul2(sp2(-0.5f), tr), un), e));
    const float2 pnn = fma2(n2, p3n, fma2(n1, p2n, mul2(n0, p1n)));
    s = make_float2(sqrtf(3.f*fmaxf(pnn.x, 0.f) / (P[0].x + eps)), sqrtf(3.f*fmaxf(pnn.y, 0.f) / (P[0].y + eps)));
  }
  float A = fabsf(un.x - s.x);
  A = fmaxf(A, fabsf(un.y - s.y)); A = fmaxf(A, fabsf(un.x + s.x)); A = fmaxf(A, fabsf(un.y + s.y));
  const float2 a = make_float2(un.x + A, un.y - A);
#pragma unroll
  for (int v = 0; v < nc; ++v) {
    const float2 t = fma2(a, C[v], Q[v]);
    f[v] = 0.5f * (t.x + t.y);
  }
}

template <int CL, typename R> __device__ __forceinline__ void rusanov(const R* p1, const R* p4, const R* n, R* f, R cp) {
  if constexpr (sizeof(R) == 4) {
    rusanov_pair<CL>(p1, p4, n, f, cp);
    return;
  }
  constexpr int nc = NC<CL>::v;
  R c1[nc], c4[nc], f1[nc], f4[nc];
  R vn1 = p1[1]*n[0] + p1[2]*n[1] + p1[3]*n[2];
  R vn4 = p4[1]*n[0] + p4[2]*n[1] + p4[3]*n[2];
  R s1 = wavespeed<CL>(p1, n), s4 = wavespeed<CL>(p4, n);
  prim2cons<CL>(p1, c1, cp); prim2cons<CL>(p4, c4, cp);
  R A = fabs(vn1 - s1);
  A = mx(A, (R)fabs(vn4 - s4)); A = mx(A, (R)fabs(vn1 + s1)); A = mx(A, (R)fabs(vn4 + s4));
  if constexpr (sizeof(R) == 4) {
    press_part<CL>(p1, n, vn1, f1); press_part<CL>(p4, n, vn4, f4);
    R a1 = vn1 + A, a4 = vn4 - A;
#pragma unroll
    for (int v = 0; v < nc; ++v) f[v] = (R)0.5 * ((a1*c1[v] + f1[v]) + (a4*c4[v] + f4[v]));
  } else {
    flux_make<CL>(p1, n, f1, cp); flux_make<CL>(p4, n, f4, cp);
#pragma unroll
    for (int v = 0; v < nc; ++v) f[v] = (R)0.5 * (f1[v] + f4[v] - A*(c4[v] - c1[v]));
  }
}

template <int CL, typename R> __device__ __forceinline__ void hlle(const R* p1, const R* p4, const R* n, R* f, R cp) {
  constexpr int nc = NC<CL>::v;
  R vn1 = p1[1]*n[0] + p1[2]*n[1] + p1[3]*n[2];
  R vn4 = p4[1]*n[0] + p4[2]*n[1] + p4[3]*n[2];
  R s1 = wavespeed<CL>(p1, n), s4 = wavespeed<CL>(p4, n);
  R r1 = sqrt(p1[0]), r4 = sqrt(p4[0]);
  R uR = (r1*p1[1] + r4*p4[1]) / (r1 + r4);
  R vR = (r1*p1[2] + r4*p4[2]) / (r1 + r4);
  R wR = (r1*p1[3] + r4*p4[3]) / (r1 + r4);
  R vnR = uR*n[0] + vR*n[1] + wR*n[2];
  R sR = (r1*s1 + r4*s4) / (r1 + r4);
  R S1 = mn(mn((R)0, vn1 - s1), vnR - sR);
  R S4 = mx(mx((R)0, vn4 + s4), vnR + sR);
  R a0 = -S1, a1 = S1*S4, a2 = S4;
  int loc = 0; R m = a0;
  if (a1 < m) { loc = 1; m = a1; }
  if (a2 < m) { loc = 2; m = a2; }
  if (loc == 0) {
    flux_make<CL>(p1, n, f, cp);
  } else if (loc == 2) {
    flux_make<CL>(p4, n, f, cp);
  } else {
    R f1[nc], f4[nc], c1[nc], c4[nc];
    prim2cons<CL>(p1, c1, cp); prim2cons<CL>(p4, c4, cp);
    if constexpr (sizeof(R) == 4) {
      press_part<CL>(p1, n, vn1, f1); press_part<CL>(p4, n, vn4, f4);
      R a1 = vn1 - S1, a4 = vn4 - S4;
#pragma unroll
      for (int v = 0; v < nc; ++v) f[v] = (S4*(a1*c1[v] + f1[v]) - S1*(a4*c4[v] + f4[v])) / (S4 - S1);
    } else {
      flux_make<CL>(p1, n, f1, cp); flux_make<CL>(p4, n, f4, cp);
#pragma unroll
      for (int v = 0; v < nc; ++v) f[v] = (S4*f1[v] - S1*f4[v] + S1*S4*(c4[v] - c1[v])) / (S4 - S1);
    }
  }
}

template <int CL, int RS, typename R> __device__ __forceinline__ void riemann(const R* p1, const R* p4, const R* n, R* f, R cp) {
  if constexpr (RS == ICE_RIEMANN_SAUREL) saurel<R>(p1, p4, n, f, cp);
  else if constexpr (RS == ICE_RIEMANN_HLLE) hlle<CL>(p1, p4, n, f, cp);
  else rusanov<CL>(p1, p4, n, f, cp);
}

// ------------------------------------------------------------------ exchange
// add_stage_source (Mod_Explicit.f90:257-280) for one cell: the source of slots 1-4 and of the energy slot
// (ie) added to the step's running sum with RK_accumulate's weights (Lib_RK.f90:28-44): stage 1 starts
// it, stage k > 1 makes it (sum + source) * c_k, so that after the last stage it holds what the update
// integrated over the step.
template <int CL>
__device__ __forceinline__ void accumulate_source(double* xstep, long long NI, long long q, const double* s, int first,
                                                  double ck) {
  constexpr int ie = NC<CL>::v == 12 ? 10 : NC<CL>::v == 7 ? 5 : 4;
  const double sv[5] = {s[0], s[1], s[2], s[3], s[ie]};
#pragma unroll
  for (int m = 0; m < 5; ++m) {
    double* a = xstep + (long long)m * NI + q;
    *a = first ? sv[m] : (*a + sv[m]) * ck;
  }
}

// ------------------------------------------------------------------ sensor
// SD_rho (Lib_Shock_Detector.f90:17-42): the Jameson weight of a cell from its density and its six
// neighbours' (r1, r2 along x, r3, r4 along y, r5, r6 along z).
template <typename R>
__device__ __forceinline__ R sd_rho(R r, R r1, R r2, R r3, R r4, R r5, R r6) {
  R kp1 = fabs((r2 - (R)2*r + r1) / (r2 + (R)2*r + r1 + (R)1e-30));
  R kp2 = fabs((r4 - (R)2*r + r3) / (r4 + (R)2*r + r3 + (R)1e-30));
  R kp3 = fabs((r6 - (R)2*r + r5) / (r6 + (R)2*r + r5 + (R)1e-30));
  R sw = mx(mx(kp1, kp2), kp3);
  if (sw < (R)(1.0/20.0)) {
    R phi = mx(sw*(R)20, (R)0);
    return (R)1 - th((R)10*phi*phi*phi);
  }
  return (R)0;
}

// ------------------------------------------------------------------ drag
template <typename R> __device__ __forceinline__ R toll_d() { return (R)(double)1e-20f; }

template <typename R> __device__ __forceinline__ R drag_wen_yu(R Re) {
  if (Re <= (R)1000) return (R)24/(Re + toll_d<R>()) * ((R)1 + (R)0.15*pw(Re, (R)0.687));
  return (R)0.43;
}
template <typename R> __device__ R henderson1(R Re, R Ma, R G, R Tr) {
  const R t = toll_d<R>();
  R sg = pw((R)0.5*G, (R)0.5);
  R X = Re + Ma*sg*((R)4.33 + ((R)3.65 - (R)1.53*Tr)/((R)1 + (R)0.353*Tr)*ex(-(R)0.247*Re/(Ma*sg + t))) + t;
  R rs = pw(Re, (R)0.5);
  return (R)24*pw(X, (R)-1)
       + ex(-(R)0.5*Ma/(rs + t))*(((R)4.5 + (R)0.38*((R)0.03*Re + (R)0.48*rs)) / ((R)1 + (R)0.03*Re + (R)0.48*rs)
                                   + (R)0.1*(Ma*Ma) + (R)0.2*pw(Ma, (R)8))
       + (R)0.6*Ma*sg*((R)1 - ex(-Ma/(Re + t)));
}
template <typename R> __device__ R henderson2(R Re, R Ma, R G, R Tr) {
  const R t = toll_d<R>();
  R q = pw(Ma/(Re + t), (R)0.5);
  return ((R)0.9 + (R)0.34/((Ma*Ma) + t) + (R)1.86*q*((R)2 + (R)2/(Ma*Ma*(R)0.5*G + t)
          + ((R)1.058/(Ma*pw((R)0.5*G, (R)0.5) + t))*pw(Tr, (R)0.5)) - (R)1/(pw(Ma, (R)4)*(G*G)*(R)0.25 + t))
         / ((R)1 + (R)1.86*q);
}
template <typename R> __device__ R drag(R Re, R Ma, R G, R Tr, int sel) {
  const R t = toll_d<R>();
  switch (sel) {
    case 1: return (R)0.45;
    case 2: return (R)24/(Re + t);
    case 3: return (R)24/(Re + t) * ((R)1 + (R)3*Re/(R)16);
    case 4: return (R)24/(Re + t) * ((R)1 + (R)0.15*pw(Re, (R)0.687));
    case 5: return drag_wen_yu(Re);
    case 6: if (Re < (R)1000) return (R)24/(Re + t) * ((R)1 + pw(Re, (R)(2.0/3.0))/(R)6); return (R)0.4392;
    case 7: return (R)24/(Re + t) * ((R)1 + (R)0.15*pw(Re, (R)0.687) + (R)0.0175*Re/((R)1 + (R)4.25*(R)1e4*pw(Re, (R)-1.16)));
    case 8: {
      R a1, a2, a3;
      if (Re <= (R)0.1) { a1 = 0; a2 = 24; a3 = 0; }
      else if (Re <= (R)1.0) { a1 = (R)3.69; a2 = (R)22.73; a3 = (R)0.0903; }
      else if (Re <= (R)10) { a1 = (R)1.222; a2 = (R)29.1667; a3 = (R)-3.8889; }
      else if (Re <= (R)100) { a1 = (R)0.6167; a2 = (R)46.5; a3 = (R)-116.67; }
      else if (Re <= (R)1000) { a1 = (R)0.3644; a2 = (R)98.33; a3 = (R)-2778; }
      else if (Re <= (R)5000) { a1 = (R)0.357; a2 = (R)148.62; a3 = (R)-4.75e+4; }
      else if (Re <= (R)10000) { a1 = (R)0.46; a2 = (R)-490.546; a3 = (R)57.87e+4; }
      else { a1 = (R)0.5191; a2 = (R)-1662.5; a3 = (R)5.4167e+6; }
      return a1 + a2/(Re + t) + a3/(Re*Re + t);
    }
    case 9: {
      R Cd0 = drag_wen_yu(Re);
      return Cd0 * ((R)1 + ex(-(R)0.427/(pw(Ma, (R)4.63) + t) - (R)3/(pw(Re, (R)0.88) + t))) /
             ((R)1 + Ma/(Re + t)*((R)3.82 + (R)1.28*ex(-(R)1.25*Re/(Ma + t))));
    }
    case 10:
      if (Ma <= (R)1) return henderson1(Re, Ma, G, Tr);
      if (Ma >= (R)1.75) return henderson2(Re, Ma, G, Tr);
      {
        R Cd1 = henderson1(Re, (R)1, G, Tr), Cd2 = henderson2(Re, (R)1.75, G, Tr);
        return Cd1 + (R)(4.0/3.0)*(Ma - (R)1)*(Cd2 - Cd1);
      }
    case 11: {
      R g = (R)1.25*((R)1 + th((R)0.77*lg10(Re + t) - (R)1.92));
      g = pw((R)10, g);
      R h = (R)2.3 + (R)1.7*pw(Tr, (R)0.5) - (R)2.3*th((R)1.17*lg10(Ma + t));
      R Cd0 = drag_wen_yu(Re);
      return (R)2 + (Cd0 - (R)2)*ex(-(R)3.07*pw(G, (R)0.5)*Ma*g/(Re + t)) + h/(Ma*pw(G, (R)0.5) + t)*ex(-Re/((R)2*Ma + t));
    }
    case 12: {
      R g = ((R)1 + Re*((R)12.278 + (R)0.548*Re)) / ((R)1 + (R)11.278*Re);
      R h = (R)5.6/((R)1 + Ma) + (R)1.7*pw(Tr, (R)0.5);
      R Cd0 = drag_wen_yu(Re);
      return (R)2 + (Cd0 - (R)2)*ex(-(R)3.07*pw(G, (R)0.5)*Ma*g/(Re + t)) + h/(Ma*pw(G, (R)0.5) + t)*ex(-Re/((R)2*Ma + t));
    }
    case 13: return (R)0;
  }
  return (R)0;
}

// ------------------------------------------------------------------ heat
template <typename R> __device__ R heat(R Re, R Pr, R Ma, int sel) {
  const R t = (R)1e-20;
  switch (sel) {
    case 1: return (R)2;
    case 2: return (R)2.5*pw(Re, (R)0.15) + (R)0.04*Re;
    case 3: return (R)2 + (R)0.37*pw(Re, (R)0.6)*pw(Pr, (R)(1.0/3.0));
    case 4: return (R)2 + (R)0.459*pw(Re, (R)0.55)*pw(Pr, (R)(1.0/3.0));
    case 5: return pw(pw((R)2 + (R)0.654*pw(Re, (R)0.5)*pw(Pr, (R)0.5), (R)-1) + (R)3.42*Ma/(Re*Pr + t), (R)-1);
    case 6: return (R)2 + (R)0.6*pw(Re, (R)0.5)*pw(Pr, (R)(1.0/3.0));
    case 7: {
      R Nu = (R)2 + (R)0.459*pw(Re, (R)0.55)*pw(Pr, (R)0.33);
      return Nu / ((R)1 + (R)3.42*Ma/(Re*Pr + t)*Nu);
    }
    case 8: return (R)0;
  }
  return (R)0;
}

// ------------------------------------------------------------------ evaporation
template <typename R> __device__ __forceinline__ R blowing(R gamma, R Rg, R mug, R kg, R rhop, R dp, R mp, R mdot) {
  if (mdot >= (R)0 || mp <= (R)0 || mug <= (R)0 || kg <= (R)0) return (R)1;
  if (dp <= (R)0 || rhop <= (R)0 || gamma <= (R)1) return (R)1;
  R cpg = gamma*Rg/(gamma - (R)1);
  R Pr = mug*cpg/kg;
  R taud = rhop*dp*dp/((R)18*mug);
  R b = -(R)1.5*Pr*taud*mdot/mp;
  if (b != b || b <= (R)1e-10) return (R)1;
  if (b > (R)500) return (R)0;
  return b/(ex(b) - (R)1);
}

template <typename R> __device__ __forceinline__ R molar2mass(R Xs, R Mv, R Mg) { return Xs*Mv/(Xs*Mv + ((R)1 - Xs)*Mg); }
template <typename R> __device__ __forceinline__ R mass2molar(R Ys, R Mv, R Mg) { return Ys*Mg/(Ys*Mg + ((R)1 - Ys)*Mv); }
template <typename R> __device__ __forceinline__ R Fcorr(R B) { return B > (R)1.0e-10 ? pw((R)1 + B, (R)0.7)*lg((R)1 + B)/B : (R)1; }

template <typename R> struct EvapEnv {
  R rhog, Tg, gamma, Rg, mug, kg, Tp, dp, cpg, p, Mg, Pr, Sc, Re05;
  R Dv, Sh;          // CEM's vapour diffusivity and Sherwood number: the same for every call of a cell
  int evap;
  const double* ep;
};

// The parts of the gas-side rate that do not depend on the surface state (every Langmuir-Knudsen
// iteration of a cell calls gas_side with the same environment): once per cell, the same expressions.
template <typename R> __device__ __forceinline__ void evap_invariants(EvapEnv<R>& e) {
  if (e.evap == 2) {
    e.Dv = e.kg/(e.rhog*e.cpg*(R)e.ep[EP_LE]);
    e.Sh = (R)2 + (R)0.6*e.Re05*pw(e.Sc, (R)(1.0/3.0));
  }
}

// gasSideRate with the five gas-side models (Lib_Evaporation.f90:205-224, 287-521)
template <typename R> __device__ void gas_side(const EvapEnv<R>& e, R Ys, R BM, R& md, R& Qd, bool& ovr) {
  const R pi = (R)kPi;
  md = (R)0; Qd = (R)0; ovr = false;
  const double* ep = e.ep;
  switch (e.evap) {
    case 1: {
      R BT = e.cpg*(e.Tg - e.Tp)/(R)ep[EP_LV];
      if (BT <= (R)0) { md = (R)0; return; }
      md = -(R)2*pi*e.dp*e.kg/e.cpg*lg((R)1 + BT);
      return;
    }
    case 2: {
      md = -pi*e.dp*e.rhog*e.Dv*e.Sh*lg((R)1 + BM);
      return;
    }
    case 3: {
      R Tf = e.Tp + (e.Tg - e.Tp)/(R)3;
      R rho_f = e.rhog*e.Tg/Tf;
      R mu_f = e.mug*pw(Tf/e.Tg, (R)0.7);
      R kl_f = e.kg*pw(Tf/e.Tg, (R)0.7);
      R cpg_f = e.cpg;
      R Le = (R)ep[EP_LE];
      R Dv_f = kl_f/(rho_f*cpg_f*Le);
      R Sc_f = mu_f*cpg_f*Le/kl_f;
      R Re_f = e.Re05*e.Re05*rho_f/e.rhog*e.mug/mu_f;
      R Sh_f = (R)2 + (R)0.6*sqrt(mx(Re_f, (R)0))*pw(Sc_f, (R)(1.0/3.0));
      md = -pi*e.dp*rho_f*Dv_f*Sh_f*lg((R)1 + BM);
      return;
    }
    case 4: {
      R Le = (R)ep[EP_LE], cpv = (R)ep[EP_CPV];
      ovr = true;
      R Dv = e.kg/(e.rhog*e.cpg*Le);
      R lnBM = lg((R)1 + BM);
      R FM = Fcorr(BM);
      R Sh0 = (R)2 + (R)0.552*e.Re05*pw(e.Sc, (R)(1.0/3.0));
      R Shs = (R)2 + (Sh0 - (R)2)/FM;
      md = -pi*e.dp*e.rhog*Dv*Shs*lnBM;
      R cpv_eff = cpv > (R)0 ? cpv : e.cpg;
      R Nu0 = (R)2 + (R)0.552*e.Re05*pw(e.Pr, (R)(1.0/3.0));
      R Nus = Nu0, BT = (R)0;
      for (int it = 1; it <= 5; ++it) {
        R phi = cpv_eff/e.cpg*Shs/Nus/Le;
        BT = pw((R)1 + BM, phi) - (R)1;
        if (BT <= (R)0) { BT = BM; Nus = Nu0; break; }
        R FT = Fcorr(BT);
        Nus = (R)2 + (Nu0 - (R)2)/FT;
      }
      Qd = BT > (R)0 ? -md*cpv_eff*(e.Tg - e.Tp)/BT : (R)0;
      return;
    }
    case 5: {
      R Le = (R)ep[EP_LE], cpv = (R)ep[EP_CPV], Yinf = (R)ep[EP_YINF], Mv = (R)ep[EP_MV];
      R Dv = e.kg/(e.rhog*e.cpg*Le);
      R cpv_eff = cpv > (R)0 ? cpv : e.cpg;
      R Xs = mn(mass2molar(Ys, Mv, e.Mg), (R)1 - (R)kXsCap);
      R Xinf = mass2molar(Yinf, Mv, e.Mg);
      R Minf = Xinf*Mv + ((R)1 - Xinf)*e.Mg;
      R rhs0 = Mv/Minf*lg(((R)1 - Xinf)/((R)1 - Xs));
      if (rhs0 <= (R)0) return;
      R Tts = e.Tp/e.Tg;
      R Lev = e.kg/(cpv_eff*Dv*e.rhog);
      R mlo = rhs0/mx(Tts, (R)1);
      R mhi = rhs0/mn(mx(Tts, (R)1.0e-3), (R)1);
      R mhat = rhs0;
      for (int it = 1; it <= 30; ++it) {
        R x = mhat/Lev, f, fp;
        if (x > (R)1.0e-6) {
          R E = ex(-x);
          f = x/((R)1 - E);
          fp = ((R)1 - E - x*E)/(((R)1 - E)*((R)1 - E));
        } else {
          f = (R)1 + (R)0.5*x + x*x/(R)12;
          fp = (R)0.5 + x/(R)6;
        }
        R G = mhat + (Tts - (R)1)*Lev*(f - (R)1) - rhs0;
        R dG = (R)1 + (Tts - (R)1)*fp;
        if (fabs(G) <= tol_newton<R>()*mx((R)1, rhs0)) break;
        if (G > (R)0) mhi = mhat; else mlo = mhat;
        mhat = mhat - G/dG;
        if (mhat <= mlo || mhat >= mhi) mhat = (R)0.5*(mlo + mhi);
      }
      R Sh = (R)2 + (R)0.6*e.Re05*pw(e.Sc, (R)(1.0/3.0));
      md = -pi*e.dp*e.rhog*Dv*Sh*mhat;
      ovr = true;
      R Nu = (R)2 + (R)0.6*e.Re05*pw(e.Pr, (R)(1.0/3.0));
      R chi = mn(-md*cpv_eff/(pi*e.dp*e.kg*Nu), (R)700);
      if (chi > (R)1.0e-9) Qd = -md*cpv_eff*(e.Tg - e.Tp)/(ex(chi) - (R)1);
      else Qd = pi*e.dp*e.kg*Nu*(e.Tg - e.Tp);
      return;
    }
  }
}

// evaporation + lkCorrection (Lib_Evaporation.f90:145-261)
template <typename R> __device__ void evaporation(R rhog, R Tg, R gamma, R Rg, R mug, R kg, R Tp, R dp, R Re,
                                                  const Mat& m, R& mdot, R& Qd, bool& ovr) {
  mdot = (R)0; Qd = (R)0; ovr = false;
  if (m.evap == 0) return;
  const double* ep = m.ep;
  EvapEnv<R> e;
  e.rhog = rhog; e.Tg = Tg; e.gamma = gamma; e.Rg = Rg; e.mug = mug; e.kg = kg; e.Tp = Tp; e.dp = dp;
  e.evap = m.evap; e.ep = ep;
  e.cpg = gamma*Rg/(gamma - (R)1);
  e.p = rhog*Rg*Tg;
  e.Mg = (R)kRu/Rg;
  R psat = (R)kPatm*ex(-(R)ep[EP_LVMVRU]*((R)1/Tp - (R)ep[EP_INVTB]));
  R Xs = psat >= e.p ? (R)1 - (R)kXsCap : mn(psat/e.p, (R)1 - (R)kXsCap);
  R Ys = molar2mass(Xs, (R)ep[EP_MV], e.Mg);
  if (Ys <= (R)ep[EP_YINF]) return;
  R BM = (Ys - (R)ep[EP_YINF])/((R)1 - Ys);
  if (BM <= (R)0) return;
  e.Re05 = sqrt(mx(Re, (R)0));
  e.Pr = mug*e.cpg/kg;
  e.Sc = e.Pr*(R)ep[EP_LE];
  evap_invariants(e);
  gas_side(e, Ys, BM, mdot, Qd, ovr);
  if (m.intf != 1) return;
  const R pi = (R)kPi;
  R LKd2 = (R)2*mug*sqrt((R)2*pi*Tp*(R)kRu/(R)ep[EP_MV])/((R)ep[EP_ALPHAE]*e.Sc*e.p)/dp;
  R diffPrev = (R)(sizeof(R) == 8 ? 1.79769313486231570e+308 : 3.40282347e+38);
  R md = mdot, mdNew = (R)0, QdNew = (R)0;
  bool ovrNew = false;
  for (int it = 1; it <= 30; ++it) {
    R beta = -md*e.Pr/((R)2*pi*mug*dp);
    R XsN = mx(Xs - LKd2*beta, (R)0);
    R YsN = molar2mass(XsN, (R)ep[EP_MV], e.Mg);
    mdNew = (R)0; QdNew = (R)0; ovrNew = false;
    if (YsN > (R)ep[EP_YINF]) {
      R BMN = (YsN - (R)ep[EP_YINF])/((R)1 - YsN);
      if (BMN > (R)0) gas_side(e, YsN, BMN, mdNew, QdNew, ovrNew);
    }
    R diff = fabs(mdNew - md);
    if (diff <= tol_picard<R>()*fabs(mdNew)) { mdot = mdNew; Qd = QdNew; ovr = ovrNew; return; }
    if (diff < diffPrev) md = mdNew; else md = (R)0.5*(md + mdNew);
    diffPrev = diff;
  }
  mdot = mdNew; Qd = QdNew; ovr = ovrNew;
}

// source_make_{MK,IG,AG}
template <int CL, typename R> __device__ __forceinline__ void source_make(const R* p, const R* F, R* s, R cp, R lv) {
  const R eps = epsv<R>();
  s[0] = -F[0];
  s[1] = -F[0]*p[1] + p[0]*F[1]/(F[5] + eps);
  s[2] = -F[0]*p[2] + p[0]*F[2]/(F[5] + eps);
  s[3] = -F[0]*p[3] + p[0]*F[3]/(F[5] + eps);
  if constexpr (CL == MK) {
    R n2 = p[1]*p[1] + p[2]*p[2] + p[3]*p[3];
    s[4] = -F[0]*((R)0.5*n2 + cp*p[4]) - F[0]*lv + F[4] + p[0]*(F[1]*p[1] + F[2]*p[2] + F[3]*p[3])/(F[5] + eps);
    s[5] = (R)0;
  } else if constexpr (CL == IG) {
    R n2 = p[1]*p[1] + p[2]*p[2] + p[3]*p[3];
    s[4] = -F[0]*(n2 + (R)3*p[4]/p[0]) + (R)2*p[0]*(F[1]*p[1] + F[2]*p[2] + F[3]*p[3])/(F[5] + eps)
           - (R)6*p[4]/(F[5] + eps);
    s[5] = -F[0]*cp*p[5] - F[0]*lv + F[4] + (R)0.5*s[4];
    s[6] = (R)0;
  } else {
    s[4] = -F[0]*(p[1]*p[1] + p[4]/p[0]) + p[0]*(F[1]*p[1] + F[1]*p[1])/(F[5] + eps) - (R)2*p[4]/(F[5] + eps);
    s[5] = -F[0]*(p[1]*p[2] + p[5]/p[0]) + p[0]*(F[2]*p[1] + F[1]*p[2])/(F[5] + eps) - (R)2*p[5]/(F[5] + eps);
    s[6] = -F[0]*(p[1]*p[3] + p[6]/p[0]) + p[0]*(F[3]*p[1] + F[1]*p[3])/(F[5] + eps) - (R)2*p[6]/(F[5] + eps);
    s[7] = -F[0]*(p[2]*p[2] + p[7]/p[0]) + p[0]*(F[2]*p[2] + F[2]*p[2])/(F[5] + eps) - (R)2*p[7]/(F[5] + eps);
    s[8] = -F[0]*(p[2]*p[3] + p[8]/p[0]) + p[0]*(F[3]*p[2] + F[2]*p[3])/(F[5] + eps) - (R)2*p[8]/(F[5] + eps);
    s[9] = -F[0]*(p[3]*p[3] + p[9]/p[0]) + p[0]*(F[3]*p[3] + F[3]*p[3])/(F[5] + eps) - (R)2*p[9]/(F[5] + eps);
    s[10] = -F[0]*cp*p[10] - F[0]*lv + F[4] + (R)0.5*s[4] + (R)0.5*s[7] + (R)0.5*s[9];
    s[11] = (R)0;
  }
}

// The per-particle quantities compute_source_ forms before the evaporation call (Mod_Sources.f90:
// 465-519), the ITC/clamp, non-burning, constant-property path.
template <typename R> struct CellPhys {
  R T, n, rho_mat, Rp, du, Re, Ma, Pr, Nu, Cd;
};
template <int CL, typename R> __device__ __forceinline__ CellPhys<R> cell_phys(const R* p, const R* gas, R gR, R ggam,
                                                                              R gk, R gmu, const Mat& m, int drag_sel,
                                                                              int heat_sel) {
  constexpr int nb = NC<CL>::v;
  const R pi = (R)kPi;
  CellPhys<R> c;
  c.T = p[nb - 2]; c.n = p[nb - 1];
  c.rho_mat = (R)m.rho;
  c.Rp = pw((R)0.75*p[0]/(c.n*pi*c.rho_mat), (R)(1.0/3.0));
  c.du = norm2_3(gas[1] - p[1], gas[2] - p[2], gas[3] - p[3]);
  c.Re = (R)2*gas[0]*c.Rp*c.du/gmu;
  c.Ma = c.du/pw(ggam*gR*gas[4], (R)0.5);
  c.Pr = ggam/(ggam - (R)1)*gR*gmu/gk;
  c.Nu = heat(c.Re, c.Pr, c.Ma, heat_sel);
  R Tr = c.T/gas[4];
  c.Cd = drag(c.Re, c.Ma, ggam, Tr, drag_sel);
  return c;
}

// The rest of compute_source_ from the mass and heat transfer rates (Mod_Sources.f90:552-622):
// mass, momentum and energy sources with radiation, the relaxation time, source_make. Returns tau
// (INF when Cd == 0).
template <int CL, typename R> __device__ __forceinline__ R cell_source_finish(const CellPhys<R>& c, const R* p,
                                                                             const R* gas, const Mat& m, R mdot,
                                                                             R Qconv, R* s) {
  const R pi = (R)kPi;
  R F[6];
  F[1] = gas[1] - p[1]; F[2] = gas[2] - p[2]; F[3] = gas[3] - p[3];
  F[0] = -mdot*c.n;
  F[4] = Qconv*c.n;
  F[4] = F[4] + (R)m.emiss*(R)kSigmaSB*(R)4*pi*c.Rp*c.Rp*c.n*(pw(gas[4], (R)4) - pw(c.T, (R)4));
  R tau;
  if (c.Cd == (R)0) tau = (R)INFINITY;
  else tau = (R)8*c.rho_mat*c.Rp/((R)3*gas[0]*c.Cd*c.du + toll_d<R>());
  F[5] = tau;
  source_make<CL>(p, F, s, (R)m.cp, (R)m.lv);
  return tau;
}

// The plain closure's mass and heat transfer rates (compute_source_'s evaporation part): heat
// correlation, evaporation with its interface model, override or blowing.
template <typename R> __device__ __forceinline__ void closure_rates(R rhog, R Tg, R gam, R gR, R gmu, R gk, R Ts, R Rp,
                                                                   R Re, R Nu, const Mat& m, int blow, R& mdot, R& Qconv) {
  const R pi = (R)kPi;
  Qconv = (R)2*Nu*gk*pi*Rp*(Tg - Ts);
  R Qevap; bool ovr;
  evaporation<R>(rhog, Tg, gam, gR, gmu, gk, Ts, (R)2*Rp, Re, m, mdot, Qevap, ovr);
  if (ovr) Qconv = Qevap;
  else if (blow == 1) Qconv = Qconv*blowing<R>(gam, gR, gmu, gk, (R)m.rho, (R)2*Rp, (R)(4.0/3.0)*pi*(Rp*Rp*Rp)*(R)m.rho, mdot);
}

// compute_source_ + cell_surface on the ITC/clamp, non-burning, constant-property path.
// gas = rho u v w T. Returns tau. INF when Cd == 0.
template <int CL, typename R> __device__ R cell_source(const R* p, const R* gas, R gR, R ggam, R gk, R gmu,
                                                      const Mat& m, int drag_sel, int heat_sel, int blow, R* s) {
  const CellPhys<R> c = cell_phys<CL, R>(p, gas, gR, ggam, gk, gmu, m, drag_sel, heat_sel);
  R mdot, Qconv;
  closure_rates<R>(gas[0], gas[4], ggam, gR, gmu, gk, c.T, c.Rp, c.Re, c.Nu, m, blow, mdot, Qconv);
  return cell_source_finish<CL, R>(c, p, gas, m, mdot, Qconv, s);
}

}  // namespace ice
