/*
 * ice_oracle_physics.h -- TEST INFRASTRUCTURE. The CPU FP64 oracle's restatement
 * of ICE's per-face and per-cell arithmetic: closures, limiters, reconstruction,
 * Riemann solvers, shock sensor, drag, heat, evaporation and the cell source.
 *
 * This file is only ever compiled into the oracle library (oracle/libice_oracle.so),
 * which the parity tests, the smoke check and the CPU-baseline leg of the bench use
 * as the checker. Nothing in the product links it.
 *
 * Every expression keeps the reference's operation order (Fortran evaluates a
 * chain of * / + - left to right) and is compiled without FMA contraction
 * (-ffp-contract=off), so that the result is the unfused IEEE result of the
 * Fortran source. Constants written in the reference as default-real (single
 * precision) literals are promoted from float exactly as gfortran does: 1e-25 in
 * the closures, 1e-20 in drag and tau, 1e+5 in compute_dt.
 *
 * The transcendentals of the sources and the sensor (exp, log, log10, pow, tanh) are the
 * deterministic functions of include/ice_math.h (within a few ulp of glibc's, tests/test_math.py),
 * the functions the device computes with, so that the FP64 forms agree to the bit; the reference
 * calls its platform's libm, which can differ from them in the last bits.
 *
 * Parity pins: tests/test_oracle_*.py check this restatement against the
 * reference's own known answers (test/unit/test_muscl_bounds.f90 B1-B5,
 * test/Riemann/AG exact solution, test/Doisneau/{MK,IG,AG} stored fields).
 */
#ifndef ICE_ORACLE_PHYSICS_H
#define ICE_ORACLE_PHYSICS_H

#include <math.h>
#include <stdint.h>
#include <string.h>
#include <float.h>
#include "../include/ice_gpu.h"
#include "../include/ice_math.h"

#define O_PI        3.14159265358979323846      /* Parameters_m.f90:41                       */
#define O_SIGMA_SB  5.670374419e-8               /* Parameters_m.f90:42                       */
#define O_RHO_EMPTY 1e-6                         /* Global_m.f90:11                           */
#define O_THETA_CAP 1.0                          /* Global_m.f90:12                           */
#define O_EPS       ((double)1e-25f)             /* eps = 1e-25 (default real), Lib_Model_*.f90 */
#define O_TOLL_DRAG ((double)1e-20f)             /* toll = 1e-20 (default real), Lib_Drag.f90:125 */
#define O_TOLL_HEAT 1e-20                        /* toll = 1.e-20_R8, Lib_Heat.f90:13          */
#define O_RU        8314.46                      /* Lib_Evaporation.f90:22                     */
#define O_PATM      101325.0                     /* Lib_Evaporation.f90:23                     */
#define O_XSCAP     1e-12                        /* Lib_Evaporation.f90:25                     */

/* ep indices, Lib_Evaporation.f90:15-19 (0-based here) */
enum { EP_MV = 0, EP_LV, EP_CPV, EP_LE, EP_YINF, EP_LVMVRU, EP_INVTB, EP_ALPHAE };

static inline int o_nbase(int closure) { return closure == ICE_CLOSURE_MK ? 6 : closure == ICE_CLOSURE_IG ? 7 : 12; }

/* NaN or Inf by the exponent bits (Finite_m.f90:66-74). */
static inline int o_not_finite(double x) {
    uint64_t u; memcpy(&u, &x, 8);
    return ((u >> 52) & 0x7FF) == 0x7FF;
}

/* gfortran's NORM2 of three values: the scaled sum of squares its front end emits
 * (scale = 0, s = 1; per non-zero |a|: rescale when it exceeds the scale; result
 * sqrt(s)*scale). compute_dt_ (Mod_dt.f90:269) and cell_surface (Mod_Sources.f90:35,39)
 * take NORM2 of 3-vectors. */
static inline double o_norm2(double a, double b, double c) {
    double v[3] = {a, b, c};
    double scale = 0.0, s = 1.0;
    for (int m = 0; m < 3; ++m) {
        if (v[m] != 0.0) {
            double ax = fabs(v[m]);
            if (scale < ax) { double q = scale / ax; s = 1.0 + s * q * q; scale = ax; }
            else            { double q = ax / scale; s = s + q * q; }
        }
    }
    return sqrt(s) * scale;
}

/* ---------------------------------------------------------------- closures */
/* Lib_Model_MK.f90:11-35, Lib_Model_IG.f90:11-37, Lib_Model_AG.f90:11-42
 * (constant-property path: mat_cp_const = cs_al) */
static inline void o_prim2cons(int cl, const double* p, double* c, const ice_gpu_family* m) {
    double n2 = p[1]*p[1] + p[2]*p[2] + p[3]*p[3];
    double cp = m->cs_al;
    c[0] = p[0];
    c[1] = p[0]*p[1]; c[2] = p[0]*p[2]; c[3] = p[0]*p[3];
    if (cl == ICE_CLOSURE_MK) {
        c[4] = p[0]*cp*p[4] + 0.5*p[0]*n2;
        c[5] = p[5];
    } else if (cl == ICE_CLOSURE_IG) {
        c[4] = p[0]*n2 + 3.0*p[4];
        c[5] = p[0]*cp*p[5] + 0.5*c[4];
        c[6] = p[6];
    } else {
        c[4] = p[0]*p[1]*p[1] + p[4];
        c[5] = p[0]*p[1]*p[2] + p[5];
        c[6] = p[0]*p[1]*p[3] + p[6];
        c[7] = p[0]*p[2]*p[2] + p[7];
        c[8] = p[0]*p[2]*p[3] + p[8];
        c[9] = p[0]*p[3]*p[3] + p[9];
        c[10] = p[0]*cp*p[10] + 0.5*(c[4] + c[7] + c[9]);
        c[11] = p[11];
    }
}

/* Lib_Model_MK.f90:38-76, Lib_Model_IG.f90:40-87, Lib_Model_AG.f90:45-124 */
static inline void o_cons2prim(int cl, const double* c, double* p, const ice_gpu_family* m) {
    const double eps = O_EPS;
    double cp = m->cs_al, n2;
    p[0] = c[0];
    p[1] = c[1] / (p[0] + eps); p[2] = c[2] / (p[0] + eps); p[3] = c[3] / (p[0] + eps);
    n2 = p[1]*p[1] + p[2]*p[2] + p[3]*p[3];
    if (cl == ICE_CLOSURE_MK) {
        p[4] = (c[4] - 0.5*p[0]*n2) / (cp*p[0] + eps);
        p[5] = c[5];
        if (p[0] < eps) for (int v = 0; v < 6; ++v) p[v] = eps;
        if (p[4] < eps) p[4] = eps;
        if (p[5] < eps) p[5] = eps;
    } else if (cl == ICE_CLOSURE_IG) {
        p[4] = 1.0/3.0 * (c[4] - p[0]*n2);
        if (p[0] <= O_RHO_EMPTY && p[4] > p[0]*O_THETA_CAP) p[4] = p[0]*O_THETA_CAP;
        p[5] = (c[5] - 0.5*c[4]) / (cp*p[0] + eps);
        p[6] = c[6];
        if (p[0] < eps) for (int v = 0; v < 7; ++v) p[v] = eps;
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
        if (p[0] <= O_RHO_EMPTY && p[4] + p[7] + p[9] > 3.0*p[0]*O_THETA_CAP) {
            double f = 3.0*p[0]*O_THETA_CAP / (p[4] + p[7] + p[9]);
            for (int v = 4; v < 10; ++v) p[v] = p[v] * f;
        }
        if (p[0] < eps) { for (int v = 0; v < 12; ++v) p[v] = eps; p[5] = 0.0; p[6] = 0.0; p[8] = 0.0; }
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

/* check_prim_{MK,IG,AG}: Lib_Model_MK.f90:79-92, IG 89-101, AG 126-140 */
static inline int o_check_prim(int cl, const double* p) {
    int nc = o_nbase(cl);
    for (int v = 0; v < nc; ++v) if (o_not_finite(p[v])) return 0;
    if (p[0] < 0.0) return 0;
    if (cl == ICE_CLOSURE_IG && p[4] < 0.0) return 0;
    if (cl == ICE_CLOSURE_AG && (p[4] < 0.0 || p[7] < 0.0 || p[9] < 0.0)) return 0;
    return 1;
}

/* wavespeed_make_*: MK 116-123, IG 140-146 (with pressure_make_IG 128-134), AG 165-178 */
static inline double o_wavespeed(int cl, const double* p, const double* n) {
    const double eps = O_EPS;
    if (cl == ICE_CLOSURE_MK) return 0.0;
    if (cl == ICE_CLOSURE_IG) {
        double pr = (p[4] + p[4] + p[4]) / 3.0;
        return sqrt(3.0*pr / (p[0] + eps));
    }
    double pnn = n[0]*(p[4]*n[0] + p[5]*n[1] + p[6]*n[2]) +
                 n[1]*(p[5]*n[0] + p[7]*n[1] + p[8]*n[2]) +
                 n[2]*(p[6]*n[0] + p[8]*n[1] + p[9]*n[2]);
    return sqrt(3.0*fmax(pnn, 0.0) / (p[0] + eps));
}

/* flux_make_*: MK 126-153, IG 149-169 (Lib_Model_IG.f90:462-491), AG 389-432 */
static inline void o_flux_make(int cl, const double* p, const double* n, double* f, const ice_gpu_family* m) {
    const double eps = O_EPS;
    double cp = m->cs_al;
    double n2 = p[1]*p[1] + p[2]*p[2] + p[3]*p[3];
    double un = p[1]*n[0] + p[2]*n[1] + p[3]*n[2];
    f[0] = p[0]*un;
    if (cl == ICE_CLOSURE_MK) {
        f[1] = f[0]*p[1]; f[2] = f[0]*p[2]; f[3] = f[0]*p[3];
        f[4] = f[0]*(0.5*n2 + cp*p[4]);
        f[5] = p[5]*un;
    } else if (cl == ICE_CLOSURE_IG) {
        f[1] = f[0]*p[1] + p[4]*n[0];
        f[2] = f[0]*p[2] + p[4]*n[1];
        f[3] = f[0]*p[3] + p[4]*n[2];
        f[4] = f[0]*n2 + 5.0*p[4]*un;
        f[5] = f[0]*(0.5*n2 + cp*p[5]) + 2.5*p[4]*un;
        f[6] = p[6]*un;
    } else {
        double p1n = p[4]*n[0] + p[5]*n[1] + p[6]*n[2];
        double p2n = p[5]*n[0] + p[7]*n[1] + p[8]*n[2];
        double p3n = p[6]*n[0] + p[8]*n[1] + p[9]*n[2];
        f[1] = f[0]*p[1] + p1n;
        f[2] = f[0]*p[2] + p2n;
        f[3] = f[0]*p[3] + p3n;
        f[4] = f[0]*p[1]*p[1] + un*p[4] + p[1]*p1n + p[1]*p1n;
        f[5] = f[0]*p[1]*p[2] + un*p[5] + p[1]*p2n + p[2]*p1n;
        f[6] = f[0]*p[1]*p[3] + un*p[6] + p[1]*p3n + p[3]*p1n;
        f[7] = f[0]*p[2]*p[2] + un*p[7] + p[2]*p2n + p[2]*p2n;
        f[8] = f[0]*p[2]*p[3] + un*p[8] + p[2]*p3n + p[3]*p2n;
        f[9] = f[0]*p[3]*p[3] + un*p[9] + p[3]*p3n + p[3]*p3n;
        f[10] = f[0]*(0.5*n2 + 0.5*(p[4] + p[7] + p[9])/(p[0] + eps) + cp*p[10])
              + p[1]*p1n + p[2]*p2n + p[3]*p3n;
        f[11] = p[11]*un;
    }
}

/* mirror_tensor_AG, Lib_Model_AG.f90:181-200: H P H, H = I - 2 n n^T */
static inline void o_mirror_tensor(const double* p, const double* n, double* pm) {
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

/* ---------------------------------------------------------------- limiters */
/* Lib_Limiters.f90:314-493. phi(r)*x, r = y/(x+1d-30), bounded by min(phi, cx, cy*r) for r > 0. */
static inline double o_min2(double a, double b) { return b < a ? b : a; }
static inline double o_max2(double a, double b) { return b > a ? b : a; }
static inline double o_limiter(int lim, double x, double y, double cx, double cy) {
    double ru, phi;
    if (lim == ICE_LIM_IORD) return 0.0;
    ru = y / (x + 1e-30);
    switch (lim) {
    case ICE_LIM_MINMOD:
        phi = o_max2(0.0, o_min2(1.0, ru));
        return phi * x;
    case ICE_LIM_VANALBADA: phi = (ru*ru + ru) / (ru*ru + 1.0); break;
    case ICE_LIM_VANLEER:   phi = (ru + fabs(ru)) / (1.0 + fabs(ru)); break;
    case ICE_LIM_OSPRE:     phi = (1.5*(ru*ru + ru)) / (ru*ru + ru + 1.0); break;
    case ICE_LIM_UMIST:
        phi = o_max2(0.0, o_min2(o_min2(o_min2(2.0*ru, 0.25 + 0.75*ru), 0.75 + 0.25*ru), 2.0)); break;
    case ICE_LIM_OSHER:     phi = o_max2(0.0, o_min2(ru, 1.5)); break;
    case ICE_LIM_SWEBY:
        phi = o_max2(o_max2(0.0, o_min2(1.5*ru, 1.0)), o_min2(ru, 1.5)); break;
    case ICE_LIM_MC:        phi = o_max2(0.0, o_min2(o_min2(2.0*ru, 0.5*(1.0 + ru)), 2.0)); break;
    case ICE_LIM_KOREN:     phi = o_max2(0.0, o_min2(2.0*ru, o_min2((1.0 + 2.0*ru)/3.0, 2.0))); break;
    case ICE_LIM_SUPERBEE:  phi = o_max2(o_max2(0.0, o_min2(2.0*ru, 1.0)), o_min2(ru, 2.0)); break;
    default: return 0.0;
    }
    if (ru > 0.0) phi = o_min2(o_min2(phi, cx), cy*ru);
    return phi * x;
}

/* -------------------------------------------------------- reconstruction */
/* state_reconstruction + slope_bounds, Lib_Reconstruction.f90:17-99 (non-solid).
 * Returns 0, or 1 when the first-order fallback is itself unphysical (report_stencil). */
static inline int o_reconstruct(int cl, int lim, const double* prev, const double* local,
                                const double* next, const double* next2,
                                double dl0, double dl1, double dl2, double dll, double dlr,
                                double* priml, double* primr, double beta) {
    int nc = o_nbase(cl);
    double cxl, cyl, cxr, cyr, limval = beta;
    if (dll > 0.0) { cxl = dl1/dll; cyl = dl0/dll; } else { cxl = 2.0; cyl = 2.0; }
    if (dlr > 0.0) { cxr = dl2/dlr; cyr = dl1/dlr; } else { cxr = 2.0; cyr = 2.0; }
    int first_l = prev[0] <= O_RHO_EMPTY || local[0] <= O_RHO_EMPTY || next[0] <= O_RHO_EMPTY;
    int first_r = local[0] <= O_RHO_EMPTY || next[0] <= O_RHO_EMPTY || next2[0] <= O_RHO_EMPTY;
    if (first_l) for (int v = 0; v < nc; ++v) priml[v] = local[v];
    if (first_r) for (int v = 0; v < nc; ++v) primr[v] = next[v];
    int st_l = first_l, st_r = first_r;
    while (!st_l || !st_r) {
        for (int v = 0; v < nc; ++v) {
            double slope1 = (next[v] - local[v]) / dl1;
            if (!first_l) {
                double slope0 = (local[v] - prev[v]) / dl0;
                double sl = o_limiter(lim, slope1, slope0, cxl, cyl) * limval;
                priml[v] = local[v] + sl*dll;
            }
            if (!first_r) {
                double slope2 = (next2[v] - next[v]) / dl2;
                double sr = o_limiter(lim, slope2, slope1, cxr, cyr) * limval;
                primr[v] = next[v] - sr*dlr;
            }
        }
        if (!first_l) st_l = o_check_prim(cl, priml);
        if (!first_r) st_r = o_check_prim(cl, primr);
        limval = 0.5*limval;
        if (limval < 1e-18 && !(st_l && st_r)) {
            for (int v = 0; v < nc; ++v) { priml[v] = local[v]; primr[v] = next[v]; }
            if (!(o_check_prim(cl, priml) && o_check_prim(cl, primr))) return 1;
            break;
        }
    }
    return 0;
}

/* ---------------------------------------------------------------- Riemann */
/* riemann_Saurel (Lib_Riemann.f90:61-109), MK slots */
static inline void o_saurel(const double* p1, const double* p4, const double* n, double* f, const ice_gpu_family* m) {
    double cp = m->cs_al;
    double vn1 = p1[1]*n[0] + p1[2]*n[1] + p1[3]*n[2];
    double vn4 = p4[1]*n[0] + p4[2]*n[1] + p4[3]*n[2];
    double vn = 0.5*(vn1 + vn4);
    if (vn > 0.0) {
        double ut = (p1[1] - vn1*n[0]), vt = (p1[2] - vn1*n[1]), wt = (p1[3] - vn1*n[2]);
        double uu = vn1*n[0] + ut, vv = vn1*n[1] + vt, ww = vn1*n[2] + wt;
        f[0] = p1[0]*vn;
        f[1] = uu*f[0]; f[2] = vv*f[0]; f[3] = ww*f[0];
        f[4] = f[0]*(0.5*(uu*uu + vv*vv + ww*ww) + cp*p1[4]);
        f[5] = p1[5]*vn;
    } else if (vn < 0.0) {
        double ut = (p4[1] - vn4*n[0]), vt = (p4[2] - vn4*n[1]), wt = (p4[3] - vn4*n[2]);
        double uu = vn4*n[0] + ut, vv = vn4*n[1] + vt, ww = vn4*n[2] + wt;
        f[0] = p4[0]*vn;
        f[1] = uu*f[0]; f[2] = vv*f[0]; f[3] = ww*f[0];
        f[4] = f[0]*(0.5*(uu*uu + vv*vv + ww*ww) + cp*p4[4]);
        f[5] = p4[5]*vn;
    } else {
        for (int v = 0; v < 6; ++v) f[v] = 0.0;
    }
}

/* riemann_Rusanov (Lib_Riemann.f90:153-186) */
static inline void o_rusanov(int cl, const double* p1, const double* p4, const double* n, double* f,
                             const ice_gpu_family* m) {
    int nc = o_nbase(cl);
    double c1[ICE_GPU_NCOND_MAX], c4[ICE_GPU_NCOND_MAX], f1[ICE_GPU_NCOND_MAX], f4[ICE_GPU_NCOND_MAX];
    double vn1 = p1[1]*n[0] + p1[2]*n[1] + p1[3]*n[2];
    double vn4 = p4[1]*n[0] + p4[2]*n[1] + p4[3]*n[2];
    double s1 = o_wavespeed(cl, p1, n), s4 = o_wavespeed(cl, p4, n);
    o_prim2cons(cl, p1, c1, m); o_prim2cons(cl, p4, c4, m);
    o_flux_make(cl, p1, n, f1, m); o_flux_make(cl, p4, n, f4, m);
    /* MAX(a,b,c,d) left to right */
    double A = fabs(vn1 - s1);
    A = o_max2(A, fabs(vn4 - s4)); A = o_max2(A, fabs(vn1 + s1)); A = o_max2(A, fabs(vn4 + s4));
    for (int v = 0; v < nc; ++v) f[v] = 0.5 * (f1[v] + f4[v] - A*(c4[v] - c1[v]));
}

/* riemann_HLLE (Lib_Riemann.f90:190-241) */
static inline void o_hlle(int cl, const double* p1, const double* p4, const double* n, double* f,
                          const ice_gpu_family* m) {
    int nc = o_nbase(cl);
    double vn1 = p1[1]*n[0] + p1[2]*n[1] + p1[3]*n[2];
    double vn4 = p4[1]*n[0] + p4[2]*n[1] + p4[3]*n[2];
    double s1 = o_wavespeed(cl, p1, n), s4 = o_wavespeed(cl, p4, n);
    double r1 = sqrt(p1[0]), r4 = sqrt(p4[0]);
    double uR = (r1*p1[1] + r4*p4[1]) / (r1 + r4);
    double vR = (r1*p1[2] + r4*p4[2]) / (r1 + r4);
    double wR = (r1*p1[3] + r4*p4[3]) / (r1 + r4);
    double vnR = uR*n[0] + vR*n[1] + wR*n[2];
    double sR = (r1*s1 + r4*s4) / (r1 + r4);
    double S1 = o_min2(o_min2(0.0, vn1 - s1), vnR - sR);
    double S4 = o_max2(o_max2(0.0, vn4 + s4), vnR + sR);
    /* minloc([-S1, S1*S4, S4]): the first smallest */
    double a0 = -S1, a1 = S1*S4, a2 = S4;
    int loc = 0; double mv = a0;
    if (a1 < mv) { loc = 1; mv = a1; }
    if (a2 < mv) { loc = 2; mv = a2; }
    if (loc == 0) {
        o_flux_make(cl, p1, n, f, m);
    } else if (loc == 2) {
        o_flux_make(cl, p4, n, f, m);
    } else {
        double f1[ICE_GPU_NCOND_MAX], f4[ICE_GPU_NCOND_MAX], c1[ICE_GPU_NCOND_MAX], c4[ICE_GPU_NCOND_MAX];
        o_flux_make(cl, p1, n, f1, m); o_flux_make(cl, p4, n, f4, m);
        o_prim2cons(cl, p1, c1, m); o_prim2cons(cl, p4, c4, m);
        for (int v = 0; v < nc; ++v) f[v] = (S4*f1[v] - S1*f4[v] + S1*S4*(c4[v] - c1[v])) / (S4 - S1);
    }
}

static inline void o_riemann(int solver, int cl, const double* p1, const double* p4, const double* n, double* f,
                             const ice_gpu_family* m) {
    if (solver == ICE_RIEMANN_SAUREL) o_saurel(p1, p4, n, f, m);
    else if (solver == ICE_RIEMANN_HLLE) o_hlle(cl, p1, p4, n, f, m);
    else o_rusanov(cl, p1, p4, n, f, m);
}

/* ------------------------------------------------------------ shock sensor */
/* SD_rho, Lib_Shock_Detector.f90:17-42 */
static inline double o_sd_rho(double r, double r1, double r2, double r3, double r4, double r5, double r6) {
    double kp1 = fabs((r2 - 2.0*r + r1) / (r2 + 2.0*r + r1 + 1e-30));
    double kp2 = fabs((r4 - 2.0*r + r3) / (r4 + 2.0*r + r3 + 1e-30));
    double kp3 = fabs((r6 - 2.0*r + r5) / (r6 + 2.0*r + r5 + 1e-30));
    double sw = o_max2(o_max2(kp1, kp2), kp3);
    if (sw < 1.0/20.0) {
        double phi = o_max2(sw*20.0, 0.0);
        return 1.0 - ice_tanh(10.0*phi*phi*phi);
    }
    return 0.0;
}

/* ------------------------------------------------------------------- drag */
/* Lib_Drag.f90:83-324 */
static inline double o_drag_wen_yu(double Re) {
    const double t = O_TOLL_DRAG;
    if (Re <= 1000) return 24.0/(Re + t) * (1.0 + 0.15*ice_pow(Re, 0.687));
    return 0.43;
}
static inline double o_henderson1(double Re, double Ma, double G, double Tr) {
    const double t = O_TOLL_DRAG;
    double sg = ice_pow(0.5*G, 0.5);
    double X = Re + Ma*sg*(4.33 + (3.65 - 1.53*Tr)/(1.0 + 0.353*Tr)*ice_exp(-0.247*Re/(Ma*sg + t))) + t;
    double rs = ice_pow(Re, 0.5);
    return 24.0*ice_pow(X, -1.0)
         + ice_exp(-0.5*Ma/(rs + t))*((4.5 + 0.38*(0.03*Re + 0.48*rs)) / (1.0 + 0.03*Re + 0.48*rs)
                                  + 0.1*(Ma*Ma) + 0.2*ice_pow(Ma, 8.0))
         + 0.6*Ma*sg*(1.0 - ice_exp(-Ma/(Re + t)));
}
static inline double o_henderson2(double Re, double Ma, double G, double Tr) {
    const double t = O_TOLL_DRAG;
    double q = ice_pow(Ma/(Re + t), 0.5);
    return (0.9 + 0.34/((Ma*Ma) + t) + 1.86*q*(2.0 + 2.0/(Ma*Ma*0.5*G + t)
            + (1.058/(Ma*ice_pow(0.5*G, 0.5) + t))*ice_pow(Tr, 0.5)) - 1.0/(ice_pow(Ma, 4.0)*(G*G)*0.25 + t))
           / (1.0 + 1.86*q);
}
static inline double o_drag(double Re, double Ma, double G, double Tr, int sel) {
    const double t = O_TOLL_DRAG;
    switch (sel) {
    case 1: return 0.45;
    case 2: return 24.0/(Re + t);
    case 3: return 24.0/(Re + t) * (1.0 + 3.0*Re/16.0);
    case 4: return 24.0/(Re + t) * (1.0 + 0.15*ice_pow(Re, 0.687));
    case 5: return o_drag_wen_yu(Re);
    case 6: if (Re < 1000) return 24.0/(Re + t) * (1.0 + ice_pow(Re, 2.0/3.0)/6.0); return 0.4392;
    case 7: return 24.0/(Re + t) * (1.0 + 0.15*ice_pow(Re, 0.687) + 0.0175*Re/(1.0 + 4.25*1e4*ice_pow(Re, -1.16)));
    case 8: {
        double a1, a2, a3;
        if (Re <= 0.1) { a1 = 0; a2 = 24; a3 = 0; }
        else if (Re <= 1.0) { a1 = 3.69; a2 = 22.73; a3 = 0.0903; }
        else if (Re <= 10) { a1 = 1.222; a2 = 29.1667; a3 = -3.8889; }
        else if (Re <= 100) { a1 = 0.6167; a2 = 46.5; a3 = -116.67; }
        else if (Re <= 1000) { a1 = 0.3644; a2 = 98.33; a3 = -2778; }
        else if (Re <= 5000) { a1 = 0.357; a2 = 148.62; a3 = -4.75e+4; }
        else if (Re <= 10000) { a1 = 0.46; a2 = -490.546; a3 = 57.87e+4; }
        else { a1 = 0.5191; a2 = -1662.5; a3 = 5.4167e+6; }
        return a1 + a2/(Re + t) + a3/(Re*Re + t);
    }
    case 9: {
        double Cd0 = o_drag_wen_yu(Re);
        return Cd0 * (1.0 + ice_exp(-0.427/(ice_pow(Ma, 4.63) + t) - 3.0/(ice_pow(Re, 0.88) + t))) /
               (1.0 + Ma/(Re + t)*(3.82 + 1.28*ice_exp(-1.25*Re/(Ma + t))));
    }
    case 10:
        if (Ma <= 1) return o_henderson1(Re, Ma, G, Tr);
        if (Ma >= 1.75) return o_henderson2(Re, Ma, G, Tr);
        {
            double Cd1 = o_henderson1(Re, 1.0, G, Tr), Cd2 = o_henderson2(Re, 1.75, G, Tr);
            return Cd1 + 4.0/3.0*(Ma - 1.0)*(Cd2 - Cd1);
        }
    case 11: {
        double g = 1.25*(1.0 + ice_tanh(0.77*ice_log10(Re + t) - 1.92));
        g = ice_pow(10.0, g);
        double h = 2.3 + 1.7*ice_pow(Tr, 0.5) - 2.3*ice_tanh(1.17*ice_log10(Ma + t));
        double Cd0 = o_drag_wen_yu(Re);
        return 2.0 + (Cd0 - 2.0)*ice_exp(-3.07*ice_pow(G, 0.5)*Ma*g/(Re + t)) + h/(Ma*ice_pow(G, 0.5) + t)*ice_exp(-Re/(2.0*Ma + t));
    }
    case 12: {
        double g = (1.0 + Re*(12.278 + 0.548*Re)) / (1.0 + 11.278*Re);
        double h = 5.6/(1.0 + Ma) + 1.7*ice_pow(Tr, 0.5);
        double Cd0 = o_drag_wen_yu(Re);
        return 2.0 + (Cd0 - 2.0)*ice_exp(-3.07*ice_pow(G, 0.5)*Ma*g/(Re + t)) + h/(Ma*ice_pow(G, 0.5) + t)*ice_exp(-Re/(2.0*Ma + t));
    }
    case 13: return 0.0;
    }
    return 0.0;
}

/* ------------------------------------------------------------------- heat */
/* Lib_Heat.f90:68-160 */
static inline double o_heat(double Re, double Pr, double Ma, int sel) {
    const double t = O_TOLL_HEAT;
    switch (sel) {
    case 1: return 2.0;
    case 2: return 2.5*ice_pow(Re, 0.15) + 0.04*Re;
    case 3: return 2.0 + 0.37*ice_pow(Re, 0.6)*ice_pow(Pr, 1.0/3.0);
    case 4: return 2.0 + 0.459*ice_pow(Re, 0.55)*ice_pow(Pr, 1.0/3.0);
    case 5: return ice_pow(ice_pow(2.0 + 0.654*ice_pow(Re, 0.5)*ice_pow(Pr, 0.5), -1.0) + 3.42*Ma/(Re*Pr + t), -1.0);
    case 6: return 2.0 + 0.6*ice_pow(Re, 0.5)*ice_pow(Pr, 1.0/3.0);
    case 7: {
        double Nu = 2.0 + 0.459*ice_pow(Re, 0.55)*ice_pow(Pr, 0.33);
        return Nu / (1.0 + 3.42*Ma/(Re*Pr + t)*Nu);
    }
    case 8: return 0.0;
    }
    return 0.0;
}

/* ------------------------------------------------------------ evaporation */
/* Lib_Evaporation.f90:129-143 */
static inline double o_blowing(double gamma, double Rg, double mug, double kg, double rhop, double dp,
                               double mp, double mdot) {
    if (mdot >= 0.0 || mp <= 0.0 || mug <= 0.0 || kg <= 0.0) return 1.0;
    if (dp <= 0.0 || rhop <= 0.0 || gamma <= 1.0) return 1.0;
    double cpg = gamma*Rg/(gamma - 1.0);
    double Pr = mug*cpg/kg;
    double taud = rhop*dp*dp/(18.0*mug);
    double b = -1.5*Pr*taud*mdot/mp;
    if (b != b || b <= 1e-10) return 1.0;
    if (b > 500.0) return 0.0;
    return b/(ice_exp(b) - 1.0);
}

static inline double o_molar2mass(double Xs, double Mv, double Mg) { return Xs*Mv/(Xs*Mv + (1.0 - Xs)*Mg); }
static inline double o_mass2molar(double Ys, double Mv, double Mg) { return Ys*Mg/(Ys*Mg + (1.0 - Ys)*Mv); }
static inline double o_Fcorr(double B) { return B > 1.0e-10 ? ice_pow(1.0 + B, 0.7)*ice_log(1.0 + B)/B : 1.0; }

typedef struct {
    double rhog, Tg, gamma, Rg, mug, kg, Tp, dp, cpg, p, Mg, Pr, Sc, Re05;
    int evap;
    const double* ep;
} o_evap_env;

/* gasSideRate (Lib_Evaporation.f90:205-224) with the five models (287-521) */
static inline void o_gas_side(const o_evap_env* e, double Ys, double BM, double* md, double* Qd, int* ovr) {
    const double pi = O_PI;
    const double* ep = e->ep;
    *md = 0.0; *Qd = 0.0; *ovr = 0;
    switch (e->evap) {
    case 1: {
        double BT = e->cpg*(e->Tg - e->Tp)/ep[EP_LV];
        if (BT <= 0.0) { *md = 0.0; return; }
        *md = -2.0*pi*e->dp*e->kg/e->cpg*ice_log(1.0 + BT);
        return;
    }
    case 2: {
        double Dv = e->kg/(e->rhog*e->cpg*ep[EP_LE]);
        double Sh = 2.0 + 0.6*e->Re05*ice_pow(e->Sc, 1.0/3.0);
        *md = -pi*e->dp*e->rhog*Dv*Sh*ice_log(1.0 + BM);
        return;
    }
    case 3: {
        double Tf = e->Tp + (e->Tg - e->Tp)/3.0;
        double rho_f = e->rhog*e->Tg/Tf;
        double mu_f = e->mug*ice_pow(Tf/e->Tg, 0.7);
        double kl_f = e->kg*ice_pow(Tf/e->Tg, 0.7);
        double cpg_f = e->cpg;
        double Dv_f = kl_f/(rho_f*cpg_f*ep[EP_LE]);
        double Sc_f = mu_f*cpg_f*ep[EP_LE]/kl_f;
        double Re_f = e->Re05*e->Re05*rho_f/e->rhog*e->mug/mu_f;
        double Sh_f = 2.0 + 0.6*sqrt(o_max2(Re_f, 0.0))*ice_pow(Sc_f, 1.0/3.0);
        *md = -pi*e->dp*rho_f*Dv_f*Sh_f*ice_log(1.0 + BM);
        return;
    }
    case 4: {
        double Le = ep[EP_LE], cpv = ep[EP_CPV];
        *ovr = 1;
        double Dv = e->kg/(e->rhog*e->cpg*Le);
        double lnBM = ice_log(1.0 + BM);
        double FM = o_Fcorr(BM);
        double Sh0 = 2.0 + 0.552*e->Re05*ice_pow(e->Sc, 1.0/3.0);
        double Shs = 2.0 + (Sh0 - 2.0)/FM;
        *md = -pi*e->dp*e->rhog*Dv*Shs*lnBM;
        double cpv_eff = cpv > 0.0 ? cpv : e->cpg;
        double Nu0 = 2.0 + 0.552*e->Re05*ice_pow(e->Pr, 1.0/3.0);
        double Nus = Nu0, BT = 0.0;
        for (int it = 1; it <= 5; ++it) {
            double phi = cpv_eff/e->cpg*Shs/Nus/Le;
            BT = ice_pow(1.0 + BM, phi) - 1.0;
            if (BT <= 0.0) { BT = BM; Nus = Nu0; break; }
            double FT = o_Fcorr(BT);
            Nus = 2.0 + (Nu0 - 2.0)/FT;
        }
        *Qd = BT > 0.0 ? -*md*cpv_eff*(e->Tg - e->Tp)/BT : 0.0;
        return;
    }
    case 5: {
        double Le = ep[EP_LE], cpv = ep[EP_CPV], Yinf = ep[EP_YINF], Mv = ep[EP_MV];
        double Dv = e->kg/(e->rhog*e->cpg*Le);
        double cpv_eff = cpv > 0.0 ? cpv : e->cpg;
        double Xs = o_min2(o_mass2molar(Ys, Mv, e->Mg), 1.0 - O_XSCAP);
        double Xinf = o_mass2molar(Yinf, Mv, e->Mg);
        double Minf = Xinf*Mv + (1.0 - Xinf)*e->Mg;
        double rhs0 = Mv/Minf*ice_log((1.0 - Xinf)/(1.0 - Xs));
        if (rhs0 <= 0.0) return;
        double Tts = e->Tp/e->Tg;
        double Lev = e->kg/(cpv_eff*Dv*e->rhog);
        double mlo = rhs0/o_max2(Tts, 1.0);
        double mhi = rhs0/o_min2(o_max2(Tts, 1.0e-3), 1.0);
        double mhat = rhs0;
        for (int it = 1; it <= 30; ++it) {
            double x = mhat/Lev, f, fp;
            if (x > 1.0e-6) {
                double E = ice_exp(-x);
                f = x/(1.0 - E);
                fp = (1.0 - E - x*E)/((1.0 - E)*(1.0 - E));
            } else {
                f = 1.0 + 0.5*x + x*x/12.0;
                fp = 0.5 + x/6.0;
            }
            double G = mhat + (Tts - 1.0)*Lev*(f - 1.0) - rhs0;
            double dG = 1.0 + (Tts - 1.0)*fp;
            if (fabs(G) <= 1.0e-13*o_max2(1.0, rhs0)) break;
            if (G > 0.0) mhi = mhat; else mlo = mhat;
            mhat = mhat - G/dG;
            if (mhat <= mlo || mhat >= mhi) mhat = 0.5*(mlo + mhi);
        }
        double Sh = 2.0 + 0.6*e->Re05*ice_pow(e->Sc, 1.0/3.0);
        *md = -pi*e->dp*e->rhog*Dv*Sh*mhat;
        *ovr = 1;
        double Nu = 2.0 + 0.6*e->Re05*ice_pow(e->Pr, 1.0/3.0);
        double chi = o_min2(-*md*cpv_eff/(pi*e->dp*e->kg*Nu), 700.0);
        if (chi > 1.0e-9) *Qd = -*md*cpv_eff*(e->Tg - e->Tp)/(ice_exp(chi) - 1.0);
        else *Qd = pi*e->dp*e->kg*Nu*(e->Tg - e->Tp);
        return;
    }
    }
}

/* evaporation + lkCorrection (Lib_Evaporation.f90:145-261), Clausius-Clapeyron psat (738-745) */
static inline void o_evaporation(double rhog, double Tg, double gamma, double Rg, double mug, double kg,
                                 double Tp, double dp, double Re, int evap, int intf, const double* ep,
                                 double* mdot, double* Qd, int* ovr) {
    const double pi = O_PI;
    *mdot = 0.0; *Qd = 0.0; *ovr = 0;
    if (evap == 0) return;
    o_evap_env e;
    e.rhog = rhog; e.Tg = Tg; e.gamma = gamma; e.Rg = Rg; e.mug = mug; e.kg = kg; e.Tp = Tp; e.dp = dp;
    e.evap = evap; e.ep = ep;
    e.cpg = gamma*Rg/(gamma - 1.0);
    e.p = rhog*Rg*Tg;
    e.Mg = O_RU/Rg;
    double psat = O_PATM*ice_exp(-ep[EP_LVMVRU]*(1.0/Tp - ep[EP_INVTB]));
    double Xs = psat >= e.p ? 1.0 - O_XSCAP : o_min2(psat/e.p, 1.0 - O_XSCAP);
    double Ys = o_molar2mass(Xs, ep[EP_MV], e.Mg);
    if (Ys <= ep[EP_YINF]) return;
    double BM = (Ys - ep[EP_YINF])/(1.0 - Ys);
    if (BM <= 0.0) return;
    e.Re05 = sqrt(o_max2(Re, 0.0));
    e.Pr = mug*e.cpg/kg;
    e.Sc = e.Pr*ep[EP_LE];
    o_gas_side(&e, Ys, BM, mdot, Qd, ovr);
    if (intf != 1) return;
    /* lkCorrection */
    double LKd2 = 2.0*mug*sqrt(2.0*pi*Tp*O_RU/ep[EP_MV])/(ep[EP_ALPHAE]*e.Sc*e.p)/dp;
    double diffPrev = DBL_MAX, md = *mdot, mdNew = 0.0, QdNew = 0.0;
    int ovrNew = 0;
    for (int it = 1; it <= 30; ++it) {
        double beta = -md*e.Pr/(2.0*pi*mug*dp);
        double XsN = o_max2(Xs - LKd2*beta, 0.0);
        double YsN = o_molar2mass(XsN, ep[EP_MV], e.Mg);
        mdNew = 0.0; QdNew = 0.0; ovrNew = 0;
        if (YsN > ep[EP_YINF]) {
            double BMN = (YsN - ep[EP_YINF])/(1.0 - YsN);
            if (BMN > 0.0) o_gas_side(&e, YsN, BMN, &mdNew, &QdNew, &ovrNew);
        }
        double diff = fabs(mdNew - md);
        if (diff <= 1.e-12*fabs(mdNew)) { *mdot = mdNew; *Qd = QdNew; *ovr = ovrNew; return; }
        if (diff < diffPrev) md = mdNew; else md = 0.5*(md + mdNew);
        diffPrev = diff;
    }
    *mdot = mdNew; *Qd = QdNew; *ovr = ovrNew;
}

/* ------------------------------------------------------------ cell source */
/* source_make_{MK,IG,AG}: Lib_Model_MK.f90:156-184, IG 172-202 (494-524), AG 248-296.
 * mat_lv = lv_al on the constant-property path. */
static inline void o_source_make(int cl, const double* p, const double* F, double* s, const ice_gpu_family* m) {
    const double eps = O_EPS;
    double cp = m->cs_al, lv = m->lv_al;
    s[0] = -F[0];
    s[1] = -F[0]*p[1] + p[0]*F[1]/(F[5] + eps);
    s[2] = -F[0]*p[2] + p[0]*F[2]/(F[5] + eps);
    s[3] = -F[0]*p[3] + p[0]*F[3]/(F[5] + eps);
    if (cl == ICE_CLOSURE_MK) {
        double n2 = p[1]*p[1] + p[2]*p[2] + p[3]*p[3];
        s[4] = -F[0]*(0.5*n2 + cp*p[4]) - F[0]*lv + F[4] + p[0]*(F[1]*p[1] + F[2]*p[2] + F[3]*p[3])/(F[5] + eps);
        s[5] = 0.0;
    } else if (cl == ICE_CLOSURE_IG) {
        double n2 = p[1]*p[1] + p[2]*p[2] + p[3]*p[3];
        s[4] = -F[0]*(n2 + 3.0*p[4]/p[0]) + 2.0*p[0]*(F[1]*p[1] + F[2]*p[2] + F[3]*p[3])/(F[5] + eps)
               - 6.0*p[4]/(F[5] + eps);
        s[5] = -F[0]*cp*p[5] - F[0]*lv + F[4] + 0.5*s[4];
        s[6] = 0.0;
    } else {
        s[4] = -F[0]*(p[1]*p[1] + p[4]/p[0]) + p[0]*(F[1]*p[1] + F[1]*p[1])/(F[5] + eps) - 2.0*p[4]/(F[5] + eps);
        s[5] = -F[0]*(p[1]*p[2] + p[5]/p[0]) + p[0]*(F[2]*p[1] + F[1]*p[2])/(F[5] + eps) - 2.0*p[5]/(F[5] + eps);
        s[6] = -F[0]*(p[1]*p[3] + p[6]/p[0]) + p[0]*(F[3]*p[1] + F[1]*p[3])/(F[5] + eps) - 2.0*p[6]/(F[5] + eps);
        s[7] = -F[0]*(p[2]*p[2] + p[7]/p[0]) + p[0]*(F[2]*p[2] + F[2]*p[2])/(F[5] + eps) - 2.0*p[7]/(F[5] + eps);
        s[8] = -F[0]*(p[2]*p[3] + p[8]/p[0]) + p[0]*(F[3]*p[2] + F[2]*p[3])/(F[5] + eps) - 2.0*p[8]/(F[5] + eps);
        s[9] = -F[0]*(p[3]*p[3] + p[9]/p[0]) + p[0]*(F[3]*p[3] + F[3]*p[3])/(F[5] + eps) - 2.0*p[9]/(F[5] + eps);
        s[10] = -F[0]*cp*p[10] - F[0]*lv + F[4] + 0.5*s[4] + 0.5*s[7] + 0.5*s[9];
        s[11] = 0.0;
    }
}

/* compute_source_ + cell_surface (Mod_Sources.f90:230-274, 465-622) on the ITC/clamp,
 * non-burning, constant-property path. gas = rho u v w T; returns tau. */
static inline double o_cell_source(int cl, const double* p, const double* gas, double gR, double ggam,
                                   double gk, double gmu, const ice_gpu_family* m, int drag_sel, int heat_sel,
                                   int blow, double* s) {
    const double pi = O_PI;
    int nb = o_nbase(cl);
    double T = p[nb - 2], n = p[nb - 1];
    double rho_mat = m->rho_al;
    double Rp = ice_pow(0.75*p[0]/(n*pi*rho_mat), 1.0/3.0);
    double du = o_norm2(gas[1] - p[1], gas[2] - p[2], gas[3] - p[3]);
    double Re = 2.0*gas[0]*Rp*du/gmu;
    double Ma = du/ice_pow(ggam*gR*gas[4], 0.5);
    double Pr = ggam/(ggam - 1.0)*gR*gmu/gk;
    double Nu = o_heat(Re, Pr, Ma, heat_sel);
    double Ts = T;                              /* ITC: drop_surface returns the mean temperature */
    double Tr = Ts/gas[4];
    double Cd = o_drag(Re, Ma, ggam, Tr, drag_sel);
    double F[6];
    F[1] = gas[1] - p[1]; F[2] = gas[2] - p[2]; F[3] = gas[3] - p[3];
    double Qconv = 2.0*Nu*gk*pi*Rp*(gas[4] - Ts);
    double mdot, Qevap; int ovr;
    o_evaporation(gas[0], gas[4], ggam, gR, gmu, gk, Ts, 2.0*Rp, Re, m->evap, m->intf, m->ep, &mdot, &Qevap, &ovr);
    if (ovr) Qconv = Qevap;
    else if (blow == 1) Qconv = Qconv*o_blowing(ggam, gR, gmu, gk, rho_mat, 2.0*Rp, 4.0/3.0*pi*(Rp*Rp*Rp)*rho_mat, mdot);
    F[0] = -mdot*n;
    F[4] = Qconv*n;
    F[4] = F[4] + m->emiss*O_SIGMA_SB*4.0*pi*Rp*Rp*n*(ice_pow(gas[4], 4.0) - ice_pow(Ts, 4.0));
    double tau;
    if (Cd == 0.0) tau = INFINITY;
    else tau = 8.0*rho_mat*Rp/(3.0*gas[0]*Cd*du + (double)1e-20f);
    F[5] = tau;
    o_source_make(cl, p, F, s, m);
    return tau;
}

#endif /* ICE_ORACLE_PHYSICS_H */
