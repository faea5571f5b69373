/*
 * ice_math.h -- the double-precision elementary functions of the solve stage: exp, expm1, log,
 * log10, pow, tanh.
 *
 * They are built from IEEE-754 additions, multiplications and divisions (never fused) and integer
 * operations on the bits, so the same source gives the same bits compiled by gcc for the host
 * (-ffp-contract=off) and by nvcc for sm_100a (--fmad=false). The sources of ICE's dispersed phase
 * (drag, heat, evaporation, radiation) and its shock sensor call these functions; with the platform
 * libraries (glibc on the host, CUDA's on the device) the last bits can differ, and in nearly empty
 * cells the step amplifies such a difference without bound. With these, the device's plain form and
 * its FP64 restatement on the host agree to the bit.
 *
 * Methods (standard numerical analysis, constants derived here from their definitions):
 *   exp:   x = k ln2 + r, |r| <= ln2/2, with ln2 split into a 29-bit head and a tail (Cody and
 *          Waite's additive reduction) so that k*ln2_hi is exact; e^r by its Taylor series to r^13
 *          (truncation < 4e-18 relative); the power of two put into the exponent bits.
 *   log:   x = 2^e m, m in [sqrt(1/2), sqrt(2)); log m = 2 atanh(s), s = (m-1)/(m+1), |s| <= 0.172,
 *          by the odd series of atanh to s^25; e ln2 added head first.
 *   pow:   x^n by binary powering for an integral exponent |n| <= 64; sqrt for y = 1/2; otherwise
 *          exp(y log x) (relative error ~ |y log x| units in the last place: 30 ulp for T^4 at
 *          1500 K, far below the physics the correlations carry).
 *   tanh:  t = expm1(2|x|), tanh = t/(t+2); expm1 by its Taylor series to u^17 below 1/2.
 * Accuracy against the platform libraries is a test (tests/test_math.py): within a few ulp.
 */
#ifndef ICE_MATH_H
#define ICE_MATH_H

#include <stdint.h>
#include <string.h>
#include <math.h>

#ifdef __CUDACC__
#define ICE_HD static __host__ __device__ __forceinline__
#else
#define ICE_HD static inline
#endif

#define ICE_LN2_HI   0.6931471806019545         /* 0x3fe62e42ff000000 */
#define ICE_LN2_LO  (-4.2009150726810846e-11)   /* ln2 - ICE_LN2_HI */
#define ICE_INV_LN2  1.4426950408889634
#define ICE_LN10     2.302585092994046
#define ICE_SQRT2    1.4142135623730951

ICE_HD double ice_bits2d(uint64_t u) {
#ifdef __CUDA_ARCH__
  return __longlong_as_double((long long)u);
#else
  double d; memcpy(&d, &u, 8); return d;
#endif
}
ICE_HD uint64_t ice_d2bits(double d) {
#ifdef __CUDA_ARCH__
  return (uint64_t)__double_as_longlong(d);
#else
  uint64_t u; memcpy(&u, &d, 8); return u;
#endif
}
ICE_HD double ice_inf(void) { return ice_bits2d(0x7FF0000000000000ULL); }
ICE_HD double ice_nan(void) { return ice_bits2d(0x7FF8000000000000ULL); }
ICE_HD int ice_isnan(double x) { return x != x; }

/* 2^k for -1074 <= k <= 1024 as a product of exact powers of two */
ICE_HD double ice_scale2(double p, int k) {
  if (k > 1023) { p = p * ice_bits2d((uint64_t)(1023 + 1023) << 52); k -= 1023; }
  if (k < -1022) { p = p * ice_bits2d((uint64_t)(1023 - 1022) << 52); k += 1022;
                   if (k < -1022) { p = p * ice_bits2d((uint64_t)(1023 - 1022) << 52); k += 1022; } }
  return p * ice_bits2d((uint64_t)(k + 1023) << 52);
}

/* nearest integer of x (ties away from zero), |x| < 2^52 */
ICE_HD double ice_round(double x) {
  double r = x >= 0.0 ? x + 0.5 : x - 0.5;
  /* truncate toward zero by clearing the fraction bits */
  uint64_t u = ice_d2bits(r);
  int e = (int)((u >> 52) & 0x7FF) - 1023;
  if (e < 0) return 0.0;
  if (e >= 52) return r;
  u &= ~((1ULL << (52 - e)) - 1ULL);
  return ice_bits2d(u);
}

ICE_HD double ice_exp(double x) {
  if (ice_isnan(x)) return x;
  if (x > 709.782712893384) return ice_inf();
  if (x < -745.1332191019412) return 0.0;
  double kd = ice_round(x * ICE_INV_LN2);
  double r = (x - kd * ICE_LN2_HI) - kd * ICE_LN2_LO;
  double p = 1.6059043836821613e-10;                    /* 1/13! */
  p = p * r + 2.08767569878681e-09;                     /* 1/12! */
  p = p * r + 2.505210838544172e-08;
  p = p * r + 2.755731922398589e-07;
  p = p * r + 2.7557319223985893e-06;
  p = p * r + 2.48015873015873e-05;
  p = p * r + 0.0001984126984126984;
  p = p * r + 0.001388888888888889;
  p = p * r + 0.008333333333333333;
  p = p * r + 0.041666666666666664;
  p = p * r + 0.16666666666666666;
  p = p * r + 0.5;
  p = p * r + 1.0;
  p = p * r + 1.0;
  return ice_scale2(p, (int)kd);
}

/* e^u - 1 without cancellation for small u */
ICE_HD double ice_expm1(double u) {
  double a = u < 0.0 ? -u : u;
  if (a < 0.5) {
    double p = 1.5619206968586225e-16;                  /* 1/18! */
    p = p * u + 2.8114572543455206e-15;
    p = p * u + 4.779477332387385e-14;
    p = p * u + 7.647163731819816e-13;
    p = p * u + 1.1470745597729725e-11;
    p = p * u + 1.6059043836821613e-10;
    p = p * u + 2.08767569878681e-09;
    p = p * u + 2.505210838544172e-08;
    p = p * u + 2.755731922398589e-07;
    p = p * u + 2.7557319223985893e-06;
    p = p * u + 2.48015873015873e-05;
    p = p * u + 0.0001984126984126984;
    p = p * u + 0.001388888888888889;
    p = p * u + 0.008333333333333333;
    p = p * u + 0.041666666666666664;
    p = p * u + 0.16666666666666666;
    p = p * u + 0.5;
    return u + (u * u) * p;
  }
  return ice_exp(u) - 1.0;
}

ICE_HD double ice_log(double x) {
  if (ice_isnan(x)) return x;
  if (x < 0.0) return ice_nan();
  if (x == 0.0) return -ice_inf();
  uint64_t u = ice_d2bits(x);
  if (((u >> 52) & 0x7FF) == 0x7FF) return x;                       /* +inf */
  int e = 0;
  if (x < ice_bits2d(0x0010000000000000ULL)) {                       /* subnormal */
    x = x * ice_bits2d((uint64_t)(1023 + 54) << 52);
    e = -54;
    u = ice_d2bits(x);
  }
  e += (int)((u >> 52) & 0x7FF) - 1023;
  double m = ice_bits2d((u & 0x000FFFFFFFFFFFFFULL) | 0x3FF0000000000000ULL);   /* [1, 2) */
  if (m > ICE_SQRT2) { m = m * 0.5; e += 1; }
  double f = m - 1.0;
  double s = f / (2.0 + f);
  double z = s * s;
  double q = 0.08;                                      /* 2/25 */
  q = q * z + 0.08695652173913043;
  q = q * z + 0.09523809523809523;
  q = q * z + 0.10526315789473684;
  q = q * z + 0.11764705882352941;
  q = q * z + 0.13333333333333333;
  q = q * z + 0.15384615384615385;
  q = q * z + 0.18181818181818182;
  q = q * z + 0.2222222222222222;
  q = q * z + 0.2857142857142857;
  q = q * z + 0.4;
  q = q * z + 0.6666666666666666;
  double lm = 2.0 * s + s * (z * q);
  double ed = (double)e;
  return (ed * ICE_LN2_LO + lm) + ed * ICE_LN2_HI;
}

ICE_HD double ice_log10(double x) { return ice_log(x) / ICE_LN10; }

ICE_HD double ice_pow(double x, double y) {
  if (ice_isnan(x) || ice_isnan(y)) return (y == 0.0) ? 1.0 : ice_nan();
  if (y == 0.0 || x == 1.0) return 1.0;
  double ay = y < 0.0 ? -y : y;
  double yi = ice_round(y);
  int integral = (ay < 4503599627370496.0) ? (yi == y) : 1;
  double sign = 1.0;
  if (x < 0.0) {
    if (!integral) return ice_nan();
    double h = ice_round(0.5 * y);
    if (h * 2.0 != y) sign = -1.0;                      /* odd integral exponent */
    x = -x;
  }
  if (x == 0.0) return y > 0.0 ? 0.0 * sign : sign * ice_inf();
  if (((ice_d2bits(x) >> 52) & 0x7FF) == 0x7FF) return y > 0.0 ? sign * ice_inf() : 0.0 * sign;
  if (integral && ay <= 64.0) {                         /* binary powering */
    long n = (long)ay;
    double b = x, r = 1.0;
    while (n > 0) { if (n & 1) r = r * b; b = b * b; n >>= 1; }
    return sign * (y < 0.0 ? 1.0 / r : r);
  }
  if (y == 0.5) return sign * sqrt(x);
  return sign * ice_exp(y * ice_log(x));
}

ICE_HD double ice_tanh(double x) {
  if (ice_isnan(x)) return x;
  double a = x < 0.0 ? -x : x;
  if (a > 22.0) return x < 0.0 ? -1.0 : 1.0;
  if (a < 3.725290298461914e-09) return x;               /* 2^-28 */
  double t = ice_expm1(2.0 * a);
  double r = t / (t + 2.0);
  return x < 0.0 ? -r : r;
}

#endif /* ICE_MATH_H */
