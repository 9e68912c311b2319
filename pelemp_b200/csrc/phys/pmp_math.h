/* pmp_math.h -- double-precision elementary functions shared, unchanged, by
 * the CUDA kernels and the CPU code of this project.
 *
 * Why a project library: the spray update spends most of its arithmetic in
 * exp/log/pow/cbrt/log1p (Source/PP_Spray/Drag.H:6-45, 199, 270, 301-329,
 * 400; Source/PP_Spray/SprayFuelData.H:192-210).  Writing them once, with
 * every multiply-add an explicit fma() and every division an IEEE division,
 * gives bit-identical results on the host and on the GPU, so the CPU oracle
 * and the kernels differ only where the kernels reorder arithmetic.
 *
 * Methods (all published, none taken from a vendor library):
 *  - exp:   Cody & Waite (1980) argument reduction x = k ln2 + r with a
 *           two-part ln2, then the degree-13 Taylor polynomial of e^r on
 *           |r| <= ln2/2 (truncation < 5e-18), then scaling by 2^k.
 *  - log:   x = 2^e m, m in [sqrt(1/2), sqrt(2)), f = m - 1, s = f/(2+f);
 *           log(1+f) = 2 atanh(s) written as f - (f^2/2 - s (f^2/2 + R(s^2)))
 *           with R the atanh series 2z/3 + 2z^2/5 + ... to z^11.
 *  - log1p: Goldberg, "What every computer scientist should know about
 *           floating-point arithmetic" (1991), Theorem 4:
 *           u = 1 + x; log1p(x) = x if u == 1 else log(u) x / (u - 1).
 *  - pow:   exp(y log x) for x > 0.
 *  - cbrt:  exp(log|x| / 3) refined by one Newton step on y^3 = |x|.
 * Accuracy (checked in the tests against 50-digit decimal values): exp, log,
 * cbrt within 1.5 ulp, log1p within 2.5 ulp; pow within 1.5 + |y log x| ulp.
 *
 * This header is valid C99 and CUDA C++.  Define PMP_USE_LIBM before
 * including it to route the PMP_* macros to the C library instead (used only
 * to compare against code compiled with the C library).
 */
#ifndef PMP_MATH_H
#define PMP_MATH_H

#include <math.h>
#include <stdint.h>
#include <string.h>

#if defined(__CUDACC__)
#define PMP_HD __host__ __device__ __forceinline__
#else
#define PMP_HD static inline
#endif

PMP_HD int64_t pmp_dbits(double x)
{
#if defined(__CUDA_ARCH__)
  return __double_as_longlong(x);
#else
  int64_t i;
  memcpy(&i, &x, sizeof(i));
  return i;
#endif
}

PMP_HD double pmp_bitsd(int64_t i)
{
#if defined(__CUDA_ARCH__)
  return __longlong_as_double(i);
#else
  double x;
  memcpy(&x, &i, sizeof(x));
  return x;
#endif
}

#define PMP_LOG2E 1.4426950408889634
#define PMP_LN2_HI 0.6931467056274414     /* ln 2, low 32 significand bits cleared */
#define PMP_LN2_LO 4.7493250390316726e-07 /* ln 2 - PMP_LN2_HI */
#define PMP_LN10 2.302585092994046
#define PMP_PI 3.141592653589793

/* 2^k as a double for -1022 <= k <= 1023 */
PMP_HD double pmp_pow2i(int k) { return pmp_bitsd((int64_t)(k + 1023) << 52); }

PMP_HD double pmp_exp(double x)
{
  if (!(x == x)) {
    return x + x; /* NaN */
  }
  if (x > 709.782712893384) {
    return HUGE_VAL;
  }
  if (x < -745.1332191019412) {
    return 0.0;
  }
  const double k = rint(x * PMP_LOG2E);
  double r = fma(-k, PMP_LN2_HI, x); /* exact: k*LN2_HI has <= 32 bits */
  r = fma(-k, PMP_LN2_LO, r);
  double p = 1.6059043836821613e-10;   /* 1/13! */
  p = fma(p, r, 2.08767569878681e-09); /* 1/12! */
  p = fma(p, r, 2.505210838544172e-08);
  p = fma(p, r, 2.755731922398589e-07);
  p = fma(p, r, 2.7557319223985893e-06);
  p = fma(p, r, 2.48015873015873e-05);
  p = fma(p, r, 1.984126984126984e-04);
  p = fma(p, r, 1.388888888888889e-03);
  p = fma(p, r, 8.333333333333333e-03);
  p = fma(p, r, 4.1666666666666664e-02);
  p = fma(p, r, 1.6666666666666666e-01);
  p = fma(p, r, 0.5);
  p = fma(p, r, 1.0);
  p = fma(p, r, 1.0);
  /* scale by 2^k in two halves so that subnormal results stay correct */
  const int ki = (int)k;
  const int k1 = ki / 2;
  return (p * pmp_pow2i(k1)) * pmp_pow2i(ki - k1);
}

PMP_HD double pmp_log(double x)
{
  if (!(x > 0.0)) {
    return (x == 0.0) ? -HUGE_VAL : (x - x) / (x - x); /* -inf or NaN */
  }
  int64_t b = pmp_dbits(x);
  int e = (int)((b >> 52) & 0x7ff);
  if (e == 0x7ff) {
    return x; /* +inf */
  }
  if (e == 0) { /* subnormal: scale by 2^54 */
    b = pmp_dbits(x * 18014398509481984.0);
    e = (int)((b >> 52) & 0x7ff) - 54;
  }
  e -= 1023;
  int64_t mb = (b & 0x000fffffffffffffLL) | 0x3ff0000000000000LL; /* m in [1,2) */
  if (mb > 0x3ff6a09e667f3bcdLL) {                                   /* m > sqrt(2) */
    mb -= 0x0010000000000000LL;                                      /* m /= 2 */
    e += 1;
  }
  const double f = pmp_bitsd(mb) - 1.0; /* exact */
  const double s = f / (2.0 + f);
  const double z = s * s;
  double R = 8.695652173913043e-02; /* 2/23 */
  R = fma(R, z, 9.523809523809523e-02);
  R = fma(R, z, 1.0526315789473684e-01);
  R = fma(R, z, 1.1764705882352941e-01);
  R = fma(R, z, 1.3333333333333333e-01);
  R = fma(R, z, 1.5384615384615385e-01);
  R = fma(R, z, 1.8181818181818182e-01);
  R = fma(R, z, 2.2222222222222222e-01);
  R = fma(R, z, 2.857142857142857e-01);
  R = fma(R, z, 4.0e-01);
  R = fma(R, z, 6.666666666666666e-01);
  R = R * z;
  const double hfsq = 0.5 * f * f;
  const double de = (double)e;
  const double lo = fma(s, hfsq + R, de * PMP_LN2_LO);
  return fma(de, PMP_LN2_HI, f - (hfsq - lo));
}

PMP_HD double pmp_log1p(double x)
{
  const double u = 1.0 + x;
  if (u == 1.0) {
    return x;
  }
  return pmp_log(u) * (x / (u - 1.0));
}

/* x^y for x > 0 (x == 0 gives 0 for y > 0, 1 for y == 0) */
PMP_HD double pmp_pow(double x, double y)
{
  if (x == 0.0) {
    return (y > 0.0) ? 0.0 : ((y == 0.0) ? 1.0 : HUGE_VAL);
  }
  return pmp_exp(y * pmp_log(x));
}

PMP_HD double pmp_cbrt(double x)
{
  if (x == 0.0 || !(x == x)) {
    return x;
  }
  const double a = fabs(x);
  double y = pmp_exp(pmp_log(a) * (1.0 / 3.0));
  /* Newton step y -= (y^3 - a) / (3 y^2) with the residual formed from the
   * exact product y*y = y2 + e2 */
  const double y2 = y * y;
  const double e2 = fma(y, y, -y2);
  double r = fma(y2, y, -a);
  r = fma(e2, y, r);
  y = y - r / (3.0 * y2);
  return (x < 0.0) ? -y : y;
}

#if defined(PMP_USE_LIBM)
#define PMP_EXP exp
#define PMP_LOG log
#define PMP_LOG1P log1p
#define PMP_POW pow
#define PMP_CBRT cbrt
#else
#define PMP_EXP pmp_exp
#define PMP_LOG pmp_log
#define PMP_LOG1P pmp_log1p
#define PMP_POW pmp_pow
#define PMP_CBRT pmp_cbrt
#endif

#endif /* PMP_MATH_H */
