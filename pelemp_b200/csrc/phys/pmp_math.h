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
 *  - exp:   Tang (ACM TOMS 15(2), 1989) table-driven: x = (128 m + j) ln2/128
 *           + r with a two-part ln2/128 (Cody & Waite), |r| <= ln2/256,
 *           exp(x) = 2^m T[j] (1 + expm1(r)), T[j] = 2^(j/128), expm1 by its
 *           degree-5 Taylor polynomial (truncation < 6e-19).  Arguments beyond
 *           |x| < 708 take a table-free path: Cody-Waite reduction by ln2 and
 *           the degree-13 Taylor polynomial, scaled in two halves.
 *  - log:   Tang (ACM TOMS 16(4), 1990) table-driven: x = 2^e m, m in
 *           [sqrt(1/2), sqrt(2)), c = 1 + j/128 with j = trunc(128 (m - 1)),
 *           log x = e ln2 + L_j + log1p(r), r = m INV_j - 1 (one fma, exact
 *           reduction, |r| < 0.0112), L_j = -log(INV_j) as hi + lo, log1p(r)
 *           by its degree-9 Taylor polynomial.  No division.  Zero,
 *           negative, subnormal and non-finite arguments take the atanh-series
 *           path (x = 2^e m, s = f/(2+f), log = 2 atanh s).
 *  - log1p: |x| < 1/128: the degree-9 series in x; otherwise u = 1 + x and
 *           log1p(x) = log(u) + (x - (u - 1))/u (Goldberg, "What every
 *           computer scientist should know about floating-point arithmetic",
 *           1991), the tiny correction multiplied by a single-precision
 *           reciprocal of u.
 *  - pow:   exp(y log x) for x > 0.
 *  - cbrt:  exp(log|x| / 3) refined by one Newton step on y^3 = |x| whose
 *           residual uses the exact product y*y = y2 + e2; the step divides
 *           by a single-precision reciprocal of 3 y^2 (the step is ~1e-15 of
 *           y, so 24 bits suffice).
 * Accuracy (checked in the tests against 50-digit decimal values): exp, log,
 * log1p, cbrt within 1.5 ulp; pow within 1.5 + 2 |y log x| ulp.
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

/* Newton iterations at most in the EOS inversion e(T, Y) -> T (pmp_eos_EY2T
 * in pmp_thermo.h and its device copy); shared so both stop alike. */
#define PMP_EY2T_MAXIT 20

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

#include "pmp_math_tables.h"

#define PMP_LOG2E 1.4426950408889634
#define PMP_LN2_HI 0.6931467056274414     /* ln 2, low 32 significand bits cleared */
#define PMP_LN2_LO 4.7493250390316726e-07 /* ln 2 - PMP_LN2_HI */
#define PMP_LN10 2.302585092994046
#define PMP_PI 3.141592653589793

/* 2^k as a double for -1022 <= k <= 1023 */
PMP_HD double pmp_pow2i(int k) { return pmp_bitsd((int64_t)(k + 1023) << 52); }

/* table-free exp (also the path for |x| >= 708, NaN, inf) */
PMP_HD double pmp_exp_cw(double x)
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

/* atanh-series log (also the path for zero, negative, subnormal, inf, NaN) */
PMP_HD double pmp_log_atanh(double x)
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

#if defined(__CUDACC__)
static __device__ double pmp_dev_exp2[PMP_EXP_N] = PMP_EXP2_TABLE;
static __device__ double pmp_dev_loginv[PMP_LOG_NTAB] = PMP_LOG_INV_TABLE;
static __device__ double pmp_dev_loglhi[PMP_LOG_NTAB] = PMP_LOG_LHI_TABLE;
static __device__ double pmp_dev_logllo[PMP_LOG_NTAB] = PMP_LOG_LLO_TABLE;
#endif
static const double pmp_host_exp2[PMP_EXP_N] = PMP_EXP2_TABLE;
static const double pmp_host_loginv[PMP_LOG_NTAB] = PMP_LOG_INV_TABLE;
static const double pmp_host_loglhi[PMP_LOG_NTAB] = PMP_LOG_LHI_TABLE;
static const double pmp_host_logllo[PMP_LOG_NTAB] = PMP_LOG_LLO_TABLE;

#if defined(__CUDA_ARCH__)
#define PMP_TAB(name, i) __ldg(&pmp_dev_##name[(i)])
#else
#define PMP_TAB(name, i) (pmp_host_##name[(i)])
#endif

PMP_HD double pmp_exp(double x)
{
  if (!(fabs(x) < 708.0)) {
    return pmp_exp_cw(x);
  }
  const double k = rint(x * PMP_INV_LN2_128);
  double r = fma(-k, PMP_LN2_128_HI, x); /* exact: k*HI has <= 52 bits */
  r = fma(-k, PMP_LN2_128_LO, r);
  const int ki = (int)k;
  const int j = ki & (PMP_EXP_N - 1);
  const int m = (ki - j) / PMP_EXP_N;
  double p = 8.333333333333333e-03; /* 1/120 */
  p = fma(p, r, 4.1666666666666664e-02);
  p = fma(p, r, 1.6666666666666666e-01);
  p = fma(p, r, 0.5);
  p = fma(p, r, 1.0);
  p = p * r; /* expm1(r) */
  const double t = PMP_TAB(exp2, j);
  return fma(t, p, t) * pmp_pow2i(m);
}

/* log1p(r) for |r| < 0.0112 (degree-9 Taylor) */
PMP_HD double pmp_log1p_core(double r)
{
  double q = 1.1111111111111111e-01; /* 1/9 */
  q = fma(q, r, -0.125);
  q = fma(q, r, 1.4285714285714285e-01);
  q = fma(q, r, -1.6666666666666666e-01);
  q = fma(q, r, 0.2);
  q = fma(q, r, -0.25);
  q = fma(q, r, 3.3333333333333331e-01);
  q = fma(q, r, -0.5);
  return fma(r * r, q, r);
}

PMP_HD double pmp_log(double x)
{
  int64_t b = pmp_dbits(x);
  /* positive normal finite only; everything else takes the atanh path */
  if (b < 0x0010000000000000LL || b >= 0x7ff0000000000000LL) {
    return pmp_log_atanh(x);
  }
  int e = (int)(b >> 52) - 1023;
  int64_t mb = (b & 0x000fffffffffffffLL) | 0x3ff0000000000000LL; /* m in [1,2) */
  if (mb > 0x3ff6a09e667f3bcdLL) {                                   /* m > sqrt(2) */
    mb -= 0x0010000000000000LL;
    e += 1;
  }
  const double m = pmp_bitsd(mb);
  const int j = (int)((m - 1.0) * 128.0) - PMP_LOG_JMIN; /* trunc toward zero */
  const double r = fma(m, PMP_TAB(loginv, j), -1.0);
  const double p = pmp_log1p_core(r);
  const double de = (double)e;
  const double hi = fma(de, PMP_LN2_HI, PMP_TAB(loglhi, j));
  const double lo = fma(de, PMP_LN2_LO, PMP_TAB(logllo, j)) + p;
  return hi + lo;
}

/* 1/u to single precision, the same bits on host and device */
PMP_HD double pmp_rcp24(double u)
{
#if defined(__CUDA_ARCH__)
  return (double)__fdiv_rn(1.0f, __double2float_rn(u));
#else
  return (double)(1.0f / (float)u);
#endif
}

/* log1p(x) given u = 1 + x and lu = pmp_log(u) (|x| >= 1/128) */
PMP_HD double pmp_log1p_from(double x, double u, double lu)
{
  const double c = x - (u - 1.0);
  if (c == 0.0) {
    return lu;
  }
  return fma(c, pmp_rcp24(u), lu);
}

PMP_HD double pmp_log1p(double x)
{
  if (fabs(x) < 0.0078125) {
    return pmp_log1p_core(x);
  }
  if (!(x > -1.0)) {
    return (x == -1.0) ? -HUGE_VAL : (x - x) / (x - x);
  }
  const double u = 1.0 + x;
  return pmp_log1p_from(x, u, pmp_log(u));
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
  const double d = 3.0 * y2;
  if (d > 1e-37 && d < 1e37) {
    y = fma(-r, pmp_rcp24(d), y);
  } else {
    y = y - r / d;
  }
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
