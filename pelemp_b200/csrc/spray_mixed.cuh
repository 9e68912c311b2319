// spray_mixed.cuh -- the mixed-precision spray update (PMP_MODE_MIXED).
//
// Same driver loop as the FP64 kernel (SprayParticles.cpp:324-481), with the
// per-droplet physics of calculateSpraySource (Drag.H:138-441) evaluated in
// FP32: gas thermo and transport, vapour state, the B_T fixed point, drag,
// Nusselt/Sherwood numbers, from FP32 copies of the tables (DevMechF,
// DevFuelF).  FP64 is kept where precision is structural:
//  - cell indices and positions (bit-exact cells, as in the FP64 form);
//  - the trilinear gather of the FP64 mesh (FP64 fused multiply-adds);
//  - the droplet state update: velocity, temperature, mass, mass fractions
//    and diameter are integrated in FP64 from the FP32 rates;
//  - the deposits: mass and species sources are FP64 differences of FP64
//    droplet masses, so the liquid + gas mass balance closes to FP64
//    round-off exactly as in the plain form;
//  - droplets that enter a call with d < 2 um (approaching complete
//    evaporation) are not touched here: their slots go to a fallback list
//    and the FP64 kernel updates them (spray_update_fp64_list).
// FP32 transcendentals use the SFU (ex2/lg2) with exact power-of-two range
// reduction: relative error ~3e-7 independent of the argument.
//
// One deliberate difference from the FP64 algorithm: the B_T fixed point
// stops when |dB_T| <= max(1e-7, 8 eps_f32 |B_T|) -- FP32 cannot resolve
// 1e-7 once B_T > 1, and the reference threshold would then run to its
// 100-iteration cap.
#pragma once

#include "spray_fp64.cuh"

namespace pmp {

constexpr double kMixedMinDia = 2e-6;  // below: FP64 path
// The learned form's threshold (PeleLMeX units): the surrogate's errors are
// largest for the small droplets that heat and evaporate fastest, and below
// 4 um (0.05% of config-2 droplets) the FP64 kernel updates them instead.
constexpr double kLearnMinDia = 4e-6;

#ifndef PMP_MIXED_FULL_RANGE_SFU
#define PMP_MIXED_FULL_RANGE_SFU 1
#endif

#if PMP_MIXED_FULL_RANGE_SFU
// 2^x, e^x, log2 x on the SFU over the full range (ex2.approx / lg2.approx);
// the relative error of e^x is ~|x| 2^-24 from rounding x log2(e), plus the
// SFU's own, well inside the form's 1e-4 budget
__device__ __forceinline__ float fexp2(float x)
{
  float r;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

__device__ __forceinline__ float fexp(float x) { return fexp2(x * 1.44269502f); }

__device__ __forceinline__ float flog2(float x)
{
  float r;
  asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
#else
// 2^x for |x| < 126: SFU ex2 on the fraction, exact 2^k scaling
__device__ __forceinline__ float fexp2(float x)
{
  const float k = rintf(x);
  const float f = x - k;
  float r;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(f));
  return r * __int_as_float((static_cast<int>(k) + 127) << 23);
}

__device__ __forceinline__ float fexp(float x)
{
  // x log2(e) with a two-part constant so the fraction keeps full precision
  const float t = x * 1.44269502f;
  const float k = rintf(t);
  float f = fmaf(x, 1.44269502f, -k);
  f = fmaf(x, 1.925963e-8f, f);
  float r;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(f));
  return r * __int_as_float((static_cast<int>(k) + 127) << 23);
}

// log2(x) for positive normal x: SFU lg2 on the mantissa in [sqrt(1/2),sqrt(2)), exact exponent
__device__ __forceinline__ float flog2(float x)
{
  const int b = __float_as_int(x);
  int e = ((b >> 23) & 0xff) - 127;
  int mb = (b & 0x007fffff) | 0x3f800000;
  if (mb > 0x3fb504f3) {  // m > sqrt(2)
    mb -= 0x00800000;
    e += 1;
  }
  float r;
  asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(__int_as_float(mb)));
  return r + static_cast<float>(e);
}

#endif

__device__ __forceinline__ float flog(float x) { return flog2(x) * 0.693147181f; }

__device__ __forceinline__ float fpow(float x, float y)
{
  return (x == 0.f) ? 0.f : fexp2(y * flog2(x));
}

__device__ __forceinline__ float fdiv(float a, float b) { return __fdividef(a, b); }

__device__ __forceinline__ float fcbrt(float x)
{
  if (x == 0.f) {
    return 0.f;
  }
  const float a = fabsf(x);
  float y = fexp2(flog2(a) * (1.f / 3.f));
  y = y - fdiv(y * y * y - a, 3.f * y * y);
  return x < 0.f ? -y : y;
}

__device__ __forceinline__ float flog1p(float x)
{
  if (fabsf(x) < 1e-2f) {
    // x - x^2/2 + x^3/3 - x^4/4 + x^5/5
    return x * fmaf(x, fmaf(x, fmaf(x, fmaf(x, 0.2f, -0.25f), 1.f / 3.f), -0.5f), 1.f);
  }
  return flog(1.f + x);
}

// 1/x in FP64 from the FP32 reciprocal estimate and one Newton step (relative
// error ~2^-44): for the gas-state gather, whose result feeds FP32 physics
__device__ __forceinline__ double drcp_from_f(double x)
{
  const double r = (double)__fdividef(1.f, (float)x);
  return r * fma(-x, r, 2.);
}

// cbrt in FP64 from an FP32 estimate and one Newton step (error ~1e-16)
__device__ __forceinline__ double dcbrt_from_f(double a)
{
  const double y = static_cast<double>(fcbrt(static_cast<float>(a)));
  const double y2 = y * y;
  const double r = fma(y2, y, -a);
  return y - r * static_cast<double>(__frcp_rn(static_cast<float>(3.0 * y2)));
}

__device__ __forceinline__ float fcubic(const float* c, float x)
{
  return fmaf(fmaf(fmaf(c[3], x, c[2]), x, c[1]), x, c[0]);
}

// Species index (in the DevMechF order) of fuel spf's liquid and of the gas
// species it deposits into: fuel spf itself when the fuels come first
template <bool FF>
__device__ __forceinline__ int fuel_sp(const DevFuel& f, int spf)
{
  return FF ? spf : f.indx[spf];
}

template <bool FF>
__device__ __forceinline__ int dep_sp(const DevFuel& f, int spf)
{
  return FF ? spf : f.dep[spf];
}

template <int N>
__device__ __forceinline__ float fsel(const float (&a)[N], int i)
{
  float v = a[0];
#pragma unroll
  for (int k = 1; k < N; ++k) {
    v = (k == i) ? a[k] : v;
  }
  return v;
}

template <int N>
__device__ __forceinline__ void fput(float (&a)[N], int i, float v)
{
#pragma unroll
  for (int k = 0; k < N; ++k) {
    a[k] = (k == i) ? v : a[k];
  }
}

__device__ __forceinline__ float cpf(const DevMechF& m, int n, float T)
{
  const float* a = m.cp[n];
  return fmaf(fmaf(fmaf(fmaf(a[4], T, a[3]), T, a[2]), T, a[1]), T, a[0]) * m.ru_w_eng[n];
}

__device__ __forceinline__ float hf(const DevMechF& m, int n, float T)
{
  const float* c = m.hc[n];
  const float hp = fmaf(fmaf(fmaf(fmaf(c[4], T, c[3]), T, c[2]), T, c[1]), T, c[0]);
  return fmaf(hp, T, c[5]) * m.ru_w_eng[n];
}

// log1p(x) and (1 + x)^0.7 from one base-2 logarithm of 1 + x: the values
// flog1p(x) and fpow(1 + x, 0.7f) give, with one SFU logarithm fewer
__device__ __forceinline__ void flog1p_pow07(float x, float& l1p, float& p07)
{
  const float u = 1.f + x;
  const float l2 = flog2(u);
  l1p = fabsf(x) < 1e-2f ? flog1p(x) : l2 * 0.693147181f;
  p07 = (u == 0.f) ? 0.f : fexp2(0.7f * l2);
}

// calcHeatCoeff (Drag.H:6-45) in FP32; lnBM1 = ln(1 + B_M)
__device__ __forceinline__ float heat_coeff_f(float ratio, float B_M, float Nu_0, float lnBM1)
{
  if (B_M <= 1e-15f) {
    return 0.f;
  }
  const float NU2 = Nu_0 - 2.f;
  float phi = fdiv(ratio, Nu_0);
  float B_T_old = fexp(phi * lnBM1) - 1.f;
  float logB, p07;
  flog1p_pow07(B_T_old, logB, p07);
  float invFT = fdiv(B_T_old, logB * p07);
  float Nu_num = 2.f + NU2 * invFT;
  phi = fdiv(ratio, Nu_num);
  float B_T = fexp(phi * lnBM1) - 1.f;
  float error = fabsf(B_T - B_T_old);
  int k = 0;
  // B_T = exp(x) - 1 in FP32 lies on a grid of one ulp of 1 + B_T (1.2e-7
  // below 1), coarser than the 1e-7 tolerance for small B_T: there the
  // iterates can settle into a 1-ulp two-cycle that never meets it.  The
  // loop also stops when the change stops shrinking (the FP32 noise floor
  // of a contracting iteration) instead of running to 100 iterations.
  float prev_error = 3.4e38f;
  while (k < 100 && error > fmaxf(1e-7f, 8.f * 1.1920929e-7f * fabsf(B_T)) && error < prev_error) {
    prev_error = error;
    B_T_old = B_T;
    flog1p_pow07(B_T, logB, p07);
    invFT = fdiv(B_T, logB * p07);
    Nu_num = 2.f + NU2 * invFT;
    phi = fdiv(ratio, Nu_num);
    B_T = fexp(phi * lnBM1) - 1.f;
    error = fabsf(B_T - B_T_old);
    k++;
  }
  flog1p_pow07(B_T, logB, p07);
  invFT = fdiv(B_T, logB * p07);
  Nu_num = 2.f + NU2 * invFT;
  return fdiv(Nu_num * logB, B_T);
}

__device__ __forceinline__ float heat_coeff_f(float ratio, float B_M, float Nu_0)
{
  return heat_coeff_f(ratio, B_M, Nu_0, flog(1.f + B_M));
}

// interpolated gas state in FP32
template <int NS>
struct GasF {
  float vel[3];
  float T;
  float rho;
  float p;
  float Y[NS];
  float mw_mix;
};

// FP64 deposits of one sub-cycle
template <int NF>
struct SrcD {
  double mom[3];
  double mass;
  double Ydot[NF];
  double eng;
};

// Liquid density of the droplet, 1 / sum_f Y_f / rhoL_f: with two fuels as
// rhoL_0 rhoL_1 / (Y_0 rhoL_1 + Y_1 rhoL_0), one FP64 division instead of
// three (the same value to FP64 round-off).
template <int NF>
__device__ __forceinline__ double mixed_rho_liquid(const DevFuel& fdat, const double* Y, double T,
                                                   const float* cBoilT)
{
  if (NF == 2) {
    constexpr int f1 = NF > 1 ? 1 : 0;
    const double r0 = rhoL(fdat, dmin(T, (double)cBoilT[0]), 0);
    const double r1 = rhoL(fdat, dmin(T, (double)cBoilT[f1]), f1);
    return (r0 * r1) / (Y[0] * r1 + Y[f1] * r0);
  }
  double s = 0.;
#pragma unroll
  for (int spf = 0; spf < NF; ++spf) {
    s += Y[spf] / rhoL(fdat, dmin(T, (double)cBoilT[spf]), spf);
  }
  return 1. / s;
}

// Liquid density and diameter after an inner sub-step (mass pmass): with
// two fuels one FP64 division, r = 1 / (P S) with P = rhoL_0 rhoL_1 and
// S = Y_0 rhoL_1 + Y_1 rhoL_0, giving rho = P^2 r and 1 / rho = S^2 r.
template <int NF>
__device__ __forceinline__ void mixed_rho_dia(const DevFuel& fdat, const double* Y, double T, const float* cBoilT,
                                              double pmass, double& rho, double& dia)
{
  if (NF == 2) {
    constexpr int f1 = NF > 1 ? 1 : 0;
    const double r0 = rhoL(fdat, dmin(T, (double)cBoilT[0]), 0);
    const double r1 = rhoL(fdat, dmin(T, (double)cBoilT[f1]), f1);
    const double Pr = r0 * r1;
    const double S = Y[0] * r1 + Y[f1] * r0;
    const double r = 1. / (Pr * S);
    rho = Pr * Pr * r;
    dia = dcbrt_from_f((6. / PMP_PI) * pmass * (S * S * r));
    return;
  }
  // one fuel: the density itself, as the reference's update takes it
  // (Drag.H:396-398)
  rho = NF == 1 ? rhoL(fdat, dmin(T, (double)cBoilT[0]), 0) : mixed_rho_liquid<NF>(fdat, Y, T, cBoilT);
  dia = dcbrt_from_f(6. * pmass / (PMP_PI * rho));
}

// Composition after an inner sub-step (Drag.H:377-396): each fuel's mass
// Y_f m + mdot_f dt over the new mass, clipped to [0, 1], zeroed below
// 1e-12, renormalised.  When no clip or zeroing applies (nearly always) that
// is a_f / sum a, one FP64 division.
template <int NF>
__device__ __forceinline__ void mixed_new_composition(double* Y, double pmass, const float* mi_dot, double part_dt,
                                                      double new_mass)
{
  double a[NF];
  double asum = 0.;
  bool plain = true;
#pragma unroll
  for (int spf = 0; spf < NF; ++spf) {
    a[spf] = Y[spf] * pmass + (double)mi_dot[spf] * part_dt;
    asum += a[spf];
    plain = plain && a[spf] > 1.E-12 * new_mass && a[spf] <= new_mass;
  }
  if (plain) {
    const double inv = 1. / asum;
#pragma unroll
    for (int spf = 0; spf < NF; ++spf) {
      Y[spf] = a[spf] * inv;
    }
    return;
  }
  const double inv_nm = 1. / new_mass;
  double sumY = 0.;
#pragma unroll
  for (int spf = 0; spf < NF; ++spf) {
    Y[spf] = dmin(1., dmax(0., a[spf] * inv_nm));
    if (Y[spf] <= 1.E-12) {
      Y[spf] = 0.;
    }
    sumY += Y[spf];
  }
  const double inv_sum = 1. / sumY;
#pragma unroll
  for (int spf = 0; spf < NF; ++spf) {
    Y[spf] *= inv_sum;
  }
}

// calculateSpraySource with FP32 physics and FP64 state (see the file header);
// PELEC: CGS units and the drag-work and evaporated kinetic-energy terms of
// the energy source (Drag.H:282-286, 418-421).
template <int NS, int NF, bool FF, bool PELEC = false>
__device__ __forceinline__ int spray_source_mixed(
  const KParams& P, double flow_dt, const GasF<NS>& g, const float* cBoilT, double* vel_io,
  double& T_io, double& dia_io, double* Y_io, double num_ppp, int& id, SrcD<NF>& src,
  double* sx, int sxs)
{
  const DevMechF& m = P.mf;
  const DevFuelF& ff = P.ff;
  const DevFuel& fdat = P.f;
  const float rule = 1.f / 3.f;
  const float C_eps = 1.E-15f;
  const double min_mass = 1.E-13 * Units<PELEC>::mass;
  const int nSubMax = 100;
  const float RU = (float)(kRuCgs * Units<PELEC>::ru);
  const float PATM = (float)(kPatmCgs * Units<PELEC>::pres);
  float Y_skin[NS];
  float Ddiag[NF];
  float L_fuel[NF];
  float mi_dot[NF];
  float X_vapor[NF];
  double Y_part[NF];
#pragma unroll
  for (int spf = 0; spf < NF; ++spf) {
    L_fuel[spf] = 0.f;
    mi_dot[spf] = 0.f;
    X_vapor[spf] = 0.f;
  }
  double vel_part[3] = {vel_io[0], vel_io[1], vel_io[2]};
  if (fdat.fixed_parts) {
    vel_part[0] = vel_part[1] = vel_part[2] = 0.;
  }
  double T_part = T_io;
  double dia_part = dia_io;
#pragma unroll
  for (int spf = 0; spf < NF; ++spf) {
    Y_part[spf] = Y_io[spf];
  }
  double rho_part = mixed_rho_liquid<NF>(fdat, Y_part, T_part, cBoilT);
  double dt = flow_dt;
  int isub = 1;
  int nsub = 1;
  double pmass = PMP_PI / 6. * rho_part * (dia_part * dia_part * dia_part);
  const double startmass = pmass;
  {
    // values needed only after the inner sub-steps: in shared memory across them
    sx[3 * sxs] = num_ppp;
    sx[4 * sxs] = startmass;
#pragma unroll
    for (int spf = 0; spf < NF; ++spf) {
      sx[(5 + spf) * sxs] = Y_io[spf];
    }
  }
  // sums over the inner sub-steps in FP32; times the parcel count in FP64 at the end
  float eng_acc = 0.f;
  float mom_acc[3] = {0.f, 0.f, 0.f};
  float T_h = (float)T_part;
  while (isub <= nsub) {
    const float Tp_f = (float)T_part;
    T_h = Tp_f;
    const float dia_f = (float)dia_part;
    float cp_part = 0.f;
    double Tboil = 0.;
    float mw_part = 0.f;
#pragma unroll
    for (int spf = 0; spf < NF; ++spf) {
      const float yp = (float)Y_part[spf];
      Tboil += Y_part[spf] * (double)cBoilT[spf];
      cp_part += yp * ff.cp[spf];
      mw_part += yp * m.inv_mw_kg[fuel_sp<FF>(fdat, spf)];
    }
    mw_part = fdiv(1.f, mw_part);
    const float delT = fmaxf(g.T - Tp_f, 0.f);
    float T_skin = g.T;
    if (fdat.mass_trans) {
      T_skin = Tp_f + rule * delT;
    }
#pragma unroll
    for (int n = 0; n < NS; ++n) {
      Y_skin[n] = 0.f;
    }
    float cp_skin = 0.f;
    float mw_skin = 0.f;
    float B_M = 0.f;
    float sumXVap = 0.f;
    if (fdat.mass_trans) {
      float mbar_vap = 0.f;
#pragma unroll
      for (int spf = 0; spf < NF; ++spf) {
        const int fspec = fuel_sp<FF>(fdat, spf);
        const float mw_fuel = m.mw_kg[fspec];
        const float Tp = fminf(Tp_f, 0.99f * cBoilT[spf]);
        const float part_latent = hf(m, fspec, Tp_f) + ff.latent[spf] - ff.cp[spf] * (Tp - ff.ref_T);
        L_fuel[spf] = part_latent;
        float pres_sat;
        if (ff.psat_d[spf] == 0.f) {
          pres_sat = PATM * fexp(part_latent * mw_fuel / RU * (ff.inv_boilT[spf] - fdiv(1.f, Tp)));
        } else {
          pres_sat = ff.psat_d[spf] * fexp2((ff.psat_a[spf] - fdiv(ff.psat_b[spf], Tp + ff.psat_c[spf])) * 3.32192809f);
        }
        const float X_fluid = fsel(g.Y, dep_sp<FF>(fdat, spf)) * g.mw_mix * m.inv_mw_kg[fspec];
        if (pres_sat > X_fluid * g.p) {
          const float Xl = (float)Y_part[spf] * mw_part * m.inv_mw_kg[fspec];
          const float Xv = fdiv(Xl * pres_sat, g.p);
          mbar_vap += Xv * mw_fuel;
          sumXVap += Xv;
          X_vapor[spf] = Xv;
        } else {
          X_vapor[spf] = 0.f;
        }
      }
      const float inv_totalmwx = fdiv(1.f, mbar_vap + (1.f - sumXVap) * g.mw_mix);
      float sumYSkin = 0.f;
      float sumYfFluid = 0.f;
      float sumYVap = 0.f;
#pragma unroll
      for (int spf = 0; spf < NF; ++spf) {
        if (X_vapor[spf] > 0.f) {
          const int fspec = fuel_sp<FF>(fdat, spf);
          const float Yfv = X_vapor[spf] * m.mw_kg[fspec] * inv_totalmwx;
          sumYVap += Yfv;
          const float gasY = fsel(g.Y, dep_sp<FF>(fdat, spf));
          sumYfFluid += gasY;
          const float Ysk = Yfv + rule * (gasY - Yfv);
          fput(Y_skin, fspec, Ysk);
          sumYSkin += Ysk;
        }
      }
      const float renorm = fdiv(1.f - sumYSkin, 1.f - sumYfFluid);
#pragma unroll
      for (int n = 0; n < NS; ++n) {
        if (Y_skin[n] == 0.f) {
          Y_skin[n] = g.Y[n] * renorm;
        }
        cp_skin += Y_skin[n] * cpf(m, n, T_skin);
        mw_skin += Y_skin[n] * m.inv_mw_kg[n];
      }
      mw_skin = fdiv(1.f, mw_skin);
      B_M = fdiv(sumYVap - sumYfFluid, fmaxf(C_eps, (1.f - sumYVap)));
      B_M = fminf(20.f, B_M);
    } else {
#pragma unroll
      for (int n = 0; n < NS; ++n) {
        Y_skin[n] = g.Y[n];
        cp_skin += g.Y[n] * cpf(m, n, T_skin);
      }
      mw_skin = g.mw_mix;
    }
    float lambda_skin = 0.f;
    float mu_skin = 0.f;
    float rho_skin = g.rho;
    if (fdat.mass_trans) {
      rho_skin = fdiv(mw_skin * g.p, RU * T_skin);
    }
    {
      float X[NS];
      float sumYW = 0.f;
#pragma unroll
      for (int k = 0; k < NS; ++k) {
        sumYW += Y_skin[k] * m.inv_mw_g[k];
      }
      const float wbar = fdiv(1.f, sumYW);
#pragma unroll
      for (int k = 0; k < NS; ++k) {
        X[k] = Y_skin[k] * wbar * m.inv_mw_g[k];
      }
      const float lnT = flog(T_skin);
      float s = 0.f;
#pragma unroll
      for (int k = 0; k < NS; ++k) {
        s = fmaf(X[k], fexp(fcubic(m.mu6[k], lnT)), s);
      }
      mu_skin = fexp(flog(s) * (1.f / 6.f));
      if (fdat.mass_trans) {
        float sl = 0.f;
#pragma unroll
        for (int k = 0; k < NS; ++k) {
          sl = fmaf(X[k], fexp(fcubic(m.lam4[k], lnT)), sl);
        }
        const float s2 = sl * sl;
        lambda_skin = s2 * s2;
        const float inv_rt = fdiv(1.f, (float)kRuCgs * T_skin);
#pragma unroll
        for (int f = 0; f < NF; ++f) {
          const int i = fuel_sp<FF>(fdat, f);
          float term1 = 0.f;
          float term2 = 0.f;
#pragma unroll
          for (int j = 0; j < NS; ++j) {
            if (j != i) {
              term1 += Y_skin[j];
              term2 = fmaf(X[j], fexp(fcubic(m.dbinm[f][j], lnT)), term2);
            }
          }
          Ddiag[f] = fdiv(m.mw_g[i] * term1 * inv_rt, term2);
        }
      }
    }
    mu_skin *= (float)Units<PELEC>::mu;
    lambda_skin *= (float)Units<PELEC>::lambda;
    float diff_vel[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      diff_vel[d] = g.vel[d] - (float)vel_part[d];
    }
    const float diff_vel_mag =
      sqrtf(diff_vel[0] * diff_vel[0] + diff_vel[1] * diff_vel[1] + diff_vel[2] * diff_vel[2]);
    const float Reyn = fdiv(rho_skin * diff_vel_mag * dia_f, mu_skin);
    const float inv_pmass = __frcp_rn((float)pmass);  // consumed in FP32
    float drag_coef = 0.f;
    if (Reyn > 1000.f) {
      drag_coef = 0.424f;
    } else if (Reyn > 1.f) {
      drag_coef = fdiv(24.f, Reyn) * (1.f + fcbrt(Reyn * Reyn) * (1.f / 6.f));
    } else if (Reyn > 0.f) {
      drag_coef = fdiv(24.f, Reyn);
    }
    const float drag_force = 0.125f * rho_skin * drag_coef * (float)PMP_PI * dia_f * dia_f * diff_vel_mag;
    const float drag_force_p = fdiv(0.75f * rho_skin * drag_coef * diff_vel_mag, dia_f * (float)rho_part);
    float part_vel_src[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      part_vel_src[d] = drag_force_p * diff_vel[d] + ff.body_force[d];
    }
    if (fdat.mom_trans) {
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        mom_acc[d] = fmaf(drag_force, diff_vel[d], mom_acc[d]);
      }
      if (PELEC) {
        // drag work on the gas, (s_d,mu . u_d)
        float S = 0.f;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          S = fmaf(diff_vel[d], (float)vel_part[d], S);
        }
        eng_acc = fmaf(drag_force, S, eng_acc);
      }
      if (isub == 1) {
        nsub = min(max(nsub, static_cast<int>((float)flow_dt * drag_force_p) + 1), nSubMax);
      }
    }
    float part_temp_src = 0.f;
    float m_dot = 0.f;
    if (fdat.mass_trans) {
      const float Pr_skin = fdiv(mu_skin * cp_skin, lambda_skin);
      const float powR = fmaxf(fpow(fminf(400.f, Reyn), 0.077f), 1.f);
      float Nu_num = 0.f;
      float sumL = 0.f;
      const float Nu_0 = 1.f + powR * fcbrt(1.f + Reyn * Pr_skin);
      if (sumXVap > 0.f) {
        float rhoDtotal = 0.f;
        float cp_fuel = 0.f;
        float sumYSkin = 0.f;
        const float inv_sumX = fdiv(1.f, sumXVap);
#pragma unroll
        for (int spf = 0; spf < NF; ++spf) {
          const int fspec = fuel_sp<FF>(fdat, spf);
          Ddiag[spf] *= mw_skin * m.inv_mw_kg[fspec] * (float)Units<PELEC>::rhod * (X_vapor[spf] * inv_sumX);
          rhoDtotal += Ddiag[spf];
          const float ysk = fsel(Y_skin, fspec);
          cp_fuel += ysk * cpf(m, fspec, T_skin);
          sumYSkin += ysk;
        }
        cp_fuel = fdiv(cp_fuel, sumYSkin);
        const float Sc_skin = fdiv(mu_skin, rhoDtotal);
        float logB, pBM07;
        flog1p_pow07(B_M, logB, pBM07);
        const float invFM = fdiv(B_M, logB * pBM07);
        const float Sh_0 = 1.f + powR * fcbrt(1.f + Reyn * Sc_skin);
        const float Sh_num = 2.f + (Sh_0 - 2.f) * invFM;
        const float mdotcoeff = (float)PMP_PI * dia_f * Sh_num * logB;
        const float ratio = fdiv(cp_fuel * Sh_num * rhoDtotal, lambda_skin);
        // ln(1 + B_M): the logarithm above where it was taken from lg2, else again
        Nu_num = heat_coeff_f(ratio, B_M, Nu_0, fabsf(B_M) < 1e-2f ? flog(1.f + B_M) : logB);
#pragma unroll
        for (int spf = 0; spf < NF; ++spf) {
          if (X_vapor[spf] > 0.f) {
            mi_dot[spf] = -fmaxf(Ddiag[spf] * mdotcoeff, 0.f);
            m_dot += mi_dot[spf];
            sumL += mi_dot[spf] * L_fuel[spf];
          }
        }
      } else {
        Nu_num = Nu_0;
      }
      const float conv_src = (float)PMP_PI * lambda_skin * dia_f * delT * Nu_num;
      eng_acc += conv_src;
      part_temp_src = fdiv((sumL + conv_src) * inv_pmass, cp_part);
      if (isub == 1 && delT > C_eps) {
        const float inv_tau_d = fdiv(-m_dot, 0.2f * (float)pmass);
        const float inv_tau_T = fdiv(conv_src * inv_pmass, cp_part * delT);
        nsub = min(max(nsub, max(static_cast<int>((float)flow_dt * inv_tau_d),
                                 static_cast<int>((float)flow_dt * inv_tau_T)) + 1),
                   nSubMax);
      }
    }
    if (isub == 1) {
      dt = nsub == 1 ? flow_dt : flow_dt / static_cast<double>(nsub);
    }
    const double part_dt = fdat.dtmod * dt;
    if (!fdat.fixed_parts) {
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        vel_part[d] += part_dt * (double)part_vel_src[d];
      }
    }
    if (fdat.mass_trans) {
      const double newT = T_part + part_dt * (double)part_temp_src;
      const double new_mass = pmass + (double)m_dot * part_dt;
      if (new_mass > min_mass && newT < Tboil) {
        T_part = newT;
        if (NF > 1) {
          mixed_new_composition<NF>(Y_part, pmass, mi_dot, part_dt, new_mass);
        }
        pmass = new_mass;
        mixed_rho_dia<NF>(fdat, Y_part, T_part, cBoilT, pmass, rho_part, dia_part);
      } else {
        pmass = 0.;
        id = -1;
        nsub = isub;
        isub = nsub + 1;
      }
    }
    ++isub;
  }
  // back from shared memory (volatile: read there, not kept in registers)
  const volatile double* vx = sx;
  num_ppp = vx[3 * sxs];
  const double startmass_ = vx[4 * sxs];
  double Y0[NF];
#pragma unroll
  for (int spf = 0; spf < NF; ++spf) {
    Y0[spf] = vx[(5 + spf) * sxs];
  }
  src.eng = num_ppp * (double)eng_acc;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    src.mom[d] = num_ppp * (double)mom_acc[d];
  }
  if (nsub > 1) {
    src.eng /= static_cast<double>(nsub);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      src.mom[d] /= static_cast<double>(nsub);
    }
  }
  // 1 / (dtmod flow_dt), computed on the host (every caller passes the sub-cycle dt)
  const double inv_dtf = P.inv_dtf;
  const double mdot_total = (pmass - startmass_) * inv_dtf;
  src.mass = num_ppp * mdot_total;
  if (PELEC) {
    // kinetic energy carried by the evaporated mass
    const double part_ke = 0.5 * (vel_part[0] * vel_part[0] + vel_part[1] * vel_part[1] + vel_part[2] * vel_part[2]);
    src.eng += num_ppp * part_ke * mdot_total;
  }
  if (fdat.mom_trans) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      src.mom[d] += num_ppp * vel_part[d] * mdot_total;
    }
  }
#pragma unroll
  for (int spf = 0; spf < NF; ++spf) {
    const double midot = (Y_part[spf] * pmass - Y0[spf] * startmass_) * inv_dtf;
    src.Ydot[spf] = num_ppp * midot;
    src.eng += num_ppp * midot * (double)hf(m, dep_sp<FF>(fdat, spf), T_h);
    Y_io[spf] = Y_part[spf];
  }
  vel_io[0] = vel_part[0];
  vel_io[1] = vel_part[1];
  vel_io[2] = vel_part[2];
  T_io = T_part;
  dia_io = dia_part;
  return nsub;
}

}  // namespace pmp
