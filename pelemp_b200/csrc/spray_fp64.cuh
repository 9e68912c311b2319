// spray_fp64.cuh -- the plain FP64 spray update kernel.
//
// One thread per droplet, droplets in the library's cell-sorted SoA, one CTA
// per chunk of a box.  Per droplet the kernel runs the device lambda of
// SprayParticleContainer::updateParticles (Source/PP_Spray/SprayParticles.cpp:324-481):
// cell location, bounds check, then for each sub-cycle the trilinear gather
// (SprayInterpolation.H:99-199), calcBoilT (SprayFuelData.H:178-200),
// calculateSpraySource (Drag.H:138-441) with calcVaporState and
// calcHeatCoeff, the atomic source scatter and the move with wall handling
// (WallFunctions.H:89-234).  All droplet state stays in registers; register
// arrays are only indexed by compile-time indices (fuel species are picked
// with unrolled selects).
//
// Exactness: this file is compiled with -fmad=false and evaluates every
// expression in the reference's order with the project math library, the
// same functions the CPU oracle uses.  Each droplet's new state and its
// deposit increments are therefore bit-identical to the oracle's; only the
// order in which atomics add the increments into a cell differs.
#pragma once

#include <cfloat>

#include "phys/pmp_math.h"
#include "pmp_device.cuh"

namespace pmp {

__device__ __forceinline__ double dmin(double a, double b) { return (b < a) ? b : a; }
__device__ __forceinline__ double dmax(double a, double b) { return (a < b) ? b : a; }

__device__ __forceinline__ double cubic(const double* c, double x)
{
  return fma(fma(fma(c[3], x, c[2]), x, c[1]), x, c[0]);
}

// a[i] for a runtime i without indexing a register array
template <int N>
__device__ __forceinline__ double sel(const double (&a)[N], int i)
{
  double v = a[0];
#pragma unroll
  for (int k = 1; k < N; ++k) {
    v = (k == i) ? a[k] : v;
  }
  return v;
}

// a[i] = v for a runtime i
template <int N>
__device__ __forceinline__ void put(double (&a)[N], int i, double v)
{
#pragma unroll
  for (int k = 0; k < N; ++k) {
    a[k] = (k == i) ? v : a[k];
  }
}

template <int NS, int NF>
struct GasVals {
  double vel[3];
  double T;
  double rho;
  double p;
  double Y[NS];
  double mw_mix;
  double mom_src[3];
  double mass_src;
  double Ydot[NF];
  double eng_src;
};

__device__ __forceinline__ double rhoL(const DevFuel& f, double T, int spf)
{
  const double a = f.rho_coef[4 * spf];
  const double b = f.rho_coef[4 * spf + 1];
  const double c = f.rho_coef[4 * spf + 2];
  const double d = f.rho_coef[4 * spf + 3];
  return a + T * (b + T * (c + T * d));
}

// log1p(x) and (1 + x)^0.7 sharing one log(1 + x); bit-identical to
// pmp_log1p(x) and pmp_pow(1. + x, 0.7) for x > -1
__device__ __forceinline__ void log1p_pow07(double x, double& l1p, double& p07)
{
  const double u = 1. + x;
  const double lu = pmp_log(u);
  l1p = (fabs(x) < 0.0078125) ? pmp_log1p_core(x) : pmp_log1p_from(x, u, lu);
  p07 = pmp_exp(0.7 * lu);
}

// calcHeatCoeff (Drag.H:6-45); pow(BM1, phi) = exp(phi log BM1) with the
// loop-invariant log hoisted (bit-identical to pmp_pow)
__device__ __forceinline__ double heat_coeff(
  double ratio, double B_M, double B_eps, double C_eps, double Nu_0)
{
  if (B_M <= C_eps) {
    return 0.;
  }
  const int maxIter = 100;
  const double NU2 = Nu_0 - 2.;
  const double BM1 = 1. + B_M;
  const double lnBM1 = pmp_log(BM1);
  double phi = ratio / Nu_0;
  double B_T_old = pmp_exp(phi * lnBM1) - 1.;
  double logB, p07;
  log1p_pow07(B_T_old, logB, p07);
  double invFT = B_T_old / (logB * p07);
  double Nu_num = 2. + NU2 * invFT;
  phi = ratio / Nu_num;
  double B_T = pmp_exp(phi * lnBM1) - 1.;
  double error = fabs(B_T - B_T_old);
  int k = 0;
  while (k < maxIter && error > B_eps) {
    B_T_old = B_T;
    log1p_pow07(B_T, logB, p07);
    invFT = B_T / (logB * p07);
    Nu_num = 2. + NU2 * invFT;
    phi = ratio / Nu_num;
    B_T = pmp_exp(phi * lnBM1) - 1.;
    error = fabs(B_T - B_T_old);
    k++;
  }
  log1p_pow07(B_T, logB, p07);
  invFT = B_T / (logB * p07);
  Nu_num = 2. + NU2 * invFT;
  return Nu_num * logB / B_T;
}

// eos.T2Cpi / eos.T2Hi of species n at T (pmp_thermo.h, same operation
// order), converted to MKS: evaluated where needed instead of kept in
// per-species register arrays
template <bool PELEC = false>
__device__ __forceinline__ double cp_mks(const DevMech& m, int n, double T)
{
  const double* a = m.cp[n];
  const double cpr = fma(fma(fma(fma(a[4], T, a[3]), T, a[2]), T, a[1]), T, a[0]);
  return (cpr * m.ru_w[n]) * Units<PELEC>::eng;
}

template <bool PELEC = false>
__device__ __forceinline__ double h_mks(const DevMech& m, int n, double T)
{
  const double* hc = m.hc[n];
  const double hp = fma(fma(fma(fma(hc[4], T, hc[3]), T, hc[2]), T, hc[1]), T, hc[0]);
  return (fma(hp, T, hc[5]) * m.ru_w[n]) * Units<PELEC>::eng;
}

// eos.EY2T of the project EOS (pmp_eos_EY2T in phys/pmp_thermo.h, the same
// operations): temperature of specific internal energy e [erg/g], Newton
// from the guess T
template <int NS>
__device__ __forceinline__ double ey2t(const DevMech& m, double e, const double* Y, double T)
{
  double t = T;
  for (int it = 0; it < PMP_EY2T_MAXIT; ++it) {
    double em = 0., cv = 0.;
#pragma unroll
    for (int k = 0; k < NS; ++k) {
      const double rw = m.ru_w[k];
      const double* a = m.hc[k];
      const double hp = fma(fma(fma(fma(a[4], t, a[3]), t, a[2]), t, a[1]), t, a[0]);
      const double hk = fma(hp, t, a[5]) * rw;
      const double* c = m.cp[k];
      const double cpr = fma(fma(fma(fma(c[4], t, c[3]), t, c[2]), t, c[1]), t, c[0]);
      const double cpk = cpr * rw;
      em = fma(Y[k], fma(-rw, t, hk), em);
      cv = fma(Y[k], cpk - rw, cv);
    }
    const double dT = (e - em) / cv;
    t = t + dT;
    if (fabs(dT) <= 1e-11 * t) {
      break;
    }
  }
  return t;
}

// calculateSpraySource (Drag.H:138-441), PeleLMeX branch.  Updates vel, T,
// dia, Y in place; returns the number of inner sub-steps taken.  With sx
// (this thread's shared-memory slots, stride sxs), the parcel count, the
// start mass and the start composition wait there across the inner
// sub-steps instead of in registers: the same values, fewer spills.
template <int NS, int NF, bool PELEC = false>
__device__ __forceinline__ int spray_source_fp64(
  const KParams& P, double flow_dt, GasVals<NS, NF>& gpv, double* vel_io, double& T_io,
  double& dia_io, double* Y_io, double num_ppp, int& id, const double* cBoilT,
  double* sx = nullptr, int sxs = 0)
{
  const DevMech& m = P.m;
  const DevFuel& fdat = P.f;
  const double rule = 1. / 3.;
  const double C_eps = 1.E-15;
  const double B_eps = 1.E-7;
  const double min_mass = 1.E-13 * Units<PELEC>::mass;
  const int nSubMax = 100;
  double Y_skin[NS];
  double T_h = T_io;  // temperature of the last h_part evaluation (Drag.H:221)
  double Ddiag[NF];  // fuel rows only
  double L_fuel[NF];
  double mi_dot[NF];
  double Y_part[NF];
  double X_vapor[NF];
#pragma unroll
  for (int spf = 0; spf < NF; ++spf) {
    L_fuel[spf] = 0.;
    mi_dot[spf] = 0.;
    X_vapor[spf] = 0.;
  }
  const double num_ppp_ = num_ppp;
  double vel_part[3] = {vel_io[0], vel_io[1], vel_io[2]};
  if (fdat.fixed_parts) {
    vel_part[0] = vel_part[1] = vel_part[2] = 0.;
  }
  double T_part = T_io;
  double dia_part = dia_io;
  double rho_part = 0.;
#pragma unroll
  for (int spf = 0; spf < NF; ++spf) {
    Y_part[spf] = Y_io[spf];
    rho_part += Y_part[spf] / rhoL(fdat, dmin(T_part, cBoilT[spf]), spf);
  }
  rho_part = 1. / rho_part;
  double dt = flow_dt;
  int isub = 1;
  int nsub = 1;
  double pmass = PMP_PI / 6. * rho_part * pmp_pow(dia_part, 3.);
  double startmass = pmass;
  if (sx) {
    sx[3 * sxs] = num_ppp_;
    sx[4 * sxs] = startmass;
#pragma unroll
    for (int spf = 0; spf < NF; ++spf) {
      sx[(5 + spf) * sxs] = Y_io[spf];
    }
  }
  // the parcel count, read back from shared memory at each use when stashed
  const volatile double* vx = sx;
  auto nppp = [&]() { return vx ? vx[3 * sxs] : num_ppp_; };
  double part_vel_src[3];
  while (isub <= nsub) {
    double cp_part = 0.;
    double Tboil = 0.;
    double mw_part = 0.;
#pragma unroll
    for (int spf = 0; spf < NF; ++spf) {
      Tboil += Y_part[spf] * cBoilT[spf];
      cp_part += Y_part[spf] * fdat.cp[spf];
      mw_part += Y_part[spf] / m.mw_kg[fdat.indx[spf]];
    }
    mw_part = 1. / mw_part;
    const double delT = dmax(gpv.T - T_part, 0.);
    double T_skin = gpv.T;
    if (fdat.mass_trans) {
      T_skin = T_part + rule * delT;
    }
    // eos.T2Cpi(T_skin) and eos.T2Hi(T_part) (Drag.H:220-226): cp_mks(n, T_skin)
    // and h_mks(n, T_part) below
    T_h = T_part;
#pragma unroll
    for (int n = 0; n < NS; ++n) {
      Y_skin[n] = 0.;
    }
    double cp_skin = 0.;
    double mw_skin = 0.;
    double B_M = 0.;
    double sumXVap = 0.;
    if (fdat.mass_trans) {
      // calcVaporState (Drag.H:48-135)
      const double RU = kRuCgs * Units<PELEC>::ru;
      const double PATM = kPatmCgs * Units<PELEC>::pres;
      double mbar_vap = 0.;
#pragma unroll
      for (int spf = 0; spf < NF; ++spf) {
        const int fspec = fdat.indx[spf];
        const int fdspec = fdat.dep[spf];
        const double boilT_ref = fdat.boilT[spf];
        const double mw_fuel = m.mw_kg[fspec];
        const double Tp = dmin(T_part, 0.99 * cBoilT[spf]);
        const double part_latent = h_mks<PELEC>(m, fspec, T_part) + fdat.latent[spf] - fdat.cp[spf] * (Tp - fdat.ref_T);
        L_fuel[spf] = part_latent;
        double pres_sat = 0.;
        if (fdat.psat_coef[4 * spf + 3] == 0.) {
          pres_sat = PATM * pmp_exp(part_latent * mw_fuel / RU * (1. / boilT_ref - 1. / Tp));
        } else {
          const double a = fdat.psat_coef[4 * spf];
          const double b = fdat.psat_coef[4 * spf + 1];
          const double c = fdat.psat_coef[4 * spf + 2];
          const double d = fdat.psat_coef[4 * spf + 3];
          pres_sat = d * pmp_exp((a - b / (Tp + c)) * fdat.ln10);
        }
        const double X_fluid = sel(gpv.Y, fdspec) * gpv.mw_mix / mw_fuel;
        if (pres_sat > X_fluid * gpv.p) {
          const double Xl = Y_part[spf] * mw_part / mw_fuel;
          const double Xv = Xl * pres_sat / gpv.p;
          mbar_vap += Xv * mw_fuel;
          sumXVap += Xv;
          X_vapor[spf] = Xv;
        } else {
          X_vapor[spf] = 0.;
        }
      }
      const double totalmwx = mbar_vap + (1. - sumXVap) * gpv.mw_mix;
      double sumYSkin = 0.;
      double sumYfFluid = 0.;
      double sumYVap = 0.;
#pragma unroll
      for (int spf = 0; spf < NF; ++spf) {
        if (X_vapor[spf] > 0.) {
          const int fspec = fdat.indx[spf];
          const double mw_fuel = m.mw_kg[fspec];
          const double Yfv = X_vapor[spf] * mw_fuel / totalmwx;
          sumYVap += Yfv;
          const double gasY = sel(gpv.Y, fdat.dep[spf]);
          sumYfFluid += gasY;
          const double Ysk = Yfv + rule * (gasY - Yfv);
          put(Y_skin, fspec, Ysk);
          sumYSkin += Ysk;
        }
      }
      const double renorm = (1. - sumYSkin) / (1. - sumYfFluid);
#pragma unroll
      for (int n = 0; n < NS; ++n) {
        if (Y_skin[n] == 0.) {
          Y_skin[n] = gpv.Y[n] * renorm;
        }
        cp_skin += Y_skin[n] * cp_mks<PELEC>(m, n, T_skin);
        mw_skin += Y_skin[n] / m.mw_kg[n];
      }
      mw_skin = 1. / mw_skin;
      B_M = (sumYVap - sumYfFluid) / dmax(C_eps, (1. - sumYVap));
      B_M = dmin(20., B_M);
    } else {
#pragma unroll
      for (int n = 0; n < NS; ++n) {
        Y_skin[n] = gpv.Y[n];
        cp_skin += gpv.Y[n] * cp_mks<PELEC>(m, n, T_skin);
      }
      mw_skin = gpv.mw_mix;
    }
    double lambda_skin = 0.;
    double mu_skin = 0.;
    double rho_skin = gpv.rho;
    if (fdat.mass_trans) {
      rho_skin = mw_skin * gpv.p / (kRuCgs * Units<PELEC>::ru * T_skin);
    }
    // trans.transport at (T_skin, Y_skin) (pmp_thermo.h), fuel rows of Ddiag
    {
      double X[NS];
      double sumYW = 0.;
#pragma unroll
      for (int k = 0; k < NS; ++k) {
        sumYW += Y_skin[k] / m.mw_g[k];
      }
      const double wbar = 1.0 / sumYW;
#pragma unroll
      for (int k = 0; k < NS; ++k) {
        X[k] = Y_skin[k] * wbar / m.mw_g[k];
      }
      const double lnT = pmp_log(T_skin);
      double s = 0.0;
#pragma unroll
      for (int k = 0; k < NS; ++k) {
        s = fma(X[k], pmp_exp(6.0 * cubic(m.mu[k], lnT)), s);
      }
      mu_skin = pmp_exp(pmp_log(s) * (1.0 / 6.0));
      if (fdat.mass_trans) {
        double sl = 0.0;
#pragma unroll
        for (int k = 0; k < NS; ++k) {
          sl = fma(X[k], pmp_exp(0.25 * cubic(m.lam[k], lnT)), sl);
        }
        const double s2 = sl * sl;
        lambda_skin = s2 * s2;
        const double rt = kRuCgs * T_skin;
#pragma unroll
        for (int f = 0; f < NF; ++f) {
          const int i = fdat.indx[f];
          double term1 = 0.0;
          double term2 = 0.0;
#pragma unroll
          for (int j = 0; j < NS; ++j) {
            if (j != i) {
              term1 += Y_skin[j];
              term2 = fma(X[j], pmp_exp(-cubic(m.dbin[f][j], lnT)), term2);
            }
          }
          Ddiag[f] = m.mw_g[i] * term1 / (term2 * rt);
        }
      }
    }
    mu_skin *= Units<PELEC>::mu;
    lambda_skin *= Units<PELEC>::lambda;
    double diff_vel[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      diff_vel[d] = gpv.vel[d] - vel_part[d];
    }
    const double diff_vel_mag =
      sqrt(diff_vel[0] * diff_vel[0] + diff_vel[1] * diff_vel[1] + diff_vel[2] * diff_vel[2]);
    const double Reyn = rho_skin * diff_vel_mag * dia_part / mu_skin;
    const double inv_pmass = 1. / pmass;
    double drag_coef = 0.;
    if (Reyn > 1000.) {
      drag_coef = 0.424;
    } else if (Reyn > 1.) {
      drag_coef = 24. / Reyn * (1. + pmp_cbrt(Reyn * Reyn) / 6.);
    } else if (Reyn > 0.) {
      drag_coef = 24. / Reyn;
    }
    drag_coef *= (1. + 2.6432 * 0.);
    const double drag_force =
      0.125 * rho_skin * drag_coef * PMP_PI * dia_part * dia_part * diff_vel_mag;
    const double drag_force_p = 0.75 * rho_skin * drag_coef * diff_vel_mag / (dia_part * rho_part);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      part_vel_src[d] = drag_force_p * diff_vel[d] + fdat.body_force[d];
    }
    if (fdat.mom_trans) {
      const double nd = nppp() * drag_force;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        gpv.mom_src[d] += nd * diff_vel[d];
      }
      if (PELEC) {
        // drag work s_d,mu . u_d (Drag.H:282-286, PeleC branch)
        const double S_dmu_dot_u =
          diff_vel[0] * vel_part[0] + diff_vel[1] * vel_part[1] + diff_vel[2] * vel_part[2];
        gpv.eng_src += nd * S_dmu_dot_u;
      }
      if (isub == 1) {
        const double inv_tau_var = drag_force_p;
        nsub = min(max(nsub, static_cast<int>(flow_dt * inv_tau_var) + 1), nSubMax);
      }
    }
    double part_temp_src = 0.;
    double m_dot = 0.;
    if (fdat.mass_trans) {
      const double Pr_skin = mu_skin * cp_skin / lambda_skin;
      const double powR = dmax(pmp_pow(dmin(400., Reyn), 0.077), 1.);
      double Nu_num = 0.;
      double sumL = 0.;
      const double Nu_0 = 1. + powR * pmp_cbrt(1. + Reyn * Pr_skin);
      if (sumXVap > 0.) {
        double rhoDtotal = 0.;
        double cp_fuel = 0.;
        double sumYSkin = 0.;
#pragma unroll
        for (int spf = 0; spf < NF; ++spf) {
          const int fspec = fdat.indx[spf];
          Ddiag[spf] *= mw_skin / m.mw_kg[fspec] * Units<PELEC>::rhod;
          const double X_norm = X_vapor[spf] / sumXVap;
          Ddiag[spf] *= X_norm;
          rhoDtotal += Ddiag[spf];
          const double ysk = sel(Y_skin, fspec);
          cp_fuel += ysk * cp_mks<PELEC>(m, fspec, T_skin);
          sumYSkin += ysk;
        }
        cp_fuel /= sumYSkin;
        const double Sc_skin = mu_skin / rhoDtotal;
        double logB, pBM07;
        log1p_pow07(B_M, logB, pBM07);
        const double invFM = B_M / (logB * pBM07);
        const double Sh_0 = 1. + powR * pmp_cbrt(1. + Reyn * Sc_skin);
        const double Sh_num = 2. + (Sh_0 - 2.) * invFM;
        const double mdotcoeff = PMP_PI * dia_part * Sh_num * logB;
        const double ratio = cp_fuel * Sh_num * rhoDtotal / lambda_skin;
        Nu_num = heat_coeff(ratio, B_M, B_eps, C_eps, Nu_0);
#pragma unroll
        for (int spf = 0; spf < NF; ++spf) {
          if (X_vapor[spf] > 0.) {
            mi_dot[spf] = -dmax(Ddiag[spf] * mdotcoeff, 0.);
            m_dot += mi_dot[spf];
            sumL += mi_dot[spf] * L_fuel[spf];
          }
        }
      } else {
        Nu_num = Nu_0;
      }
      const double conv_src = PMP_PI * lambda_skin * dia_part * delT * Nu_num;
      gpv.eng_src += nppp() * conv_src;
      part_temp_src = (sumL + conv_src) * inv_pmass / cp_part;
      if (isub == 1 && delT > C_eps) {
        const double inv_tau_d = -m_dot / (0.2 * pmass);
        const double inv_tau_T = conv_src * inv_pmass / (cp_part * delT);
        nsub = min(
          max(nsub, max(static_cast<int>(flow_dt * inv_tau_d), static_cast<int>(flow_dt * inv_tau_T)) + 1),
          nSubMax);
      }
    }
    if (isub == 1) {
      dt = nsub == 1 ? flow_dt : flow_dt / static_cast<double>(nsub);  // the same value
    }
    const double part_dt = fdat.dtmod * dt;
    if (!fdat.fixed_parts) {
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        vel_part[d] += part_dt * part_vel_src[d];
      }
    }
    if (fdat.mass_trans) {
      const double newT = T_part + part_dt * part_temp_src;
      const double new_mass = pmass + m_dot * part_dt;
      if (new_mass > min_mass && newT < Tboil) {
        T_part = newT;
        if (NF > 1) {
          rho_part = 0.;
          double sumY = 0.;
#pragma unroll
          for (int spf = 0; spf < NF; ++spf) {
            Y_part[spf] = dmin(1., dmax(0., (Y_part[spf] * pmass + mi_dot[spf] * part_dt) / new_mass));
            if (Y_part[spf] <= 1.E-12) {
              Y_part[spf] = 0.;
            }
            sumY += Y_part[spf];
          }
#pragma unroll
          for (int spf = 0; spf < NF; ++spf) {
            Y_part[spf] /= sumY;
            rho_part += Y_part[spf] / rhoL(fdat, dmin(T_part, cBoilT[spf]), spf);
          }
          rho_part = 1. / rho_part;
        } else {
          rho_part = rhoL(fdat, dmin(T_part, cBoilT[0]), 0);
        }
        pmass = new_mass;
        dia_part = pmp_cbrt(6. * pmass / (PMP_PI * rho_part));
      } else {
        pmass = 0.;
        id = -1;
        nsub = isub;
        isub = nsub + 1;
      }
    }
    ++isub;
  }
  if (nsub > 1) {
    gpv.eng_src /= static_cast<double>(nsub);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      gpv.mom_src[d] /= static_cast<double>(nsub);
    }
  }
  double Y0[NF];
#pragma unroll
  for (int spf = 0; spf < NF; ++spf) {
    Y0[spf] = vx ? vx[(5 + spf) * sxs] : Y_io[spf];
  }
  if (vx) {
    startmass = vx[4 * sxs];
  }
  const double np_end = nppp();
  const double mdot_total = (pmass - startmass) / (fdat.dtmod * flow_dt);
  gpv.mass_src = np_end * mdot_total;
  if (PELEC) {
    // kinetic energy of the exchanged mass (Drag.H:418-421, PeleC branch)
    const double part_ke =
      0.5 * (vel_part[0] * vel_part[0] + vel_part[1] * vel_part[1] + vel_part[2] * vel_part[2]);
    gpv.eng_src += np_end * part_ke * mdot_total;
  }
  if (fdat.mom_trans) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      gpv.mom_src[d] += np_end * vel_part[d] * mdot_total;
    }
  }
#pragma unroll
  for (int spf = 0; spf < NF; ++spf) {
    const double oldY = Y0[spf];
    const double newY = Y_part[spf];
    const double midot = (newY * pmass - oldY * startmass) / (fdat.dtmod * flow_dt);
    gpv.Ydot[spf] = np_end * midot;
    gpv.eng_src += np_end * midot * h_mks<PELEC>(m, fdat.dep[spf], T_h);
    Y_io[spf] = Y_part[spf];
  }
  vel_io[0] = vel_part[0];
  vel_io[1] = vel_part[1];
  vel_io[2] = vel_part[2];
  T_io = T_part;
  dia_io = dia_part;
  return nsub;
}

// check_bounds (SprayInterpolation.H:64-97)
__device__ __forceinline__ bool check_bounds(const KParams& P, const double* pos, int* bflags)
{
#pragma unroll
  for (int hilo = 0; hilo < 2; ++hilo) {
    const int fact = (hilo == 0) ? 1 : -1;
#pragma unroll
    for (int dir = 0; dir < 3; ++dir) {
      const double dom_loc = (hilo == 0) ? P.plo[dir] : P.phi[dir];
      const int bflag = (hilo == 0) ? P.bndry_lo[dir] : P.bndry_hi[dir];
      if (bflag != 0) {
        const double diff = static_cast<double>(fact) * (pos[dir] - dom_loc);
        if (diff < 0.) {
          if (bflag == 1) {
            bflags[dir] = -fact;
          } else {
            return true;
          }
        } else if (diff < 0.5 * P.dx[dir]) {
          bflags[dir] = -2 * fact;
        }
      }
    }
  }
  return false;
}

// impose_wall without splash or EB (WallFunctions.H:89-234)
__device__ __forceinline__ void impose_wall(const KParams& P, double* pos, double* vel, const int* bflags)
{
  double normpos[3];
  int ijkc[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    normpos[d] = (pos[d] - P.plo[d]) / P.dx[d];
    ijkc[d] = static_cast<int>(floor(normpos[d]));
  }
  bool wall_check = false;
  double normal[3];
  double bcentv[3];
#pragma unroll
  for (int dir = 0; dir < 3; ++dir) {
    if ((bflags[dir] == -1 || bflags[dir] == 1) && !wall_check) {
      normal[dir] = -static_cast<double>(bflags[dir]);
      bcentv[dir] = static_cast<double>(ijkc[dir]) + 0.5 * static_cast<double>(1 - bflags[dir]);
      wall_check = true;
    } else {
      normal[dir] = 0.;
      bcentv[dir] = 0.;
    }
  }
  if (!wall_check) {
    return;
  }
  const double par_dot = (normpos[0] - bcentv[0]) * P.dx[0] * normal[0] +
                         (normpos[1] - bcentv[1]) * P.dx[1] * normal[1] +
                         (normpos[2] - bcentv[2]) * P.dx[2] * normal[2];
  if (par_dot < DBL_EPSILON) {
    const double Nw_Vp = normal[0] * vel[0] + normal[1] * vel[1] + normal[2] * vel[2];
#pragma unroll
    for (int dir = 0; dir < 3; ++dir) {
      vel[dir] -= 2. * Nw_Vp * normal[dir];
      pos[dir] -= 2. * par_dot * normal[dir];
    }
  }
}

__device__ __forceinline__ void set_error(const KParams& P, int code, int box, long long slot)
{
  if (atomicCAS(&P.status->code, 0, code) == 0) {
    P.status->box = box;
    P.status->slot = slot;
    if (P.err_host) {
      *reinterpret_cast<volatile int*>(P.err_host) = code;
    }
  }
}

// True when a call of the handle failed since the host last cleared the
// status: the CTA then leaves the droplets as they are, so that the state the
// host reads after pmp_spray_sync is the failing call's.  CTA-uniform (read
// once, shared), as the callers end in CTA- or warp-wide operations.
__device__ __forceinline__ bool cta_call_failed(const KParams& P)
{
  __shared__ int s_failed;
  if (threadIdx.x == 0) {
    s_failed = *reinterpret_cast<volatile const int*>(&P.status->code);
  }
  __syncthreads();
  return s_failed != 0;
}

// Append slot s to the call's FP64 fallback list.
__device__ __forceinline__ void push_fallback(const KParams& P, long long s)
{
  const unsigned long long k = atomicAdd(&P.status->fb_count, 1ULL);
  P.fb_list[k] = s;
  atomicAdd(&P.status->fallback, 1ULL);
}

// Append slot s to the learned form's list of gate rejections, which grows
// from the end of the fallback list (a droplet is on one of the two lists at
// most, so they never meet).
__device__ __forceinline__ void push_fallback_back(const KParams& P, long long s)
{
  const unsigned long long k = atomicAdd(&P.status->fb_gate, 1ULL);
  P.fb_list[P.fb_cap - 1 - (long long)k] = s;
  atomicAdd(&P.status->fallback, 1ULL);
}

// Off by default: on config 2 (16M droplets, 7-8 per cell, cell-sorted) the
// aggregation's shuffles cost more issue slots than the reductions it saves
// (mixed form 7.40e9 -> 7.18e9 droplet-substeps/s, FP64 2.26e9 -> 2.24e9).
#ifndef PMP_WARP_AGG_DEPOSITS
#define PMP_WARP_AGG_DEPOSITS 0
#endif

// One droplet's source increments of a sub-cycle, coef * {momentum (with
// mom_trans), density and the fuels' species (with mass_trans), energy},
// added into its source cell q (SprayParticles.cpp:419-441; nstride: the
// view's component stride).  Warp-aggregated: the lanes of the warp that
// deposit at the same time match on the cell; when every such group is a run
// of consecutive lanes (the droplets are sorted by cell, so they usually
// are), a segmented shuffle reduction sums each group's increments into its
// first lane, which alone issues the FP64 reductions -- one per cell and
// component instead of one per droplet.  Otherwise every lane issues its own.
// The sum order differs from lane-by-lane atomics only in rounding, as
// atomics are unordered anyway.
template <int NF>
__device__ __forceinline__ void deposit(const KParams& P, double* q, int nstride, double coef,
                                        const double* mom, double mass, const double* Ydot, double eng)
{
  constexpr int NC = 5 + NF;
  double v[NC];
  int off[NC];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    v[d] = coef * mom[d];
    off[d] = (P.s_mom + d) * nstride;
  }
  v[3] = coef * mass;
  off[3] = P.s_rho * nstride;
#pragma unroll
  for (int f = 0; f < NF; ++f) {
    v[4 + f] = coef * Ydot[f];
    off[4 + f] = (P.s_spec + f) * nstride;
  }
  v[4 + NF] = coef * eng;
  off[4 + NF] = P.s_eng * nstride;
  const bool mom_on = P.f.mom_trans != 0;
  const bool mass_on = P.f.mass_trans != 0;
#if PMP_WARP_AGG_DEPOSITS
  const unsigned act = __activemask();
  const unsigned peers = __match_any_sync(act, reinterpret_cast<unsigned long long>(q));
  const int lane = threadIdx.x & 31;
  const int first = __ffs(peers) - 1;
  const int last = 31 - __clz(peers);
  const bool run = __popc(peers) == last - first + 1;
  if (__all_sync(act, run)) {
    const int width = (int)__reduce_max_sync(act, (unsigned)(last - first + 1));
    for (int o = 1; o < width; o <<= 1) {
      const bool take = lane + o <= last;
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        const double t = __shfl_down_sync(act, v[c], o);
        v[c] = take ? v[c] + t : v[c];
      }
    }
    if (lane != first) {
      return;
    }
  }
#endif
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    const bool on = c < 3 ? mom_on : (c < 4 + NF ? mass_on : true);
    if (on) {
      red_add(q + off[c], v[c]);
    }
  }
}

__device__ __forceinline__ bool in_box(const int* lo, const int* hi, int i, int j, int k)
{
  return i >= lo[0] && i <= hi[0] && j >= lo[1] && j <= hi[1] && k >= lo[2] && k <= hi[2];
}

}  // namespace pmp
