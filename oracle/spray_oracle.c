/* spray_oracle.c -- CPU FP64 oracle of the spray particle update.
 * TEST INFRASTRUCTURE: see spray_oracle.h for scope, sources and parity pin.
 * Build with -ffp-contract=off so that a*b+c stays two roundings, as in the
 * reference built without contraction.
 */
#include "spray_oracle.h"

#include <float.h>
#include <stdio.h>
#include <stdlib.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* SprayUnits, PeleLMeX branch (Source/PP_Spray/SprayFuelData.H:44-54,66) */
/* SprayUnits (SprayFuelData.H:42-67): PeleLMeX (PELELM_USE_SPRAY, MKS at
 * the interface) or PeleC (CGS throughout), chosen by
 * pmp_oracle_set_coupling; set before any other call, read-only after. */
typedef struct {
  double ru, eng, rho, mass, rhod, mu, lambda, pres;
} units_t;
static const units_t k_units_lmex = {1.E-7, 1.E-4, 1.E3, 1.E-3, 0.1, 0.1, 1.E-5, 0.1};
static const units_t k_units_pelec = {1., 1., 1., 1., 1., 1., 1., 1.};
static units_t g_units = {1.E-7, 1.E-4, 1.E3, 1.E-3, 0.1, 0.1, 1.E-5, 0.1};
static int g_pelec = 0;
#define U_RU_CONV (g_units.ru)
#define U_ENG_CONV (g_units.eng)
#define U_RHO_CONV (g_units.rho)
#define U_MASS_CONV (g_units.mass)
#define U_RHOD_CONV (g_units.rhod)
#define U_MU_CONV (g_units.mu)
#define U_LAMBDA_CONV (g_units.lambda)
#define U_PRES_CONV (g_units.pres)

void pmp_oracle_set_coupling(int pelec)
{
  g_pelec = pelec != 0;
  g_units = g_pelec ? k_units_pelec : k_units_lmex;
}

/* std::min / std::max semantics (amrex::min/max forward to them) */
static inline double dmin(double a, double b) { return (b < a) ? b : a; }
static inline double dmax(double a, double b) { return (a < b) ? b : a; }
static inline int imin(int a, int b) { return (b < a) ? b : a; }
static inline int imax(int a, int b) { return (a < b) ? b : a; }

/* GasPhaseVals (SprayFuelData.H:71-112) */
typedef struct {
  double vel_fluid[3];
  double T_fluid;
  double rho_fluid;
  double p_fluid;
  double Y_fluid[PMP_MAX_SPEC];
  double mw_mix;
  double mw[PMP_MAX_SPEC];
  double fluid_mom_src[3];
  double fluid_mass_src;
  double fluid_Y_dot[PMP_MAX_FUEL];
  double fluid_eng_src;
} gpv_t;

static void gpv_reset(gpv_t* g, int ns, int nf)
{
  for (int d = 0; d < 3; ++d) {
    g->fluid_mom_src[d] = 0.;
    g->vel_fluid[d] = 0.;
  }
  g->T_fluid = 0.;
  g->rho_fluid = 0.;
  g->fluid_eng_src = 0.;
  g->fluid_mass_src = 0.;
  for (int n = 0; n < ns; ++n) {
    g->Y_fluid[n] = 0.;
  }
  for (int n = 0; n < nf; ++n) {
    g->fluid_Y_dot[n] = 0.;
  }
}

static void gpv_define(gpv_t* g, int ns)
{
  g->mw_mix = 0.;
  for (int n = 0; n < ns; ++n) {
    g->mw_mix += g->Y_fluid[n] / g->mw[n];
  }
  g->p_fluid = g->rho_fluid * PMP_RU_CGS * g->mw_mix * g->T_fluid * U_RU_CONV;
  g->mw_mix = 1. / g->mw_mix;
}

/* SprayData member functions (SprayFuelData.H:144-211) */
static double rhoL(const pmp_spray_data* f, double T, int spf)
{
  const double a = f->rho_coef[4 * spf];
  const double b = f->rho_coef[4 * spf + 1];
  const double c = f->rho_coef[4 * spf + 2];
  const double d = f->rho_coef[4 * spf + 3];
  return a + T * (b + T * (c + T * d));
}

static void calcBoilT(const pmp_spray_data* f, const gpv_t* g, double* cBoilT)
{
  const double RU = PMP_RU_CGS * U_RU_CONV;
  const double PATM = PMP_PATM_CGS * U_PRES_CONV;
  for (int spf = 0; spf < f->nfuel; ++spf) {
    const int fspec = f->indx[spf];
    const double mw_fuel = g->mw[fspec];
    const double Hboil_ref =
      f->ref_latent[spf] *
      PMP_POW((f->critT[spf] - f->ref_T) / (f->critT[spf] - f->boilT[spf]), -0.38);
    cBoilT[spf] =
      1. / (PMP_LOG(PATM / g->p_fluid) * RU / (Hboil_ref * mw_fuel) + 1. / f->boilT[spf]);
    cBoilT[spf] = dmin(f->critT[spf], cBoilT[spf]);
  }
}

static double psat(const pmp_spray_data* f, double T, int spf)
{
  const double a = f->psat_coef[4 * spf];
  const double b = f->psat_coef[4 * spf + 1];
  const double c = f->psat_coef[4 * spf + 2];
  const double d = f->psat_coef[4 * spf + 3];
  return d * PMP_POW(10., a - b / (T + c));
}

/* calcHeatCoeff (Drag.H:6-45) */
static double calcHeatCoeff(
  double ratio, double B_M, double B_eps, double C_eps, double Nu_0)
{
  if (B_M <= C_eps) {
    return 0.;
  }
  const int maxIter = 100;
  const double NU2 = Nu_0 - 2.;
  const double BM1 = 1. + B_M;
  double phi = ratio / Nu_0;
  double B_T_old = PMP_POW(BM1, phi) - 1.;
  double logB = PMP_LOG1P(B_T_old);
  double invFT = B_T_old / (logB * PMP_POW(1. + B_T_old, 0.7));
  double Nu_num = 2. + NU2 * invFT;
  phi = ratio / Nu_num;
  double B_T = PMP_POW(BM1, phi) - 1.;
  double error = fabs(B_T - B_T_old);
  int k = 0;
  while (k < maxIter && error > B_eps) {
    B_T_old = B_T;
    logB = PMP_LOG1P(B_T);
    invFT = B_T / (logB * PMP_POW(1. + B_T, 0.7));
    Nu_num = 2. + NU2 * invFT;
    phi = ratio / Nu_num;
    B_T = PMP_POW(BM1, phi) - 1.;
    error = fabs(B_T - B_T_old);
    k++;
  }
  logB = PMP_LOG1P(B_T);
  invFT = B_T / (logB * PMP_POW(1. + B_T, 0.7));
  Nu_num = 2. + NU2 * invFT;
  return Nu_num * logB / B_T;
}

/* calcVaporState (Drag.H:48-135) */
static void calcVaporState(
  const pmp_mech* mech, const pmp_spray_data* fdat, const gpv_t* gpv,
  double rule, double T_in, double C_eps, double mw_part, const double* Y_l,
  const double* h_part, const double* cp_n, const double* cBoilT,
  double* Y_skin, double* X_vapor, double* L_fuel, double* B_M,
  double* sumXVap, double* cp_skin, double* mw_skin)
{
  const int NF = fdat->nfuel;
  const int NS = mech->nspec;
  const double RU = PMP_RU_CGS * U_RU_CONV;
  const double PATM = PMP_PATM_CGS * U_PRES_CONV;
  double mbar_vap = 0.;
  for (int spf = 0; spf < NF; ++spf) {
    const int fspec = fdat->indx[spf];
    const int fdspec = fdat->dep_indx[spf];
    const double boilT_ref = fdat->boilT[spf];
    const double mw_fuel = gpv->mw[fspec];
    const double T_part = dmin(T_in, 0.99 * cBoilT[spf]);
    const double part_latent =
      h_part[fspec] + fdat->latent[spf] - fdat->cp[spf] * (T_part - fdat->ref_T);
    L_fuel[spf] = part_latent;
    double pres_sat = 0.;
    if (fdat->psat_coef[4 * spf + 3] == 0.) {
      pres_sat = PATM * PMP_EXP(part_latent * mw_fuel / RU * (1. / boilT_ref - 1. / T_part));
    } else {
      pres_sat = psat(fdat, T_part, spf);
    }
    const double X_fluid = gpv->Y_fluid[fdspec] * gpv->mw_mix / mw_fuel;
    if (pres_sat > X_fluid * gpv->p_fluid) {
      const double Xl = Y_l[spf] * mw_part / mw_fuel;
      const double Xv = Xl * pres_sat / gpv->p_fluid;
      mbar_vap += Xv * mw_fuel;
      *sumXVap += Xv;
      X_vapor[spf] = Xv;
    } else {
      X_vapor[spf] = 0.;
    }
  }
  const double totalmwx = mbar_vap + (1. - *sumXVap) * gpv->mw_mix;
  double sumYSkin = 0.;
  double sumYfFluid = 0.;
  double sumYVap = 0.;
  for (int spf = 0; spf < NF; ++spf) {
    if (X_vapor[spf] > 0.) {
      const int fspec = fdat->indx[spf];
      const int fdspec = fdat->dep_indx[spf];
      const double mw_fuel = gpv->mw[fspec];
      const double Yfv = X_vapor[spf] * mw_fuel / totalmwx;
      sumYVap += Yfv;
      const double gasY = gpv->Y_fluid[fdspec];
      sumYfFluid += gasY;
      const double Ysk = Yfv + rule * (gasY - Yfv);
      Y_skin[fspec] = Ysk;
      sumYSkin += Ysk;
    }
  }
  const double renorm = (1. - sumYSkin) / (1. - sumYfFluid);
  for (int n = 0; n < NS; ++n) {
    if (Y_skin[n] == 0.) {
      Y_skin[n] = gpv->Y_fluid[n] * renorm;
    }
    *cp_skin += Y_skin[n] * cp_n[n];
    *mw_skin += Y_skin[n] / gpv->mw[n];
  }
  *mw_skin = 1. / *mw_skin;
  *B_M = (sumYVap - sumYfFluid) / dmax(C_eps, (1. - sumYVap));
  *B_M = dmin(20., *B_M);
}

/* calculateSpraySource (Drag.H:138-441), PeleLMeX branch (no KE terms).
 * rdata = droplet real components; returns the Reynolds number. */
/* calculateSpraySource (Drag.H:138-441).
 *
 * eres (may be NULL) accumulates the droplet's term of the energy identity of
 * the explicit scheme (PeleLMeX coupling): the liquid enthalpy change plus the
 * enthalpy the gas receives equals, per parcel of num_ppp droplets,
 *   sum_i sum_f [ dM_fi cp_f (T_{i+1} - T_i)                 explicit update
 *               + (p mdot_fi - dM_fi) L_fi                   composition clip
 *               + p mdot_fi (L'_fi - L_fi)                   latent heat below boiling
 *               + dM_fi (h_f(T_i) - h_dep(f)(T_last)) ]      vapour enthalpy at T_last
 *   + sum_f M_fk L_fk - p conv_k                             kill at step k
 *   - (nsub / k - 1) sum_{i<=k} p conv_i                     average over k steps
 * with i the inner sub-steps (part_dt p, droplet temperature T_i, fuel masses
 * M_fi = m Y_f, their change dM_fi, the evaporation rates mdot_fi that enter
 * the temperature update, convective heat conv_i), the liquid enthalpy
 * h_L,f(T) = cp_f (T - ref_T) - latent_f and the latent heat it implies
 * L_fi = h_f(T_i) - h_L,f(T_i); the temperature update uses L'_fi, the same
 * expression at min(T_i, 0.99 cBoilT) (Drag.H:79-83); the vapour enthalpy the
 * gas receives is taken at the last sub-step's droplet temperature T_last
 * (Drag.H:425-434), the convective heat averaged over nsub (Drag.H:410-413),
 * and when the droplet dies at sub-step k (Drag.H:401-406) its remaining
 * mass passes to the gas as vapour with the heat of that sub-step unabsorbed. */
static double calculateSpraySource(
  const pmp_mech* mech, double flow_dt, gpv_t* gpv, const pmp_spray_data* fdat,
  double* rdata, int* id, double* cBoilT, double* eres)
{
  const int NF = fdat->nfuel;
  const int NS = mech->nspec;
  const double rule = 1. / 3.;
  const double C_eps = 1.E-15;
  const double B_eps = 1.E-7;
  const double min_mass = 1.E-13 * U_MASS_CONV;
  const int nSubMax = 100;
  int get_Ddiag = 1;
  int get_lambda = 1;
  const int get_mu = 1;
  if (!fdat->mass_trans) {
    get_Ddiag = 0;
    get_lambda = 0;
  }
  double Y_skin[PMP_MAX_SPEC];
  double h_part[PMP_MAX_SPEC];
  double cp_n[PMP_MAX_SPEC];
  double Ddiag[PMP_MAX_SPEC];
  double L_fuel[PMP_MAX_FUEL] = {0.0};
  double mi_dot[PMP_MAX_FUEL] = {0.0};
  double Y_part[PMP_MAX_FUEL];
  double X_vapor[PMP_MAX_FUEL] = {0.0};
  const double num_ppp = rdata[PMP_PSTATE_NUMDENS(NF)];
  double vel_part[3] = {rdata[0], rdata[1], rdata[2]};
  double y_tab = 0.;
  if (fdat->do_breakup == 1) {
    y_tab = rdata[PMP_PSTATE_BM1(NF)];
  }
  if (fdat->fixed_parts) {
    vel_part[0] = vel_part[1] = vel_part[2] = 0.;
  }
  double T_part = rdata[PMP_PSTATE_T];
  double dia_part = rdata[PMP_PSTATE_DIA];
  double rho_part = 0.;
  for (int spf = 0; spf < NF; ++spf) {
    Y_part[spf] = rdata[PMP_PSTATE_Y + spf];
    rho_part += Y_part[spf] / rhoL(fdat, dmin(T_part, cBoilT[spf]), spf);
  }
  rho_part = 1. / rho_part;
  double dt = flow_dt;
  int isub = 1;
  int nsub = 1;
  double pmass = PMP_PI / 6. * rho_part * PMP_POW(dia_part, 3);
  const double startmass = pmass;
  double Reyn = 0.;
  double part_vel_src[3];
  /* energy identity terms (eres) */
  double e_expl = 0., e_clip = 0., e_lat = 0., e_vap = 0., e_kill = 0., e_conv = 0.;
  double dM_tot[PMP_MAX_FUEL] = {0.0};
  int nsub_first = 1, k_kill = 0;
  while (isub <= nsub) {
    double cp_part = 0.;
    double Tboil = 0.;
    double mw_part = 0.;
    for (int spf = 0; spf < NF; ++spf) {
      Tboil += Y_part[spf] * cBoilT[spf];
      cp_part += Y_part[spf] * fdat->cp[spf];
      mw_part += Y_part[spf] / gpv->mw[fdat->indx[spf]];
    }
    mw_part = 1. / mw_part;
    const double delT = dmax(gpv->T_fluid - T_part, 0.);
    double T_skin = gpv->T_fluid;
    if (fdat->mass_trans) {
      T_skin = T_part + rule * delT;
    }
    pmp_eos_T2Cpi(mech, T_skin, cp_n);
    pmp_eos_T2Hi(mech, T_part, h_part);
    for (int n = 0; n < NS; ++n) {
      Y_skin[n] = 0.;
      h_part[n] *= U_ENG_CONV;
      cp_n[n] *= U_ENG_CONV;
    }
    double cp_skin = 0.;
    double mw_skin = 0.;
    double B_M = 0.;
    double sumXVap = 0.;
    if (fdat->mass_trans) {
      calcVaporState(
        mech, fdat, gpv, rule, T_part, C_eps, mw_part, Y_part, h_part, cp_n,
        cBoilT, Y_skin, X_vapor, L_fuel, &B_M, &sumXVap, &cp_skin, &mw_skin);
    } else {
      for (int n = 0; n < NS; ++n) {
        Y_skin[n] = gpv->Y_fluid[n];
        cp_skin += gpv->Y_fluid[n] * cp_n[n];
      }
      mw_skin = gpv->mw_mix;
    }
    double lambda_skin = 0.;
    double mu_skin = 0.;
    double rho_skin = gpv->rho_fluid;
    if (fdat->mass_trans) {
      rho_skin = mw_skin * gpv->p_fluid / (PMP_RU_CGS * U_RU_CONV * T_skin);
    }
    const double rho_cgs = rho_skin / U_RHO_CONV;
    pmp_transport(
      mech, get_mu, get_lambda, get_Ddiag, T_skin, rho_cgs, Y_skin, Ddiag,
      &mu_skin, &lambda_skin);
    mu_skin *= U_MU_CONV;
    lambda_skin *= U_LAMBDA_CONV;
    double diff_vel[3];
    for (int d = 0; d < 3; ++d) {
      diff_vel[d] = gpv->vel_fluid[d] - vel_part[d];
    }
    const double diff_vel_mag = sqrt(
      diff_vel[0] * diff_vel[0] + diff_vel[1] * diff_vel[1] + diff_vel[2] * diff_vel[2]);
    Reyn = rho_skin * diff_vel_mag * dia_part / mu_skin;

    const double inv_pmass = 1. / pmass;
    double drag_coef = 0.;
    if (Reyn > 1000.) {
      drag_coef = 0.424;
    } else if (Reyn > 1.) {
      drag_coef = 24. / Reyn * (1. + PMP_CBRT(Reyn * Reyn) / 6.);
    } else if (Reyn > 0.) {
      drag_coef = 24. / Reyn;
    }
    drag_coef *= (1. + 2.6432 * y_tab);
    const double drag_force =
      0.125 * rho_skin * drag_coef * PMP_PI * dia_part * dia_part * diff_vel_mag;
    const double drag_force_p =
      0.75 * rho_skin * drag_coef * diff_vel_mag / (dia_part * rho_part);
    for (int d = 0; d < 3; ++d) {
      part_vel_src[d] = drag_force_p * diff_vel[d] + fdat->body_force[d];
    }
    if (fdat->mom_trans) {
      const double nd = num_ppp * drag_force;
      for (int d = 0; d < 3; ++d) {
        gpv->fluid_mom_src[d] += nd * diff_vel[d];
      }
      if (g_pelec) {
        /* drag work s_d,mu . u_d, PeleC branch (Drag.H:282-286) */
        const double S_dmu_dot_u = diff_vel[0] * vel_part[0] + diff_vel[1] * vel_part[1] +
                                   diff_vel[2] * vel_part[2];
        gpv->fluid_eng_src += nd * S_dmu_dot_u;
      }
      if (isub == 1) {
        const double inv_tau_var = drag_force_p;
        nsub = imin(imax(nsub, (int)(flow_dt * inv_tau_var) + 1), nSubMax);
      }
    }

    double part_temp_src = 0.;
    double m_dot = 0.;
    double conv_i = 0.;                    /* this sub-step's convective heat */
    double mL[PMP_MAX_FUEL] = {0.0};      /* the rates in its temperature update */
    if (fdat->mass_trans) {
      const double Pr_skin = mu_skin * cp_skin / lambda_skin;
      const double powR = dmax(PMP_POW(dmin(400., Reyn), 0.077), 1.);
      double Nu_num = 0.;
      double sumL = 0.;
      const double Nu_0 = 1. + powR * PMP_CBRT(1. + Reyn * Pr_skin);
      if (sumXVap > 0.) {
        double rhoDtotal = 0.;
        double cp_fuel = 0.;
        double sumYSkin = 0.;
        for (int spf = 0; spf < NF; ++spf) {
          const int fspec = fdat->indx[spf];
          Ddiag[fspec] *= mw_skin / gpv->mw[fspec] * U_RHOD_CONV;
          const double X_norm = X_vapor[spf] / sumXVap;
          Ddiag[fspec] *= X_norm;
          rhoDtotal += Ddiag[fspec];
          cp_fuel += Y_skin[fspec] * cp_n[fspec];
          sumYSkin += Y_skin[fspec];
        }
        cp_fuel /= sumYSkin;
        const double Sc_skin = mu_skin / rhoDtotal;
        const double logB = PMP_LOG1P(B_M);
        const double invFM = B_M / (logB * PMP_POW(1. + B_M, 0.7));
        const double Sh_0 = 1. + powR * PMP_CBRT(1. + Reyn * Sc_skin);
        const double Sh_num = 2. + (Sh_0 - 2.) * invFM;
        const double mdotcoeff = PMP_PI * dia_part * Sh_num * logB;
        const double ratio = cp_fuel * Sh_num * rhoDtotal / lambda_skin;
        Nu_num = calcHeatCoeff(ratio, B_M, B_eps, C_eps, Nu_0);
        for (int spf = 0; spf < NF; ++spf) {
          const int fspec = fdat->indx[spf];
          if (X_vapor[spf] > 0.) {
            mi_dot[spf] = -dmax(Ddiag[fspec] * mdotcoeff, 0.);
            m_dot += mi_dot[spf];
            sumL += mi_dot[spf] * L_fuel[spf];
            mL[spf] = mi_dot[spf];
          }
        }
      } else {
        Nu_num = Nu_0;
      }
      const double conv_src = PMP_PI * lambda_skin * dia_part * delT * Nu_num;
      conv_i = conv_src;
      gpv->fluid_eng_src += num_ppp * conv_src;
      part_temp_src = (sumL + conv_src) * inv_pmass / cp_part;
      if (isub == 1 && delT > C_eps) {
        const double inv_tau_d = -m_dot / (0.2 * pmass);
        const double inv_tau_T = conv_src * inv_pmass / (cp_part * delT);
        nsub = imin(
          imax(nsub, imax((int)(flow_dt * inv_tau_d), (int)(flow_dt * inv_tau_T)) + 1),
          nSubMax);
      }
    }
    if (isub == 1) {
      dt = flow_dt / (double)nsub;
      nsub_first = nsub;
    }
    const double part_dt = fdat->dtmod * dt;
    if (!fdat->fixed_parts) {
      for (int d = 0; d < 3; ++d) {
        vel_part[d] += part_dt * part_vel_src[d];
      }
    }
    /* the sub-step's start state, for the energy identity */
    const double T_i = T_part;
    const double pm_i = pmass;
    double Y_i[PMP_MAX_FUEL];
    for (int spf = 0; spf < NF; ++spf) {
      Y_i[spf] = Y_part[spf];
    }
    if (fdat->mass_trans) {
      const double newT = T_part + part_dt * part_temp_src;
      const double new_mass = pmass + m_dot * part_dt;
      e_conv += part_dt * conv_i;
      if (new_mass > min_mass && newT < Tboil) {
        T_part = newT;
        if (NF > 1) {
          rho_part = 0.;
          double sumY = 0.;
          for (int spf = 0; spf < NF; ++spf) {
            Y_part[spf] = dmin(
              1., dmax(0., (Y_part[spf] * pmass + mi_dot[spf] * part_dt) / new_mass));
            if (Y_part[spf] <= 1.E-12) {
              Y_part[spf] = 0.;
            }
            sumY += Y_part[spf];
          }
          for (int spf = 0; spf < NF; ++spf) {
            Y_part[spf] /= sumY;
            rho_part += Y_part[spf] / rhoL(fdat, dmin(T_part, cBoilT[spf]), spf);
          }
          rho_part = 1. / rho_part;
        } else {
          rho_part = rhoL(fdat, dmin(T_part, cBoilT[0]), 0);
        }
        pmass = new_mass;
        dia_part = PMP_CBRT(6. * pmass / (PMP_PI * rho_part));
        if (eres) {
          for (int spf = 0; spf < NF; ++spf) {
            const double dM = pmass * Y_part[spf] - pm_i * Y_i[spf];
            const double L = h_part[fdat->indx[spf]] + fdat->latent[spf] - fdat->cp[spf] * (T_i - fdat->ref_T);
            e_expl += dM * fdat->cp[spf] * (T_part - T_i);
            e_clip += (part_dt * mL[spf] - dM) * L;
            e_lat += part_dt * mL[spf] * (L_fuel[spf] - L);
            e_vap += dM * h_part[fdat->indx[spf]];
            dM_tot[spf] += dM;
          }
        }
      } else {
        if (eres) {
          for (int spf = 0; spf < NF; ++spf) {
            const double M = pm_i * Y_i[spf];
            const double L = h_part[fdat->indx[spf]] + fdat->latent[spf] - fdat->cp[spf] * (T_i - fdat->ref_T);
            e_vap -= M * h_part[fdat->indx[spf]];
            dM_tot[spf] -= M;
            e_kill += M * L;
          }
          e_kill -= part_dt * conv_i;
          k_kill = isub;
        }
        pmass = 0.;
        *id = -1;
        nsub = isub;
        isub = nsub + 1;
      }
    }
    ++isub;
  }
  if (eres && fdat->mass_trans) {
    /* the gas receives the vapour at the last sub-step's enthalpies */
    for (int spf = 0; spf < NF; ++spf) {
      e_vap -= dM_tot[spf] * h_part[fdat->dep_indx[spf]];
    }
    const double avg = k_kill > 0 ? -((double)nsub_first / (double)k_kill - 1.) * e_conv : 0.;
    *eres += num_ppp * (e_expl + e_clip + e_lat + e_vap + e_kill + avg);
  }
  if (nsub > 1) {
    gpv->fluid_eng_src /= (double)nsub;
    for (int d = 0; d < 3; ++d) {
      gpv->fluid_mom_src[d] /= (double)nsub;
    }
  }
  const double mdot_total = (pmass - startmass) / (fdat->dtmod * flow_dt);
  gpv->fluid_mass_src = num_ppp * mdot_total;
  if (g_pelec) {
    /* kinetic energy of the mass exchanged, PeleC branch (Drag.H:418-421) */
    const double part_ke =
      0.5 * (vel_part[0] * vel_part[0] + vel_part[1] * vel_part[1] + vel_part[2] * vel_part[2]);
    gpv->fluid_eng_src += num_ppp * part_ke * mdot_total;
  }
  if (fdat->mom_trans) {
    for (int d = 0; d < 3; ++d) {
      gpv->fluid_mom_src[d] += num_ppp * vel_part[d] * mdot_total;
    }
  }
  for (int spf = 0; spf < NF; ++spf) {
    const int fdspec = fdat->dep_indx[spf];
    const double oldY = rdata[PMP_PSTATE_Y + spf];
    const double newY = Y_part[spf];
    const double midot = (newY * pmass - oldY * startmass) / (fdat->dtmod * flow_dt);
    gpv->fluid_Y_dot[spf] = num_ppp * midot;
    gpv->fluid_eng_src += num_ppp * midot * h_part[fdspec];
    rdata[PMP_PSTATE_Y + spf] = Y_part[spf];
  }
  rdata[0] = vel_part[0];
  rdata[1] = vel_part[1];
  rdata[2] = vel_part[2];
  rdata[PMP_PSTATE_T] = T_part;
  rdata[PMP_PSTATE_DIA] = dia_part;
  return Reyn;
}

/* check_bounds (SprayInterpolation.H:64-97) */
static int check_bounds(
  const double* pos, const double* plo, const double* phi, const double* dx,
  const int* bndry_lo, const int* bndry_hi, int* bflags)
{
  for (int hilo = 0; hilo < 2; ++hilo) {
    const int fact = (hilo == 0) ? 1 : -1;
    for (int dir = 0; dir < 3; ++dir) {
      const double dom_loc = (hilo == 0) ? plo[dir] : phi[dir];
      const int bflag = (hilo == 0) ? bndry_lo[dir] : bndry_hi[dir];
      if (bflag != 0) {
        const double diff = (double)fact * (pos[dir] - dom_loc);
        if (diff < 0.) {
          if (bflag == 1) {
            bflags[dir] = -fact;
          } else {
            return 1;
          }
        } else if (diff < 0.5 * dx[dir]) {
          bflags[dir] = -2 * fact;
        }
      }
    }
  }
  return 0;
}

/* trilinear_interp (SprayInterpolation.H:158-199) */
static void trilinear_interp(
  const int* ijk, const double* lx, int (*indx)[3], double* w, const int* bflags)
{
  double ssv[2][3];
  for (int dir = 0; dir < 3; ++dir) {
    const double sx_hi = lx[dir] - (double)ijk[dir];
    const double sx_lo = 1. - sx_hi;
    if (bflags[dir] > 1) {
      ssv[0][dir] = 1.;
      ssv[1][dir] = 0.;
    } else if (bflags[dir] < -1) {
      ssv[0][dir] = 0.;
      ssv[1][dir] = 1.;
    } else {
      ssv[0][dir] = sx_lo;
      ssv[1][dir] = sx_hi;
    }
  }
  int cc = 0;
  for (int kk = -1; kk < 1; kk++) {
    for (int jj = -1; jj < 1; jj++) {
      for (int ii = -1; ii < 1; ii++) {
        indx[cc][0] = ijk[0] + ii;
        indx[cc][1] = ijk[1] + jj;
        indx[cc][2] = ijk[2] + kk;
        w[cc] = ssv[ii + 1][0] * ssv[jj + 1][1] * ssv[kk + 1][2];
        cc++;
      }
    }
  }
}

static inline double* vat(const pmp_box_view* v, int i, int j, int k, int n)
{
  return v->p + (long long)(i - v->lo[0]) + (long long)(j - v->lo[1]) * v->jstride +
         (long long)(k - v->lo[2]) * v->kstride + (long long)n * v->nstride;
}

static inline int box_contains(const int* lo, const int* hi, const int* iv)
{
  return iv[0] >= lo[0] && iv[0] <= hi[0] && iv[1] >= lo[1] && iv[1] <= hi[1] &&
         iv[2] >= lo[2] && iv[2] <= hi[2];
}

/* tile_at_bndry (WallFunctions.H:8-35) */
static int tile_at_bndry(const pmp_box* b, const pmp_geometry* g)
{
  int grown_inside = 1;
  for (int d = 0; d < 3; ++d) {
    if (b->lo[d] - 1 < g->domain_lo[d] || b->hi[d] + 1 > g->domain_hi[d]) {
      grown_inside = 0;
    }
  }
  if (grown_inside) {
    return 0;
  }
  int at = 0;
  for (int d = 0; d < 3; ++d) {
    const int lo_out = b->lo[d] - 1 < g->domain_lo[d];
    const int hi_out = b->hi[d] + 1 > g->domain_hi[d];
    /* box grown low in d leaves the domain iff lo-1 < dlo (other directions
     * of the valid box are inside the domain) */
    if ((lo_out && g->bndry_lo[d] != 0) || (hi_out && g->bndry_hi[d] != 0)) {
      at = 1;
    }
  }
  return at;
}

/* impose_wall without splash or EB (WallFunctions.H:89-234) */
static void impose_wall(
  double* pos, double* vel, const double* dx, const double* plo, const int* bflags)
{
  double normpos[3];
  int ijkc[3];
  for (int d = 0; d < 3; ++d) {
    normpos[d] = (pos[d] - plo[d]) / dx[d];
    ijkc[d] = (int)floor(normpos[d]);
  }
  int wall_check = 0;
  double normal[3];
  double bcentv[3];
  for (int dir = 0; dir < 3; ++dir) {
    if ((bflags[dir] == -1 || bflags[dir] == 1) && !wall_check) {
      normal[dir] = -(double)bflags[dir];
      bcentv[dir] = (double)ijkc[dir] + 0.5 * (double)(1 - bflags[dir]);
      wall_check = 1;
    } else {
      normal[dir] = 0.;
      bcentv[dir] = 0.;
    }
  }
  if (!wall_check) {
    return;
  }
  const double par_dot = (normpos[0] - bcentv[0]) * dx[0] * normal[0] +
                         (normpos[1] - bcentv[1]) * dx[1] * normal[1] +
                         (normpos[2] - bcentv[2]) * dx[2] * normal[2];
  if (par_dot < DBL_EPSILON) {
    const double Nw_Vp = normal[0] * vel[0] + normal[1] * vel[1] + normal[2] * vel[2];
    for (int dir = 0; dir < 3; ++dir) {
      vel[dir] -= 2. * Nw_Vp * normal[dir];
      pos[dir] -= 2. * par_dot * normal[dir];
    }
  }
}

typedef struct {
  const pmp_mech* mech;
  const pmp_spray_data* fdat;
  const pmp_spray_comps* comps;
  const pmp_geometry* geom;
  const pmp_box_view* st;
  const pmp_box_view* sr;
  int state_lo[3], state_hi[3];
  int src_lo[3], src_hi[3];
  double dxi[3], inv_vol;
  double flow_dt, sub_dt;
  int num_iter, do_move, is_ghost, at_bounds, atomic;
} ctx_t;

static inline void dep(const ctx_t* c, double* p, double v)
{
  if (c->atomic) {
#pragma omp atomic
    *p += v;
  } else {
    *p += v;
  }
}

/* The per-droplet body of updateParticles (SprayParticles.cpp:324-481).
 * Returns 0 or an error code. */
static int update_droplet(const ctx_t* c, double* pos, double* rdata, int* id, long long* nsubsteps,
                          double* eres)
{
  const pmp_spray_data* fdat = c->fdat;
  const pmp_geometry* g = c->geom;
  const int NF = fdat->nfuel;
  const int NS = c->mech->nspec;
  if (!(*id > 0)) {
    return 0;
  }
  gpv_t gpv;
  double cBoilT[PMP_MAX_FUEL];
  pmp_eos_molecular_weight(c->mech, gpv.mw);
  for (int n = 0; n < NS; ++n) {
    gpv.mw[n] *= U_MASS_CONV;
  }
  int indx_array[8][3];
  double weights[8];
  double lx[3], lxc[3];
  int ijk[3], ijkc[3];
  for (int d = 0; d < 3; ++d) {
    lx[d] = (pos[d] - g->plo[d]) * c->dxi[d] + 0.5;
    ijk[d] = (int)floor(lx[d]);
    lxc[d] = (pos[d] - g->plo[d]) * c->dxi[d];
    ijkc[d] = (int)floor(lxc[d]);
  }
  int bflags[3] = {0, 0, 0};
  if (c->at_bounds) {
    if (check_bounds(pos, g->plo, g->phi, g->dx, g->bndry_lo, g->bndry_hi, bflags)) {
      return PMP_ERR_LEFT_DOMAIN;
    }
  }
  const pmp_spray_comps* sc = c->comps;
  for (int cur_iter = 0; cur_iter < c->num_iter && *id > 0; ++cur_iter) {
    if (rdata[PMP_PSTATE_FILMHGHT(NF)] > 0.) {
      return PMP_ERR_UNSUPPORTED; /* wall film needs the splash model */
    }
    trilinear_interp(ijk, lx, indx_array, weights, bflags);
    gpv_reset(&gpv, NS, NF);
    /* InterpolateGasPhase (SprayInterpolation.H:99-150): PeleLMeX branch
     * (velocity and T read directly) or PeleC branch (velocity = mom / rho,
     * T from the internal energy through eos.EY2T, the cell's T the guess) */
    for (int a = 0; a < 8; ++a) {
      const double cw = weights[a];
      if (cw > 0.) {
        const int* ci = indx_array[a];
        if (!box_contains(c->state_lo, c->state_hi, ci)) {
          return PMP_ERR_STATE_BOX;
        }
        const double cur_rho = *vat(c->st, ci[0], ci[1], ci[2], sc->rhoIndx);
        gpv.rho_fluid += cw * cur_rho;
        double inv_rho = 1. / cur_rho;
        double mass_frac[PMP_MAX_SPEC];
        for (int n = 0; n < NS; ++n) {
          const double cur_mf = *vat(c->st, ci[0], ci[1], ci[2], sc->specIndx + n) * inv_rho;
          gpv.Y_fluid[n] += cw * cur_mf;
          mass_frac[n] = cur_mf;
        }
        if (!g_pelec) {
          inv_rho = 1.;
        }
        double ke = 0.;
        for (int dir = 0; dir < 3; ++dir) {
          const double vel = *vat(c->st, ci[0], ci[1], ci[2], sc->momIndx + dir) * inv_rho;
          gpv.vel_fluid[dir] += cw * vel;
          ke += vel * vel / 2.;
        }
        double T_i = *vat(c->st, ci[0], ci[1], ci[2], sc->utempIndx);
        if (g_pelec) {
          const double intEng = *vat(c->st, ci[0], ci[1], ci[2], sc->engIndx) * inv_rho - ke;
          pmp_eos_EY2T(c->mech, intEng, mass_frac, &T_i);
        }
        gpv.T_fluid += cw * T_i;
      }
    }
    gpv_define(&gpv, NS);
    calcBoilT(fdat, &gpv, cBoilT);
    calculateSpraySource(c->mech, c->sub_dt, &gpv, fdat, rdata, id, cBoilT, eres);
    if (nsubsteps) {
      *nsubsteps += 1;
    }
    const int* cur = ijkc;
    const double cur_coef = -c->inv_vol * c->sub_dt / c->flow_dt;
    if (!box_contains(c->src_lo, c->src_hi, cur)) {
      if (!c->is_ghost) {
        return PMP_ERR_SOURCE_BOX;
      }
      if (!(cur[0] >= c->sr->lo[0] && cur[0] <= c->sr->hi[0] && cur[1] >= c->sr->lo[1] &&
            cur[1] <= c->sr->hi[1] && cur[2] >= c->sr->lo[2] && cur[2] <= c->sr->hi[2])) {
        return PMP_ERR_SOURCE_BOX;
      }
    }
    if (fdat->mom_trans) {
      for (int dir = 0; dir < 3; ++dir) {
        dep(c, vat(c->sr, cur[0], cur[1], cur[2], sc->momSrcIndx + dir),
            cur_coef * gpv.fluid_mom_src[dir]);
      }
    }
    if (fdat->mass_trans) {
      dep(c, vat(c->sr, cur[0], cur[1], cur[2], sc->rhoSrcIndx), cur_coef * gpv.fluid_mass_src);
      for (int spf = 0; spf < NF; ++spf) {
        dep(c, vat(c->sr, cur[0], cur[1], cur[2], sc->specSrcIndx + spf),
            cur_coef * gpv.fluid_Y_dot[spf]);
      }
    }
    dep(c, vat(c->sr, cur[0], cur[1], cur[2], sc->engSrcIndx), cur_coef * gpv.fluid_eng_src);
    if (c->do_move && !fdat->fixed_parts && *id > 0) {
      for (int dir = 0; dir < 3; ++dir) {
        const double cvel = rdata[PMP_PSTATE_VEL + dir];
        pos[dir] += c->sub_dt * cvel;
      }
      if (c->at_bounds) {
        if (check_bounds(pos, g->plo, g->phi, g->dx, g->bndry_lo, g->bndry_hi, bflags)) {
          *id = -1;
        } else {
          impose_wall(pos, rdata + PMP_PSTATE_VEL, g->dx, g->plo, bflags);
        }
      }
      for (int d = 0; d < 3; ++d) {
        lx[d] = (pos[d] - g->plo[d]) * c->dxi[d] + 0.5;
        ijk[d] = (int)floor(lx[d]);
        lxc[d] = (pos[d] - g->plo[d]) * c->dxi[d];
        ijkc[d] = (int)floor(lxc[d]);
      }
    }
    if (c->is_ghost && !box_contains(c->src_lo, c->src_hi, ijkc)) {
      *id = -1;
    }
  }
  return 0;
}

static double** eres_box = NULL;

void pmp_oracle_set_energy_out(double** per_box) { eres_box = per_box; }

int pmp_oracle_update(
  const pmp_mech* mech, const pmp_spray_data* fdat,
  const pmp_spray_comps* comps, const pmp_geometry* geom, int nboxes,
  const pmp_box* boxes, pmp_particles* parts, const pmp_box_view* state,
  const pmp_box_view* source, double flow_dt, int state_ghosts,
  int source_ghosts, int is_virt, int is_ghost, int do_move,
  double spray_cfl_lev, int nthreads, pmp_error_info* err,
  long long* substeps)
{
  (void)is_virt;
  if (err) {
    memset(err, 0, sizeof(*err));
    err->particle = -1;
  }
  if (substeps) {
    *substeps = 0;
  }
  if (fdat->do_breakup != 0 || fdat->do_splash) {
    if (err) {
      err->code = PMP_ERR_UNSUPPORTED;
    }
    return PMP_ERR_UNSUPPORTED;
  }
  const int NF = fdat->nfuel;
  ctx_t c;
  memset(&c, 0, sizeof(c));
  c.mech = mech;
  c.fdat = fdat;
  c.comps = comps;
  c.geom = geom;
  for (int d = 0; d < 3; ++d) {
    c.dxi[d] = 1. / geom->dx[d];
  }
  const double vol = geom->dx[0] * geom->dx[1] * geom->dx[2];
  c.inv_vol = 1. / vol;
  c.flow_dt = flow_dt;
  const double sub_cfl = 0.5;
  c.sub_dt = flow_dt;
  c.num_iter = 1;
  if (do_move && spray_cfl_lev > sub_cfl) {
    c.num_iter = (int)ceil(spray_cfl_lev / sub_cfl);
    c.sub_dt = flow_dt / (double)c.num_iter;
  }
  c.do_move = do_move;
  c.is_ghost = is_ghost;
  c.atomic = nthreads > 1;
  int status = PMP_OK;
  long long total = 0;
  for (int b = 0; b < nboxes && status == PMP_OK; ++b) {
    c.st = &state[b];
    c.sr = &source[b];
    for (int d = 0; d < 3; ++d) {
      c.state_lo[d] = boxes[b].lo[d] - state_ghosts;
      c.state_hi[d] = boxes[b].hi[d] + state_ghosts;
      c.src_lo[d] = boxes[b].lo[d] - source_ghosts;
      c.src_hi[d] = boxes[b].hi[d] + source_ghosts;
    }
    c.at_bounds = tile_at_bndry(&boxes[b], geom);
    pmp_particles* P = &parts[b];
    const long long Np = P->n;
    long long first_bad = -1;
    int bad_code = 0;
    long long nsubs = 0;
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 256) num_threads(nthreads > 1 ? nthreads : 1) reduction(+ : nsubs)
#endif
    for (long long i = 0; i < Np; ++i) {
      double pos[3];
      double rd[PMP_MAX_RCOMP];
      const int nr = PMP_PSTATE_NUM(NF);
      for (int d = 0; d < 3; ++d) {
        pos[d] = P->pos[d][i];
      }
      for (int r = 0; r < nr; ++r) {
        rd[r] = P->rdata[r][i];
      }
      int id = P->id[i];
      long long ns = 0;
      const int rc = update_droplet(&c, pos, rd, &id, &ns, eres_box ? eres_box[b] + i : NULL);
      nsubs += ns;
      if (rc != 0) {
#ifdef _OPENMP
#pragma omp critical
#endif
        {
          if (first_bad < 0 || i < first_bad) {
            first_bad = i;
            bad_code = rc;
          }
        }
      }
      for (int d = 0; d < 3; ++d) {
        P->pos[d][i] = pos[d];
      }
      for (int r = 0; r < nr; ++r) {
        P->rdata[r][i] = rd[r];
      }
      P->id[i] = id;
    }
    total += nsubs;
    if (first_bad >= 0) {
      status = bad_code;
      if (err) {
        err->code = bad_code;
        err->box = b;
        err->particle = first_bad;
        for (int d = 0; d < 3; ++d) {
          err->pos[d] = P->pos[d][first_bad];
        }
        snprintf(err->message, sizeof(err->message), "oracle: error %d at box %d droplet %lld",
                 bad_code, b, first_bad);
      }
    }
  }
  if (substeps) {
    *substeps = total;
  }
  return status;
}

double pmp_oracle_droplet_source(
  const pmp_mech* mech, const pmp_spray_data* fdat, double flow_dt,
  const double* gas, double* rdata, int* id, double* src)
{
  const int NS = mech->nspec;
  const int NF = fdat->nfuel;
  gpv_t gpv;
  double cBoilT[PMP_MAX_FUEL];
  pmp_eos_molecular_weight(mech, gpv.mw);
  for (int n = 0; n < NS; ++n) {
    gpv.mw[n] *= U_MASS_CONV;
  }
  gpv_reset(&gpv, NS, NF);
  gpv.rho_fluid = gas[0];
  gpv.T_fluid = gas[1];
  for (int d = 0; d < 3; ++d) {
    gpv.vel_fluid[d] = gas[2 + d];
  }
  for (int n = 0; n < NS; ++n) {
    gpv.Y_fluid[n] = gas[5 + n];
  }
  gpv_define(&gpv, NS);
  calcBoilT(fdat, &gpv, cBoilT);
  const double re = calculateSpraySource(mech, flow_dt, &gpv, fdat, rdata, id, cBoilT, NULL);
  for (int d = 0; d < 3; ++d) {
    src[d] = gpv.fluid_mom_src[d];
  }
  src[3] = gpv.fluid_mass_src;
  src[4] = gpv.fluid_eng_src;
  for (int f = 0; f < NF; ++f) {
    src[5 + f] = gpv.fluid_Y_dot[f];
  }
  return re;
}

int pmp_oracle_mech(pmp_mech* mech, int nspec, const char (*names)[PMP_NAME_LEN])
{
  int idx[PMP_MAX_SPEC];
  if (nspec < 1 || nspec > PMP_MAX_SPEC) {
    return -1;
  }
  for (int k = 0; k < nspec; ++k) {
    idx[k] = pmp_db_lookup(names[k]);
    if (idx[k] < 0) {
      return -1;
    }
  }
  return pmp_mech_build(mech, nspec, idx);
}

/* readSprayParams + spraySetup (SpraySetup.cpp:73-297) */
int pmp_oracle_setup(
  const pmp_mech* mech, const char (*names)[PMP_NAME_LEN],
  const pmp_spray_inputs* in, pmp_spray_data* out)
{
  memset(out, 0, sizeof(*out));
  const int NF = in->nfuel;
  if (NF < 1 || NF > PMP_MAX_FUEL) {
    return PMP_ERR_INVALID;
  }
  out->nfuel = NF;
  out->mass_trans = in->mass_transfer;
  out->mom_trans = in->mom_transfer;
  out->fixed_parts = in->fixed_parts;
  out->min_eb_vfrac = 0.05;
  out->sigma = -1.;
  out->wall_T = -1.;
  out->theta_c = -1.;
  out->dtmod = 0.5;
  if (in->cfl > 2.) {
    return PMP_ERR_INVALID;
  }
  if (in->use_breakup_model != 0 || in->use_splash_model) {
    return PMP_ERR_UNSUPPORTED;
  }
  for (int f = 0; f < NF; ++f) {
    out->critT[f] = in->crit_temp[f];
    out->boilT[f] = in->boil_temp[f];
    out->cp[f] = in->cp[f];
    out->ref_latent[f] = in->latent[f];
    const int* nc[4] = {in->ncoef_lambda, in->ncoef_psat, in->ncoef_rho, in->ncoef_mu};
    const double(*src[4])[4] = {in->lambda, in->psat, in->rho, in->mu};
    double* dst[4] = {out->lambda_coef, out->psat_coef, out->rho_coef, out->mu_coef};
    for (int q = 0; q < 4; ++q) {
      if (nc[q][f] == 4) {
        for (int i = 0; i < 4; ++i) {
          dst[q][4 * f + i] = src[q][f][i];
        }
      } else if (nc[q][f] == 1) {
        for (int i = 0; i < 4; ++i) {
          dst[q][4 * f + i] = 0.;
        }
        dst[q][4 * f] = src[q][f][0];
      } else if (q == 2) {
        return PMP_ERR_INVALID; /* rho is required */
      }
    }
    out->latent[f] = out->ref_latent[f];
  }
  out->ref_T = in->fuel_ref_temp;
  for (int f = 0; f < NF; ++f) {
    out->indx[f] = -1;
    out->dep_indx[f] = -1;
    const char* dep = in->dep_fuel_species[f][0] ? in->dep_fuel_species[f] : in->fuel_species[f];
    for (int ns = 0; ns < mech->nspec; ++ns) {
      if (strcmp(names[ns], in->fuel_species[f]) == 0) {
        out->indx[f] = ns;
      }
      if (strcmp(names[ns], dep) == 0) {
        out->dep_indx[f] = ns;
      }
    }
    if (out->indx[f] < 0 || out->dep_indx[f] < 0) {
      return PMP_ERR_INVALID;
    }
  }
  double fuelEnth[PMP_MAX_SPEC];
  pmp_eos_T2Hi(mech, out->ref_T, fuelEnth);
  for (int ns = 0; ns < NF; ++ns) {
    const int fspec = out->indx[ns];
    out->latent[ns] -= fuelEnth[fspec] * U_ENG_CONV;
  }
  for (int d = 0; d < 3; ++d) {
    out->body_force[d] = in->body_force[d];
  }
  return PMP_OK;
}

/* ---- test hooks: elementary functions, thermo, transport, ABI sizes ---- */

/* fn: 0 exp, 1 log, 2 log1p, 3 pow, 4 cbrt (project library, or the C
 * library in the libm build) */
void pmp_oracle_math(int fn, const double* x, const double* y, double* out, long long n)
{
  for (long long i = 0; i < n; ++i) {
    switch (fn) {
      case 0: out[i] = PMP_EXP(x[i]); break;
      case 1: out[i] = PMP_LOG(x[i]); break;
      case 2: out[i] = PMP_LOG1P(x[i]); break;
      case 3: out[i] = PMP_POW(x[i], y[i]); break;
      default: out[i] = PMP_CBRT(x[i]); break;
    }
  }
}

void pmp_oracle_thermo(const pmp_mech* m, double T, double* cp, double* h)
{
  pmp_eos_T2Cpi(m, T, cp);
  pmp_eos_T2Hi(m, T, h);
}

void pmp_oracle_transport(
  const pmp_mech* m, double T, const double* Y, double* Ddiag, double* mu, double* lam)
{
  pmp_transport(m, 1, 1, 1, T, 0.0, Y, Ddiag, mu, lam);
}

/* sizeof of the C ABI structs, in the order the tests list them */
void pmp_oracle_abi_sizes(long long* out)
{
  out[0] = (long long)sizeof(pmp_geometry);
  out[1] = (long long)sizeof(pmp_box);
  out[2] = (long long)sizeof(pmp_box_view);
  out[3] = (long long)sizeof(pmp_spray_comps);
  out[4] = (long long)sizeof(pmp_spray_data);
  out[5] = (long long)sizeof(pmp_spray_inputs);
  out[6] = (long long)sizeof(pmp_particles);
  out[7] = (long long)sizeof(pmp_spray_config);
  out[8] = (long long)sizeof(pmp_error_info);
  out[9] = (long long)sizeof(pmp_stats);
  out[10] = (long long)sizeof(pmp_mech);
  out[11] = (long long)sizeof(pmp_launch_config);
  out[12] = (long long)sizeof(pmp_tune_report);
  out[13] = (long long)sizeof(pmp_learn_config);
  out[14] = (long long)sizeof(pmp_learn_report);
}
