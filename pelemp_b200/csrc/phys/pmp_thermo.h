/* pmp_thermo.h -- the project's gas equation of state and transport model.
 *
 * Stands in for the PelePhysics calls the spray update makes (PeleMP call
 * sites: eos.molecular_weight at Source/PP_Spray/SprayParticles.cpp:332,
 * eos.T2Cpi / eos.T2Hi at Source/PP_Spray/Drag.H:220-221 and
 * Source/PP_Spray/SpraySetup.cpp:286, trans.transport at
 * Source/PP_Spray/Drag.H:252-256).  Same units as that interface: CGS
 * (g/mol, erg/g/K, erg/g, g/cm/s, erg/cm/s/K, g/cm/s for rho*D).
 *
 * Data: pmp_thermo_data.h (written by gen_thermo.py).  A "mechanism" is an
 * ordered subset of the species database; the spray code indexes species by
 * their position in the mechanism.
 *
 * Mixture rules of transport():
 *   mu     = (sum_k X_k mu_k^6)^(1/6)
 *   lambda = (sum_k X_k lambda_k^(1/4))^4
 *   Ddiag_i = W_i/(R T) * (sum_{j!=i} Y_j) / (sum_{j!=i} X_j / (P D_ij)),
 *            i.e. (W_i/Wbar) rho D_i,mix with the Hirschfelder-Curtiss
 *            mixture-averaged diffusivity D_i,mix.
 * Valid C99 and CUDA C++; the math goes through the PMP_* macros of
 * pmp_math.h.
 */
#ifndef PMP_THERMO_H
#define PMP_THERMO_H

#include "pmp_math.h"
#include "pmp_thermo_data.h"

#define PMP_MAX_SPEC 8
#define PMP_RU_CGS 8.31446261815324e7 /* erg/(mol K) */
#define PMP_PATM_CGS 1013250.0        /* dyn/cm^2 */

typedef struct pmp_mech {
  int nspec;
  int db_index[PMP_MAX_SPEC];
  double mw[PMP_MAX_SPEC];       /* g/mol */
  double cp[PMP_MAX_SPEC][5];    /* cp/R = sum cp[n] T^n */
  double hc[PMP_MAX_SPEC][6];    /* h/(R T) = sum hc[n] T^n (n<5) + hc[5]/T */
  double mu[PMP_MAX_SPEC][4];    /* ln mu(lnT) */
  double lam[PMP_MAX_SPEC][4];   /* ln lambda(lnT) */
  double dbin[PMP_MAX_SPEC][PMP_MAX_SPEC][4]; /* ln(P D_jk)(lnT) */
} pmp_mech;

/* Build a mechanism from database indices (host).  Returns 0 on success. */
static inline int pmp_mech_build(pmp_mech* m, int nspec, const int* db_index)
{
  if (nspec < 1 || nspec > PMP_MAX_SPEC) {
    return -1;
  }
  memset(m, 0, sizeof(*m));
  m->nspec = nspec;
  for (int k = 0; k < nspec; ++k) {
    const int d = db_index[k];
    if (d < 0 || d >= PMP_DB_NSPEC) {
      return -1;
    }
    m->db_index[k] = d;
    m->mw[k] = pmp_db_mw[d];
    for (int n = 0; n < 5; ++n) {
      m->cp[k][n] = pmp_db_cp[d][n];
      m->hc[k][n] = pmp_db_cp[d][n] / (double)(n + 1);
    }
    m->hc[k][5] = pmp_db_cp[d][5];
    for (int n = 0; n < 4; ++n) {
      m->mu[k][n] = pmp_db_mu[d][n];
      m->lam[k][n] = pmp_db_lam[d][n];
    }
  }
  for (int j = 0; j < nspec; ++j) {
    for (int k = 0; k < nspec; ++k) {
      for (int n = 0; n < 4; ++n) {
        m->dbin[j][k][n] = pmp_db_dbin[m->db_index[j]][m->db_index[k]][n];
      }
    }
  }
  return 0;
}

/* Database index of a species name, -1 if unknown (host). */
static inline int pmp_db_lookup(const char* name)
{
  for (int d = 0; d < PMP_DB_NSPEC; ++d) {
    if (strcmp(name, pmp_db_names[d]) == 0) {
      return d;
    }
  }
  return -1;
}

PMP_HD void pmp_eos_molecular_weight(const pmp_mech* m, double* mw)
{
  for (int k = 0; k < m->nspec; ++k) {
    mw[k] = m->mw[k];
  }
}

/* per-species cp [erg/(g K)] */
PMP_HD void pmp_eos_T2Cpi(const pmp_mech* m, double T, double* cpi)
{
  for (int k = 0; k < m->nspec; ++k) {
    const double* a = m->cp[k];
    const double cpr = fma(fma(fma(fma(a[4], T, a[3]), T, a[2]), T, a[1]), T, a[0]);
    cpi[k] = cpr * (PMP_RU_CGS / m->mw[k]);
  }
}

/* per-species enthalpy [erg/g] */
PMP_HD void pmp_eos_T2Hi(const pmp_mech* m, double T, double* hi)
{
  for (int k = 0; k < m->nspec; ++k) {
    const double* a = m->hc[k];
    const double p = fma(fma(fma(fma(a[4], T, a[3]), T, a[2]), T, a[1]), T, a[0]);
    hi[k] = fma(p, T, a[5]) * (PMP_RU_CGS / m->mw[k]);
  }
}

/* eos.EY2T: the temperature at which the mixture's specific internal energy
 * sum_k Y_k (h_k(T) - R T / W_k) [erg/g] equals e, by Newton iteration from
 * the guess in *T (at most 20 steps; stops once |dT| <= 1e-11 T).  PelePhysics'
 * own EY2T is not part of PeleMP; this is the project's EOS inversion, used by
 * the PeleC coupling's gas-state gather (SprayInterpolation.H:111-146). */
PMP_HD void pmp_eos_EY2T(const pmp_mech* m, double e, const double* Y, double* T)
{
  double t = *T;
  for (int it = 0; it < PMP_EY2T_MAXIT; ++it) {
    double em = 0., cv = 0.;
    for (int k = 0; k < m->nspec; ++k) {
      const double rw = PMP_RU_CGS / m->mw[k];
      const double* a = m->hc[k];
      const double hp = fma(fma(fma(fma(a[4], t, a[3]), t, a[2]), t, a[1]), t, a[0]);
      const double hk = fma(hp, t, a[5]) * rw;
      const double* c = m->cp[k];
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
  *T = t;
}

PMP_HD double pmp_cubic(const double* c, double x)
{
  return fma(fma(fma(c[3], x, c[2]), x, c[1]), x, c[0]);
}

/* Mixture transport.  rho is accepted for interface parity and unused. */
PMP_HD void pmp_transport(
  const pmp_mech* m, int get_mu, int get_lam, int get_Ddiag, double T,
  double rho, const double* Y, double* Ddiag, double* mu, double* lam)
{
  (void)rho;
  const int ns = m->nspec;
  double X[PMP_MAX_SPEC];
  double sumYW = 0.0;
  for (int k = 0; k < ns; ++k) {
    sumYW += Y[k] / m->mw[k];
  }
  const double wbar = 1.0 / sumYW;
  for (int k = 0; k < ns; ++k) {
    X[k] = Y[k] * wbar / m->mw[k];
  }
  const double lnT = PMP_LOG(T);
  if (get_mu) {
    double s = 0.0;
    for (int k = 0; k < ns; ++k) {
      s = fma(X[k], PMP_EXP(6.0 * pmp_cubic(m->mu[k], lnT)), s);
    }
    *mu = PMP_EXP(PMP_LOG(s) * (1.0 / 6.0));
  }
  if (get_lam) {
    double s = 0.0;
    for (int k = 0; k < ns; ++k) {
      s = fma(X[k], PMP_EXP(0.25 * pmp_cubic(m->lam[k], lnT)), s);
    }
    const double s2 = s * s;
    *lam = s2 * s2;
  }
  if (get_Ddiag) {
    const double rt = PMP_RU_CGS * T;
    for (int i = 0; i < ns; ++i) {
      double term1 = 0.0;
      double term2 = 0.0;
      for (int j = 0; j < ns; ++j) {
        if (j != i) {
          term1 += Y[j];
          term2 = fma(X[j], PMP_EXP(-pmp_cubic(m->dbin[i][j], lnT)), term2);
        }
      }
      Ddiag[i] = m->mw[i] * term1 / (term2 * rt);
    }
  }
}

#endif /* PMP_THERMO_H */
