// learn_common.cuh -- the learned form's surrogate: its inputs, its targets,
// the FP64 teacher that produces the targets, and the closed-form vapor state
// the learned kernel evaluates beside the network.
//
// What the surrogate replaces: the skin-state transport and the heat/mass
// transfer correlations of one inner sub-step of calculateSpraySource
// (Source/PP_Spray/Drag.H:212-360): the mixture viscosity, conductivity and
// fuel diffusivities at the skin state, the Sherwood number with the
// film-thickness correction, and the B_T fixed point of calcHeatCoeff with
// the Nusselt number.  Kept exact (FP32 closed form): calcVaporState's
// saturation pressures, Raoult mole fractions, surface vapor mass fractions
// and Spalding number B_M -- the steep, exponential part -- and then, as in
// the mixed form, the drag law, the sub-step count, the explicit FP64 update
// of velocity, temperature, mass and composition, the deposits and the move.
//
// Inputs (10, FP32, normalised by the training set's mean / std):
//   0 ln d            1 T_d               2 T_gas             3 ln(p / 1 atm)
//   4 Y_gas of fuel 0's deposit species    5 same for fuel 1 (0 with one fuel)
//   6 ln(rho_gas |u_gas - u_d| d + 1e-12)  (slip Reynolds number times mu_gas)
//   7 Y_liq of fuel 0 (that of fuel 1 is 1 - Y_liq0 with two fuels)
//   8, 9 surface vapor mass fraction Y_fv of fuel 0 / fuel 1 (0 with one fuel)
// Targets (5), logarithms so that the network's absolute error is a relative
// error of the physical factor:
//   0, 1  ln(rhoD_f * Sh*)  per fuel: with the closed-form vapor state the
//         fuel mass flux is mdot_f = -pi d rhoD_f Sh* (X_v,f / sum X_v) ln(1 + B_M)
//   2     ln(lambda_skin * Nu*): the convective heat flux is pi d (T_gas - T_d) times this
//   3     ln mu_skin    4 ln rho_skin: film viscosity and density of the drag law
// The film temperature is the explicit one-third rule T_d + (T_gas - T_d)/3.
#pragma once

#include "../spray_fp64.cuh"
#include "../spray_mixed.cuh"

namespace pmp {

constexpr int kLearnIn = 10;
constexpr int kLearnOut = 5;
constexpr int kLearnHidden = 64;

// Baseline of the targets.  The network predicts each target's residual
// about a polynomial in the inputs, fitted by least squares over the
// training tuples.  The network's error is set by its bf16 weights and
// activations and is a near-constant fraction (a few 1e-3) of the spread of
// what it predicts; the polynomial leaves the network a residual with 0.1-3 %
// of each target's spread, so the same network error is that much smaller in
// the target.  Terms: the inputs that vary in a spray (ln d, T_d, T_gas,
// ln(Re mu), Y_liq, Y_fv x2) linear and quadratic, the gas pressure and fuel
// vapour in the gas linear, ell = ln(1 + B_M) and its square (the transfer
// rates' steep dependence near boiling, where Y_fv -> 1), and the
// Frossling-shaped g = (1 + c Re)^(1/3) with its square and its products
// with the quadratic inputs (the Sherwood and Nusselt numbers' dependence on
// the Reynolds number).
constexpr int kBaseQ = 7;                                   // quadratic inputs
constexpr int kBaseL = 3;                                   // linear-only inputs
constexpr int kBaseEll = 1 + kBaseQ + kBaseL;               // first ell term
constexpr int kBaseG = kBaseEll + 2;                        // first g term
constexpr int kBaseQuad = kBaseG + 2 + kBaseQ;              // first product z_i z_j
constexpr int kBaseTerms = kBaseQuad + kBaseQ * (kBaseQ + 1) / 2;  // 50
__host__ __device__ constexpr int base_q_input(int i)
{
  return i < 3 ? i : i + 3;  // 0 1 2 6 7 8 9
}
__host__ __device__ constexpr int base_l_input(int i) { return 3 + i; }  // 3 4 5

// Normalisation and gate, FP32, in the kernel parameters of the learned form
struct LearnNorm {
  float x_mean[kLearnIn];
  float x_inv_std[kLearnIn];
  float x_lo[kLearnIn];   // gate: accepted input range (training range widened by the margin)
  float x_hi[kLearnIn];
  float y_mean[kLearnOut];  // of the residual about the baseline
  float y_std[kLearnOut];
  // baseline coefficients per target: [0] constant, [1..7] linear in the
  // quadratic inputs z, [8..10] linear in the linear-only inputs, [11] ell,
  // [12] ell^2, [13] g, [14] g^2, [15..21] g z_i, then the products z_i z_j
  // (i <= j) row by row
  float base[kLearnOut][kBaseTerms];
  // residual gate: the accepted range of each normalised network output
  // (the training residuals' range widened by the gate margin)
  float r_lo[kLearnOut];
  float r_hi[kLearnOut];
};

// The baseline's two derived variables of a droplet.
struct BaseVars {
  float ell;  // ln(1 + B_M)
  float g;    // (1 + c Re)^(1/3) - 2
};

#ifdef __CUDACC__
// From the raw surrogate inputs, the same function in training and
// inference.  (1 + B_M) = (1 - sum Y_gas,fuel) / (1 - sum Y_fv), B_M capped at
// 20 as in calcVaporState (Drag.H:134).  c Re = exp(x6 - mean(x6) + 2),
// input 6 being ln(Re mu_gas): the cube root's knee sits at e^-2 of the
// training set's typical Re mu (chosen on labelled config-2 tuples, where
// moving the knee 8x changed the fitted residual by under 15 %).
__device__ __forceinline__ BaseVars base_vars(const float* x, const LearnNorm& nrm)
{
  const float num = fmaxf(1.f - x[4] - x[5], 1e-30f);
  const float den = fmaxf(1.f - x[8] - x[9], 1e-6f);
  BaseVars v;
  v.ell = fminf(flog(num / den), 3.04452244f);  // ln 21
  v.g = fcbrt(1.f + fexp(fminf(x[6] - nrm.x_mean[6] + 2.f, 60.f))) - 2.f;  // centred near its mean
  return v;
}
#endif

// Features of the baseline (the polynomial's terms) of normalised inputs xn.
template <typename R>
__host__ __device__ __forceinline__ void base_features(const float* xn, BaseVars v, R* f)
{
  f[0] = R(1);
  for (int i = 0; i < kBaseQ; ++i) {
    f[1 + i] = R(xn[base_q_input(i)]);
  }
  for (int i = 0; i < kBaseL; ++i) {
    f[1 + kBaseQ + i] = R(xn[base_l_input(i)]);
  }
  f[kBaseEll] = R(v.ell);
  f[kBaseEll + 1] = R(v.ell) * R(v.ell);
  f[kBaseG] = R(v.g);
  f[kBaseG + 1] = R(v.g) * R(v.g);
  for (int i = 0; i < kBaseQ; ++i) {
    f[kBaseG + 2 + i] = R(v.g) * R(xn[base_q_input(i)]);
  }
  int t = kBaseQuad;
  for (int i = 0; i < kBaseQ; ++i) {
    for (int j = i; j < kBaseQ; ++j) {
      f[t++] = R(xn[base_q_input(i)]) * R(xn[base_q_input(j)]);
    }
  }
}

// Baseline of target o, FP32, in nested form: the g terms as
// g (c_g + c_gg g + sum_i c_gi z_i), the quadratic part as
// sum_i z_i (b_i + sum_{j >= i} c_ij z_j).
__host__ __device__ __forceinline__ float learn_base(const LearnNorm& nrm, int o, const float* xn, BaseVars v)
{
  const float* c = nrm.base[o];
  float acc = fmaf(fmaf(c[kBaseEll + 1], v.ell, c[kBaseEll]), v.ell, c[0]);
#pragma unroll
  for (int i = 0; i < kBaseL; ++i) {
    acc = fmaf(c[1 + kBaseQ + i], xn[base_l_input(i)], acc);
  }
  float sg = fmaf(c[kBaseG + 1], v.g, c[kBaseG]);
#pragma unroll
  for (int i = 0; i < kBaseQ; ++i) {
    sg = fmaf(c[kBaseG + 2 + i], xn[base_q_input(i)], sg);
  }
  acc = fmaf(sg, v.g, acc);
  int t = kBaseQuad;
#pragma unroll
  for (int i = 0; i < kBaseQ; ++i) {
    float s = c[1 + i];
#pragma unroll
    for (int j = i; j < kBaseQ; ++j) {
      s = fmaf(c[t++], xn[base_q_input(j)], s);
    }
    acc = fmaf(s, xn[base_q_input(i)], acc);
  }
  return acc;
}

// Raw (un-normalised) surrogate inputs of a droplet.
template <int NF>
__device__ __forceinline__ void learn_inputs(
  float* x, double dia, double T_d, double T_g, double p, double Yg0, double Yg1, double rho_g,
  double slip, const double* Y_l, const double* Yfv)
{
  x[0] = (float)log(dia);
  x[1] = (float)T_d;
  x[2] = (float)T_g;
  x[3] = (float)log(p / (kPatmCgs * kPresConv));
  x[4] = (float)Yg0;
  x[5] = (float)Yg1;
  x[6] = (float)log(rho_g * slip * dia + 1e-12);
  x[7] = (float)Y_l[0];
  x[8] = (float)Yfv[0];
  x[9] = NF > 1 ? (float)Yfv[NF > 1 ? 1 : 0] : 0.f;
}

// The teacher: targets of an inner sub-step of calculateSpraySource for a
// droplet (T_part, dia_part, Y_part, vel_part) in the gas gpv, FP64, mass
// transfer on; mirrors spray_source_fp64 up to the rates.  Also returns the
// surface vapor mass fractions (inputs 8, 9).  Returns false when no fuel
// evaporates (sum X_v = 0): the learned kernel sends such droplets to the
// FP64 kernel and no tuple is made.
template <int NS, int NF>
__device__ __forceinline__ bool learn_teacher(
  const KParams& P, const GasVals<NS, NF>& gpv, const double* cBoilT, double T_part,
  double dia_part, const double* Y_part, const double* vel_part, float* y, double* Yfv_out)
{
  const DevMech& m = P.m;
  const DevFuel& fdat = P.f;
  const double rule = 1. / 3.;
  const double C_eps = 1.E-15;
  const double B_eps = 1.E-7;
  const double RU = kRuCgs * kRuConv;
  const double PATM = kPatmCgs * kPresConv;
  double Y_skin[NS];
  double Ddiag[NF], X_vapor[NF];
#pragma unroll
  for (int f = 0; f < NF; ++f) {
    Ddiag[f] = 0.;
    X_vapor[f] = 0.;
    Yfv_out[f] = 0.;
  }
  double mw_part = 0.;
#pragma unroll
  for (int spf = 0; spf < NF; ++spf) {
    mw_part += Y_part[spf] / m.mw_kg[fdat.indx[spf]];
  }
  mw_part = 1. / mw_part;
  const double delT = dmax(gpv.T - T_part, 0.);
  const double T_skin = T_part + rule * delT;
#pragma unroll
  for (int n = 0; n < NS; ++n) {
    Y_skin[n] = 0.;
  }
  double cp_skin = 0., mw_skin = 0., B_M = 0., sumXVap = 0.;
  {
    double mbar_vap = 0.;
#pragma unroll
    for (int spf = 0; spf < NF; ++spf) {
      const int fspec = fdat.indx[spf];
      const double mw_fuel = m.mw_kg[fspec];
      const double Tp = dmin(T_part, 0.99 * cBoilT[spf]);
      const double part_latent = h_mks(m, fspec, T_part) + fdat.latent[spf] - fdat.cp[spf] * (Tp - fdat.ref_T);
      double pres_sat;
      if (fdat.psat_coef[4 * spf + 3] == 0.) {
        pres_sat = PATM * pmp_exp(part_latent * mw_fuel / RU * (1. / fdat.boilT[spf] - 1. / Tp));
      } else {
        const double a = fdat.psat_coef[4 * spf], b = fdat.psat_coef[4 * spf + 1];
        const double c = fdat.psat_coef[4 * spf + 2], d = fdat.psat_coef[4 * spf + 3];
        pres_sat = d * pmp_exp((a - b / (Tp + c)) * fdat.ln10);
      }
      const double X_fluid = sel(gpv.Y, fdat.dep[spf]) * gpv.mw_mix / mw_fuel;
      if (pres_sat > X_fluid * gpv.p) {
        const double Xv = Y_part[spf] * mw_part / mw_fuel * pres_sat / gpv.p;
        mbar_vap += Xv * mw_fuel;
        sumXVap += Xv;
        X_vapor[spf] = Xv;
      }
    }
    if (!(sumXVap > 0.)) {
      return false;
    }
    const double totalmwx = mbar_vap + (1. - sumXVap) * gpv.mw_mix;
    double sumYSkin = 0., sumYfFluid = 0., sumYVap = 0.;
#pragma unroll
    for (int spf = 0; spf < NF; ++spf) {
      if (X_vapor[spf] > 0.) {
        const int fspec = fdat.indx[spf];
        const double Yfv = X_vapor[spf] * m.mw_kg[fspec] / totalmwx;
        Yfv_out[spf] = Yfv;
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
      cp_skin += Y_skin[n] * cp_mks(m, n, T_skin);
      mw_skin += Y_skin[n] / m.mw_kg[n];
    }
    mw_skin = 1. / mw_skin;
    B_M = dmin(20., (sumYVap - sumYfFluid) / dmax(C_eps, (1. - sumYVap)));
  }
  const double rho_skin = mw_skin * gpv.p / (RU * T_skin);
  double mu_skin, lambda_skin;
  {
    double X[NS];
    double sumYW = 0.;
#pragma unroll
    for (int k = 0; k < NS; ++k) {
      sumYW += Y_skin[k] / m.mw_g[k];
    }
    const double wbar = 1. / sumYW;
#pragma unroll
    for (int k = 0; k < NS; ++k) {
      X[k] = Y_skin[k] * wbar / m.mw_g[k];
    }
    const double lnT = pmp_log(T_skin);
    double s = 0., sl = 0.;
#pragma unroll
    for (int k = 0; k < NS; ++k) {
      s = fma(X[k], pmp_exp(6.0 * cubic(m.mu[k], lnT)), s);
      sl = fma(X[k], pmp_exp(0.25 * cubic(m.lam[k], lnT)), sl);
    }
    mu_skin = pmp_exp(pmp_log(s) * (1.0 / 6.0)) * kMuConv;
    lambda_skin = sl * sl * sl * sl * kLambdaConv;
    const double rt = kRuCgs * T_skin;
#pragma unroll
    for (int f = 0; f < NF; ++f) {
      const int i = fdat.indx[f];
      double term1 = 0., term2 = 0.;
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
  double diff_mag = 0.;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double dv = gpv.vel[d] - vel_part[d];
    diff_mag += dv * dv;
  }
  diff_mag = sqrt(diff_mag);
  const double Reyn = rho_skin * diff_mag * dia_part / mu_skin;
  const double Pr_skin = mu_skin * cp_skin / lambda_skin;
  const double powR = dmax(pmp_pow(dmin(400., Reyn), 0.077), 1.);
  const double Nu_0 = 1. + powR * pmp_cbrt(1. + Reyn * Pr_skin);
  double rhoD[NF];
  double rhoDtotal = 0., cp_fuel = 0., sumYSkin = 0.;
#pragma unroll
  for (int spf = 0; spf < NF; ++spf) {
    const int fspec = fdat.indx[spf];
    rhoD[spf] = Ddiag[spf] * (mw_skin / m.mw_kg[fspec] * kRhodConv);
    rhoDtotal += rhoD[spf] * (X_vapor[spf] / sumXVap);
    const double ysk = sel(Y_skin, fspec);
    cp_fuel += ysk * cp_mks(m, fspec, T_skin);
    sumYSkin += ysk;
  }
  cp_fuel /= sumYSkin;
  const double Sc_skin = mu_skin / rhoDtotal;
  const double logB = pmp_log1p(B_M);
  const double invFM = B_M / (logB * pmp_pow(1. + B_M, 0.7));
  const double Sh_0 = 1. + powR * pmp_cbrt(1. + Reyn * Sc_skin);
  const double Sh_num = 2. + (Sh_0 - 2.) * invFM;
  const double ratio = cp_fuel * Sh_num * rhoDtotal / lambda_skin;
  const double Nu_num = heat_coeff(ratio, B_M, B_eps, C_eps, Nu_0);
  y[0] = (float)log(rhoD[0] * Sh_num);
  y[1] = NF > 1 ? (float)log(rhoD[NF > 1 ? 1 : 0] * Sh_num) : 0.f;
  y[2] = (float)log(lambda_skin * Nu_num);
  y[3] = (float)log(mu_skin);
  y[4] = (float)log(rho_skin);
  return true;
}

// calcVaporState's closed-form part in FP32 (Drag.H:232-288): fuel latent
// heats, saturation pressures, Raoult vapor mole fractions, surface vapor mass
// fractions and the Spalding number B_M, for the learned kernel.
template <int NS, int NF, bool FF>
__device__ __forceinline__ void vapor_state_f(
  const DevMechF& m, const DevFuelF& ff, const DevFuel& fdat, const GasF<NS>& g, const float* cBoilT,
  float Tp_f, const double* Y_part, float* L_fuel, float* X_vapor, float* Yfv, float& sumXVap, float& B_M)
{
  const float RU = (float)(kRuCgs * kRuConv);
  const float PATM = (float)(kPatmCgs * kPresConv);
  float mw_part = 0.f;
#pragma unroll
  for (int spf = 0; spf < NF; ++spf) {
    mw_part += (float)Y_part[spf] * m.inv_mw_kg[fuel_sp<FF>(fdat, spf)];
  }
  mw_part = fdiv(1.f, mw_part);
  float mbar_vap = 0.f;
  sumXVap = 0.f;
#pragma unroll
  for (int spf = 0; spf < NF; ++spf) {
    const int fspec = fuel_sp<FF>(fdat, spf);
    const float mw_fuel = m.mw_kg[fspec];
    const float Tp = fminf(Tp_f, 0.99f * cBoilT[spf]);
    L_fuel[spf] = hf(m, fspec, Tp_f) + ff.latent[spf] - ff.cp[spf] * (Tp - ff.ref_T);
    float pres_sat;
    if (ff.psat_d[spf] == 0.f) {
      pres_sat = PATM * fexp(L_fuel[spf] * mw_fuel / RU * (ff.inv_boilT[spf] - fdiv(1.f, Tp)));
    } else {
      pres_sat = ff.psat_d[spf] * fexp2((ff.psat_a[spf] - fdiv(ff.psat_b[spf], Tp + ff.psat_c[spf])) * 3.32192809f);
    }
    const float X_fluid = fsel(g.Y, dep_sp<FF>(fdat, spf)) * g.mw_mix * m.inv_mw_kg[fspec];
    X_vapor[spf] = 0.f;
    if (pres_sat > X_fluid * g.p) {
      const float Xv = fdiv((float)Y_part[spf] * mw_part * m.inv_mw_kg[fspec] * pres_sat, g.p);
      mbar_vap += Xv * mw_fuel;
      sumXVap += Xv;
      X_vapor[spf] = Xv;
    }
  }
  const float inv_totalmwx = fdiv(1.f, mbar_vap + (1.f - sumXVap) * g.mw_mix);
  float sumYVap = 0.f, sumYfFluid = 0.f;
#pragma unroll
  for (int spf = 0; spf < NF; ++spf) {
    Yfv[spf] = 0.f;
    if (X_vapor[spf] > 0.f) {
      Yfv[spf] = X_vapor[spf] * m.mw_kg[fuel_sp<FF>(fdat, spf)] * inv_totalmwx;
      sumYVap += Yfv[spf];
      sumYfFluid += fsel(g.Y, dep_sp<FF>(fdat, spf));
    }
  }
  B_M = fminf(20.f, fdiv(sumYVap - sumYfFluid, fmaxf(1.E-15f, 1.f - sumYVap)));
}

// FP64 gas state at a droplet (trilinear gather, define): the teacher's input.
// Returns false if a stencil cell lies outside the grown state box.
template <int NS, int NF>
__device__ __forceinline__ bool learn_gas_fp64(
  const KParams& P, const BoxEntry& B, const double* pos, GasVals<NS, NF>& gpv, double* cBoilT)
{
  double lx[3];
  int ijk[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    lx[d] = (pos[d] - P.plo[d]) * P.dxi[d] + 0.5;
    ijk[d] = static_cast<int>(floor(lx[d]));
  }
  gpv.rho = 0.;
  gpv.T = 0.;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    gpv.vel[d] = 0.;
  }
#pragma unroll
  for (int n = 0; n < NS; ++n) {
    gpv.Y[n] = 0.;
  }
#pragma unroll
  for (int kk = -1; kk < 1; ++kk) {
#pragma unroll
    for (int jj = -1; jj < 1; ++jj) {
#pragma unroll
      for (int ii = -1; ii < 1; ++ii) {
        const double wx = ii == 0 ? lx[0] - ijk[0] : 1. - (lx[0] - ijk[0]);
        const double wy = jj == 0 ? lx[1] - ijk[1] : 1. - (lx[1] - ijk[1]);
        const double wz = kk == 0 ? lx[2] - ijk[2] : 1. - (lx[2] - ijk[2]);
        const double cw = wx * wy * wz;
        if (cw > 0.) {
          const int ci = ijk[0] + ii, cj = ijk[1] + jj, ck = ijk[2] + kk;
          if (!in_box(B.state_lo, B.state_hi, ci, cj, ck)) {
            return false;
          }
          const double* q = B.st + ((ci - B.st_lo[0]) + (cj - B.st_lo[1]) * B.st_j32 + (ck - B.st_lo[2]) * B.st_k32);
          const double r = q[P.c_rho * B.st_n32];
          gpv.rho += cw * r;
#pragma unroll
          for (int n = 0; n < NS; ++n) {
            gpv.Y[n] += cw * q[(P.c_spec + n) * B.st_n32] / r;
          }
#pragma unroll
          for (int d = 0; d < 3; ++d) {
            gpv.vel[d] += cw * q[(P.c_mom + d) * B.st_n32];
          }
          gpv.T += cw * q[P.c_T * B.st_n32];
        }
      }
    }
  }
  double mw_mix = 0.;
#pragma unroll
  for (int n = 0; n < NS; ++n) {
    mw_mix += gpv.Y[n] / P.m.mw_kg[n];
  }
  gpv.p = gpv.rho * kRuCgs * mw_mix * gpv.T * kRuConv;
  gpv.mw_mix = 1. / mw_mix;
  const double lp = pmp_log(kPatmCgs * kPresConv / gpv.p);
#pragma unroll
  for (int spf = 0; spf < NF; ++spf) {
    const double mw_fuel = P.m.mw_kg[P.f.indx[spf]];
    cBoilT[spf] = dmin(P.f.critT[spf], 1. / (lp * kRuCgs * kRuConv / (P.f.hboil_ref[spf] * mw_fuel) + 1. / P.f.boilT[spf]));
  }
  return true;
}

}  // namespace pmp
