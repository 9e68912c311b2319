"""Generate the project's gas thermodynamics and transport tables.

The spray update calls a gas equation of state and a transport model through
four functions: molecular weights, per-species c_p(T), per-species h(T) and a
mixture transport routine returning viscosity, thermal conductivity and the
mixture-averaged diagonal diffusion coefficients (PeleMP call sites:
Source/PP_Spray/SprayParticles.cpp:332, Source/PP_Spray/Drag.H:220-221,
Source/PP_Spray/Drag.H:252-256).  In the reference those come from the
PelePhysics library and a generated mechanism header, neither of which ships
with PeleMP.  This script builds the project's own stand-in, written from
published physics:

* c_p/R of each species is a quartic in T (the NASA 7-coefficient form,
  a single temperature range 250-3000 K), least-squares fitted to tabulated
  ideal-gas heat capacities; the enthalpy constant a5 places h(298.15 K) at the
  species' standard enthalpy of formation.
* Lennard-Jones parameters come from the corresponding-states correlation of
  Chung, Ajlan, Lee & Starling (Ind. Eng. Chem. Res. 27, 671, 1988):
  eps/k = Tc / 1.2593, sigma = 0.809 Vc^(1/3).
* Pure-species viscosity is Chapman-Enskog with the Omega(2,2)* fit of
  Neufeld, Janzen & Aziz (J. Chem. Phys. 57, 1100, 1972); conductivity is the
  modified Eucken relation lambda = mu/W (c_p,molar + 5/4 R); binary diffusion
  is Chapman-Enskog with Neufeld's Omega(1,1)* and Lorentz-Berthelot rules.
* ln(mu), ln(lambda) and ln(P*D_jk) are fitted as cubics in ln T over
  250-3000 K, the storage form a reduced ("simple") transport model uses.

Units are CGS at this interface (g, cm, s, erg, dyn), as the spray code
expects before it applies its unit conversions.

Run:  python gen_thermo.py  (rewrites pmp_thermo_data.h beside this file).
"""
import os

import numpy as np

RU_CGS = 8.31446261815324e7  # erg / (mol K)
RU_SI = 8.31446261815324     # J / (mol K)
PATM_CGS = 1013250.0         # dyn / cm^2

T_ANCHOR = np.array([300., 400., 500., 600., 800., 1000., 1500., 2000., 2500.])

# name, W [g/mol], Hf(298.15) [J/mol], Tc [K], Vc [cm^3/mol], cp anchors [J/(mol K)]
SPECIES = [
    ("N2", 28.0134, 0.0, 126.2, 89.8,
     [29.12, 29.25, 29.58, 30.11, 31.43, 32.70, 34.85, 36.00, 36.60]),
    ("O2", 31.9988, 0.0, 154.6, 73.4,
     [29.38, 30.11, 31.09, 32.09, 33.74, 34.88, 36.56, 37.78, 38.90]),
    ("NC7H16", 100.2019, -187.8e3, 540.2, 428.0,
     [166.0, 209.0, 248.0, 281.0, 333.0, 373.0, 427.0, 452.0, 465.0]),
    ("NC10H22", 142.2817, -249.5e3, 617.7, 624.0,
     [234.0, 296.0, 350.0, 396.0, 467.0, 520.0, 600.0, 632.0, 648.0]),
    ("CO2", 44.0095, -393.51e3, 304.1, 94.1,
     [37.22, 41.33, 44.63, 47.32, 51.43, 54.31, 58.38, 60.35, 61.50]),
]

T0 = 298.15
T_FIT = np.exp(np.linspace(np.log(250.0), np.log(3000.0), 240))


def fit_cp(cp_anchor):
    """Least-squares quartic of cp/R in T (columns scaled by 1000^n)."""
    y = np.asarray(cp_anchor) / RU_SI
    s = T_ANCHOR / 1000.0
    A = np.vander(s, 5, increasing=True)
    c, *_ = np.linalg.lstsq(A, y, rcond=None)
    return c / (1000.0 ** np.arange(5))


def h_over_rt_poly(a, T):
    return (a[0] + a[1] * T / 2 + a[2] * T**2 / 3 + a[3] * T**3 / 4
            + a[4] * T**4 / 5)


def omega22(ts):
    return (1.16145 * ts ** -0.14874 + 0.52487 * np.exp(-0.77320 * ts)
            + 2.16178 * np.exp(-2.43787 * ts))


def omega11(ts):
    return (1.06036 * ts ** -0.15610 + 0.19300 * np.exp(-0.47635 * ts)
            + 1.03587 * np.exp(-1.52996 * ts) + 1.76474 * np.exp(-3.89411 * ts))


def lj(tc, vc):
    return tc / 1.2593, 0.809 * vc ** (1.0 / 3.0)


def cp_molar_cgs(a, T):
    return RU_CGS * np.polyval(a[::-1], T)


def main():
    ns = len(SPECIES)
    cp_coef = np.zeros((ns, 6))
    mu_fit = np.zeros((ns, 4))
    lam_fit = np.zeros((ns, 4))
    dbin_fit = np.zeros((ns, ns, 4))
    mw = np.array([s[1] for s in SPECIES])
    eps = np.zeros(ns)
    sig = np.zeros(ns)
    lnT = np.log(T_FIT)
    for k, (name, W, hf, tc, vc, cpa) in enumerate(SPECIES):
        a = fit_cp(cpa)
        a5 = hf / RU_SI - T0 * h_over_rt_poly(a, T0)
        cp_coef[k, :5] = a
        cp_coef[k, 5] = a5
        eps[k], sig[k] = lj(tc, vc)
        mu = 2.6693e-5 * np.sqrt(W * T_FIT) / (sig[k] ** 2 * omega22(T_FIT / eps[k]))
        lam = mu / W * (cp_molar_cgs(a, T_FIT) + 1.25 * RU_CGS)
        mu_fit[k] = np.polyfit(lnT, np.log(mu), 3)[::-1]
        lam_fit[k] = np.polyfit(lnT, np.log(lam), 3)[::-1]
    for j in range(ns):
        for k in range(ns):
            s_jk = 0.5 * (sig[j] + sig[k])
            e_jk = np.sqrt(eps[j] * eps[k])
            d_atm = (0.0018583 * np.sqrt(T_FIT**3 * (1 / mw[j] + 1 / mw[k]))
                     / (s_jk**2 * omega11(T_FIT / e_jk)))
            pd = d_atm * PATM_CGS
            dbin_fit[j, k] = np.polyfit(lnT, np.log(pd), 3)[::-1]

    def arr(v):
        return ", ".join(repr(float(x)) for x in np.ravel(v))

    lines = [
        "/* Generated by gen_thermo.py; do not edit by hand.",
        " * Gas thermodynamic and transport tables of the project's species",
        " * database, CGS units.  Species order:",
        " *   " + ", ".join(s[0] for s in SPECIES),
        " * cp/R = a0 + a1 T + a2 T^2 + a3 T^3 + a4 T^4 ; h/(R T) adds a5/T.",
        " * ln mu, ln lambda, ln(P D_jk) = c0 + c1 lnT + c2 lnT^2 + c3 lnT^3.",
        " */",
        "#ifndef PMP_THERMO_DATA_H",
        "#define PMP_THERMO_DATA_H",
        f"#define PMP_DB_NSPEC {ns}",
    ]
    for k, s in enumerate(SPECIES):
        lines.append(f"#define PMP_SP_{s[0]} {k}")
    lines += [
        "static const char* const pmp_db_names[PMP_DB_NSPEC] = {"
        + ", ".join(f'"{s[0]}"' for s in SPECIES) + "};",
        f"static const double pmp_db_mw[PMP_DB_NSPEC] = {{{arr(mw)}}};",
        f"static const double pmp_db_cp[PMP_DB_NSPEC][6] = {{{arr(cp_coef)}}};",
        f"static const double pmp_db_mu[PMP_DB_NSPEC][4] = {{{arr(mu_fit)}}};",
        f"static const double pmp_db_lam[PMP_DB_NSPEC][4] = {{{arr(lam_fit)}}};",
        "static const double pmp_db_dbin[PMP_DB_NSPEC][PMP_DB_NSPEC][4] = {"
        + arr(dbin_fit) + "};",
        "#endif",
        "",
    ]
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "pmp_thermo_data.h")
    with open(out, "w") as f:
        f.write("\n".join(lines))
    # fit quality report
    for k, s in enumerate(SPECIES):
        a = cp_coef[k, :5]
        err = np.max(np.abs(np.polyval(a[::-1], T_ANCHOR) * RU_SI - np.array(s[5]))
                     / np.array(s[5]))
        print(f"{s[0]:8s} cp fit max rel err {err:.2e}  eps/k {eps[k]:.1f} sigma {sig[k]:.3f}")


if __name__ == "__main__":
    main()
