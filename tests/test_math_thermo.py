"""The project math library and the gas thermo/transport model.

pmp_math.h is checked in ulps against correctly rounded values (50-digit
decimal arithmetic) and against the C library over the argument ranges the
spray update uses; the thermo/transport tables are
checked against the kinetic-theory formulas they were fitted to
(pelemp_b200/csrc/phys/gen_thermo.py) and evaluated exactly against a numpy
restatement of the fitted forms.
"""
import importlib.util
import os

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _truth(fn, x, y=None):
    """Correctly rounded values from 50-digit decimal arithmetic."""
    from decimal import Decimal, getcontext
    getcontext().prec = 50
    out = np.empty_like(x)
    for i, v in enumerate(x):
        d = Decimal(float(v))
        if fn == "exp":
            r = d.exp()
        elif fn == "log":
            r = d.ln()
        elif fn == "log1p":
            r = (1 + d).ln()
        elif fn == "cbrt":
            r = d ** (Decimal(1) / Decimal(3))
        else:
            r = (Decimal(float(y[i])) * d.ln()).exp()
        out[i] = float(r)
    return out


def ulps(ours, truth):
    return np.abs(ours - truth) / np.spacing(np.abs(truth))


@pytest.mark.parametrize("fn,lo,hi", [
    ("exp", -30.0, 30.0), ("exp", -700.0, 700.0), ("log", 1e-300, 1e300), ("log", 0.5, 2.0),
    ("log1p", -0.9, 20.0), ("log1p", -1e-10, 1e-10), ("cbrt", 1e-30, 1e6),
])
def test_math_ulps(fn, lo, hi, oracle):
    rng = np.random.default_rng(1)
    if lo > 0 and hi / lo > 1e3:
        x = np.exp(rng.uniform(np.log(lo), np.log(hi), 3000))
    else:
        x = rng.uniform(lo, hi, 3000)
    bound = 2.5 if fn == "log1p" else 1.5
    assert np.max(ulps(oracle.math(fn, x), _truth(fn, x))) <= bound, fn


def test_pow_ulps(oracle):
    rng = np.random.default_rng(2)
    x = np.exp(rng.uniform(np.log(1e-3), np.log(1e3), 3000))
    y = rng.uniform(-3.0, 3.0, 3000)
    bound = 1.5 + 2.0 * np.abs(y * np.log(x))
    assert np.all(ulps(oracle.math("pow", x, y), _truth("pow", x, y)) <= bound)


def test_math_close_to_c_library(oracle, oracle_libm):
    rng = np.random.default_rng(3)
    x = np.exp(rng.uniform(np.log(1e-6), np.log(1e6), 100_000))
    for fn in ("exp", "log", "log1p", "cbrt"):
        xx = np.log(x) if fn == "exp" else x
        a, b = oracle.math(fn, xx), oracle_libm.math(fn, xx)
        assert np.max(np.abs(a - b) / np.abs(b)) <= 1e-15, fn


def test_math_special_values(oracle):
    assert oracle.math("exp", np.array([0.0]))[0] == 1.0
    assert oracle.math("log", np.array([1.0]))[0] == 0.0
    assert oracle.math("cbrt", np.array([27.0]))[0] == 3.0
    assert oracle.math("cbrt", np.array([-8.0]))[0] == -2.0
    assert oracle.math("exp", np.array([-800.0]))[0] == 0.0
    assert np.isinf(oracle.math("exp", np.array([800.0]))[0])
    assert oracle.math("pow", np.array([0.0]), np.array([2.0]))[0] == 0.0


def _gen():
    spec = importlib.util.spec_from_file_location(
        "gen_thermo", os.path.join(ROOT, "pelemp_b200", "csrc", "phys", "gen_thermo.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_thermo_tables_match_kinetic_theory(oracle):
    g = _gen()
    names = [s[0] for s in g.SPECIES]
    mech = oracle.mech(names)
    for T in (300.0, 600.0, 1000.0, 2000.0):
        cp, h = oracle.thermo(mech, T)
        for k, s in enumerate(g.SPECIES):
            W = s[1]
            cp_anchor = np.interp(T, g.T_ANCHOR, s[5])  # J/(mol K)
            assert abs(cp[k] * W * 1e-7 - cp_anchor) <= 0.02 * cp_anchor
    # h(298.15) = standard enthalpy of formation
    _, h = oracle.thermo(mech, 298.15)
    for k, s in enumerate(g.SPECIES):
        assert abs(h[k] * s[1] * 1e-7 - s[2]) <= 1e-6 * max(1.0, abs(s[2]))


def test_transport_matches_formulas(oracle):
    g = _gen()
    names = ["N2", "O2", "NC7H16"]
    mech = oracle.mech(names)
    sp = {s[0]: s for s in g.SPECIES}
    for T in (320.0, 700.0, 1200.0):
        # pure N2: mixture rules reduce to the species value
        mu, lam, _ = oracle.transport(mech, T, [1.0, 0.0, 0.0])
        W, tc, vc = sp["N2"][1], sp["N2"][3], sp["N2"][4]
        eps, sig = g.lj(tc, vc)
        mu_kt = 2.6693e-5 * np.sqrt(W * T) / (sig ** 2 * g.omega22(T / eps))
        assert abs(mu - mu_kt) <= 0.01 * mu_kt
        a = g.fit_cp(sp["N2"][5])
        lam_kt = mu_kt / W * (g.cp_molar_cgs(a, T) + 1.25 * g.RU_CGS)
        assert abs(lam - lam_kt) <= 0.01 * lam_kt
        # trace heptane in N2: Ddiag -> (W_f/Wbar) rho D_fN2 with D from Chapman-Enskog
        Y = [1.0 - 1e-9, 0.0, 1e-9]
        _, _, Dd = oracle.transport(mech, T, Y)
        e2, s2 = g.lj(sp["NC7H16"][3], sp["NC7H16"][4])
        sjk, ejk = 0.5 * (sig + s2), np.sqrt(eps * e2)
        Wf = sp["NC7H16"][1]
        d_atm = 0.0018583 * np.sqrt(T ** 3 * (1 / W + 1 / Wf)) / (sjk ** 2 * g.omega11(T / ejk))
        rhoD = (101325.0 * 10 * W / (g.RU_CGS * T)) * d_atm   # rho D at 1 atm, CGS
        expect = Wf / W * rhoD
        assert abs(Dd[2] - expect) <= 0.02 * expect


def test_transport_exact_form(oracle):
    """The mixture rules as documented in pmp_thermo.h, evaluated in numpy."""
    import ctypes
    names = ["N2", "O2", "NC10H22", "NC7H16", "CO2"]
    mech = oracle.mech(names)
    T = 640.0
    Y = np.array([0.6, 0.2, 0.1, 0.05, 0.05])
    mu, lam, Dd = oracle.transport(mech, T, Y)
    W = np.array(mech.mw[:5])
    X = Y / W / np.sum(Y / W)
    lnT = np.log(T)
    P = lambda c: c[0] + c[1] * lnT + c[2] * lnT ** 2 + c[3] * lnT ** 3
    mu_k = np.array([np.exp(P(mech.mu[k])) for k in range(5)])
    lam_k = np.array([np.exp(P(mech.lam[k])) for k in range(5)])
    assert abs(mu - np.sum(X * mu_k ** 6) ** (1 / 6)) <= 1e-13 * mu
    assert abs(lam - np.sum(X * lam_k ** 0.25) ** 4) <= 1e-13 * lam
    for i in range(5):
        t1 = sum(Y[j] for j in range(5) if j != i)
        t2 = sum(X[j] / np.exp(P(mech.dbin[i][j])) for j in range(5) if j != i)
        expect = W[i] * t1 / (t2 * 8.31446261815324e7 * T)
        assert abs(Dd[i] - expect) <= 1e-13 * expect
