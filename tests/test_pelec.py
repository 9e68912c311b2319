"""The PeleC coupling (CGS units, energy state) of the oracle, on CPU.

* oracle built with the C library's math == PeleMP's headers compiled
  without PELELM_USE_SPRAY (oracle/_ref/libref_pelec_*), bit for bit: the
  gas temperature from the energy (SprayInterpolation.H:111-146), the drag
  work and the evaporated kinetic energy in the energy source
  (Drag.H:282-286, 418-421), the CGS units (SprayFuelData.H:41-70);
* the project-math oracle within the FP64 tolerance of it;
* the same physical problem in both couplings: the droplets and the mass and
  momentum deposits agree after the unit change; the energy deposits differ
  by the two PeleC terms.
"""
import numpy as np
import pytest

from pelemp_b200 import capi
from pelemp_b200 import workloads as W
from oracle.pyoracle import Oracle, Reference
from tests.parity import assert_parts_close, source_errors
from tests.test_oracle import SMALL, run_calls


def pelec_problem(name, oracle, **kw):
    prob = W.CONFIGS[name](**(kw or SMALL[name]))
    return prob, W.to_pelec(prob, oracle.mech(prob.species))


@pytest.fixture(scope="module")
def oracle_pelec_libm():
    return Oracle(libm=True, pelec=True)


@pytest.fixture(scope="module")
def oracle_pelec():
    return Oracle(libm=False, pelec=True)


@pytest.mark.parametrize("name", list(SMALL))
def test_pelec_oracle_matches_reference_bitwise(name, oracle_pelec_libm):
    _, prob = pelec_problem(name, oracle_pelec_libm)
    if not Reference.available(prob.nspec, prob.nfuel, pelec=True):
        pytest.skip("PeleC reference build not present (needs the PeleMP sources at build time)")
    ref = Reference(prob.nspec, prob.nfuel, pelec=True)
    mech = oracle_pelec_libm.mech(prob.species)
    rc, fdat = oracle_pelec_libm.setup(prob, mech)
    assert rc == 0
    pr, sr = run_calls(ref, prob, mech, fdat, prob.steps)
    po, so = run_calls(oracle_pelec_libm, prob, mech, fdat, prob.steps)
    for a, b in zip(pr, po):
        for k in a:
            assert np.array_equal(a[k], b[k]), k
    for a, b in zip(sr, so):
        for x, y in zip(a, b):
            assert np.array_equal(x, y)


@pytest.mark.parametrize("name", ["config1", "config2"])
def test_pelec_project_math_within_fp64_tolerance(name, oracle_pelec, oracle_pelec_libm):
    _, prob = pelec_problem(name, oracle_pelec)
    mech = oracle_pelec.mech(prob.species)
    _, fdat = oracle_pelec.setup(prob, mech)
    pl, sl = run_calls(oracle_pelec_libm, prob, mech, fdat, prob.steps)
    pp, sp = run_calls(oracle_pelec, prob, mech, fdat, prob.steps)
    assert_parts_close(pl, pp, prob.nfuel, prob.dx)
    for a, b in zip(sl, sp):
        assert source_errors(a, b) <= 1e-9


def test_pelec_setup_units(oracle, oracle_pelec):
    """spraySetup's latent shift uses the coupling's energy unit: the CGS
    latent heat is 1e4 x the MKS one."""
    lm, pc = pelec_problem("config1", oracle_pelec, n=10)
    _, fm = oracle.setup(lm)
    _, fp = oracle_pelec.setup(pc)
    assert fp.latent[0] == pytest.approx(fm.latent[0] * 1e4, rel=1e-13)
    assert fp.ref_latent[0] == pytest.approx(fm.ref_latent[0] * 1e4, rel=1e-15)


def test_pelec_same_physics_as_lmex(oracle, oracle_pelec):
    """One MKD + MK of the same flow in both couplings: the droplets agree
    after the unit change (the gas temperature of the PeleC run comes from
    the energy by Newton iteration from a guess 7 K off), and so do the mass
    and momentum deposits (g/cm^3/s = 1e3 kg/m^3/s; g/cm^2/s^2 = 10 kg/m^2/s^2)."""
    lm, pc = pelec_problem("config1", oracle_pelec, n=3000, steps=1)
    ml = oracle.mech(lm.species)
    _, fl = oracle.setup(lm, ml)
    mp = oracle_pelec.mech(pc.species)
    _, fp = oracle_pelec.setup(pc, mp)
    pl, sl = run_calls(oracle, lm, ml, fl, 1)
    pp, sp = run_calls(oracle_pelec, pc, mp, fp, 1)
    nf = lm.nfuel
    for a, b in zip(pl, pp):
        assert np.array_equal(a["id"], b["id"])
        np.testing.assert_allclose(b["pos"] / 100.0, a["pos"], rtol=1e-12)
        rl, rp = a["rdata"], b["rdata"]
        np.testing.assert_allclose(rp[0:3] / 100.0, rl[0:3], rtol=1e-9, atol=1e-12)
        np.testing.assert_allclose(rp[capi.PSTATE_T], rl[capi.PSTATE_T], rtol=1e-9)
        np.testing.assert_allclose(rp[capi.PSTATE_DIA] / 100.0, rl[capi.PSTATE_DIA], rtol=1e-9)
    scale = {lm.comps().rhoSrcIndx: 1e3, lm.comps().momSrcIndx: 10.0}
    for call_l, call_p in zip(sl, sp):
        for bl, bp in zip(call_l, call_p):
            for c, f in scale.items():
                top = np.abs(bl[c]).max()
                assert top > 0
                assert np.abs(bp[c] * f - bl[c]).max() <= 1e-8 * top
            # the PeleC energy deposit (erg/cm^3/s = 0.1 J/m^3/s) adds the drag
            # work and the vapour's kinetic energy to the same enthalpy
            # exchange: present, and small beside it at these slip speeds
            e = 4 + nf
            diff = np.abs(bp[e] * 0.1 - bl[e]).max() / np.abs(bl[e]).max()
            assert 1e-6 < diff < 1e-3
