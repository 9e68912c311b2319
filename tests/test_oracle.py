"""The CPU oracle against the reference's own code, known answers and identities.

* oracle built with the C library's math == PeleMP's Drag.H / SprayFuelData.H /
  SprayInterpolation.H / WallFunctions.H compiled here (oracle/_ref), bit for
  bit, on the configured workloads and on the error paths;
* oracle with the project math library within the FP64 tolerance of it;
* oracle built with the C library's math == the committed golden vectors
  (tests/golden, made by the reference build with tests/golden/make_golden.py),
  bit for bit, so the pin holds where the reference sources are absent;
* known answers: Stokes drag, saturated gas, kill below min_mass, boiling
  temperature at 1 atm, latent-heat adjustment of spraySetup;
* mass conservation of the deposits.
"""
import numpy as np
import pytest

from pelemp_b200 import capi
from pelemp_b200 import workloads as W
from oracle.pyoracle import Reference
from tests.parity import assert_parts_close, droplet_mass, source_errors


def run_calls(lib, prob, mech, fdat, steps, **kw):
    parts = prob.copy_parts()
    srcs = []
    for _ in range(steps):
        for do_move in (1, 0):
            src = prob.new_sources()
            rc, err, _ = lib.update(prob, mech, fdat, parts, src, do_move, **kw)
            assert rc == 0, (rc, err.box, err.particle, err.message)
            srcs.append(src)
    return parts, srcs


SMALL = {
    "config1": dict(n=6000, steps=2),
    "config2": dict(n=6000, steps=2, ncells=(32, 32, 32), box=(16, 16, 16)),
    "walls": dict(n=3000),
}


@pytest.mark.parametrize("name", list(SMALL))
def test_oracle_libm_matches_reference_bitwise(name, oracle_libm):
    prob = W.CONFIGS[name](**SMALL[name])
    if not Reference.available(prob.nspec, prob.nfuel):
        pytest.skip("reference build not present (needs the PeleMP sources at build time)")
    ref = Reference(prob.nspec, prob.nfuel)
    mech = oracle_libm.mech(prob.species)
    rc, fdat = oracle_libm.setup(prob, mech)
    assert rc == 0
    pr, sr = run_calls(ref, prob, mech, fdat, prob.steps)
    po, so = run_calls(oracle_libm, prob, mech, fdat, prob.steps)
    for a, b in zip(pr, po):
        for k in a:
            assert np.array_equal(a[k], b[k]), k
    for a, b in zip(sr, so):
        for x, y in zip(a, b):
            assert np.array_equal(x, y)


@pytest.mark.parametrize("name", list(SMALL))
def test_project_math_within_fp64_tolerance(name, oracle, oracle_libm):
    prob = W.CONFIGS[name](**SMALL[name])
    mech = oracle.mech(prob.species)
    _, fdat = oracle.setup(prob, mech)
    pl, sl = run_calls(oracle_libm, prob, mech, fdat, prob.steps)
    pp, sp = run_calls(oracle, prob, mech, fdat, prob.steps)
    assert_parts_close(pl, pp, prob.nfuel, prob.dx)
    # The mass, species and enthalpy deposits are formed as (m_new - m_old)/dt
    # (Drag.H:416-432): the ~1e-16 relative difference between two math
    # libraries in m is amplified by m/dm ~ 1e4-1e5, so the deposits of the two
    # builds agree to ~1e-11 of the largest deposit, not 1e-12.
    for a, b in zip(sl, sp):
        assert source_errors(a, b) <= 1e-9


def test_error_paths_match_reference(oracle_libm):
    prob = W.walls(n=500)
    if not Reference.available(prob.nspec, prob.nfuel):
        pytest.skip("reference build not present")
    ref = Reference(prob.nspec, prob.nfuel)
    mech = oracle_libm.mech(prob.species)
    _, fdat = oracle_libm.setup(prob, mech)
    # droplet outside the outflow (z) boundary at entry
    parts = prob.copy_parts()
    parts[0]["pos"][2, 7] = -0.5 * prob.dx[2]
    for lib in (ref, oracle_libm):
        p = [{k: v.copy() for k, v in q.items()} for q in parts]
        rc, err, _ = lib.update(prob, mech, fdat, p, prob.new_sources(), 1)
        assert rc == capi.PMP_ERR_LEFT_DOMAIN and err.box == 0 and err.particle == 7
    # film height > 0 needs the splash model
    parts = prob.copy_parts()
    parts[1]["rdata"][capi.pstate_filmhght(1), 3] = 1e-6
    for lib in (ref, oracle_libm):
        p = [{k: v.copy() for k, v in q.items()} for q in parts]
        rc, err, _ = lib.update(prob, mech, fdat, p, prob.new_sources(), 1)
        assert rc == capi.PMP_ERR_UNSUPPORTED and err.box == 1 and err.particle == 3


def test_state_and_source_box_errors(oracle_libm):
    prob = W.config1(n=200, steps=1)
    mech = oracle_libm.mech(prob.species)
    _, fdat = oracle_libm.setup(prob, mech)
    refs = [oracle_libm]
    if Reference.available(prob.nspec, prob.nfuel):
        refs.append(Reference(prob.nspec, prob.nfuel))
    # a droplet 2.7 cells outside its box needs stencil cells beyond 2 ghosts
    parts = prob.copy_parts()
    parts[0]["pos"][0, 11] = -2.7 * prob.dx[0]
    prob2 = W.config1(n=200, steps=1)
    prob2.state_ghosts = 2
    prob2.state = [s[:, 1:-1, 1:-1, 1:-1].copy() for s in prob.state]
    for lib in refs:
        p = [{k: v.copy() for k, v in q.items()} for q in parts]
        rc, err, _ = lib.update(prob2, mech, fdat, p, prob2.new_sources(), 0)
        assert rc == capi.PMP_ERR_STATE_BOX and err.particle == 11
    # deposit cell two cells out with one source ghost cell
    parts = prob.copy_parts()
    parts[0]["pos"][1, 5] = -1.5 * prob.dx[1]
    prob3 = W.config1(n=200, steps=1)
    prob3.source_ghosts = 1
    for lib in refs:
        p = [{k: v.copy() for k, v in q.items()} for q in parts]
        rc, err, _ = lib.update(prob3, mech, fdat, p, prob3.new_sources(), 0)
        assert rc == capi.PMP_ERR_SOURCE_BOX and err.particle == 5


def test_setup_latent_adjustment(oracle):
    """spraySetup subtracts h_fuel(ref_T) from the latent heat (SpraySetup.cpp:284-290)."""
    prob = W.config2(n=10, ncells=(16, 16, 16), box=(16, 16, 16))
    mech = oracle.mech(prob.species)
    rc, fdat = oracle.setup(prob, mech)
    assert rc == 0
    _, h = oracle.thermo(mech, prob.ref_T)
    for f, name in enumerate(prob.fuels):
        k = prob.species.index(name)
        assert fdat.indx[f] == k and fdat.dep_indx[f] == k
        assert fdat.ref_latent[f] == W.LIQUIDS[name]["latent"]
        assert fdat.latent[f] == W.LIQUIDS[name]["latent"] - h[k] * 1e-4
        assert fdat.rho_coef[4 * f] == W.LIQUIDS[name]["rho"]
        assert fdat.psat_coef[4 * f + 3] == 1e5
    assert fdat.dtmod == 0.5


def test_setup_rejects_breakup_and_unknown_fuel(oracle):
    prob = W.config1(n=10)
    mech = oracle.mech(prob.species)
    inp = prob.inputs()
    inp.use_breakup_model = 1
    rc, _ = oracle.setup(prob, mech, inp)
    assert rc == capi.PMP_ERR_UNSUPPORTED
    inp = prob.inputs()
    inp.fuel_species[0].value = b"NC12H26"
    rc, _ = oracle.setup(prob, mech, inp)
    assert rc == capi.PMP_ERR_INVALID


def _one(oracle, mech, fdat, gas, rd, dt=1e-6):
    return oracle.droplet_source(mech, fdat, dt, gas, rd)


def _gas(prob, T=900.0, vel=(0.0, 0.0, 0.0), Y=None, p=101325.0):
    W_ = np.array([W.MW[s] for s in prob.species])
    Y = np.array(Y if Y is not None else [0.767, 0.233] + [0.0] * (prob.nspec - 2))
    rho = p / (W.RU_SI * T * np.sum(Y / W_))
    return np.concatenate([[rho, T], vel, Y])


def _rdata(nf, d=20e-6, T=300.0, vel=(0.0, 0.0, 0.0), Y=(1.0,)):
    rd = np.zeros(capi.pstate_num(nf))
    rd[0:3] = vel
    rd[capi.PSTATE_T] = T
    rd[capi.PSTATE_DIA] = d
    rd[capi.PSTATE_Y:capi.PSTATE_Y + nf] = Y
    rd[capi.pstate_numdens(nf)] = 1.0
    return rd


def test_stokes_drag_known_answer(oracle):
    """mass_transfer off, Re < 1: C_D = 24/Re (Drag.H:271-273) gives the Stokes
    relaxation rate 18 mu / (rho_l d^2)."""
    prob = W.config1(n=10)
    prob.mass_trans = 0
    mech = oracle.mech(prob.species)
    _, fdat = oracle.setup(prob, mech)
    gas = _gas(prob, T=900.0, vel=(0.05, 0.0, 0.0))
    rd = _rdata(1, d=10e-6)
    dt = 1e-6
    re, out, _, src = _one(oracle, mech, fdat, gas, rd, dt)
    assert 0 < re < 1
    # viscosity of the gas at T (mass transfer off: T_skin = T_gas, Y_skin = Y_gas)
    mu, _, _ = oracle.transport(mech, 900.0, gas[5:8])
    mu_si = mu * 0.1
    rate = 18.0 * mu_si / (681.4 * 10e-6 ** 2)
    expect = 0.5 * dt * rate * 0.05
    assert abs(out[0] - expect) <= 1e-12 * abs(expect)
    assert out[1] == 0.0 and out[2] == 0.0
    assert out[capi.PSTATE_T] == 300.0 and out[capi.PSTATE_DIA] == 10e-6
    assert src[3] == 0.0   # no mass source
    # momentum given to the gas: N drag_force (u_g - u_d) = N 3 pi mu d (u_g - u_d) (Drag.H:281)
    assert abs(src[0] - 3 * np.pi * mu_si * 10e-6 * 0.05) <= 1e-12 * abs(src[0])


def test_zero_slip_zero_drag(oracle):
    prob = W.config1(n=10)
    mech = oracle.mech(prob.species)
    _, fdat = oracle.setup(prob, mech)
    gas = _gas(prob, T=900.0, vel=(1.0, -2.0, 0.5))
    rd = _rdata(1, vel=(1.0, -2.0, 0.5))
    re, out, _, src = _one(oracle, mech, fdat, gas, rd)
    assert re == 0.0
    # velocity changes only by the mass-loss term: none on the droplet itself
    assert np.array_equal(out[0:3], rd[0:3])


def test_saturated_gas_no_evaporation(oracle):
    """Fuel vapour above saturation: X_vapor = 0, mdot = 0, Nu = Nu_0 (Drag.H:95,341-344)."""
    prob = W.config1(n=10)
    mech = oracle.mech(prob.species)
    _, fdat = oracle.setup(prob, mech)
    gas = _gas(prob, T=320.0, Y=[0.2, 0.1, 0.7])
    rd = _rdata(1, T=300.0)
    _, out, pid, src = _one(oracle, mech, fdat, gas, rd)
    assert pid == 1
    assert src[3] == 0.0 and src[5] == 0.0           # no mass, no species source
    # no mass loss; d is recomputed as cbrt(6 m / (pi rho_l)) (Drag.H:400)
    assert abs(out[capi.PSTATE_DIA] - rd[capi.PSTATE_DIA]) <= 1e-15 * rd[capi.PSTATE_DIA]
    assert out[capi.PSTATE_T] > 300.0                   # still heated by convection


def test_kill_below_min_mass(oracle):
    """A droplet whose new mass is <= 1e-16 kg is removed and its whole mass
    goes to the gas (Drag.H:373-406,416-417)."""
    prob = W.config1(n=10)
    mech = oracle.mech(prob.species)
    _, fdat = oracle.setup(prob, mech)
    gas = _gas(prob, T=950.0)
    d = 0.6e-6
    rd = _rdata(1, d=d)
    dt = 1e-6
    _, out, pid, src = _one(oracle, mech, fdat, gas, rd, dt)
    assert pid == -1
    m0 = np.pi / 6 * 681.4 * d ** 3
    assert abs(src[3] + m0 / (0.5 * dt)) <= 1e-12 * m0 / (0.5 * dt)
    assert src[5] == src[3]


def test_mass_conservation_identity(oracle):
    """sum_cells S_rho V (dtmod dt) = -sum_droplets N (m_new - m_old) per call."""
    prob = W.config2(n=20000, steps=1, ncells=(32, 32, 32), box=(16, 16, 16))
    mech = oracle.mech(prob.species)
    _, fdat = oracle.setup(prob, mech)
    rho_l = [W.LIQUIDS[f]["rho"] for f in prob.fuels]
    parts = prob.copy_parts()
    vol = float(np.prod(prob.dx))
    for do_move in (1, 0):
        m0 = droplet_mass(prob, parts, rho_l)
        src = prob.new_sources()
        rc, err, nsub = oracle.update(prob, mech, fdat, parts, src, do_move)
        assert rc == 0
        m1 = droplet_mass(prob, parts, rho_l)
        gas = sum(float(np.sum(s[3])) for s in src) * vol * 0.5 * prob.flow_dt
        liq = sum(float(np.sum(b - a)) for a, b in zip(m0, m1))
        scale = sum(float(np.sum(np.abs(b - a))) for a, b in zip(m0, m1))
        assert scale > 0
        assert abs(gas + liq) <= 1e-9 * scale
        # species: the fuel deposit equals the mass deposit (single-species liquid pieces)
        fuel = sum(float(np.sum(s[4] + s[5])) for s in src)
        assert abs(fuel - sum(float(np.sum(s[3])) for s in src)) <= 1e-9 * abs(fuel)


@pytest.mark.parametrize("case", ["config1_n400", "config2_n400", "walls_n400", "pelec_config1_n400"])
def test_oracle_libm_matches_golden(case):
    """The libm oracle reproduces the reference build's committed outputs bit for bit."""
    import os
    from oracle.pyoracle import Oracle
    from tests.golden import make_golden as G
    g = np.load(os.path.join(os.path.dirname(G.__file__), case + ".npz"))
    pelec = G.CASES[case][2]
    orc = Oracle(libm=True, pelec=pelec)
    prob, _ = G.problem(case, orc.mech)
    assert str(g["input_sha256"]) == G.input_digest(prob), "workload generator changed"
    mech = orc.mech(prob.species)
    rc, fdat = orc.setup(prob, mech)
    assert rc == 0
    parts, calls = G.run(orc, prob, mech, fdat)
    for b, p in enumerate(parts):
        for k in ("pos", "rdata", "id"):
            assert np.array_equal(p[k], g[f"b{b}_{k}"]), (b, k)
    gold = G.unpack_sources(g, prob, int(g["ncalls"]))
    assert len(gold) == len(calls)
    for a, b in zip(calls, gold):
        for x, y in zip(a, b):
            assert np.array_equal(x, y)


def _energy_run(orc, prob, steps):
    mech = orc.mech(prob.species)
    rc, fdat = orc.setup(prob, mech)
    assert rc == 0
    parts = prob.copy_parts()
    res = [np.zeros(p["id"].size) for p in parts]
    calls = []
    for _ in range(steps):
        for do_move in (1, 0):
            src = prob.new_sources()
            rc, err, _ = orc.update_energy(prob, mech, fdat, parts, src, do_move, res)
            assert rc == 0, err.message
            calls.append(src)
    return fdat, parts, calls, res


@pytest.mark.parametrize("name", ["config1", "config2", "kills"])
def test_energy_identity_of_the_explicit_scheme(name, oracle):
    """Liquid enthalpy change + gas enthalpy gain == the sum of the scheme's
    named residual terms (explicit update, composition clip, vapour enthalpy at
    the last sub-step, droplet death, average over the sub-steps), to
    round-off of the exchanged enthalpy; PeleLMeX coupling, periodic domain."""
    from tests.parity import energy_identity
    if name == "kills":
        prob = W.config1(n=3000, steps=2)
        # a fifth of the droplets near min_mass (1e-16 kg): they die in the call
        p = prob.parts[0]
        p["rdata"][capi.PSTATE_DIA, ::5] = 0.75e-6
    else:
        prob = W.CONFIGS[name](**SMALL[name])
    rho_l = [W.LIQUIDS[f]["rho"] for f in prob.fuels]
    fdat, parts, calls, res = _energy_run(oracle, prob, prob.steps)
    err, rel_res = energy_identity(prob, fdat, prob.parts, parts, calls, res, rho_l)
    print(f"{name}: energy identity closes to {err:.2e} of the exchange; scheme residual {rel_res:.2e}")
    assert abs(err) <= 1e-10
    if name == "kills":
        assert sum(int(np.sum(q["id"] <= 0)) for q in parts) > 0
