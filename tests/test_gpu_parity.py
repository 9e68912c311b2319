"""FP64 kernel parity against the CPU oracle, through the C ABI, on a B200.

The plain FP64 kernel evaluates the oracle's arithmetic in the same order
with the same math library, so each droplet's state after every call must
be bit-identical to the oracle's (cell indices, ids and box assignment
included).  Mesh deposits differ only by the order of the atomic additions:
per component |gpu - oracle| <= 1e-12 max|deposit|.
"""
import numpy as np
import pytest

from pelemp_b200 import capi
from pelemp_b200 import workloads as W
from pelemp_b200.spray import SprayError, from_problem, views
from tests.gpu_util import assert_bitwise, device_sources, device_state, gpu_run, oracle_run
from tests.parity import assert_parts_close, droplet_mass, source_errors

pytestmark = pytest.mark.gpu

CASES = {
    "config1": dict(n=100_000, steps=10),
    "config2": dict(n=40_000, steps=3, ncells=(32, 32, 32), box=(16, 16, 16)),
    "walls": dict(n=8000),
}


@pytest.mark.parametrize("name", list(CASES))
def test_fp64_bitwise_vs_oracle(name, oracle):
    prob = W.CONFIGS[name](**CASES[name])
    pg, sg, sp = gpu_run(prob, prob.steps)
    po, so = oracle_run(oracle, prob, prob.steps)
    assert_bitwise(pg, po)
    for a, b in zip(sg, so):
        assert source_errors(a, b) <= 1e-12
    st = sp.stats()
    assert st.substeps > 0


def test_ghost_particles_vs_oracle(oracle):
    prob = W.config1(n=20_000, steps=2)
    pg, sg, _ = gpu_run(prob, 2, is_ghost=1)
    po, so = oracle_run(oracle, prob, 2, is_ghost=1)
    assert_bitwise(pg, po)
    for a, b in zip(sg, so):
        assert source_errors(a, b) <= 1e-12


def test_host_views_match_device_views():
    import torch
    prob = W.config2(n=20_000, steps=1, ncells=(32, 32, 32), box=(16, 16, 16))
    pg, sg, _ = gpu_run(prob, 1)
    sp = from_problem(prob)
    st_h = [np.ascontiguousarray(s) for s in prob.state]
    st_v = views(st_h, [prob.grown(b, prob.state_ghosts)[0] for b in range(len(prob.boxes))])
    srcs = []
    for do_move in (1, 0):
        src = prob.new_sources()
        src_v = views(src, [prob.grown(b, prob.source_ghosts)[0] for b in range(len(prob.boxes))])
        sp.update_particles_host(st_v, src_v, prob.flow_dt, 0.0, prob.state_ghosts,
                                 prob.source_ghosts, 0, 0, do_move, prob.spray_cfl_lev)
        srcs.append(src)
    ph = [sp.get_particles(b) for b in range(len(prob.boxes))]
    assert_bitwise(pg, ph)
    for a, b in zip(sg, srcs):
        assert source_errors(a, b) <= 1e-12


def test_caller_order_and_aos_round_trip():
    prob = W.config1(n=5000)
    sp = from_problem(prob)
    back = sp.get_particles(0)
    p = prob.parts[0]
    for k in ("pos", "rdata", "id"):
        assert np.array_equal(back[k], p[k])
    # AoS in, AoS out: { pos[3], rdata[10+F], id, cpu }
    n = p["id"].shape[0]
    nr = capi.pstate_num(1)
    rec = np.zeros((n, 3 + nr + 1), dtype=np.float64)
    rec[:, 0:3] = p["pos"].T
    rec[:, 3:3 + nr] = p["rdata"].T
    ids = rec[:, 3 + nr:].view(np.int32)
    ids[:, 0] = p["id"]
    ids[:, 1] = 7
    sp.set_particles_aos(0, rec, n)
    out = sp.get_particles_aos(0).view(np.float64).reshape(n, 3 + nr + 1)
    assert np.array_equal(out[:, :3 + nr], rec[:, :3 + nr])
    assert np.array_equal(out[:, 3 + nr:].view(np.int32)[:, 0], p["id"])


def _expect_error(prob, code, particle, box=0, do_move=1):
    import torch
    sp = from_problem(prob)
    st, st_v = device_state(prob)
    src, src_v = device_sources(prob)
    with pytest.raises(SprayError) as e:
        sp.update_particles(st_v, src_v, prob.flow_dt, 0.0, prob.state_ghosts, prob.source_ghosts,
                            0, 0, do_move, prob.spray_cfl_lev,
                            torch.cuda.current_stream().cuda_stream)
    assert e.value.code == code
    assert e.value.info.box == box and e.value.info.particle == particle
    # the handle stays usable
    sp.close()


def test_error_left_domain():
    prob = W.walls(n=500)
    prob.parts[0]["pos"][2, 7] = -0.5 * prob.dx[2]
    _expect_error(prob, capi.PMP_ERR_LEFT_DOMAIN, 7)


def test_error_state_box():
    prob = W.config1(n=200, steps=1)
    prob.parts[0]["pos"][0, 11] = -2.7 * prob.dx[0]
    prob.state_ghosts = 2
    prob.state = [s[:, 1:-1, 1:-1, 1:-1].copy() for s in prob.state]
    _expect_error(prob, capi.PMP_ERR_STATE_BOX, 11, do_move=0)


def test_error_source_box():
    prob = W.config1(n=200, steps=1)
    prob.parts[0]["pos"][1, 5] = -1.5 * prob.dx[1]
    prob.source_ghosts = 1
    _expect_error(prob, capi.PMP_ERR_SOURCE_BOX, 5, do_move=0)


def test_error_film_unsupported():
    prob = W.walls(n=500)
    prob.parts[1]["rdata"][capi.pstate_filmhght(1), 3] = 1e-6
    _expect_error(prob, capi.PMP_ERR_UNSUPPORTED, 3, box=1)


def test_host_pointer_rejected_by_device_entry_point():
    """Plain host arrays given to pmp_spray_update are refused before launch."""
    import torch
    prob = W.config1(n=100, steps=1)
    sp = from_problem(prob)
    st_h = views(prob.state, [prob.grown(0, prob.state_ghosts)[0]])
    src, src_v = device_sources(prob)
    with pytest.raises(SprayError) as e:
        sp.update_particles(st_h, src_v, prob.flow_dt, 0.0, prob.state_ghosts, prob.source_ghosts,
                            0, 0, 1, prob.spray_cfl_lev, torch.cuda.current_stream().cuda_stream)
    assert e.value.code == capi.PMP_ERR_INVALID
    sp.close()


def test_empty_boxes_and_zero_droplets():
    prob = W.config2(n=0, steps=1, ncells=(32, 32, 32), box=(16, 16, 16))
    pg, sg, sp = gpu_run(prob, 1)
    assert sp.stats().substeps == 0
    assert all(np.all(s == 0) for call in sg for s in call)


def test_full_size_config2_sampled_parity_and_mass(oracle):
    """16M droplets, 8 boxes of 64^3: every droplet's state after a step is
    compared bit for bit with the oracle on a random sample (droplets are
    independent given the gas state), and the mass deposits close the liquid
    mass balance of all 16M droplets to round-off."""
    prob = W.config2(n=16_000_000, steps=1)
    rho_l = [W.LIQUIDS[f]["rho"] for f in prob.fuels]
    m0 = droplet_mass(prob, prob.parts, rho_l)
    pg, sg, sp = gpu_run(prob, 1)
    assert sp.stats().substeps > 0
    m1 = droplet_mass(prob, pg, rho_l)
    vol = float(np.prod(prob.dx))
    gas = sum(float(np.sum(s[3])) for call in sg for s in call) * vol * 0.5 * prob.flow_dt
    liq = sum(float(np.sum(b - a)) for a, b in zip(m0, m1))
    scale = sum(float(np.sum(np.abs(b - a))) for a, b in zip(m0, m1))
    assert abs(gas + liq) <= 1e-9 * scale
    # sampled bitwise parity
    rng = np.random.default_rng(5)
    sub = W.config2(n=0, steps=1)
    sub.state = prob.state
    sub.parts = []
    picks = []
    for b, p in enumerate(prob.parts):
        sel = np.sort(rng.choice(p["id"].shape[0], size=2500, replace=False))
        picks.append(sel)
        sub.parts.append({k: np.ascontiguousarray(v[..., sel]) for k, v in p.items()})
    po, _ = oracle_run(oracle, sub, 1)
    for b, sel in enumerate(picks):
        for k in ("pos", "rdata", "id"):
            assert np.array_equal(pg[b][k][..., sel], po[b][k]), (b, k)


@pytest.mark.parametrize("case", ["config1_n400", "config2_n400", "walls_n400"])
def test_fp64_vs_reference_golden(case):
    """The FP64 kernel against the reference build's committed outputs
    (tests/golden): the kernel runs the project math library, the reference
    the C library's, so droplets agree within the FP64 tolerances of
    tests/parity.py and deposits, (m_new - m_old)/dt differences, within 1e-9
    of the largest."""
    import os
    from oracle.pyoracle import Oracle
    from tests.golden import make_golden as G
    g = np.load(os.path.join(os.path.dirname(G.__file__), case + ".npz"))
    prob, _ = G.problem(case, Oracle(libm=True).mech)
    assert str(g["input_sha256"]) == G.input_digest(prob)
    pg, sg, sp = gpu_run(prob, prob.steps)
    gold_parts = [{k: g[f"b{b}_{k}"] for k in ("pos", "rdata", "id")} for b in range(len(prob.boxes))]
    assert_parts_close(pg, gold_parts, prob.nfuel, prob.dx)
    gold = G.unpack_sources(g, prob, int(g["ncalls"]))
    for a, b in zip(sg, gold):
        assert source_errors(b, a) <= 1e-9
    sp.close()


@pytest.mark.parametrize("name", ["config1", "config2", "kills"])
def test_fp64_energy_identity(name, oracle):
    """Global liquid + gas energy: the GPU's liquid enthalpy change plus the
    enthalpy its deposits give the gas equals the explicit scheme's residual
    (summed over the droplets by the oracle, Drag.H:345-434) to round-off;
    the mass balance closes exactly (liquid loss == gas gain)."""
    from tests.gpu_util import oracle_energy_residual
    from tests.parity import energy_identity
    if name == "kills":
        prob = W.config1(n=20_000, steps=2)
        prob.parts[0]["rdata"][capi.PSTATE_DIA, ::5] = 0.75e-6
    elif name == "config1":
        prob = W.config1(n=100_000, steps=3)
    else:
        prob = W.config2(n=40_000, steps=3, ncells=(32, 32, 32), box=(16, 16, 16))
    rho_l = [W.LIQUIDS[f]["rho"] for f in prob.fuels]
    fdat, _, _, res = oracle_energy_residual(oracle, prob, prob.steps)
    pg, sg, sp = gpu_run(prob, prob.steps)
    err, rel = energy_identity(prob, fdat, prob.parts, pg, sg, res, rho_l)
    print(f"{name}: FP64 energy identity {err:.2e} of the exchange (scheme residual {rel:.2e})")
    assert abs(err) <= 1e-10
    m0 = sum(float(np.sum(m)) for m in droplet_mass(prob, prob.parts, rho_l))
    m1 = sum(float(np.sum(m)) for m in droplet_mass(prob, pg, rho_l))
    vol = float(np.prod(prob.dx))
    gas = sum(float(np.sum(s[prob.comps().rhoSrcIndx])) for call in sg for s in call) * vol * fdat.dtmod * prob.flow_dt
    assert abs(gas + (m1 - m0)) <= 1e-10 * abs(m1 - m0)
    sp.close()


@pytest.mark.parametrize("mode", [capi.PMP_MODE_FP64, capi.PMP_MODE_MIXED])
def test_counters_exact_per_call(mode, oracle):
    """The update counters, summed by the host over their device slots: every
    call's droplet-substeps equal the oracle's count, and its kills equal
    the droplets the call removed (a fifth of box 0's droplets start at
    0.75 um and evaporate within the call; the mixed form hands them to its
    FP64 kernel, so its kills match the oracle's too)."""
    import torch
    prob = W.config1(n=20_000, steps=2)
    prob.parts[0]["rdata"][capi.PSTATE_DIA, ::5] = 0.75e-6
    mech = oracle.mech(prob.species)
    rc, fdat = oracle.setup(prob, mech)
    assert rc == 0
    parts = prob.copy_parts()
    sp = from_problem(prob, mode=mode)
    st_keep, st_v = device_state(prob)
    killed_total = 0
    for _step in range(prob.steps):
        for do_move in (1, 0):
            alive0 = sum(int(np.sum(p["id"] > 0)) for p in parts)
            rc, err, n_or = oracle.update(prob, mech, fdat, parts, prob.new_sources(), do_move)
            assert rc == 0, err.message
            alive1 = sum(int(np.sum(p["id"] > 0)) for p in parts)
            _src, src_v = device_sources(prob)
            sp.update_particles(st_v, src_v, prob.flow_dt, 0.0, prob.state_ghosts, prob.source_ghosts,
                                0, 0, do_move, prob.spray_cfl_lev, torch.cuda.current_stream().cuda_stream)
            s = sp.stats()
            assert s.substeps == n_or
            assert s.killed == alive0 - alive1
            assert s.inner_steps >= s.substeps
            killed_total += s.killed
    assert killed_total > 0
    del st_keep
    sp.close()
