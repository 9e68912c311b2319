"""Mixed-precision form (PMP_MODE_MIXED) against the FP64 oracle.

Bounds (after several MKD+MK steps):
* droplet temperature, diameter, liquid mass: 1e-4 relative (the headline
  accuracy target); measured errors are far smaller and printed;
* droplet velocity: 1e-4 of max(|u|, 1 m/s);
* deposits per component: 1e-4 of the component's largest deposit;
* liquid + gas mass balance: closes to FP64 round-off (1e-9 of the mass
  exchanged), because masses and deposits stay FP64;
* droplets that enter a call with d < 2 um are updated by the FP64 kernel:
  bit-identical to the oracle.
"""
import numpy as np
import pytest

from pelemp_b200 import capi
from pelemp_b200 import workloads as W
from tests.gpu_util import gpu_run, oracle_run
from tests.parity import droplet_mass

pytestmark = pytest.mark.gpu

TOL = 1e-4


def errors(pg, po, nfuel):
    e = {"T": 0.0, "dia": 0.0, "vel": 0.0, "Y": 0.0}
    for a, b in zip(pg, po):
        alive = (b["id"] > 0) & (a["id"] > 0)
        ra, rb = a["rdata"][:, alive], b["rdata"][:, alive]
        for key, row in (("T", capi.PSTATE_T), ("dia", capi.PSTATE_DIA)):
            e[key] = max(e[key], float(np.max(np.abs(ra[row] - rb[row]) / np.abs(rb[row]), initial=0)))
        sp = np.maximum(np.sqrt(np.sum(rb[0:3] ** 2, axis=0)), 1.0)
        e["vel"] = max(e["vel"], float(np.max(np.sqrt(np.sum((ra[0:3] - rb[0:3]) ** 2, axis=0)) / sp,
                                              initial=0)))
        e["Y"] = max(e["Y"], float(np.max(np.abs(ra[5:5 + nfuel] - rb[5:5 + nfuel]), initial=0)))
    return e


@pytest.mark.parametrize("name,kw", [
    ("config1", dict(n=50_000, steps=5)),
    ("config2", dict(n=40_000, steps=4, ncells=(32, 32, 32), box=(16, 16, 16))),
])
def test_mixed_accuracy_vs_fp64_oracle(name, kw, oracle):
    prob = W.CONFIGS[name](**kw)
    pg, sg, sp = gpu_run(prob, prob.steps, mode=capi.PMP_MODE_MIXED)
    po, so = oracle_run(oracle, prob, prob.steps)
    ids_g = np.concatenate([p["id"] for p in pg])
    ids_o = np.concatenate([p["id"] for p in po])
    assert np.mean(ids_g == ids_o) > 0.9999
    e = errors(pg, po, prob.nfuel)
    print(name, "mixed vs FP64 errors:", e)
    for k in ("T", "dia", "vel", "Y"):
        assert e[k] <= TOL, (k, e)
    worst = 0.0
    for a, b in zip(sg, so):
        for x, y in zip(a, b):
            for c in range(x.shape[0]):
                scale = np.max(np.abs(y[c]))
                if scale > 0:
                    worst = max(worst, float(np.max(np.abs(x[c] - y[c])) / scale))
    print(name, "mixed vs FP64 deposit error:", worst)
    assert worst <= TOL


def test_mixed_mass_balance_closes():
    prob = W.config2(n=40_000, steps=1, ncells=(32, 32, 32), box=(16, 16, 16))
    rho_l = [W.LIQUIDS[f]["rho"] for f in prob.fuels]
    m0 = droplet_mass(prob, prob.parts, rho_l)
    pg, sg, _ = gpu_run(prob, 1, mode=capi.PMP_MODE_MIXED)
    m1 = droplet_mass(prob, pg, rho_l)
    vol = float(np.prod(prob.dx))
    gas = sum(float(np.sum(s[3])) for call in sg for s in call) * vol * 0.5 * prob.flow_dt
    liq = sum(float(np.sum(b - a)) for a, b in zip(m0, m1))
    scale = sum(float(np.sum(np.abs(b - a))) for a, b in zip(m0, m1))
    assert abs(gas + liq) <= 1e-9 * scale


def test_small_droplets_take_the_fp64_path(oracle):
    prob = W.config1(n=20_000, steps=1)
    p = prob.parts[0]
    small = np.arange(0, p["id"].shape[0], 7)
    p["rdata"][capi.PSTATE_DIA, small] = 1.5e-6
    pg, _, sp = gpu_run(prob, 1, mode=capi.PMP_MODE_MIXED)
    assert sp.stats().fallback == small.size  # the MK call's fallback count
    po, _ = oracle_run(oracle, prob, 1)
    for k in ("pos", "rdata", "id"):
        a, b = pg[0][k], po[0][k]
        assert np.array_equal(a[..., small], b[..., small]), k


def test_mixed_graph_and_side_stream_match_plain_launch(oracle):
    """The mixed form's FP64 list kernel runs on a side stream beside the mixed
    kernel; replayed from a CUDA graph (use_graph), the forked work gives the
    same droplets bit for bit and the same deposits up to atomic order, and
    the small droplets still match the FP64 oracle exactly."""
    from tests.gpu_util import assert_bitwise
    from tests.parity import source_errors
    prob = W.config2(n=30_000, steps=2, ncells=(32, 32, 32), box=(16, 16, 16))
    small = []
    for p in prob.parts:
        idx = np.arange(0, p["id"].shape[0], 11)
        p["rdata"][capi.PSTATE_DIA, idx] = 1.5e-6
        small.append(idx)
    pa, sa, _ = gpu_run(prob, prob.steps, mode=capi.PMP_MODE_MIXED)
    pb, sb, spb = gpu_run(prob, prob.steps, mode=capi.PMP_MODE_MIXED,
                          setup=lambda sp: sp.set_launch(use_graph=True))
    assert spb.stats().graph != 0
    assert_bitwise(pa, pb)
    for a, b in zip(sa, sb):
        assert source_errors(b, a) <= 1e-12
    po, _ = oracle_run(oracle, prob, prob.steps)
    for b, idx in enumerate(small):
        for k in ("pos", "rdata", "id"):
            assert np.array_equal(pa[b][k][..., idx], po[b][k][..., idx]), (b, k)


def test_mixed_energy_identity(oracle):
    """Global energy drift of the mixed form: its liquid enthalpy change plus
    the enthalpy its deposits give the gas, against the FP64 scheme's residual
    (the oracle's): within 1e-5 of the enthalpy exchanged (the FP64 form closes
    it to round-off)."""
    from tests.gpu_util import oracle_energy_residual
    from tests.parity import energy_identity
    prob = W.config2(n=40_000, steps=3, ncells=(32, 32, 32), box=(16, 16, 16))
    rho_l = [W.LIQUIDS[f]["rho"] for f in prob.fuels]
    fdat, _, _, res = oracle_energy_residual(oracle, prob, prob.steps)
    pg, sg, sp = gpu_run(prob, prob.steps, mode=capi.PMP_MODE_MIXED)
    err, rel = energy_identity(prob, fdat, prob.parts, pg, sg, res, rho_l)
    print(f"mixed energy drift {err:.2e} of the exchange (FP64 scheme residual {rel:.2e})")
    assert abs(err) <= 1e-5
    sp.close()
