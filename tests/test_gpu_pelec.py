"""The PeleC coupling against the CPU oracle, on a B200.

FP64 form: the same bar as the PeleLMeX coupling, every droplet
bit-identical to the oracle's after each call (the gas temperature found from
the energy by the same Newton iteration), mesh deposits within 1e-12 of the
largest deposit (order of the atomic additions only).  Mixed form: the
PeleLMeX mixed form's bounds (1e-4), droplets below 2 um (2e-4 cm) on the FP64
path bit-identical.
"""
import numpy as np
import pytest

from pelemp_b200 import capi
from pelemp_b200 import workloads as W
from pelemp_b200.spray import SprayError, SprayParticleContainer, from_problem
from oracle.pyoracle import Oracle
from tests.gpu_util import assert_bitwise, device_sources, device_state, gpu_run, oracle_run
from tests.parity import source_errors

pytestmark = pytest.mark.gpu

CASES = {
    "config1": dict(n=60_000, steps=2),
    "config2": dict(n=40_000, steps=2, ncells=(32, 32, 32), box=(16, 16, 16)),
    "walls": dict(n=8000),
}


@pytest.fixture(scope="module")
def oracle_pelec():
    return Oracle(pelec=True)


@pytest.mark.parametrize("name", list(CASES))
def test_pelec_fp64_bitwise_vs_oracle(name, oracle_pelec):
    lm = W.CONFIGS[name](**CASES[name])
    prob = W.to_pelec(lm, oracle_pelec.mech(lm.species))
    pg, sg, sp = gpu_run(prob, prob.steps)
    assert sp.coupling == capi.PMP_COUPLING_PELEC
    po, so = oracle_run(oracle_pelec, prob, prob.steps)
    assert_bitwise(pg, po)
    for a, b in zip(sg, so):
        assert source_errors(a, b) <= 1e-12


def test_pelec_rules(oracle_pelec):
    import torch
    lm = W.config1(n=2000, steps=1)
    prob = W.to_pelec(lm, oracle_pelec.mech(lm.species))
    # the coupling is fixed once the spray data is set
    sp = SprayParticleContainer(lm.species, lm.nfuel)
    sp.spray_setup(lm.inputs())
    with pytest.raises(SprayError) as e:
        sp.set_coupling(capi.PMP_COUPLING_PELEC)
    assert e.value.code == capi.PMP_ERR_INVALID
    sp.close()
    # the PeleC coupling runs the FP64 and mixed forms, not the learned one
    sp = from_problem(prob, mode=capi.PMP_MODE_LEARNED)
    st_keep, st_v = device_state(prob)
    src, src_v = device_sources(prob)
    with pytest.raises(SprayError) as e:
        sp.update_particles(st_v, src_v, prob.flow_dt, 0.0, prob.state_ghosts,
                            prob.source_ghosts, 0, 0, 1, prob.spray_cfl_lev,
                            torch.cuda.current_stream().cuda_stream)
    assert e.value.code == capi.PMP_ERR_UNSUPPORTED
    del st_keep, src


def test_pelec_mixed_vs_oracle(oracle_pelec):
    lm = W.config2(n=40_000, steps=3, ncells=(32, 32, 32), box=(16, 16, 16))
    prob = W.to_pelec(lm, oracle_pelec.mech(lm.species))
    small = []
    for p in prob.parts:
        idx = np.arange(0, p["id"].shape[0], 13)
        p["rdata"][capi.PSTATE_DIA, idx] = 1.5e-4  # 1.5 um in cm
        small.append(idx)
    pg, sg, sp = gpu_run(prob, prob.steps, mode=capi.PMP_MODE_MIXED)
    po, so = oracle_run(oracle_pelec, prob, prob.steps)
    worst = {"T": 0.0, "dia": 0.0, "vel": 0.0}
    for b, (a, o) in enumerate(zip(pg, po)):
        alive = (a["id"] > 0) & (o["id"] > 0)
        ra, ro = a["rdata"][:, alive], o["rdata"][:, alive]
        for key, row in (("T", capi.PSTATE_T), ("dia", capi.PSTATE_DIA)):
            worst[key] = max(worst[key], float(np.max(np.abs(ra[row] / ro[row] - 1))))
        spd = np.maximum(np.sqrt(np.sum(ro[0:3] ** 2, axis=0)), 100.0)  # cm/s
        worst["vel"] = max(worst["vel"], float(np.max(np.sqrt(np.sum((ra[0:3] - ro[0:3]) ** 2, axis=0)) / spd)))
        for k in ("pos", "rdata", "id"):
            assert np.array_equal(a[k][..., small[b]], o[k][..., small[b]]), (b, k)
    print("PeleC mixed vs FP64 oracle:", worst)
    assert max(worst.values()) <= 1e-4
    dep = 0.0
    for a, b in zip(sg, so):
        for x, y in zip(a, b):
            for c in range(x.shape[0]):
                scale = np.max(np.abs(y[c]))
                if scale > 0:
                    dep = max(dep, float(np.max(np.abs(x[c] - y[c])) / scale))
    print("PeleC mixed deposit error:", dep)
    assert dep <= 1e-4
