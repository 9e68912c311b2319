"""Properties of the CPU oracle of the operations around the update
(oracle/mesh_oracle.py), without a GPU: the periodic ghost fold conserves
the total, re-binning keeps every live droplet exactly once inside the
domain, and the time-step estimate follows its definition."""
import numpy as np

from oracle import mesh_oracle as MO
from pelemp_b200 import workloads as W


def test_fold_conserves_total_on_a_periodic_domain():
    prob = W.config2(n=2000, steps=1, ncells=(16, 16, 16), box=(8, 8, 8))
    rng = np.random.default_rng(0)
    g = prob.source_ghosts
    nb = len(prob.boxes)
    tmp_lo = [prob.grown(b, g)[0] for b in range(nb)]
    tmp = [rng.standard_normal(s.shape) for s in prob.new_sources()]
    total = sum(float(t.sum()) for t in tmp)
    act = [np.zeros_like(t) for t in tmp]
    MO.transfer_source(tmp, tmp_lo, act, tmp_lo, prob.boxes, prob.domain_lo, prob.domain_hi, [True] * 3, g, 0)
    # every ghost cell of a periodic domain lands in some valid cell
    assert abs(sum(float(a.sum()) for a in act) - total) < 1e-9 * sum(float(np.abs(t).sum()) for t in act) + 1e-9
    assert all(np.all(t == 0.0) for t in tmp)


def test_redistribute_keeps_live_droplets_once():
    prob = W.config2(n=5000, steps=1, ncells=(16, 16, 16), box=(8, 8, 8))
    rng = np.random.default_rng(1)
    L = prob.phi - prob.plo
    for p in prob.parts:
        p["pos"] += (rng.random(p["pos"].shape) - 0.5) * 2.5 * L[:, None]
        p["id"][::50] = -1
    live = sorted(int(i) for p in prob.parts for i in p["id"] if i > 0)
    out = MO.redistribute(prob.parts, prob.boxes, prob.plo, prob.phi, prob.dx, prob.domain_lo,
                          prob.domain_hi, [True] * 3)
    got = sorted(int(i) for p in out for i in p["id"])
    assert got == live
    for b, p in enumerate(out):
        lo, hi = prob.boxes[b]
        c = MO.cells_of(p["pos"], prob.plo, prob.dx)
        assert np.all((c >= np.asarray(lo)[:, None]) & (c <= np.asarray(hi)[:, None]))
        assert np.all((p["pos"] >= prob.plo[:, None]) & (p["pos"] < prob.phi[:, None]))


def test_est_timestep_definition():
    prob = W.config1(n=100, steps=1)
    p = prob.parts[0]
    v = np.abs(p["rdata"][0:3]) * (1.0 / prob.dx)[:, None]
    assert MO.est_timestep(prob.parts, prob.dx, 0.5) == float(np.min(0.5 / v.max(axis=0)))
    assert MO.est_timestep(prob.parts, prob.dx, 0.5, fixed_parts=True) == -1.0
