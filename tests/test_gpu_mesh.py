"""The operations on either side of the update against the numpy oracle
(oracle/mesh_oracle.py):

* estTimestep: bit-identical (a min reduction), including the reference's -1
  for a dead droplet still held and the injection-jet bound;
* computeDerivedVars: every field within 1e-12 of its component's largest
  value (atomic deposits reorder sums), ghost cells included;
* transferSource: the periodic ghost fold, the add (same component count
  and addSpraySrc's mapping) and the reset, within 1e-12;
* redistribute: per box, the same droplets (by id) bit for bit, periodic
  wraps included, dead and out-of-domain droplets dropped; droplets of each
  box in cell order afterwards; a following update still runs.
"""
import numpy as np
import pytest

from oracle import mesh_oracle as MO
from pelemp_b200 import capi
from pelemp_b200 import workloads as W
from pelemp_b200.spray import from_problem, views
from tests.gpu_util import device_sources, device_state

pytestmark = pytest.mark.gpu

SMALL2 = dict(n=60_000, steps=1, ncells=(32, 32, 32), box=(16, 16, 16))


def rel_close(a, b, tol=1e-12):
    for x, y in zip(a, b):
        for c in range(x.shape[0]):
            scale = max(float(np.max(np.abs(y[c]))), 1e-300)
            assert float(np.max(np.abs(x[c] - y[c]))) <= tol * scale, c


def test_est_timestep():
    prob = W.config2(**SMALL2)
    prob.parts[3]["rdata"][0:3, 7] = 0.0  # a droplet at rest: 1e50
    sp = from_problem(prob)
    dt = sp.est_timestep(0.5)
    assert dt == MO.est_timestep(prob.parts, prob.dx, 0.5)
    dtj = sp.est_timestep(0.5, max_jet_vel=2000.0)
    assert dtj == MO.est_timestep(prob.parts, prob.dx, 0.5, max_jet_vel=2000.0) == 0.5 * prob.dx[0] / 2000.0
    prob.parts[1]["id"][5] = -1  # a dead droplet still held
    sp2 = from_problem(prob)
    assert sp2.est_timestep(0.5) == -1.0 == MO.est_timestep(prob.parts, prob.dx, 0.5)


@pytest.mark.parametrize("species", [True, False])
def test_compute_derived_vars(species):
    import torch
    prob = W.config2(**SMALL2)
    p = prob.parts[2]
    p["rdata"][9 + prob.nfuel, ::11] = 3e-6  # some wall-film droplets
    sp = from_problem(prob)
    start = 2
    nvar = 15 + (prob.nfuel if species else 0)
    g = 1
    shapes = []
    for b in range(len(prob.boxes)):
        lo, hi = prob.grown(b, g)
        shapes.append((start + nvar,) + tuple(hi[d] - lo[d] + 1 for d in (2, 1, 0)))
    dev = [torch.zeros(s, dtype=torch.float64, device="cuda") for s in shapes]
    sp.compute_derived_vars(views(dev, [prob.grown(b, g)[0] for b in range(len(prob.boxes))]), start, species)
    got = [d.cpu().numpy() for d in dev]
    want = [np.zeros(s) for s in shapes]
    rho_coef = np.zeros(16)
    for f, name in enumerate(prob.fuels):
        rho_coef[4 * f] = W.LIQUIDS[name]["rho"]
    MO.derive(prob.parts, want, [prob.grown(b, g)[0] for b in range(len(prob.boxes))], start, prob.nfuel,
              species, rho_coef, prob.plo, prob.dx)
    assert np.all(got[0][:start] == 0.0)
    rel_close([x[start:] for x in got], [x[start:] for x in want])
    no_film = sum(int(np.sum(q["rdata"][9 + prob.nfuel] == 0.0)) for q in prob.parts)
    assert sum(float(np.sum(x[start + 11])) for x in got) == no_film


@pytest.mark.parametrize("case", ["config1-same", "config2-add"])
def test_transfer_source(case):
    import torch
    rng = np.random.default_rng(4)
    if case == "config1-same":
        prob = W.config1(n=1000, steps=1)
    else:
        prob = W.config2(**SMALL2)
    sp = from_problem(prob)
    g = prob.source_ghosts
    nb = len(prob.boxes)
    tmp_lo = [prob.grown(b, g)[0] for b in range(nb)]
    tmp = [rng.standard_normal(s.shape) for s in prob.new_sources()]
    act_g = 1
    act_lo = [prob.grown(b, act_g)[0] for b in range(nb)]
    nact = prob.n_src_comp if case == "config1-same" else prob.n_state_comp
    act = []
    for b in range(nb):
        lo, hi = prob.grown(b, act_g)
        act.append(rng.standard_normal((nact,) + tuple(hi[d] - lo[d] + 1 for d in (2, 1, 0))))
    d_tmp = [torch.from_numpy(t.copy()).cuda() for t in tmp]
    d_act = [torch.from_numpy(a.copy()).cuda() for a in act]
    sp.transfer_source(views(d_tmp, tmp_lo), views(d_act, act_lo), g, act_g)
    periodic = [prob.bndry_lo[d] == 0 for d in range(3)]
    dep = list(sp.spray_data().dep_indx)[:prob.nfuel]
    MO.transfer_source(tmp, tmp_lo, act, act_lo, prob.boxes, prob.domain_lo, prob.domain_hi, periodic, g, act_g,
                       comps=prob.comps(), nfuel=prob.nfuel, dep_indx=dep)
    for t in d_tmp:
        assert torch.all(t == 0.0)
    rel_close([a.cpu().numpy() for a in d_act], act)


def test_redistribute_then_update():
    import torch
    prob = W.config2(**SMALL2)
    rng = np.random.default_rng(9)
    L = prob.phi - prob.plo
    n_dead = 0
    for p in prob.parts:
        n = p["id"].shape[0]
        move = rng.random(n) < 0.3
        p["pos"][:, move] += (rng.random((3, int(move.sum()))) - 0.5) * 1.5 * L[:, None]
        dead = rng.random(n) < 0.02
        p["id"][dead] = -1
        n_dead += int(dead.sum())
    sp = from_problem(prob)
    before = [sp.get_particles(b) for b in range(len(prob.boxes))]
    periodic = [prob.bndry_lo[d] == 0 for d in range(3)]
    want = MO.redistribute(before, prob.boxes, prob.plo, prob.phi, prob.dx, prob.domain_lo, prob.domain_hi, periodic)
    removed = sp.redistribute()
    assert removed == n_dead
    for b in range(len(prob.boxes)):
        got = sp.get_particles(b)
        order = np.argsort(got["id"], kind="stable")
        for k in ("pos", "rdata", "id"):
            assert np.array_equal(got[k][..., order], want[b][k]), (b, k)
        c = MO.cells_of(got["pos"], prob.plo, prob.dx)
        lo, hi = prob.boxes[b]
        assert np.all((c >= np.asarray(lo)[:, None]) & (c <= np.asarray(hi)[:, None]))
        # cell order: x-fastest rows, or 2x2x2 bricks (bricks x fastest, cells
        # x fastest in a brick) when the library is built with PMP_SORT_BRICKS
        r = c - np.asarray(lo)[:, None]
        ex, ey = hi[0] - lo[0] + 1, hi[1] - lo[1] + 1
        rows = (r[2] * ey + r[1]) * ex + r[0]
        brick = ((r[2] // 2) * ((ey + 1) // 2) + r[1] // 2) * ((ex + 1) // 2) + r[0] // 2
        bricks = brick * 8 + ((r[2] % 2) * 2 + r[1] % 2) * 2 + r[0] % 2
        assert np.all(np.diff(rows) >= 0) or np.all(np.diff(bricks) >= 0)
    # the re-binned droplets go through an update (stencils inside their boxes)
    st_keep, st_v = device_state(prob)
    _src, src_v = device_sources(prob)
    sp.update_particles(st_v, src_v, prob.flow_dt, 0.0, prob.state_ghosts, prob.source_ghosts, 0, 0, 1,
                        prob.spray_cfl_lev, torch.cuda.current_stream().cuda_stream)
    assert sp.stats().substeps > 0
    assert sp.est_timestep(0.5) > 0.0
    del st_keep


def test_redistribute_repeated():
    """Re-binning several times in a row: the second call gathers into the
    store the first one left as its spare, the third runs after an update
    moved the droplets; every time the boxes hold what the oracle's
    re-binning of the droplets before the call gives."""
    import torch
    prob = W.config2(**SMALL2)
    rng = np.random.default_rng(11)
    L = prob.phi - prob.plo
    for p in prob.parts:
        n = p["id"].shape[0]
        move = rng.random(n) < 0.2
        p["pos"][:, move] += (rng.random((3, int(move.sum()))) - 0.5) * L[:, None]
        p["id"][rng.random(n) < 0.03] = -1
    sp = from_problem(prob)
    periodic = [prob.bndry_lo[d] == 0 for d in range(3)]
    st_keep, st_v = device_state(prob)
    for it in range(3):
        if it == 2:
            _src, src_v = device_sources(prob)
            sp.update_particles(st_v, src_v, prob.flow_dt, 0.0, prob.state_ghosts, prob.source_ghosts, 0, 0, 1,
                                prob.spray_cfl_lev, torch.cuda.current_stream().cuda_stream)
        cur = [sp.get_particles(b) for b in range(len(prob.boxes))]
        want = MO.redistribute(cur, prob.boxes, prob.plo, prob.phi, prob.dx, prob.domain_lo, prob.domain_hi,
                               periodic)
        removed = sp.redistribute()
        assert removed == sum(int(np.sum(p["id"] <= 0)) for p in cur)
        for b in range(len(prob.boxes)):
            got = sp.get_particles(b)
            order = np.argsort(got["id"], kind="stable")
            for k in ("pos", "rdata", "id"):
                assert np.array_equal(got[k][..., order], want[b][k]), (it, b, k)
    del st_keep
