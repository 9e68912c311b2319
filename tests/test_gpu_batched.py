"""Batched form: launch shapes, CUDA-graph replay and the autotuner on the
config-3 workload (many boxes, capped-Zipf droplet counts), scaled down.

* every launch shape (grid / persistent, 64-256 threads, 96 or 128
  registers, one launch per box) gives droplets bit-identical to the default
  launch, and deposits within 1e-12 of each component's largest (only the
  order of the atomic additions differs);
* an update replayed from a captured CUDA graph gives the same droplets as
  direct launches, and alternating MKD / MK calls both replay;
* the autotuner times every candidate, leaves droplets and the caller's
  source untouched, and a second handle reads its choice back from the
  cache file;
* one launch for all boxes beats one launch per box.
"""
import os

import numpy as np
import pytest

from pelemp_b200 import capi
from pelemp_b200 import workloads as W
from pelemp_b200.spray import from_problem
from tests.gpu_util import assert_bitwise, device_sources, device_state, gpu_run

pytestmark = pytest.mark.gpu

SHAPES = [
    dict(kind=capi.PMP_LAUNCH_GRID, block=64, regs=96),
    dict(kind=capi.PMP_LAUNCH_GRID, block=128, regs=128),
    dict(kind=capi.PMP_LAUNCH_GRID, block=256, regs=128),
    dict(kind=capi.PMP_LAUNCH_PERSISTENT, block=128, regs=96, chunk=128),
    dict(kind=capi.PMP_LAUNCH_PERSISTENT, block=128, regs=96, chunk=2048),
    dict(kind=capi.PMP_LAUNCH_PERSISTENT, block=64, regs=96, chunk=512, ctas_per_sm=3),
    dict(kind=capi.PMP_LAUNCH_PERSISTENT, block=256, regs=128, chunk=1024),
    dict(kind=capi.PMP_LAUNCH_PER_BOX, block=128, regs=96),
]


def small_config3(total=150_000):
    return W.config3(total=total, steps=2, nbox_xyz=(4, 4, 4), box=16)


def close_sources(sa, sb, tol=1e-12):
    for a, b in zip(sa, sb):
        for x, y in zip(a, b):
            for c in range(x.shape[0]):
                scale = np.max(np.abs(y[c]))
                assert np.max(np.abs(x[c] - y[c])) <= tol * max(scale, 1e-300), c


@pytest.fixture(scope="module")
def reference_run():
    prob = small_config3()
    pg, sg, _ = gpu_run(prob, prob.steps)
    return prob, pg, sg


@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: "%d-%d-%d-%d" % (
    s["kind"], s["block"], s["regs"], s.get("chunk", 0)))
def test_launch_shape_matches_default(shape, reference_run):
    prob, p_ref, s_ref = reference_run
    pg, sg, sp = gpu_run(prob, prob.steps, setup=lambda s: s.set_launch(**shape))
    cfg = sp.launch()
    assert (cfg.kind, cfg.block, cfg.regs) == (shape["kind"], shape["block"], shape["regs"])
    assert_bitwise(pg, p_ref)
    close_sources(sg, s_ref)


def _run_same_buffers(prob, steps, setup):
    """MKD + MK steps with the same state and source buffers every call."""
    import torch
    sp = from_problem(prob)
    setup(sp)
    st_keep, st_v = device_state(prob)
    src, src_v = device_sources(prob)
    stream = torch.cuda.current_stream().cuda_stream
    graph_states, sources = [], []
    for _ in range(steps):
        for do_move in (1, 0):
            for s in src:
                s.zero_()
            sp.update_particles(st_v, src_v, prob.flow_dt, 0.0, prob.state_ghosts, prob.source_ghosts,
                                0, 0, do_move, prob.spray_cfl_lev, stream)
            graph_states.append(sp.stats().graph)
            sources.append([s.cpu().numpy() for s in src])
    parts = [sp.get_particles(b) for b in range(len(prob.boxes))]
    del st_keep
    return parts, sources, graph_states


@pytest.mark.parametrize("shape", [dict(), dict(kind=capi.PMP_LAUNCH_PERSISTENT, block=128, regs=96,
                                                chunk=512)], ids=["grid", "persistent"])
def test_graph_replay(shape):
    prob = W.config3(total=100_000, steps=3, nbox_xyz=(4, 4, 2), box=16)
    p0, s0, g0 = _run_same_buffers(prob, 3, lambda sp: sp.set_launch(**shape))
    p1, s1, g1 = _run_same_buffers(prob, 3, lambda sp: sp.set_launch(use_graph=True, **shape))
    assert g0 == [0] * 6
    # the MKD and MK calls are captured once each, then replayed
    assert g1 == [2, 2, 1, 1, 1, 1]
    assert_bitwise(p1, p0)
    close_sources(s1, s0)


def test_autotune_and_cache(tmp_path):
    import torch
    prob = small_config3()
    cache = str(tmp_path / "tune.txt")
    sp = from_problem(prob)
    st_keep, st_v = device_state(prob)
    src, src_v = device_sources(prob)
    for s in src:
        s.fill_(1.5)
    before = [sp.get_particles(b) for b in range(len(prob.boxes))]
    stream = torch.cuda.current_stream().cuda_stream
    rep = sp.autotune(st_v, src_v, prob.flow_dt, prob.state_ghosts, prob.source_ghosts, 0, 1,
                      prob.spray_cfl_lev, cache_path=cache, stream=stream)
    print("autotune: candidates %d best %.3f ms (kind %d block %d regs %d chunk %d) default %.3f ms "
          "per-box %.3f ms" % (rep.ncandidates, rep.best_ms, rep.best.kind, rep.best.block, rep.best.regs,
                               rep.best.chunk, rep.default_ms, rep.per_box_ms))
    assert rep.cached == 0 and rep.ncandidates == 10
    assert 0 < rep.best_ms <= rep.default_ms
    assert rep.per_box_ms > 0
    cfg = sp.launch()
    assert (cfg.kind, cfg.block, cfg.regs, cfg.chunk) == (rep.best.kind, rep.best.block, rep.best.regs,
                                                          rep.best.chunk)
    after = [sp.get_particles(b) for b in range(len(prob.boxes))]
    assert_bitwise(after, before)
    for s in src:
        assert torch.all(s == 1.5)
    assert os.path.exists(cache)
    sp2 = from_problem(prob)
    rep2 = sp2.autotune(st_v, src_v, prob.flow_dt, prob.state_ghosts, prob.source_ghosts, 0, 1,
                        prob.spray_cfl_lev, cache_path=cache, stream=stream)
    assert rep2.cached == 1
    assert (rep2.best.kind, rep2.best.block, rep2.best.regs, rep2.best.chunk) == (
        rep.best.kind, rep.best.block, rep.best.regs, rep.best.chunk)
    del st_keep


def test_one_launch_beats_per_box():
    import torch
    prob = W.config3(total=2_000_000, steps=1, nbox_xyz=(8, 8, 4), box=16)
    times = {}
    for kind in (capi.PMP_LAUNCH_GRID, capi.PMP_LAUNCH_PER_BOX):
        sp = from_problem(prob)
        sp.set_launch(kind=kind)
        st_keep, st_v = device_state(prob)
        src, src_v = device_sources(prob)
        stream = torch.cuda.current_stream().cuda_stream
        ms = []
        for _ in range(3):
            sp.update_particles(st_v, src_v, prob.flow_dt, 0.0, prob.state_ghosts, prob.source_ghosts,
                                0, 0, 0, prob.spray_cfl_lev, stream)
            ms.append(sp.stats().kernel_ms)
        times[kind] = min(ms)
        del st_keep
        sp.close()
    print("256 boxes, 2M droplets: one launch %.3f ms, per box %.3f ms" % (
        times[capi.PMP_LAUNCH_GRID], times[capi.PMP_LAUNCH_PER_BOX]))
    assert times[capi.PMP_LAUNCH_GRID] < times[capi.PMP_LAUNCH_PER_BOX]
