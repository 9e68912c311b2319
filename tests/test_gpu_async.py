"""Stream-ordered updates through the C ABI, on a B200.

pmp_spray_update enqueues and returns; pmp_spray_sync waits, reports the
first device error of the calls since the previous sync and their summed
counters.  These tests check that
* steps enqueued without any host wait give the same droplets (bit for bit)
  and deposits as the oracle;
* a whole MKD+MK step captured by the caller into one CUDA graph and replayed
  gives the same droplets as eager steps;
* a device error surfaces at pmp_spray_sync with the reference's box and
  droplet, and at the next update call once the failing call has finished;
  calls enqueued after the failing one leave the droplets untouched until the
  error has been reported, and the handle runs again afterwards.
"""
import numpy as np
import pytest

from pelemp_b200 import capi
from pelemp_b200 import workloads as W
from pelemp_b200.spray import SprayError, from_problem
from tests.gpu_util import assert_bitwise, device_sources, device_state, oracle_run
from tests.parity import source_errors

pytestmark = pytest.mark.gpu


def _async_steps(prob, steps, mode=capi.PMP_MODE_FP64):
    """steps x (MKD + MK), each call's deposits into its own source arrays,
    no host wait until the end."""
    import torch
    sp = from_problem(prob, mode=mode)
    st_keep, st_v = device_state(prob)
    stream = torch.cuda.current_stream().cuda_stream
    keep = []
    for _ in range(steps):
        for do_move in (1, 0):
            src, src_v = device_sources(prob)
            keep.append(src)
            sp.update_particles(st_v, src_v, prob.flow_dt, 0.0, prob.state_ghosts, prob.source_ghosts,
                                0, 0, do_move, prob.spray_cfl_lev, stream, sync=False)
    sp.sync()
    srcs = [[s.cpu().numpy() for s in call] for call in keep]
    parts = [sp.get_particles(b) for b in range(len(prob.boxes))]
    del st_keep
    return parts, srcs, sp


def test_enqueued_steps_match_oracle(oracle):
    prob = W.config2(n=20_000, steps=3, ncells=(32, 32, 32), box=(16, 16, 16))
    pg, sg, sp = _async_steps(prob, prob.steps)
    # counters summed over the 6 calls since the previous sync
    assert sp.stats().substeps > 0
    po, so = oracle_run(oracle, prob, prob.steps)
    assert_bitwise(pg, po)
    for a, b in zip(sg, so):
        assert source_errors(a, b) <= 1e-12
    sp.close()


@pytest.mark.parametrize("mode", [capi.PMP_MODE_FP64, capi.PMP_MODE_MIXED])
def test_captured_step_graph_matches_eager(mode):
    """One CUDA graph of a whole step (zero the sources, MKD, MK), captured by
    the caller after one eager step, replayed: the same droplets as eager steps."""
    import torch
    prob = W.config2(n=20_000, steps=4, ncells=(32, 32, 32), box=(16, 16, 16))
    st_keep, st_v = device_state(prob)
    src, src_v = device_sources(prob)

    def step(sp, stream):
        for s in src:
            s.zero_()
        for do_move in (1, 0):
            sp.update_particles(st_v, src_v, prob.flow_dt, 0.0, prob.state_ghosts, prob.source_ghosts,
                                0, 0, do_move, prob.spray_cfl_lev, stream, sync=False)

    eager = from_problem(prob, mode=mode)
    for _ in range(prob.steps):
        step(eager, torch.cuda.current_stream().cuda_stream)
    eager.sync()
    pe = [eager.get_particles(b) for b in range(len(prob.boxes))]
    se = [s.cpu().numpy() for s in src]
    n_eager = eager.stats().substeps

    sp = from_problem(prob, mode=mode)
    step(sp, torch.cuda.current_stream().cuda_stream)  # outside the capture first
    sp.sync()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        step(sp, torch.cuda.current_stream().cuda_stream)
    for _ in range(prob.steps - 1):
        g.replay()
    torch.cuda.synchronize()
    sp.sync()
    # the replays' counters accumulate in the handle's status
    assert sp.stats().substeps > 0
    pgr = [sp.get_particles(b) for b in range(len(prob.boxes))]
    assert_bitwise(pgr, pe)
    assert source_errors([s.cpu().numpy() for s in src], se) <= 1e-12
    del g
    assert n_eager > 0
    sp.close()
    eager.close()
    del st_keep


def test_device_error_reported_by_sync_and_next_call():
    import torch
    prob = W.walls(n=500)
    prob.parts[0]["pos"][2, 7] = -0.5 * prob.dx[2]  # outside a non-periodic face
    sp = from_problem(prob)
    st_keep, st_v = device_state(prob)
    src, src_v = device_sources(prob)
    stream = torch.cuda.current_stream().cuda_stream
    args = (st_v, src_v, prob.flow_dt, 0.0, prob.state_ghosts, prob.source_ghosts, 0, 0, 1,
            prob.spray_cfl_lev, stream)
    # enqueued: no error yet
    sp.update_particles(*args, sync=False)
    torch.cuda.synchronize()
    # the failing call has finished: the next call reports its error at once
    with pytest.raises(SprayError) as e:
        sp.update_particles(*args, sync=False)
    assert e.value.code == capi.PMP_ERR_LEFT_DOMAIN
    assert e.value.info.box == 0 and e.value.info.particle == 7
    # reported once: the next sync is clean
    sp.sync()

    # a failing call A with a call B enqueued behind it before A runs: B
    # leaves the droplets as A left them, and sync reports A's error.  Both
    # handles first take one reported failing call (a handle's first call
    # allocates its buffers, which waits for the device); then the GPU is
    # held busy so that A and B are both enqueued before A runs.
    def failed_once(h):
        with pytest.raises(SprayError):
            h.update_particles(*args)

    ref = from_problem(prob)
    failed_once(ref)
    with pytest.raises(SprayError):
        ref.update_particles(*args)  # A alone
    want = [ref.get_particles(b) for b in range(len(prob.boxes))]
    sp2 = from_problem(prob)
    failed_once(sp2)
    torch.cuda._sleep(200_000_000)
    sp2.update_particles(*args, sync=False)  # A
    sp2.update_particles(*args, sync=False)  # B
    with pytest.raises(SprayError) as e2:
        sp2.sync()
    assert e2.value.code == capi.PMP_ERR_LEFT_DOMAIN
    assert e2.value.info.box == 0 and e2.value.info.particle == 7
    after = [sp2.get_particles(b) for b in range(len(prob.boxes))]
    assert_bitwise(after, want)
    sp.close()
    ref.close()
    sp2.close()
    del st_keep


def test_handle_runs_after_reported_error(oracle):
    """After an error has been reported, the handle's next calls run: the
    droplets given again by set_particles step like the oracle's."""
    import torch
    prob = W.walls(n=500)
    bad = W.walls(n=500)
    bad.parts[0]["pos"][2, 7] = -0.5 * bad.dx[2]
    sp = from_problem(bad)
    st_keep, st_v = device_state(prob)
    src, src_v = device_sources(prob)
    stream = torch.cuda.current_stream().cuda_stream
    with pytest.raises(SprayError):
        sp.update_particles(st_v, src_v, prob.flow_dt, 0.0, prob.state_ghosts, prob.source_ghosts,
                            0, 0, 1, prob.spray_cfl_lev, stream)
    for b, p in enumerate(prob.parts):
        sp.set_particles(b, p["pos"], p["rdata"], p["id"])
    for do_move in (1, 0):
        for s in src:
            s.zero_()
        sp.update_particles(st_v, src_v, prob.flow_dt, 0.0, prob.state_ghosts, prob.source_ghosts,
                            0, 0, do_move, prob.spray_cfl_lev, stream)
    po, _ = oracle_run(oracle, prob, 1)
    assert_bitwise([sp.get_particles(b) for b in range(len(prob.boxes))], po)
    sp.close()
    del st_keep


def test_host_views_enqueued(oracle):
    """pmp_spray_update_host without a host wait between calls: each call's
    copies are ordered after the previous call's copy-back."""
    import torch
    from pelemp_b200.spray import views
    prob = W.config2(n=20_000, steps=2, ncells=(32, 32, 32), box=(16, 16, 16))
    sp = from_problem(prob, mode=capi.PMP_MODE_FP64)

    def pinned(a):
        return torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()

    st_h = [pinned(s) for s in prob.state]
    st_v = views(st_h, [prob.grown(b, prob.state_ghosts)[0] for b in range(len(prob.boxes))])
    src_h = [pinned(s) for s in prob.new_sources()]
    src_v = views(src_h, [prob.grown(b, prob.source_ghosts)[0] for b in range(len(prob.boxes))])
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(prob.steps):
        for do_move in (1, 0):
            sp.update_particles_host(st_v, src_v, prob.flow_dt, 0.0, prob.state_ghosts, prob.source_ghosts,
                                     0, 0, do_move, prob.spray_cfl_lev, stream, sync=False)
    sp.sync()
    po, so = oracle_run(oracle, prob, prob.steps)
    assert_bitwise([sp.get_particles(b) for b in range(len(prob.boxes))], po)
    # the host sources accumulated every call's deposits
    total = [sum(call[b] for call in so) for b in range(len(prob.boxes))]
    assert source_errors(src_h, total) <= 1e-12
    sp.close()
