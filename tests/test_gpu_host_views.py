"""pmp_spray_update_host (host views; the copies overlap the update, in groups
of boxes) against pmp_spray_update (device views) on a B200.

Each droplet bit-identical after every call; deposits equal up to the order
of the atomic additions (1e-12 of the component's largest).  Cases: the FP64
form (several box groups, uneven and empty boxes), the mixed form, the PeleC
coupling, page-locked and pageable host memory, the FP64 form with a
non-default launch shape (copies, update and copy-back in sequence), and a
host source taken as zero on entry (not copied in, overwritten).
"""
import numpy as np
import pytest

from pelemp_b200 import capi
from pelemp_b200 import workloads as W
from tests.gpu_util import assert_bitwise, gpu_run, host_run
from tests.parity import source_errors

pytestmark = pytest.mark.gpu


def uneven(total=120_000):
    """32 boxes of 16^3 with capped-Zipf counts; boxes 3 and 17 emptied."""
    prob = W.config3(total=total, steps=2, nbox_xyz=(4, 4, 2), box=16)
    nr = prob.parts[0]["rdata"].shape[0]
    for b in (3, 17):
        prob.parts[b] = dict(pos=np.zeros((3, 0)), rdata=np.zeros((nr, 0)),
                             id=np.zeros(0, dtype=np.int32))
    return prob


def compare(prob, mode=capi.PMP_MODE_FP64, setup=None, pinned=True, host_setup=None, src_fill=0.0):
    pd, sd, _ = gpu_run(prob, prob.steps, mode=mode, setup=setup)
    ph, sh, sp = host_run(prob, prob.steps, mode=mode, setup=host_setup or setup, pinned=pinned,
                          src_fill=src_fill)
    assert_bitwise(pd, ph)
    for a, b in zip(sd, sh):
        assert source_errors(b, a) <= 1e-12
    assert sp.stats().substeps > 0
    return sp


@pytest.mark.parametrize("mode", [capi.PMP_MODE_FP64, capi.PMP_MODE_MIXED])
def test_host_views_uneven_boxes(mode):
    compare(uneven(), mode)


def test_host_views_config2_pageable():
    prob = W.config2(n=60_000, steps=2, ncells=(32, 32, 32), box=(16, 16, 16))
    compare(prob, capi.PMP_MODE_MIXED, pinned=False)


def test_host_views_pelec():
    from oracle.pyoracle import Oracle
    lm = W.config2(n=40_000, steps=2, ncells=(32, 32, 32), box=(16, 16, 16))
    compare(W.to_pelec(lm, Oracle(pelec=True).mech(lm.species)))


def test_host_views_sequential_launch_shape():
    def persistent(sp):
        sp.set_launch(kind=capi.PMP_LAUNCH_PERSISTENT, block=128, regs=96, chunk=512)
    compare(uneven(60_000), setup=persistent)


@pytest.mark.parametrize("mode", [capi.PMP_MODE_FP64, capi.PMP_MODE_MIXED])
def test_host_source_taken_as_zero(mode):
    """set_host_source_in(False): the host source is not copied in, the call
    writes the deposits over it.  Host sources pre-filled with 3.0 end equal
    to the device-view update's deposits into zeroed sources."""
    def no_copy_in(sp):
        sp.set_host_source_in(False)
    compare(uneven(60_000), mode, host_setup=no_copy_in, src_fill=3.0)


def test_host_views_copy_only_the_components_used():
    """The host-view update copies the state components the update reads and
    the source components it deposits into: an unread state component may hold
    NaN, and an extra source component keeps its host value."""
    import torch
    from pelemp_b200.spray import from_problem, views
    prob = W.config1(n=20_000, steps=1)
    pd, sd, _ = gpu_run(prob, 1)
    ns = prob.nspec
    st_h = []
    for s in prob.state:
        a = torch.from_numpy(s.copy()).pin_memory().numpy()
        a[4 + ns] = np.nan  # rhoH: not read in the PeleLMeX coupling
        st_h.append(a)
    sp = from_problem(prob)
    st_v = views(st_h, [prob.grown(b, prob.state_ghosts)[0] for b in range(len(prob.boxes))])
    srcs = []
    for do_move in (1, 0):
        src = []
        for s in prob.new_sources():
            a = torch.zeros((s.shape[0] + 1,) + s.shape[1:], dtype=torch.float64).pin_memory().numpy()
            a[-1] = 7.0
            src.append(a)
        src_v = views(src, [prob.grown(b, prob.source_ghosts)[0] for b in range(len(prob.boxes))])
        sp.update_particles_host(st_v, src_v, prob.flow_dt, 0.0, prob.state_ghosts, prob.source_ghosts,
                                 0, 0, do_move, prob.spray_cfl_lev, torch.cuda.current_stream().cuda_stream)
        for a in src:
            assert np.all(a[-1] == 7.0)
        srcs.append([a[:-1].copy() for a in src])
    ph = [sp.get_particles(b) for b in range(len(prob.boxes))]
    assert_bitwise(pd, ph)
    for a, b in zip(sd, srcs):
        assert source_errors(b, a) <= 1e-12
