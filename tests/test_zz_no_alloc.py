"""pmp_spray_update_static: the update for callers that cannot allocate device
memory while it runs (their device memory is all in their own pre-sized pool,
or their solver forbids device allocations after initialisation).  The entry
point takes the caller's own device arrays and keeps
its working data in a fixed array inside the library.

Checked here through the C ABI against pmp_spray_update on the same inputs,
over two calls in a row (MKD then MK): every droplet's state bit-identical,
deposits within 1e-12 of the component's largest deposit (atomic ordering);
on the two-fuel slice, the walled domain, ghost droplets and the single-fuel
mechanism.  The call is synchronous, so a stream capture is refused.
This file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

from pelemp_b200 import capi
from pelemp_b200 import spray
from pelemp_b200 import workloads as W
from tests.gpu_util import assert_bitwise, gpu_run
from tests.parity import source_errors

pytestmark = pytest.mark.gpu


def _bind():
    f = spray.lib().pmp_spray_update_static
    f.restype = C.c_int
    f.argtypes = [C.POINTER(capi.SprayConfig), C.POINTER(capi.SprayData),
                  C.POINTER(capi.SprayComps), C.POINTER(capi.Geometry), C.c_int,
                  C.POINTER(capi.Box), C.POINTER(capi.Particles), C.POINTER(capi.BoxView),
                  C.POINTER(capi.BoxView), C.c_double, C.c_double, C.c_int, C.c_int, C.c_int,
                  C.c_int, C.c_int, C.c_double, C.c_void_p, C.POINTER(capi.ErrorInfo)]
    return f


def _config(prob):
    cfg = capi.SprayConfig()
    cfg.nfuel = prob.nfuel
    cfg.nspec = prob.nspec
    for i, s in enumerate(prob.species):
        cfg.species[i].value = s.encode()
    return cfg


def _static_two_calls(prob, is_ghost=0):
    """MKD then MK through pmp_spray_update_static on device copies of the
    problem's droplets; returns (droplets per box, sources per call)."""
    import torch
    f = _bind()
    nb = len(prob.boxes)
    handle = spray.from_problem(prob)
    data = handle.spray_data()
    handle.close()
    dev_parts = [{k: torch.from_numpy(v.copy()).cuda() for k, v in p.items()} for p in prob.parts]
    parts = (capi.Particles * nb)()
    for b, p in enumerate(dev_parts):
        parts[b].layout = capi.PMP_LAYOUT_SOA
        parts[b].where = capi.PMP_WHERE_DEVICE
        parts[b].n = p["id"].shape[0]
        for d in range(3):
            parts[b].pos[d] = p["pos"][d].data_ptr()
        for r in range(p["rdata"].shape[0]):
            parts[b].rdata[r] = p["rdata"][r].data_ptr()
        parts[b].id = p["id"].data_ptr()
    st = [torch.from_numpy(s).cuda() for s in prob.state]
    st_v = spray.views(st, [prob.grown(b, prob.state_ghosts)[0] for b in range(nb)])
    stream = torch.cuda.current_stream().cuda_stream
    srcs = []
    for do_move in (1, 0):
        src = [torch.zeros(s.shape, dtype=torch.float64, device="cuda") for s in prob.new_sources()]
        src_v = spray.views(src, [prob.grown(b, prob.source_ghosts)[0] for b in range(nb)])
        err = capi.ErrorInfo()
        rc = f(C.byref(_config(prob)), C.byref(data), C.byref(prob.comps()),
               C.byref(prob.geometry()), nb, prob.box_array(), parts, st_v, src_v,
               prob.flow_dt, 0.0, prob.state_ghosts, prob.source_ghosts, 0, is_ghost, do_move,
               prob.spray_cfl_lev, C.c_void_p(stream), C.byref(err))
        assert rc == capi.PMP_OK, err.message
        srcs.append([s.cpu().numpy() for s in src])
    got = [{k: v.cpu().numpy() for k, v in p.items()} for p in dev_parts]
    return got, srcs


def test_static_entry_matches_update_on_two_calls():
    prob = W.config2(n=30_000, steps=1, ncells=(32, 32, 32), box=(16, 16, 16))
    ref_parts, ref_srcs, handle = gpu_run(prob, 1)
    handle.close()
    got, srcs = _static_two_calls(prob)
    assert_bitwise(ref_parts, got)
    for a, b in zip(ref_srcs, srcs):
        assert source_errors(a, b) <= 1e-12


@pytest.mark.parametrize("case", ["walls", "ghost", "config1"])
def test_static_entry_matches_update_other_cases(case):
    """Reflective / outflow walls (bounds checks and impose_wall), ghost
    droplets (deposits into the grown source view, killed on leaving the
    source box) and the single-fuel, 3-species mechanism."""
    is_ghost = 1 if case == "ghost" else 0
    prob = {"walls": lambda: W.walls(n=6000),
            "ghost": lambda: W.config1(n=20_000, steps=1),
            "config1": lambda: W.config1(n=20_000, steps=1)}[case]()
    ref_parts, ref_srcs, handle = gpu_run(prob, 1, is_ghost=is_ghost)
    handle.close()
    got, srcs = _static_two_calls(prob, is_ghost=is_ghost)
    assert_bitwise(ref_parts, got)
    for a, b in zip(ref_srcs, srcs):
        assert source_errors(a, b) <= 1e-12


def test_static_entry_refuses_stream_capture():
    """The entry point is synchronous: under an active capture it refuses."""
    import torch
    prob = W.config1(n=100, steps=1)
    f = _bind()
    handle = spray.from_problem(prob)
    data = handle.spray_data()
    handle.close()
    nb = len(prob.boxes)
    parts = (capi.Particles * nb)()
    st = [torch.from_numpy(s).cuda() for s in prob.state]
    st_v = spray.views(st, [prob.grown(b, prob.state_ghosts)[0] for b in range(nb)])
    src = [torch.zeros(s.shape, dtype=torch.float64, device="cuda") for s in prob.new_sources()]
    src_v = spray.views(src, [prob.grown(b, prob.source_ghosts)[0] for b in range(nb)])
    err = capi.ErrorInfo()
    g = torch.cuda.CUDAGraph()
    rc = None
    with torch.cuda.graph(g):
        src[0].zero_()
        rc = f(C.byref(_config(prob)), C.byref(data), C.byref(prob.comps()), C.byref(prob.geometry()),
               nb, prob.box_array(), parts, st_v, src_v, prob.flow_dt, 0.0, prob.state_ghosts,
               prob.source_ghosts, 0, 0, 1, prob.spray_cfl_lev,
               C.c_void_p(torch.cuda.current_stream().cuda_stream), C.byref(err))
    assert rc == capi.PMP_ERR_INVALID
    assert b"captured" in err.message
    del g


def test_static_entry_rejects_too_many_boxes():
    prob = W.config1(n=10, steps=1)
    f = _bind()
    n = capi_max = 257
    boxes = (capi.Box * n)()
    parts = (capi.Particles * n)()
    views = (capi.BoxView * n)()
    src = (capi.BoxView * n)()
    err = capi.ErrorInfo()
    import torch
    data = capi.SprayData()
    data.nfuel = 1
    rc = f(C.byref(_config(prob)), C.byref(data), C.byref(prob.comps()), C.byref(prob.geometry()),
           capi_max, boxes, parts, views, src, prob.flow_dt, 0.0, 3, 2, 0, 0, 1, 0.1,
           C.c_void_p(torch.cuda.current_stream().cuda_stream), C.byref(err))
    assert rc == capi.PMP_ERR_INVALID
    assert b"at most" in err.message
