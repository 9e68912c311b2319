"""Helpers for the GPU tests: run a workloads.Problem through the C ABI."""
import numpy as np

from pelemp_b200 import capi
from pelemp_b200.spray import from_problem, views


def device_state(prob):
    import torch
    st = [torch.from_numpy(s).cuda() for s in prob.state]
    return st, views(st, [prob.grown(b, prob.state_ghosts)[0] for b in range(len(prob.boxes))])


def device_sources(prob):
    import torch
    src = [torch.zeros(s.shape, dtype=torch.float64, device="cuda") for s in prob.new_sources()]
    return src, views(src, [prob.grown(b, prob.source_ghosts)[0] for b in range(len(prob.boxes))])


def gpu_run(prob, steps, mode=capi.PMP_MODE_FP64, is_ghost=0, keep=None, setup=None):
    """steps x (MKD + MK) on the GPU; returns (parts per box, sources per call, container).

    setup(sp), if given, runs on the new container before the first update."""
    import torch
    sp = from_problem(prob, mode=mode)
    if setup is not None:
        setup(sp)
    st_keep, st_v = device_state(prob)  # keep the tensors alive while the views are used
    srcs = []
    for _step in range(steps):
        for do_move in (1, 0):
            src, src_v = device_sources(prob)
            sp.update_particles(st_v, src_v, prob.flow_dt, 0.0, prob.state_ghosts,
                                prob.source_ghosts, 0, is_ghost, do_move, prob.spray_cfl_lev,
                                torch.cuda.current_stream().cuda_stream)
            srcs.append([s.cpu().numpy() for s in src])
    parts = [sp.get_particles(b) for b in range(len(prob.boxes))]
    del st_keep
    return parts, srcs, sp


def host_run(prob, steps, mode=capi.PMP_MODE_FP64, setup=None, pinned=True, src_fill=0.0):
    """gpu_run through pmp_spray_update_host: state and sources in host memory
    (page-locked when pinned), the host sources filled with src_fill before
    each call."""
    import torch
    sp = from_problem(prob, mode=mode)
    if setup is not None:
        setup(sp)

    def host(a):
        t = torch.from_numpy(np.ascontiguousarray(a))
        return (t.pin_memory() if pinned else t.clone()).numpy()

    st_h = [host(s) for s in prob.state]
    st_v = views(st_h, [prob.grown(b, prob.state_ghosts)[0] for b in range(len(prob.boxes))])
    srcs = []
    for _step in range(steps):
        for do_move in (1, 0):
            src = [host(np.full_like(s, src_fill)) for s in prob.new_sources()]
            src_v = views(src, [prob.grown(b, prob.source_ghosts)[0] for b in range(len(prob.boxes))])
            sp.update_particles_host(st_v, src_v, prob.flow_dt, 0.0, prob.state_ghosts,
                                     prob.source_ghosts, 0, 0, do_move, prob.spray_cfl_lev,
                                     torch.cuda.current_stream().cuda_stream)
            srcs.append([s.copy() for s in src])
    parts = [sp.get_particles(b) for b in range(len(prob.boxes))]
    return parts, srcs, sp


def oracle_run(oracle, prob, steps, is_ghost=0):
    mech = oracle.mech(prob.species)
    rc, fdat = oracle.setup(prob, mech)
    assert rc == 0
    parts = prob.copy_parts()
    srcs = []
    for _ in range(steps):
        for do_move in (1, 0):
            src = prob.new_sources()
            rc, err, _ = oracle.update(prob, mech, fdat, parts, src, do_move, is_ghost=is_ghost)
            assert rc == 0, (rc, err.message)
            srcs.append(src)
    return parts, srcs


def assert_bitwise(pa, pb):
    for a, b in zip(pa, pb):
        for k in ("pos", "rdata", "id"):
            if not np.array_equal(a[k], b[k]):
                diff = np.nonzero(~np.all(a[k] == b[k], axis=0) if a[k].ndim > 1 else a[k] != b[k])[0]
                raise AssertionError(f"{k} differs at {diff[:10]} (of {diff.size})")


def oracle_energy_residual(oracle, prob, steps):
    """The oracle's run with the energy-identity residual of every parcel:
    returns (fdat, parts, sources per call, residual per box)."""
    mech = oracle.mech(prob.species)
    rc, fdat = oracle.setup(prob, mech)
    assert rc == 0
    parts = prob.copy_parts()
    res = [np.zeros(p["id"].size) for p in parts]
    srcs = []
    for _ in range(steps):
        for do_move in (1, 0):
            src = prob.new_sources()
            rc, err, _ = oracle.update_energy(prob, mech, fdat, parts, src, do_move, res)
            assert rc == 0, (rc, err.message)
            srcs.append(src)
    return fdat, parts, srcs, res
