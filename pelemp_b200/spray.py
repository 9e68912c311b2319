"""Python mirror of PeleMP's SprayParticleContainer update surface over the C ABI.

Method names follow the reference (Source/PP_Spray/SprayParticles.H:195-243,
SpraySetup.cpp:73-297): ``spray_setup`` (readSprayParams + spraySetup),
``assign_spray_comps``, ``update_particles``, ``move_kick_drift``,
``move_kick``.  Errors the reference reports with amrex::Abort raise
``SprayError`` carrying the library's status code.

The native library (pelemp_b200/libpmpspray.so, sm_100a) is required: there
is no CPU path behind this class.
"""
import ctypes as C
import os

import numpy as np

from . import capi
from .workloads import view_of

_LIB = None
_LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libpmpspray.so")

# exported C ABI functions and their argument types
_SIGS = {
    "pmp_spray_create": [C.POINTER(capi.SprayConfig), C.POINTER(C.c_void_p)],
    "pmp_spray_destroy": [C.c_void_p],
    "pmp_spray_setup": [C.c_void_p, C.POINTER(capi.SprayInputs)],
    "pmp_spray_set_data": [C.c_void_p, C.POINTER(capi.SprayData)],
    "pmp_spray_get_data": [C.c_void_p, C.POINTER(capi.SprayData)],
    "pmp_spray_set_comps": [C.c_void_p, C.POINTER(capi.SprayComps)],
    "pmp_spray_set_geometry": [C.c_void_p, C.POINTER(capi.Geometry)],
    "pmp_spray_set_grids": [C.c_void_p, C.c_int, C.POINTER(capi.Box)],
    "pmp_spray_set_particles": [C.c_void_p, C.c_int, C.POINTER(capi.Particles)],
    "pmp_spray_get_particles": [C.c_void_p, C.c_int, C.POINTER(capi.Particles)],
    "pmp_spray_num_particles": [C.c_void_p, C.c_int, C.POINTER(C.c_longlong)],
    "pmp_spray_update": [C.c_void_p, C.POINTER(capi.BoxView), C.POINTER(capi.BoxView), C.c_int,
                         C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                         C.c_double, C.c_void_p],
    "pmp_spray_update_host": [C.c_void_p, C.POINTER(capi.BoxView), C.POINTER(capi.BoxView),
                              C.c_int, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int,
                              C.c_int, C.c_int, C.c_double, C.c_void_p],
    "pmp_spray_move_kick_drift": [C.c_void_p, C.POINTER(capi.BoxView), C.POINTER(capi.BoxView),
                                  C.c_int, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int,
                                  C.c_int, C.c_int, C.c_double, C.c_void_p],
    "pmp_spray_move_kick": [C.c_void_p, C.POINTER(capi.BoxView), C.POINTER(capi.BoxView),
                            C.c_int, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int,
                            C.c_double, C.c_void_p],
    "pmp_spray_set_host_source_in": [C.c_void_p, C.c_int],
    "pmp_spray_set_mode": [C.c_void_p, C.c_int],
    "pmp_spray_set_coupling": [C.c_void_p, C.c_int],
    "pmp_spray_get_coupling": [C.c_void_p, C.POINTER(C.c_int)],
    "pmp_spray_sync": [C.c_void_p],
    "pmp_spray_last_error": [C.c_void_p, C.POINTER(capi.ErrorInfo)],
    "pmp_spray_get_stats": [C.c_void_p, C.POINTER(capi.Stats)],
    "pmp_spray_version": [],
    "pmp_spray_est_timestep": [C.c_void_p, C.c_double, C.c_double, C.POINTER(C.c_double), C.c_void_p],
    "pmp_spray_derive": [C.c_void_p, C.POINTER(capi.BoxView), C.c_int, C.c_int, C.c_int, C.c_void_p],
    "pmp_spray_transfer_source": [C.c_void_p, C.POINTER(capi.BoxView), C.POINTER(capi.BoxView), C.c_int,
                                  C.c_int, C.c_int, C.c_void_p],
    "pmp_spray_redistribute": [C.c_void_p, C.POINTER(C.c_longlong), C.c_void_p],
    "pmp_spray_set_launch": [C.c_void_p, C.POINTER(capi.LaunchConfig)],
    "pmp_spray_get_launch": [C.c_void_p, C.POINTER(capi.LaunchConfig)],
    "pmp_spray_autotune": [C.c_void_p, C.POINTER(capi.BoxView), C.POINTER(capi.BoxView), C.c_int,
                           C.c_double, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_char_p,
                           C.POINTER(capi.TuneReport), C.c_void_p],
    "pmp_spray_learn_generate": [C.c_void_p, C.POINTER(capi.BoxView), C.c_int, C.c_double, C.c_int,
                                 C.c_int, C.c_double, C.c_longlong, C.c_int, C.c_ulonglong,
                                 C.c_void_p],
    "pmp_spray_learn_count": [C.c_void_p, C.POINTER(C.c_longlong)],
    "pmp_spray_learn_tuples": [C.c_void_p, C.c_void_p, C.POINTER(C.c_longlong)],
    "pmp_spray_learn_train": [C.c_void_p, C.POINTER(capi.LearnConfig), C.POINTER(capi.LearnReport)],
    "pmp_spray_learn_weights": [C.c_void_p, C.c_int, C.c_void_p, C.POINTER(C.c_longlong)],
    "pmp_spray_learn_set_audit": [C.c_void_p, C.c_double],
    "pmp_spray_learn_audit": [C.c_void_p, C.POINTER(C.c_longlong), C.POINTER(C.c_double)],
    "pmp_learn_debug_grad": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p,
                             C.POINTER(C.c_double)],
    "pmp_learn_debug_infer": [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p],
    "pmp_learn_debug_infer_tc": [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p],
    "pmp_learn_debug_wait_timeout": [C.POINTER(C.c_longlong)],
    "pmp_learn_param_count": [],
    "pmp_learn_base_terms": [],
    "pmp_learn_debug_base": [C.c_void_p, C.c_float, C.c_float, C.c_void_p, C.c_void_p, C.POINTER(C.c_float)],
    "pmp_learn_debug_solve_baseline": [C.c_void_p, C.c_void_p],
    "pmp_measure_peaks": [C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double)],
}


class SprayError(RuntimeError):
    def __init__(self, code, info=None):
        self.code = code
        self.info = info
        msg = capi.STATUS_NAMES.get(code, str(code))
        if info is not None:
            msg += f" (box {info.box}, droplet {info.particle}: {info.message.decode(errors='replace')})"
        super().__init__(msg)


def lib():
    """Load libpmpspray.so (raises if it is not built)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(_LIB_PATH):
            raise RuntimeError(f"{_LIB_PATH} is not built: run `python -m pelemp_b200.build`")
        L = C.CDLL(_LIB_PATH)
        for name, args in _SIGS.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = C.c_char_p if name == "pmp_spray_version" else C.c_int
        _LIB = L
    return _LIB


def _ptr(a):
    """Data pointer of a numpy array or a torch tensor."""
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    return a.ctypes.data


def _is_cuda(a):
    return hasattr(a, "is_cuda") and a.is_cuda


def views(arrays, los):
    """pmp_box_view array of per-box (ncomp, nz, ny, nx) arrays (numpy or torch)."""
    out = (capi.BoxView * len(arrays))()
    for b, (a, lo) in enumerate(zip(arrays, los)):
        if hasattr(a, "data_ptr"):
            nc, nz, ny, nx = a.shape
            v = out[b]
            v.p = a.data_ptr()
            for d in range(3):
                v.lo[d] = int(lo[d])
            v.hi[0], v.hi[1], v.hi[2] = lo[0] + nx - 1, lo[1] + ny - 1, lo[2] + nz - 1
            st = a.stride()
            v.nstride, v.kstride, v.jstride = st[0], st[1], st[2]
            v.ncomp = nc
        else:
            out[b] = view_of(a, lo)
    return out


class SprayParticleContainer:
    """One level's spray droplets on one GPU (the reference's container, update path)."""

    def __init__(self, species, nfuel, device=0):
        L = lib()
        cfg = capi.SprayConfig()
        cfg.nfuel = nfuel
        cfg.nspec = len(species)
        for i, s in enumerate(species):
            cfg.species[i].value = s.encode()
        cfg.device = device
        h = C.c_void_p()
        rc = L.pmp_spray_create(C.byref(cfg), C.byref(h))
        if rc != 0:
            raise SprayError(rc)
        self._h = h
        self.species = list(species)
        self.nfuel = nfuel
        self.nboxes = 0

    def close(self):
        if getattr(self, "_h", None):
            lib().pmp_spray_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != 0:
            info = capi.ErrorInfo()
            lib().pmp_spray_last_error(self._h, C.byref(info))
            raise SprayError(rc, info)

    # --- setup (SpraySetup.cpp) -------------------------------------------
    def spray_setup(self, inputs):
        self._check(lib().pmp_spray_setup(self._h, C.byref(inputs)))

    def set_spray_data(self, data):
        self._check(lib().pmp_spray_set_data(self._h, C.byref(data)))

    def spray_data(self):
        d = capi.SprayData()
        self._check(lib().pmp_spray_get_data(self._h, C.byref(d)))
        return d

    def assign_spray_comps(self, comps):
        self._check(lib().pmp_spray_set_comps(self._h, C.byref(comps)))

    def set_geometry(self, geom):
        self._check(lib().pmp_spray_set_geometry(self._h, C.byref(geom)))

    def set_grids(self, boxes):
        arr = (capi.Box * len(boxes))()
        for b, (lo, hi) in enumerate(boxes):
            for d in range(3):
                arr[b].lo[d] = int(lo[d])
                arr[b].hi[d] = int(hi[d])
        self.nboxes = len(boxes)
        self._check(lib().pmp_spray_set_grids(self._h, len(boxes), arr))

    def set_mode(self, mode):
        self._check(lib().pmp_spray_set_mode(self._h, mode))

    def set_coupling(self, coupling):
        """capi.PMP_COUPLING_LMEX (default) or PMP_COUPLING_PELEC; before setup."""
        self._check(lib().pmp_spray_set_coupling(self._h, coupling))

    @property
    def coupling(self):
        c = C.c_int(0)
        self._check(lib().pmp_spray_get_coupling(self._h, C.byref(c)))
        return c.value

    # --- droplets ---------------------------------------------------------
    def set_particles(self, box, pos, rdata, ids):
        """pos (3,n), rdata (10+F,n) float64, ids (n,) int32: numpy or CUDA tensors."""
        p = capi.Particles()
        p.layout = capi.PMP_LAYOUT_SOA
        p.where = capi.PMP_WHERE_DEVICE if _is_cuda(pos) else capi.PMP_WHERE_HOST
        p.n = int(ids.shape[0])
        for d in range(3):
            p.pos[d] = _ptr(pos[d])
        for r in range(rdata.shape[0]):
            p.rdata[r] = _ptr(rdata[r])
        p.id = _ptr(ids)
        self._check(lib().pmp_spray_set_particles(self._h, box, C.byref(p)))

    def set_particles_aos(self, box, aos, n, on_device=False):
        p = capi.Particles()
        p.layout = capi.PMP_LAYOUT_AOS
        p.where = capi.PMP_WHERE_DEVICE if on_device else capi.PMP_WHERE_HOST
        p.n = n
        p.aos = _ptr(aos)
        self._check(lib().pmp_spray_set_particles(self._h, box, C.byref(p)))

    def num_particles(self, box):
        n = C.c_longlong()
        self._check(lib().pmp_spray_num_particles(self._h, box, C.byref(n)))
        return n.value

    def get_particles(self, box):
        """Droplets of `box` in the caller's order as host numpy arrays."""
        n = self.num_particles(box)
        nr = capi.pstate_num(self.nfuel)
        pos = np.zeros((3, n))
        rdata = np.zeros((nr, n))
        ids = np.zeros(n, dtype=np.int32)
        p = capi.Particles()
        p.layout = capi.PMP_LAYOUT_SOA
        p.where = capi.PMP_WHERE_HOST
        p.n = n
        for d in range(3):
            p.pos[d] = pos[d].ctypes.data
        for r in range(nr):
            p.rdata[r] = rdata[r].ctypes.data
        p.id = ids.ctypes.data
        self._check(lib().pmp_spray_get_particles(self._h, box, C.byref(p)))
        return dict(pos=pos, rdata=rdata, id=ids)

    def get_particles_aos(self, box):
        n = self.num_particles(box)
        rec = 8 * (3 + capi.pstate_num(self.nfuel)) + 8
        buf = np.zeros(n * rec, dtype=np.uint8)
        p = capi.Particles()
        p.layout = capi.PMP_LAYOUT_AOS
        p.where = capi.PMP_WHERE_HOST
        p.n = n
        p.aos = buf.ctypes.data
        self._check(lib().pmp_spray_get_particles(self._h, box, C.byref(p)))
        return buf

    # --- the update (SprayParticles.cpp:37-87,142-502) --------------------
    # The C ABI's update calls are stream-ordered (they enqueue and return);
    # with sync=True (the default here) the mirror then waits for the call
    # and raises its device error, as the reference's per-box synchronisation
    # (SprayParticles.cpp:499) would abort.  sync=False leaves the call in
    # flight: errors and stats come from sync().
    def update_particles(self, state, source, flow_dt, time, state_ghosts, source_ghosts,
                         is_virt, is_ghost, do_move, spray_cfl_lev, stream=0, sync=True):
        """state/source: pmp_box_view arrays (device memory)."""
        self._check(lib().pmp_spray_update(
            self._h, state, source, len(state), flow_dt, time, state_ghosts, source_ghosts,
            int(is_virt), int(is_ghost), int(do_move), spray_cfl_lev, C.c_void_p(stream)))
        if sync:
            self.sync()

    def update_particles_host(self, state, source, flow_dt, time, state_ghosts, source_ghosts,
                              is_virt, is_ghost, do_move, spray_cfl_lev, stream=0, sync=True):
        """Same call with host-memory views (copies inside)."""
        self._check(lib().pmp_spray_update_host(
            self._h, state, source, len(state), flow_dt, time, state_ghosts, source_ghosts,
            int(is_virt), int(is_ghost), int(do_move), spray_cfl_lev, C.c_void_p(stream)))
        if sync:
            self.sync()

    def set_host_source_in(self, copy_in):
        """update_particles_host: add the deposits to the host source (True,
        default) or take it as zero on entry and write the deposits over it
        (False; saves its host-to-device copy)."""
        self._check(lib().pmp_spray_set_host_source_in(self._h, int(bool(copy_in))))

    def move_kick_drift(self, state, source, dt, time, is_virt, is_ghost, state_ghosts,
                        source_ghosts, do_move=True, spray_cfl_lev=-1.0, stream=0, sync=True):
        self._check(lib().pmp_spray_move_kick_drift(
            self._h, state, source, len(state), dt, time, int(is_virt), int(is_ghost),
            state_ghosts, source_ghosts, int(do_move), spray_cfl_lev, C.c_void_p(stream)))
        if sync:
            self.sync()

    def move_kick(self, state, source, dt, time, is_virt, is_ghost, state_ghosts, source_ghosts,
                  spray_cfl_lev=-1.0, stream=0, sync=True):
        self._check(lib().pmp_spray_move_kick(
            self._h, state, source, len(state), dt, time, int(is_virt), int(is_ghost),
            state_ghosts, source_ghosts, spray_cfl_lev, C.c_void_p(stream)))
        if sync:
            self.sync()

    def sync(self):
        """Wait for the enqueued updates; raise SprayError for a device error."""
        self._check(lib().pmp_spray_sync(self._h))

    def last_error(self):
        info = capi.ErrorInfo()
        lib().pmp_spray_last_error(self._h, C.byref(info))
        return info

    def stats(self):
        s = capi.Stats()
        lib().pmp_spray_get_stats(self._h, C.byref(s))
        return s

    # --- around the update (SprayParticles.cpp:89-140, SprayDerive.cpp,
    #     SprayParticles.H:250-319, Redistribute) ---------------------------
    def est_timestep(self, cfl, max_jet_vel=0.0, stream=0):
        dt = C.c_double(0.0)
        self._check(lib().pmp_spray_est_timestep(self._h, cfl, max_jet_vel, C.byref(dt),
                                                 C.c_void_p(stream)))
        return dt.value

    def compute_derived_vars(self, var_views, start_indx=0, with_species=True, stream=0):
        self._check(lib().pmp_spray_derive(self._h, var_views, len(var_views), start_indx,
                                           int(with_species), C.c_void_p(stream)))

    def transfer_source(self, tmp_views, act_views, source_ghosts, act_ghosts, stream=0):
        self._check(lib().pmp_spray_transfer_source(self._h, tmp_views, act_views, len(tmp_views),
                                                    source_ghosts, act_ghosts, C.c_void_p(stream)))

    def redistribute(self, stream=0):
        """Re-bin droplets to boxes (periodic wrap, dead dropped); returns the count dropped."""
        n = C.c_longlong(0)
        self._check(lib().pmp_spray_redistribute(self._h, C.byref(n), C.c_void_p(stream)))
        return n.value

    # --- launch shape, CUDA graph, autotuner (batched form) ---------------
    def set_launch(self, kind=capi.PMP_LAUNCH_GRID, block=128, regs=96, chunk=512, ctas_per_sm=0,
                   use_graph=False):
        cfg = capi.LaunchConfig(kind, block, regs, chunk, ctas_per_sm, int(use_graph))
        self._check(lib().pmp_spray_set_launch(self._h, C.byref(cfg)))

    def launch(self):
        cfg = capi.LaunchConfig()
        self._check(lib().pmp_spray_get_launch(self._h, C.byref(cfg)))
        return cfg

    def autotune(self, state, source, flow_dt, state_ghosts, source_ghosts, is_ghost, do_move,
                 spray_cfl_lev, cache_path=None, stream=0):
        """Pick the fastest launch shape of the FP64 update for these views."""
        rep = capi.TuneReport()
        self._check(lib().pmp_spray_autotune(
            self._h, state, source, len(state), flow_dt, state_ghosts, source_ghosts, int(is_ghost),
            int(do_move), spray_cfl_lev, cache_path.encode() if cache_path else None, C.byref(rep),
            C.c_void_p(stream)))
        return rep

    # --- learned form (no counterpart in the reference) -------------------
    def learn_generate(self, state, flow_dt, state_ghosts, do_move=True, spray_cfl_lev=-1.0,
                       sample_stride=1, augment=0, seed=1, stream=0):
        """Label droplets at this state with the FP64 teacher (tuples accumulate)."""
        self._check(lib().pmp_spray_learn_generate(
            self._h, state, len(state), flow_dt, state_ghosts, int(do_move), spray_cfl_lev,
            int(sample_stride), int(augment), int(seed), C.c_void_p(stream)))

    def learn_count(self):
        n = C.c_longlong(0)
        self._check(lib().pmp_spray_learn_count(self._h, C.byref(n)))
        return n.value

    def learn_tuples(self):
        """(n, 16) float32: 10 raw inputs, 5 targets, pad."""
        n = C.c_longlong(0)
        self._check(lib().pmp_spray_learn_tuples(self._h, None, C.byref(n)))
        buf = np.empty((n.value, 16), np.float32)
        self._check(lib().pmp_spray_learn_tuples(self._h, buf.ctypes.data, C.byref(n)))
        return buf[:n.value]

    def learn_train(self, epochs=0, batch=0, lr=0.0, gate_margin=0.0, audit_fraction=0.0,
                    no_quant=False, seed=0):
        cfg = capi.LearnConfig(epochs, batch, lr, gate_margin, audit_fraction, int(no_quant), seed)
        rep = capi.LearnReport()
        self._check(lib().pmp_spray_learn_train(self._h, C.byref(cfg), C.byref(rep)))
        return rep

    def learn_weights(self):
        """Flat float32 vector: parameters, then the normalisation and gate."""
        n = C.c_longlong(0)
        self._check(lib().pmp_spray_learn_weights(self._h, 1, None, C.byref(n)))
        buf = np.empty(n.value, np.float32)
        self._check(lib().pmp_spray_learn_weights(self._h, 1, buf.ctypes.data, C.byref(n)))
        return buf

    def set_learn_weights(self, buf):
        buf = np.ascontiguousarray(buf, np.float32)
        n = C.c_longlong(buf.size)
        self._check(lib().pmp_spray_learn_weights(self._h, 0, buf.ctypes.data, C.byref(n)))

    def learn_set_audit(self, fraction):
        self._check(lib().pmp_spray_learn_set_audit(self._h, float(fraction)))

    def learn_audit(self):
        """(droplets audited, RMS error per surrogate output) of the last learned update."""
        n = C.c_longlong(0)
        e = (C.c_double * 5)()
        self._check(lib().pmp_spray_learn_audit(self._h, C.byref(n), e))
        return n.value, np.array(e[:])


def learn_param_count():
    return lib().pmp_learn_param_count()


def learn_base_terms():
    return lib().pmp_learn_base_terms()


def learn_debug_base(xn, ell, g, coef):
    """(terms, value): the baseline's terms for normalised inputs xn[10] and
    derived variables ell, g, and the FP32 polynomial with coefficients coef,
    from the library's host code (no GPU)."""
    nt = learn_base_terms()
    xn = np.ascontiguousarray(xn, np.float32)
    coef = np.ascontiguousarray(coef, np.float32)
    assert xn.size == capi.LEARN_IN and coef.size == nt
    feats = np.zeros(nt)
    val = C.c_float(0.0)
    rc = lib().pmp_learn_debug_base(xn.ctypes.data, float(ell), float(g), coef.ctypes.data,
                                    feats.ctypes.data, C.byref(val))
    if rc != capi.PMP_OK:
        raise SprayError(rc)
    return feats, val.value


def learn_debug_solve_baseline(acc):
    """coef[5, terms] from the normal equations in k_base_normal's layout (no GPU)."""
    nt = learn_base_terms()
    acc = np.ascontiguousarray(acc, np.float64)
    assert acc.size == nt * (nt + 1) // 2 + nt * capi.LEARN_OUT
    coef = np.zeros((capi.LEARN_OUT, nt), np.float32)
    rc = lib().pmp_learn_debug_solve_baseline(acc.ctypes.data, coef.ctypes.data)
    if rc != capi.PMP_OK:
        raise SprayError(rc)
    return coef


def learn_debug_grad(params, x, y, quant=True):
    """Loss and gradient of the training kernels (see pmp_learn_debug_grad)."""
    params = np.ascontiguousarray(params, np.float32)
    x = np.ascontiguousarray(x, np.float32)
    y = np.ascontiguousarray(y, np.float32)
    n = x.shape[0]
    assert params.size == learn_param_count() and x.shape == (n, capi.LEARN_IN)
    assert y.shape == (n, capi.LEARN_OUT)
    g = np.zeros_like(params)
    loss = C.c_double(0.0)
    rc = lib().pmp_learn_debug_grad(params.ctypes.data, x.ctypes.data, y.ctypes.data, n,
                                    int(quant), g.ctypes.data, C.byref(loss))
    if rc != capi.PMP_OK:
        raise SprayError(rc)
    return loss.value, g


def from_problem(prob, device=0, mode=capi.PMP_MODE_FP64, set_droplets=True):
    """Container set up for a workloads.Problem (droplets copied from host)."""
    sp = SprayParticleContainer(prob.species, prob.nfuel, device)
    if getattr(prob, "pelec", False):
        sp.set_coupling(capi.PMP_COUPLING_PELEC)
    sp.spray_setup(prob.inputs())
    sp.assign_spray_comps(prob.comps())
    sp.set_geometry(prob.geometry())
    sp.set_grids(prob.boxes)
    sp.set_mode(mode)
    if set_droplets:
        for b, p in enumerate(prob.parts):
            sp.set_particles(b, p["pos"], p["rdata"], p["id"])
    return sp


def learn_debug_infer(params, xn, engine="mma"):
    """Outputs of the tensor-core network for normalised inputs: engine "mma"
    (warp-level mma.sync) or "tc" (CTA-level tcgen05, accumulators in TMEM)."""
    params = np.ascontiguousarray(params, np.float32)
    xn = np.ascontiguousarray(xn, np.float32)
    n = xn.shape[0]
    y = np.zeros((n, capi.LEARN_OUT), np.float32)
    fn = lib().pmp_learn_debug_infer_tc if engine == "tc" else lib().pmp_learn_debug_infer
    rc = fn(params.ctypes.data, xn.ctypes.data, n, y.ctypes.data)
    if rc != capi.PMP_OK:
        raise SprayError(rc)
    return y


def learn_debug_wait_timeout():
    """(status, cycles) of a tcgen05 wait on an mbarrier nothing arrives on."""
    cycles = C.c_longlong(0)
    rc = lib().pmp_learn_debug_wait_timeout(C.byref(cycles))
    return rc, cycles.value


def measure_peaks(device=0):
    """Measured FP64 / FP32 FMA (TFLOP/s) and SFU ex2 (G op/s) rates of the device."""
    a, b, c = C.c_double(), C.c_double(), C.c_double()
    rc = lib().pmp_measure_peaks(device, C.byref(a), C.byref(b), C.byref(c))
    if rc != 0:
        raise SprayError(rc, capi.ErrorInfo())
    return {"fp64_tflops": a.value, "fp32_tflops": b.value, "sfu_gops": c.value}
