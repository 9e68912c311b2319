"""ctypes bindings of the CPU oracle and of the reference build.

TEST INFRASTRUCTURE: imported only by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, to compare against.  The product never imports it.

* ``Oracle(libm=False)`` -- oracle/liboracle.so (project math, the functions
  the CUDA kernels use); ``Oracle(libm=True)`` -- oracle/liboracle_libm.so
  (C library math).
* ``Reference(nspec, nfuel)`` -- oracle/_ref/libref_n{S}_f{F}.so, PeleMP's own
  physics headers compiled in this repository (C library math).

``pelec=True`` selects the PeleC coupling (CGS units, energy state, drag work
and kinetic-energy source terms): the oracle's process-wide coupling switch is
set before each call, and the reference build is the one compiled without
PELELM_USE_SPRAY (oracle/_ref/libref_pelec_n{S}_f{F}.so).
"""
import ctypes as C
import os

import numpy as np

from pelemp_b200 import capi
from pelemp_b200.workloads import view_of

HERE = os.path.dirname(os.path.abspath(__file__))


def _parts_array(prob, parts):
    arr = (capi.Particles * len(parts))()
    for b, p in enumerate(parts):
        a = arr[b]
        a.layout = capi.PMP_LAYOUT_SOA
        a.where = capi.PMP_WHERE_HOST
        a.n = p["id"].shape[0]
        for d in range(3):
            a.pos[d] = p["pos"][d].ctypes.data
        for r in range(p["rdata"].shape[0]):
            a.rdata[r] = p["rdata"][r].ctypes.data
        a.id = p["id"].ctypes.data
    return arr


def _views(prob, arrays, ghosts):
    arr = (capi.BoxView * len(arrays))()
    for b, a in enumerate(arrays):
        lo, _ = prob.grown(b, ghosts)
        arr[b] = view_of(a, lo)
    return arr


class _Base:
    _update_name = None
    pelec = False

    def _couple(self):
        pass

    def _bind_update(self):
        f = getattr(self.lib, self._update_name)
        f.restype = C.c_int
        f.argtypes = [C.POINTER(capi.Mech), C.POINTER(capi.SprayData),
                      C.POINTER(capi.SprayComps), C.POINTER(capi.Geometry), C.c_int,
                      C.POINTER(capi.Box), C.POINTER(capi.Particles),
                      C.POINTER(capi.BoxView), C.POINTER(capi.BoxView), C.c_double,
                      C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_int,
                      C.POINTER(capi.ErrorInfo), C.POINTER(C.c_longlong)]
        self._update = f

    def update(self, prob, mech, fdat, parts, sources, do_move, is_ghost=0, is_virt=0,
               nthreads=1, flow_dt=None, state=None):
        """One updateParticles call over all boxes; parts/sources updated in place.
        Returns (status, ErrorInfo, substeps)."""
        err = capi.ErrorInfo()
        nsub = C.c_longlong(0)
        pa = _parts_array(prob, parts)
        st = _views(prob, state if state is not None else prob.state, prob.state_ghosts)
        sr = _views(prob, sources, prob.source_ghosts)
        self._couple()
        rc = self._update(
            C.byref(mech), C.byref(fdat), C.byref(prob.comps()), C.byref(prob.geometry()),
            len(prob.boxes), prob.box_array(), pa, st, sr,
            prob.flow_dt if flow_dt is None else flow_dt, prob.state_ghosts,
            prob.source_ghosts, is_virt, is_ghost, do_move, prob.spray_cfl_lev, nthreads,
            C.byref(err), C.byref(nsub))
        return rc, err, nsub.value


class Oracle(_Base):
    _update_name = "pmp_oracle_update"

    def __init__(self, libm=False, pelec=False):
        name = "liboracle_libm.so" if libm else "liboracle.so"
        path = os.path.join(HERE, name)
        if not os.path.exists(path):
            raise RuntimeError(f"{path} missing: run `make -C oracle`")
        self.lib = C.CDLL(path)
        self.pelec = bool(pelec)
        self.lib.pmp_oracle_set_coupling.restype = None
        self.lib.pmp_oracle_set_coupling.argtypes = [C.c_int]
        self._bind_update()
        self.lib.pmp_oracle_mech.restype = C.c_int
        self.lib.pmp_oracle_mech.argtypes = [C.POINTER(capi.Mech), C.c_int, C.c_void_p]
        self.lib.pmp_oracle_setup.restype = C.c_int
        self.lib.pmp_oracle_setup.argtypes = [C.POINTER(capi.Mech), C.c_void_p,
                                              C.POINTER(capi.SprayInputs),
                                              C.POINTER(capi.SprayData)]
        f = self.lib.pmp_oracle_droplet_source
        f.restype = C.c_double
        f.argtypes = [C.POINTER(capi.Mech), C.POINTER(capi.SprayData), C.c_double,
                      C.c_void_p, C.c_void_p, C.POINTER(C.c_int), C.c_void_p]
        L = self.lib
        L.pmp_oracle_thermo.restype = None
        L.pmp_oracle_thermo.argtypes = [C.POINTER(capi.Mech), C.c_double, C.c_void_p, C.c_void_p]
        L.pmp_oracle_transport.restype = None
        L.pmp_oracle_transport.argtypes = [C.POINTER(capi.Mech), C.c_double, C.c_void_p,
                                           C.c_void_p, C.c_void_p, C.c_void_p]
        L.pmp_oracle_math.restype = None
        L.pmp_oracle_math.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_longlong]
        L.pmp_oracle_abi_sizes.restype = None
        L.pmp_oracle_abi_sizes.argtypes = [C.c_void_p]

    def _couple(self):
        self.lib.pmp_oracle_set_coupling(1 if self.pelec else 0)

    def update_energy(self, prob, mech, fdat, parts, sources, do_move, residual, **kw):
        """update() that also adds each parcel's energy-identity residual of the
        call to residual[b][i] (float64 arrays, one per box; PeleLMeX coupling)."""
        ptrs = (C.c_void_p * len(residual))(*[r.ctypes.data for r in residual])
        self.lib.pmp_oracle_set_energy_out.restype = None
        self.lib.pmp_oracle_set_energy_out.argtypes = [C.c_void_p]
        self.lib.pmp_oracle_set_energy_out(C.cast(ptrs, C.c_void_p))
        try:
            return self.update(prob, mech, fdat, parts, sources, do_move, **kw)
        finally:
            self.lib.pmp_oracle_set_energy_out(None)

    def math(self, fn, x, y=None):
        """fn in ('exp','log','log1p','pow','cbrt') over float64 arrays."""
        code = ("exp", "log", "log1p", "pow", "cbrt").index(fn)
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.ascontiguousarray(y if y is not None else np.zeros_like(x), dtype=np.float64)
        out = np.empty_like(x)
        self.lib.pmp_oracle_math(code, x.ctypes.data, y.ctypes.data, out.ctypes.data, x.size)
        return out

    def thermo(self, mech, T):
        cp = np.zeros(capi.PMP_MAX_SPEC)
        h = np.zeros(capi.PMP_MAX_SPEC)
        self.lib.pmp_oracle_thermo(C.byref(mech), T, cp.ctypes.data, h.ctypes.data)
        return cp[:mech.nspec], h[:mech.nspec]

    def transport(self, mech, T, Y):
        Yb = np.zeros(capi.PMP_MAX_SPEC)
        Yb[:len(Y)] = Y
        Dd = np.zeros(capi.PMP_MAX_SPEC)
        mu = np.zeros(1)
        lam = np.zeros(1)
        self.lib.pmp_oracle_transport(C.byref(mech), T, Yb.ctypes.data, Dd.ctypes.data,
                                      mu.ctypes.data, lam.ctypes.data)
        return mu[0], lam[0], Dd[:mech.nspec]

    def abi_sizes(self):
        out = np.zeros(15, dtype=np.int64)
        self.lib.pmp_oracle_abi_sizes(out.ctypes.data)
        return out

    def mech(self, species):
        m = capi.Mech()
        names = capi.names_array(species)
        rc = self.lib.pmp_oracle_mech(C.byref(m), len(species), C.cast(names, C.c_void_p))
        if rc != 0:
            raise ValueError(f"unknown species in {species}")
        return m

    def setup(self, prob, mech=None, inputs=None):
        mech = mech if mech is not None else self.mech(prob.species)
        names = capi.names_array(prob.species)
        out = capi.SprayData()
        inp = inputs if inputs is not None else prob.inputs()
        self._couple()
        rc = self.lib.pmp_oracle_setup(C.byref(mech), C.cast(names, C.c_void_p),
                                       C.byref(inp), C.byref(out))
        return rc, out

    def droplet_source(self, mech, fdat, flow_dt, gas, rdata, pid=1):
        gas = np.ascontiguousarray(gas, dtype=np.float64)
        rd = np.ascontiguousarray(rdata, dtype=np.float64).copy()
        src = np.zeros(5 + fdat.nfuel)
        idv = C.c_int(pid)
        self._couple()
        re = self.lib.pmp_oracle_droplet_source(
            C.byref(mech), C.byref(fdat), flow_dt, gas.ctypes.data, rd.ctypes.data,
            C.byref(idv), src.ctypes.data)
        return re, rd, idv.value, src


class Reference(_Base):
    _update_name = "pmp_ref_update"

    def __init__(self, nspec, nfuel, pelec=False):
        path = self._path(nspec, nfuel, pelec)
        if not os.path.exists(path):
            raise RuntimeError(f"{path} missing (needs the PeleMP sources at build time)")
        self.lib = C.CDLL(path)
        self.pelec = bool(pelec)
        self._bind_update()

    @staticmethod
    def _path(nspec, nfuel, pelec):
        tag = "pelec_" if pelec else ""
        return os.path.join(HERE, "_ref", f"libref_{tag}n{nspec}_f{nfuel}.so")

    @staticmethod
    def available(nspec, nfuel, pelec=False):
        return os.path.exists(Reference._path(nspec, nfuel, pelec))
