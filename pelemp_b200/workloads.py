"""Seeded synthetic spray workloads (mesh state + droplets) of the named shapes.

The reference ships no benchmark data for its spray update, so every input is
generated here from a seed with numpy's PCG64 generator:

* ``config1`` -- plain FP64, one 32^3 periodic box, dx = 1e-4 m, gas
  [N2, O2, NC7H16] at 1 atm with T ~ U[800,1000] K and u ~ U[-5,5]^3 m/s per
  cell, 100k n-heptane droplets (d lognormal, median 20 um, sigma 0.3,
  clipped to [2,80] um; T = 300 K; u ~ U[-10,10]^3), dt = 1e-6 s, 10 steps.
* ``config2`` -- plain FP64 at scale: 128^3 cells as 8 boxes of 64^3, gas
  [N2, O2, NC10H22, NC7H16, CO2] with T = 900 + 100 sin sin sin K, 16M
  two-component droplets (n-decane fraction ~ U[0,1]), d lognormal median
  15 um sigma 0.4, T ~ U[290,350] K, dt = 5e-7 s, spray_cfl_lev = 2 (four
  sub-cycles per move), 20 steps.
* ``config3`` -- config 1's physics on 256 boxes of 32^3 with capped-Zipf
  droplet counts (s = 1.2, at most 400k per box, 16M total).
* ``config4`` -- config 1's distributions, 32M droplets on 256x128x128.
* ``walls``   -- a small non-periodic case (reflective x, outflow z) used to
  exercise the boundary branches.
* ``to_pelec(prob, mech)`` -- any of the above restated for the PeleC
  coupling: CGS units, momentum and total energy in the state.

Liquid properties: n-heptane from Exec/SprayTests/PeleC/heptane_evap/input2d:64-77
(converted to MKS), n-decane from Exec/SprayTests/PeleLMeX/abramzon_test/inputs_2d:65-77.
The gas density is set so that the ideal-gas pressure is 101325 Pa per cell.
Ghost widths are 3 (state) and 2 (source) cells so that several steps run
without re-binning droplets that drift out of their box.

Mesh layout (AMReX Array4, x fastest): a box's state is a numpy array of
shape (ncomp, nz, ny, nx) over the box grown by its ghost width.  State
components: vel 0..2 (PeleLMeX stores velocity), rho 3, rhoY 4..4+NSP-1,
rhoH 4+NSP (not read on this path), T 5+NSP.  Source components: mom 0..2,
rho 3, rhoY_fuel 4..4+F-1, energy 4+F.  In the PeleC restatement the same
slots hold rho*u 0..2, rho 3, rhoY, rho*E 4+NSP and the temperature guess.
"""
from dataclasses import dataclass, field

import numpy as np

from . import capi

RU_SI = 8.31446261815324
PATM = 101325.0

# W [kg/mol] of the project's species database (pmp_thermo_data.h order)
MW = {"N2": 28.0134e-3, "O2": 31.9988e-3, "NC7H16": 100.2019e-3,
      "NC10H22": 142.2817e-3, "CO2": 44.0095e-3}

LIQUIDS = {
    # crit_temp, boil_temp, latent [J/kg], cp [J/(kg K)], rho [kg/m^3], Antoine a b c d[Pa]
    "NC7H16": dict(crit_temp=540.0, boil_temp=371.6, latent=3.63e5, cp=2248.3,
                   rho=681.4, psat=(4.02832, 1268.636, -56.199, 1.0e5)),
    "NC10H22": dict(crit_temp=617.8, boil_temp=447.27, latent=3.5899e5, cp=2192.1,
                    rho=640.0, psat=(4.07857, 1501.268, -78.67, 1.0e5)),
}


@dataclass
class Problem:
    name: str
    species: list
    fuels: list
    ref_T: float
    plo: np.ndarray
    phi: np.ndarray
    dx: np.ndarray
    domain_lo: tuple
    domain_hi: tuple
    bndry_lo: tuple
    bndry_hi: tuple
    boxes: list              # [(lo(3), hi(3))] valid boxes
    state_ghosts: int
    source_ghosts: int
    state: list              # per box (ncomp, nz, ny, nx) float64
    parts: list              # per box dict(pos=(3,n), rdata=(nr,n), id=(n,))
    flow_dt: float
    spray_cfl_lev: float
    steps: int
    mass_trans: int = 1
    mom_trans: int = 1
    fixed_parts: int = 0
    body_force: tuple = (0.0, 0.0, 0.0)
    pelec: bool = False      # CGS units and the PeleC state (to_pelec)
    meta: dict = field(default_factory=dict)

    @property
    def nspec(self):
        return len(self.species)

    @property
    def nfuel(self):
        return len(self.fuels)

    @property
    def n_state_comp(self):
        return 6 + self.nspec

    @property
    def n_src_comp(self):
        return 5 + self.nfuel

    @property
    def n_droplets(self):
        return int(sum(p["id"].shape[0] for p in self.parts))

    def comps(self):
        ns, nf = self.nspec, self.nfuel
        return capi.SprayComps(rhoIndx=3, momIndx=0, engIndx=4 + ns, utempIndx=5 + ns,
                               specIndx=4, rhoSrcIndx=3, momSrcIndx=0,
                               engSrcIndx=4 + nf, specSrcIndx=4)

    def geometry(self):
        g = capi.Geometry()
        for d in range(3):
            g.plo[d] = float(self.plo[d])
            g.phi[d] = float(self.phi[d])
            g.dx[d] = float(self.dx[d])
            g.domain_lo[d] = int(self.domain_lo[d])
            g.domain_hi[d] = int(self.domain_hi[d])
            g.bndry_lo[d] = int(self.bndry_lo[d])
            g.bndry_hi[d] = int(self.bndry_hi[d])
        return g

    def box_array(self):
        arr = (capi.Box * len(self.boxes))()
        for b, (lo, hi) in enumerate(self.boxes):
            for d in range(3):
                arr[b].lo[d] = int(lo[d])
                arr[b].hi[d] = int(hi[d])
        return arr

    def inputs(self, cfl=None):
        """The particles.* inputs of this problem (pmp_spray_inputs)."""
        s = capi.SprayInputs()
        s.nfuel = self.nfuel
        # CGS for PeleC: erg/g = 1e4 J/kg, g/cm^3 = 1e3 kg/m^3, dyn/cm^2 = 0.1 Pa
        eng, rho, pres = (1e4, 1e-3, 10.0) if self.pelec else (1.0, 1.0, 1.0)
        for f, name in enumerate(self.fuels):
            liq = LIQUIDS[name]
            s.fuel_species[f].value = name.encode()
            s.crit_temp[f] = liq["crit_temp"]
            s.boil_temp[f] = liq["boil_temp"]
            s.latent[f] = liq["latent"] * eng
            s.cp[f] = liq["cp"] * eng
            s.ncoef_rho[f] = 1
            s.rho[f][0] = liq["rho"] * rho
            s.ncoef_psat[f] = 4
            for i in range(3):
                s.psat[f][i] = liq["psat"][i]
            s.psat[f][3] = liq["psat"][3] * pres
        s.mass_transfer = self.mass_trans
        s.mom_transfer = self.mom_trans
        s.fixed_parts = self.fixed_parts
        s.cfl = 0.5 if cfl is None else cfl
        s.fuel_ref_temp = self.ref_T
        for d in range(3):
            s.body_force[d] = self.body_force[d] * (100.0 if self.pelec else 1.0)
        return s

    def grown(self, b, g):
        lo, hi = self.boxes[b]
        return tuple(l - g for l in lo), tuple(h + g for h in hi)

    def new_sources(self):
        out = []
        for b in range(len(self.boxes)):
            lo, hi = self.grown(b, self.source_ghosts)
            shape = (self.n_src_comp,) + tuple(hi[d] - lo[d] + 1 for d in (2, 1, 0))
            out.append(np.zeros(shape))
        return out

    def copy_parts(self):
        return [{k: v.copy() for k, v in p.items()} for p in self.parts]


def view_of(arr, lo):
    """pmp_box_view of a (ncomp, nz, ny, nx) array whose (0,0,0) is cell lo."""
    v = capi.BoxView()
    nc, nz, ny, nx = arr.shape
    v.p = arr.ctypes.data
    for d in range(3):
        v.lo[d] = int(lo[d])
    v.hi[0] = lo[0] + nx - 1
    v.hi[1] = lo[1] + ny - 1
    v.hi[2] = lo[2] + nz - 1
    v.jstride = nx
    v.kstride = nx * ny
    v.nstride = nx * ny * nz
    v.ncomp = nc
    return v


def _gas_state(prob, T_fn, vel_fn, Y):
    """Fill each box's grown state from global per-cell fields."""
    ns = prob.nspec
    W = np.array([MW[s] for s in prob.species])
    Wbar = 1.0 / np.sum(np.asarray(Y) / W)
    nglob = tuple(prob.domain_hi[d] - prob.domain_lo[d] + 1 for d in range(3))
    Tg = T_fn(nglob)          # (nz, ny, nx)
    Ug = vel_fn(nglob)        # (3, nz, ny, nx)
    states = []
    for b in range(len(prob.boxes)):
        lo, hi = prob.grown(b, prob.state_ghosts)
        idx = []
        for d in range(3):
            r = np.arange(lo[d], hi[d] + 1) - prob.domain_lo[d]
            if prob.bndry_lo[d] == 0:
                r = np.mod(r, nglob[d])
            else:
                r = np.clip(r, 0, nglob[d] - 1)
            idx.append(r)
        ix = np.ix_(idx[2], idx[1], idx[0])
        T = Tg[ix]
        rho = PATM * Wbar / (RU_SI * T)
        st = np.zeros((prob.n_state_comp,) + T.shape)
        for d in range(3):
            st[d] = Ug[d][ix]
        st[3] = rho
        for k in range(ns):
            st[4 + k] = rho * Y[k]
        st[4 + ns] = 0.0
        st[5 + ns] = T
        states.append(np.ascontiguousarray(st))
    return states


def _droplets(prob, rng, n, dia_median, dia_sigma, T_fn, Yl_fn, vmax=10.0, counts=None):
    """Uniform droplets over the domain (or `counts` per box), binned to boxes."""
    nf = prob.nfuel
    nr = capi.pstate_num(nf)
    plo, phi, dx = prob.plo, prob.phi, prob.dx
    dxi = 1.0 / dx
    if counts is None:
        pos = plo[:, None] + rng.random((3, n)) * (phi - plo)[:, None]
    else:
        chunks = []
        for b, cnt in enumerate(counts):
            lo, hi = prob.boxes[b]
            blo = plo + np.asarray(lo) * dx
            bhi = plo + (np.asarray(hi) + 1) * dx
            chunks.append(blo[:, None] + rng.random((3, cnt)) * (bhi - blo)[:, None])
        pos = np.concatenate(chunks, axis=1)
        n = pos.shape[1]
    dia = np.clip(dia_median * np.exp(dia_sigma * rng.standard_normal(n)), 2e-6, 80e-6)
    vel = rng.uniform(-vmax, vmax, (3, n))
    T = T_fn(n)
    Yl = Yl_fn(n)
    rdata = np.zeros((nr, n))
    rdata[0:3] = vel
    rdata[capi.PSTATE_T] = T
    rdata[capi.PSTATE_DIA] = dia
    rdata[capi.PSTATE_Y:capi.PSTATE_Y + nf] = Yl
    rdata[capi.pstate_numdens(nf)] = 1.0
    rdata[6 + nf] = 1.0   # N0
    ids = np.arange(1, n + 1, dtype=np.int32)
    # bin by the cell containing the droplet, computed as the kernel does
    ijkc = np.floor((pos - plo[:, None]) * dxi[:, None]).astype(np.int64)
    box_of = np.full(n, -1, dtype=np.int64)
    for b, (lo, hi) in enumerate(prob.boxes):
        inside = np.ones(n, dtype=bool)
        for d in range(3):
            inside &= (ijkc[d] >= lo[d]) & (ijkc[d] <= hi[d])
        box_of[inside] = b
    assert (box_of >= 0).all(), "droplet outside every box"
    parts = []
    for b in range(len(prob.boxes)):
        sel = np.nonzero(box_of == b)[0]
        parts.append(dict(pos=np.ascontiguousarray(pos[:, sel]),
                          rdata=np.ascontiguousarray(rdata[:, sel]),
                          id=np.ascontiguousarray(ids[sel])))
    return parts


def _boxes(ncells, box_size):
    nb = [ncells[d] // box_size[d] for d in range(3)]
    out = []
    for k in range(nb[2]):
        for j in range(nb[1]):
            for i in range(nb[0]):
                lo = (i * box_size[0], j * box_size[1], k * box_size[2])
                hi = tuple(lo[d] + box_size[d] - 1 for d in range(3))
                out.append((lo, hi))
    return out


def _base(name, species, fuels, ref_T, ncells, box_size, dx, ghosts, flow_dt,
          cfl_lev, steps, bndry=((0, 0, 0), (0, 0, 0))):
    dxv = np.array([dx, dx, dx])
    plo = np.zeros(3)
    phi = plo + np.array(ncells) * dxv
    return Problem(
        name=name, species=list(species), fuels=list(fuels), ref_T=ref_T,
        plo=plo, phi=phi, dx=dxv, domain_lo=(0, 0, 0),
        domain_hi=tuple(n - 1 for n in ncells), bndry_lo=bndry[0], bndry_hi=bndry[1],
        boxes=_boxes(ncells, box_size), state_ghosts=ghosts[0],
        source_ghosts=ghosts[1], state=[], parts=[], flow_dt=flow_dt,
        spray_cfl_lev=cfl_lev, steps=steps)


def config1(n=100_000, seed=0, steps=10):
    """Plain FP64, CPU-runnable: 32^3, 100k n-heptane droplets."""
    rng = np.random.default_rng(seed)
    prob = _base("config1", ["N2", "O2", "NC7H16"], ["NC7H16"], 300.0, (32, 32, 32),
                 (32, 32, 32), 1e-4, (3, 2), 1e-6, 0.1, steps)
    prob.state = _gas_state(
        prob, lambda s: rng.uniform(800.0, 1000.0, s[::-1]),
        lambda s: rng.uniform(-5.0, 5.0, (3,) + s[::-1]), [0.767, 0.233, 0.0])
    prob.parts = _droplets(prob, rng, n, 20e-6, 0.3, lambda m: np.full(m, 300.0),
                           lambda m: np.ones((1, m)))
    return prob


def _sin_T(shape, mean=900.0, amp=100.0):
    nx, ny, nz = shape
    x = (np.arange(nx) + 0.5) / nx
    y = (np.arange(ny) + 0.5) / ny
    z = (np.arange(nz) + 0.5) / nz
    return mean + amp * (np.sin(2 * np.pi * z)[:, None, None]
                         * np.sin(2 * np.pi * y)[None, :, None]
                         * np.sin(2 * np.pi * x)[None, None, :])


def config2(n=16_000_000, seed=0, steps=20, ncells=(128, 128, 128), box=(64, 64, 64)):
    """Plain FP64 at scale: 128^3 as 8 boxes of 64^3, 16M two-fuel droplets."""
    rng = np.random.default_rng(seed)
    prob = _base("config2", ["N2", "O2", "NC10H22", "NC7H16", "CO2"],
                 ["NC10H22", "NC7H16"], 298.15, ncells, box, 1e-4, (3, 2), 5e-7, 2.0, steps)
    prob.state = _gas_state(prob, _sin_T, lambda s: rng.uniform(-5.0, 5.0, (3,) + s[::-1]),
                            [0.767, 0.233, 0.0, 0.0, 0.0])

    def yl(m):
        yd = rng.random(m)
        return np.stack([yd, 1.0 - yd])

    prob.parts = _droplets(prob, rng, n, 15e-6, 0.4, lambda m: rng.uniform(290.0, 350.0, m), yl)
    return prob


def zipf_counts(nbox=256, total=16_000_000, s=1.2, cap=400_000):
    """Capped Zipf droplet counts per box: min(cap, C k^-s) with sum = total."""
    k = np.arange(1, nbox + 1, dtype=np.float64)
    w = k ** -s
    lo, hi = 0.0, float(total) * 10
    for _ in range(200):
        c = 0.5 * (lo + hi)
        tot = np.minimum(cap, np.floor(c * w)).sum()
        if tot > total:
            hi = c
        else:
            lo = c
    cnt = np.minimum(cap, np.floor(lo * w)).astype(np.int64)
    rem = total - int(cnt.sum())
    i = 0
    while rem > 0:
        if cnt[i] < cap:
            cnt[i] += 1
            rem -= 1
        i = (i + 1) % nbox
    return cnt


def config3(total=16_000_000, seed=0, steps=10, nbox_xyz=(8, 8, 4), box=32):
    """Batched: 256 boxes of 32^3, capped-Zipf droplet counts, config-1 physics."""
    rng = np.random.default_rng(seed)
    ncells = tuple(n * box for n in nbox_xyz)
    prob = _base("config3", ["N2", "O2", "NC7H16"], ["NC7H16"], 300.0, ncells,
                 (box, box, box), 1e-4, (3, 2), 1e-6, 0.1, steps)
    prob.state = _gas_state(
        prob, lambda s: rng.uniform(800.0, 1000.0, s[::-1]),
        lambda s: rng.uniform(-5.0, 5.0, (3,) + s[::-1]), [0.767, 0.233, 0.0])
    nbox = len(prob.boxes)
    counts = zipf_counts(nbox, total) if total >= nbox else np.full(nbox, total // nbox)
    counts = counts[rng.permutation(nbox)]
    prob.parts = _droplets(prob, rng, 0, 20e-6, 0.3, lambda m: np.full(m, 300.0),
                           lambda m: np.ones((1, m)), counts=counts)
    prob.meta["counts"] = counts
    return prob


def config4(n=32_000_000, seed=0, steps=10):
    """Mixed precision: config-1 distributions, 32M droplets on 256x128x128."""
    rng = np.random.default_rng(seed)
    prob = _base("config4", ["N2", "O2", "NC7H16"], ["NC7H16"], 300.0, (256, 128, 128),
                 (64, 64, 64), 1e-4, (3, 2), 1e-6, 0.1, steps)
    prob.state = _gas_state(
        prob, lambda s: rng.uniform(800.0, 1000.0, s[::-1]),
        lambda s: rng.uniform(-5.0, 5.0, (3,) + s[::-1]), [0.767, 0.233, 0.0])
    prob.parts = _droplets(prob, rng, n, 20e-6, 0.3, lambda m: np.full(m, 300.0),
                           lambda m: np.ones((1, m)))
    return prob


def config5(n=16_000_000, seed=0, steps=10):
    """Learned-surrogate workload: config-1 distributions (heptane droplets of
    20 um median at 300 K in 800-1000 K air) at 16M or 64M droplets, on
    config 4's 256x128x128 mesh of 64^3 boxes."""
    prob = config4(n=n, seed=seed, steps=steps)
    prob.name = "config5"
    return prob


def walls(n=20_000, seed=0, steps=2):
    """Non-periodic case: reflective x walls, outflow z, periodic y; 2 boxes."""
    rng = np.random.default_rng(seed)
    prob = _base("walls", ["N2", "O2", "NC7H16"], ["NC7H16"], 300.0, (16, 16, 16),
                 (8, 16, 16), 1e-4, (3, 2), 2e-6, 2.0, steps,
                 bndry=((1, 0, -1), (1, 0, -1)))
    prob.state = _gas_state(
        prob, lambda s: rng.uniform(800.0, 1000.0, s[::-1]),
        lambda s: rng.uniform(-5.0, 5.0, (3,) + s[::-1]), [0.767, 0.233, 0.0])
    prob.parts = _droplets(prob, rng, n, 20e-6, 0.3, lambda m: np.full(m, 300.0),
                           lambda m: np.ones((1, m)), vmax=40.0)
    return prob


CONFIGS = {"config1": config1, "config2": config2, "config3": config3,
           "config4": config4, "config5": config5, "walls": walls}


RU_CGS = 8.31446261815324e7   # erg/(mol K)


def internal_energy(mech, T, Y):
    """Mixture specific internal energy [erg/g] of the mechanism's NASA fits:
    sum_k Y_k (h_k(T) - R T / W_k), h_k = (R/W_k)(sum_n hc_n T^(n+1) + hc_5).
    T: array; Y: (nspec,) + T.shape."""
    e = np.zeros_like(T)
    for k in range(mech.nspec):
        a = [mech.hc[k][n] for n in range(6)]
        rw = RU_CGS / mech.mw[k]
        p = (((a[4] * T + a[3]) * T + a[2]) * T + a[1]) * T + a[0]
        e += Y[k] * ((p * T + a[5]) * rw - rw * T)
    return e


def to_pelec(prob, mech, guess_offset=-7.0):
    """The same flow and droplets restated for the PeleC coupling (CGS).

    The state keeps its component slots but holds rho*u [g/(cm^2 s)] in
    0..2, rho [g/cm^3] in 3, rho*Y in 4.., rho*E = rho (e(T, Y) + |u|^2/2)
    [erg/cm^3] in 4+NSP and T + guess_offset in 5+NSP: the stored temperature
    is only the starting guess of the EOS inversion, so the gathered gas
    temperature comes from the energy.  Lengths x 100, velocities x 100,
    liquid properties in CGS (Problem.inputs)."""
    ns = prob.nspec
    out = Problem(**{k: getattr(prob, k) for k in prob.__dataclass_fields__})
    out.name = prob.name + "_pelec"
    out.pelec = True
    out.plo = prob.plo * 100.0
    out.phi = prob.phi * 100.0
    out.dx = prob.dx * 100.0
    out.meta = dict(prob.meta)
    states = []
    for st in prob.state:
        rho = st[3] * 1e-3
        vel = st[0:3] * 100.0
        Y = st[4:4 + ns] / st[3]
        T = st[5 + ns]
        q = np.zeros_like(st)
        q[0:3] = rho * vel
        q[3] = rho
        q[4:4 + ns] = rho * Y
        q[4 + ns] = rho * (internal_energy(mech, T, Y) + 0.5 * np.sum(vel * vel, axis=0))
        q[5 + ns] = T + guess_offset
        states.append(np.ascontiguousarray(q))
    out.state = states
    nf = prob.nfuel
    parts = []
    for p in prob.parts:
        rd = p["rdata"].copy()
        rd[0:3] *= 100.0
        rd[capi.PSTATE_DIA] *= 100.0
        rd[capi.pstate_filmhght(nf)] *= 100.0
        parts.append(dict(pos=p["pos"] * 100.0, rdata=rd, id=p["id"].copy()))
    out.parts = parts
    return out
