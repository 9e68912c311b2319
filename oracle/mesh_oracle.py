"""CPU oracle of the operations around the update (numpy restatement).

Test infrastructure: only the tests use this module, to check
pmp_spray_est_timestep, pmp_spray_derive, pmp_spray_transfer_source and
pmp_spray_redistribute.  Each function follows the reference lines it cites.
Arrays are per box (ncomp, nz, ny, nx) with a lower corner `lo` (x, y, z);
droplets are dicts pos (3, n), rdata (10+F, n), id (n,).
"""
import numpy as np

PSTATE_VEL, PSTATE_T, PSTATE_DIA, PSTATE_Y = 0, 3, 4, 5


def est_timestep(parts, dx, cfl, max_jet_vel=0.0, fixed_parts=False):
    """SprayParticleContainer::estTimestep, SprayParticles.cpp:89-140."""
    if fixed_parts:
        return -1.0
    dxi = 1.0 / np.asarray(dx, np.float64)
    dt = np.finfo(np.float64).max
    for p in parts:
        if p["id"].size == 0:
            continue
        v = np.abs(p["rdata"][PSTATE_VEL:PSTATE_VEL + 3]) * dxi[:, None]
        mv = np.max(v, axis=0)
        with np.errstate(divide="ignore"):
            dtp = np.where(mv > 0.0, cfl / np.where(mv > 0.0, mv, 1.0), 1.0e50)
        dtp = np.where(p["id"] > 0, dtp, -1.0)
        dt = min(dt, float(np.min(dtp)))
    if max_jet_vel > 0.0:
        dt = min(dt, cfl * dx[0] / max_jet_vel)
    return dt


def cells_of(pos, plo, dx):
    """floor((x - plo) * (1/dx)), SprayDerive.cpp:87-88 / SprayParticles.cpp:340-343."""
    dxi = 1.0 / np.asarray(dx, np.float64)
    return np.floor((pos - np.asarray(plo)[:, None]) * dxi[:, None]).astype(np.int64)


def derive(parts, views, los, start, nfuel, with_species, rho_coef, plo, dx):
    """computeDerivedVars, SprayDerive.cpp:9-155 (3D, no EB).  views[b] is
    modified in place (the caller zeroes it first)."""
    dx = np.asarray(dx, np.float64)
    cell_vol = dx[0] * dx[1] * dx[2]
    face_area = dx[0] * dx[0]
    species = with_species and nfuel > 1
    for p, V, lo in zip(parts, views, los):
        live = p["id"] > 0
        r = p["rdata"][:, live]
        c = cells_of(p["pos"][:, live], plo, dx)
        ii, jj, kk = c[0] - lo[0], c[1] - lo[1], c[2] - lo[2]
        T = r[PSTATE_T]
        d = r[PSTATE_DIA]
        inv = np.zeros_like(T)
        for f in range(nfuel):
            a, b, cc, dd = rho_coef[4 * f:4 * f + 4]
            inv += r[PSTATE_Y + f] / (a + T * (b + T * (cc + T * dd)))
        rho = 1.0 / inv
        surf = np.pi * d * d
        vol = np.pi / 6.0 * (d * d * d)
        pmass = vol * rho
        num = r[5 + nfuel]
        film = r[9 + nfuel]
        dep = film == 0.0

        def add(comp, val, sel):
            np.add.at(V[start + comp], (kk[sel], jj[sel], ii[sel]), val[sel])
        add(0, num * pmass, dep)
        add(1, num * pmass / cell_vol, dep)
        add(2, num, dep)
        add(3, num * vol, dep)
        add(4, num * surf, dep)
        add(5, num * vol / cell_vol, dep)
        add(6, num * d, dep)
        add(7, num * vol * 6.0, dep)
        add(10, num * pmass * T, dep)
        add(11, np.ones_like(num), dep)
        for q in range(3):
            add(12 + q, num * pmass * r[PSTATE_VEL + q], dep)
        if species:
            for f in range(nfuel):
                add(15 + f, r[PSTATE_Y + f] * pmass, dep)
        fl = ~dep
        rad2 = (0.5 * d) ** 2
        cur_vol = np.pi / 6.0 * film * (3.0 * rad2 + film * film)
        add(8, cur_vol / face_area, fl)
        add(9, rho * cur_vol, fl)
        for den, numr in ((2, 6), (4, 7), (0, 10), (0, 12), (0, 13), (0, 14)):
            D = V[start + den]
            nz = D != 0.0
            V[start + numr][nz] = V[start + numr][nz] / D[nz]


def transfer_source(tmp, tmp_lo, act, act_lo, boxes, domain_lo, domain_hi, periodic, g, act_ghosts,
                    comps=None, nfuel=0, dep_indx=()):
    """transferSource level 0, SprayParticles.H:250-295: SumBoundary (ghost
    cells add into the valid cell owning their periodically wrapped location;
    ghost cells keep their values), act += tmp over boxes grown by
    min(act_ghosts, g) (all components, or addSpraySrc's mapping,
    SprayParticles.H:299-319, when the component counts differ), tmp = 0.
    Arrays are modified in place."""
    dlo = np.asarray(domain_lo)
    n = np.asarray(domain_hi) - dlo + 1
    owner = {}
    for b, (lo, hi) in enumerate(boxes):
        owner[b] = (np.asarray(lo), np.asarray(hi))
    orig = [t.copy() for t in tmp]
    for b, (lo, hi) in enumerate(boxes):
        lo, hi = np.asarray(lo), np.asarray(hi)
        glo, ghi = lo - g, hi + g
        zz, yy, xx = np.meshgrid(np.arange(glo[2], ghi[2] + 1), np.arange(glo[1], ghi[1] + 1),
                                 np.arange(glo[0], ghi[0] + 1), indexing="ij")
        cells = np.stack([xx.ravel(), yy.ravel(), zz.ravel()])
        valid = np.all((cells >= lo[:, None]) & (cells <= hi[:, None]), axis=0)
        cells = cells[:, ~valid]
        w = cells.copy()
        keep = np.ones(w.shape[1], dtype=bool)
        for d in range(3):
            r = w[d] - dlo[d]
            if periodic[d]:
                r = np.mod(r, n[d])
            else:
                keep &= (r >= 0) & (r < n[d])
            w[d] = dlo[d] + r
        cells, w = cells[:, keep], w[:, keep]
        src = orig[b][:, cells[2] - tmp_lo[b][2], cells[1] - tmp_lo[b][1], cells[0] - tmp_lo[b][0]]
        for o, (olo, ohi) in owner.items():
            sel = np.all((w >= olo[:, None]) & (w <= ohi[:, None]), axis=0)
            if not sel.any():
                continue
            tl = tmp_lo[o]
            for comp in range(tmp[o].shape[0]):
                np.add.at(tmp[o][comp], (w[2, sel] - tl[2], w[1, sel] - tl[1], w[0, sel] - tl[0]),
                          src[comp, sel])
    ng = min(act_ghosts, g)
    for b, (lo, hi) in enumerate(boxes):
        lo, hi = np.asarray(lo), np.asarray(hi)
        sl_t = tuple(slice(lo[d] - ng - tmp_lo[b][d], hi[d] + ng + 1 - tmp_lo[b][d]) for d in (2, 1, 0))
        sl_a = tuple(slice(lo[d] - ng - act_lo[b][d], hi[d] + ng + 1 - act_lo[b][d]) for d in (2, 1, 0))
        if act[b].shape[0] == tmp[b].shape[0]:
            act[b][(slice(None),) + sl_a] += tmp[b][(slice(None),) + sl_t]
        else:
            c = comps
            for q in range(3):
                act[b][(c.momIndx + q,) + sl_a] += tmp[b][(c.momSrcIndx + q,) + sl_t]
            act[b][(c.rhoIndx,) + sl_a] += tmp[b][(c.rhoSrcIndx,) + sl_t]
            act[b][(c.engIndx,) + sl_a] += tmp[b][(c.engSrcIndx,) + sl_t]
            for f in range(nfuel):
                act[b][(c.specIndx + dep_indx[f],) + sl_a] += tmp[b][(c.specSrcIndx + f,) + sl_t]
    for t in tmp:
        t[...] = 0.0


def redistribute(parts, boxes, plo, phi, dx, domain_lo, domain_hi, periodic):
    """Re-binning after a move as pmp_spray_redistribute restates AMReX's
    Redistribute: periodic wrap (while x >= phi: x -= L; while x < plo: x += L),
    box = the one whose valid region holds floor((x - plo)/dx), droplets with
    id <= 0 or in no box dropped.  Returns new per-box dicts ordered by id."""
    allp = {k: np.concatenate([p[k] for p in parts], axis=-1) for k in ("pos", "rdata", "id")}
    live = allp["id"] > 0
    pos = allp["pos"][:, live].copy()
    for d in range(3):
        if periodic[d]:
            L = phi[d] - plo[d]
            x = pos[d]
            for _ in range(64):
                m = x >= phi[d]
                if not m.any():
                    break
                x[m] = x[m] - L
            for _ in range(64):
                m = x < plo[d]
                if not m.any():
                    break
                x[m] = x[m] + L
    c = cells_of(pos, plo, dx)
    dlo = np.asarray(domain_lo)
    n = np.asarray(domain_hi) - dlo + 1
    for d in range(3):
        r = c[d] - dlo[d]
        if periodic[d]:
            r = np.mod(r, n[d])
        c[d] = dlo[d] + r
    box_of = np.full(pos.shape[1], -1)
    for b, (lo, hi) in enumerate(boxes):
        inside = np.all((c >= np.asarray(lo)[:, None]) & (c <= np.asarray(hi)[:, None]), axis=0)
        box_of[inside] = b
    rdata, ids = allp["rdata"][:, live], allp["id"][live]
    out = []
    for b in range(len(boxes)):
        sel = np.nonzero(box_of == b)[0]
        sel = sel[np.argsort(ids[sel], kind="stable")]
        out.append({"pos": pos[:, sel], "rdata": rdata[:, sel], "id": ids[sel]})
    return out
