"""Comparison helpers shared by the parity tests.

Tolerances (FP64 forms):
* droplet temperature, diameter: |a-b| <= 1e-12 |a|
* droplet velocity: |a-b| <= 1e-12 max(|u|, 1 m/s) (vector norm of the droplet's
  velocity; components near zero carry the absolute error of the whole vector)
* liquid mass fractions: |a-b| <= 1e-12 (they are in [0, 1])
* position: |a-b| <= 1e-12 dx
* cell indices, ids, box assignment: exact
* mesh sources: per component |a-b| <= 1e-12 max_cells |s| (deposits are
  summed with atomics in an unspecified order on the GPU)
"""
import numpy as np

from pelemp_b200 import capi

RTOL = 1e-12


def compare_parts(a, b, nfuel, dx, rtol=RTOL):
    """Return dict of max normalised errors between two per-box droplet lists."""
    out = {"T": 0.0, "dia": 0.0, "vel": 0.0, "Y": 0.0, "pos": 0.0, "id_mismatch": 0,
           "cell_mismatch": 0}
    for pa, pb in zip(a, b):
        ra, rb = pa["rdata"], pb["rdata"]
        alive = pa["id"] > 0
        out["id_mismatch"] += int(np.sum(pa["id"] != pb["id"]))
        for key, row in (("T", capi.PSTATE_T), ("dia", capi.PSTATE_DIA)):
            den = np.abs(ra[row])
            err = np.abs(ra[row] - rb[row]) / np.where(den > 0, den, 1.0)
            out[key] = max(out[key], float(np.max(err, initial=0.0)))
        speed = np.sqrt(np.sum(ra[0:3] ** 2, axis=0))
        verr = np.sqrt(np.sum((ra[0:3] - rb[0:3]) ** 2, axis=0)) / np.maximum(speed, 1.0)
        out["vel"] = max(out["vel"], float(np.max(verr, initial=0.0)))
        yerr = np.abs(ra[capi.PSTATE_Y:capi.PSTATE_Y + nfuel] - rb[capi.PSTATE_Y:capi.PSTATE_Y + nfuel])
        out["Y"] = max(out["Y"], float(np.max(yerr, initial=0.0)))
        perr = np.abs(pa["pos"] - pb["pos"]) / dx[:, None]
        out["pos"] = max(out["pos"], float(np.max(perr, initial=0.0)))
        ca = np.floor(pa["pos"] / dx[:, None])
        cb = np.floor(pb["pos"] / dx[:, None])
        out["cell_mismatch"] += int(np.sum(np.any(ca != cb, axis=0) & alive))
    return out


def assert_parts_close(a, b, nfuel, dx, rtol=RTOL):
    e = compare_parts(a, b, nfuel, dx, rtol)
    assert e["id_mismatch"] == 0, e
    assert e["cell_mismatch"] == 0, e
    for k in ("T", "dia", "vel", "Y", "pos"):
        assert e[k] <= rtol, (k, e)
    return e


def source_errors(sa, sb):
    worst = 0.0
    for a, b in zip(sa, sb):
        for c in range(a.shape[0]):
            scale = np.max(np.abs(a[c]))
            if scale == 0:
                assert np.max(np.abs(b[c])) == 0
                continue
            worst = max(worst, float(np.max(np.abs(a[c] - b[c])) / scale))
    return worst


def droplet_mass(prob, parts, rho_l):
    """Per-droplet liquid mass with constant liquid densities rho_l[f] (kg/m^3)."""
    out = []
    nf = prob.nfuel
    for p in parts:
        Y = p["rdata"][capi.PSTATE_Y:capi.PSTATE_Y + nf]
        inv_rho = np.sum(Y / np.asarray(rho_l)[:, None], axis=0)
        d = p["rdata"][capi.PSTATE_DIA]
        m = np.pi / 6.0 * d ** 3 / inv_rho
        m = np.where(p["id"] > 0, m, 0.0)
        out.append(m * p["rdata"][capi.pstate_numdens(nf)])
    return out


def liquid_enthalpy(prob, fdat, parts, rho_l):
    """Sum over live droplets of N m h_L, h_L = sum_f Y_f (cp_f (T - ref_T) - latent_f)
    (the liquid enthalpy the scheme's latent heat implies: L_f = h_f - h_L,f)."""
    nf = prob.nfuel
    masses = droplet_mass(prob, parts, rho_l)  # N m, zero for dead droplets
    total = 0.0
    for p, m in zip(parts, masses):
        Y = p["rdata"][capi.PSTATE_Y:capi.PSTATE_Y + nf]
        T = p["rdata"][capi.PSTATE_T]
        hL = np.zeros_like(T)
        for f in range(nf):
            hL += Y[f] * (fdat.cp[f] * (T - fdat.ref_T) - fdat.latent[f])
        total += float(np.sum(m * hL))
    return total


def gas_enthalpy_gain(prob, fdat, calls):
    """Enthalpy the gas receives from the energy deposits of the given calls
    (each call's source times cell volume times dtmod * flow_dt), and the same
    sum of magnitudes (the scale of the exchange)."""
    vol = float(np.prod(prob.dx))
    c = prob.comps().engSrcIndx
    gain, scale = 0.0, 0.0
    for call in calls:
        for s in call:
            gain += float(np.sum(s[c])) * vol * fdat.dtmod * prob.flow_dt
            scale += float(np.sum(np.abs(s[c]))) * vol * fdat.dtmod * prob.flow_dt
    return gain, scale


def energy_identity(prob, fdat, parts0, parts1, calls, residual, rho_l):
    """(liquid enthalpy change + gas enthalpy gain - sum of the scheme's
    residual terms) / exchange scale, and the residual / scale."""
    dH = liquid_enthalpy(prob, fdat, parts1, rho_l) - liquid_enthalpy(prob, fdat, parts0, rho_l)
    G, scale = gas_enthalpy_gain(prob, fdat, calls)
    R = float(sum(np.sum(r) for r in residual))
    return (dH + G - R) / scale, R / scale
