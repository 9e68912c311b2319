"""Golden vectors of the spray update, made by the reference build.

The reference build (oracle/_ref: PeleMP's own Drag.H, SprayFuelData.H,
SprayInterpolation.H and WallFunctions.H compiled in this repository from the
reference sources, against the stand-in headers in oracle/ref_shim) runs
MKD + MK steps on small seeded workloads; the droplets after the last call
and every call's deposits (the non-zero entries) are written to
tests/golden/<case>.npz, with a SHA-256 of the inputs so that a change of the
workload generator is caught.  The committed files let the oracle be checked
against the reference where the reference sources are absent.

Usage (where oracle/_ref was built): python tests/golden/make_golden.py
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from pelemp_b200 import workloads as W  # noqa: E402

# (generator, arguments, PeleC coupling)
CASES = {
    "config1_n400": ("config1", dict(n=400, steps=3), False),
    "config2_n400": ("config2", dict(n=400, steps=2, ncells=(32, 32, 32), box=(16, 16, 16)), False),
    "walls_n400": ("walls", dict(n=400, steps=2), False),
    "pelec_config1_n400": ("config1", dict(n=400, steps=2), True),
}


def problem(name, mech_of):
    gen, kw, pelec = CASES[name]
    prob = W.CONFIGS[gen](**kw)
    if pelec:
        prob = W.to_pelec(prob, mech_of(prob.species))
    return prob, pelec


def input_digest(prob):
    h = hashlib.sha256()
    for s in prob.state:
        h.update(np.ascontiguousarray(s).tobytes())
    for p in prob.parts:
        for k in ("pos", "rdata", "id"):
            h.update(np.ascontiguousarray(p[k]).tobytes())
    h.update(repr((prob.flow_dt, prob.spray_cfl_lev, prob.state_ghosts, prob.source_ghosts)).encode())
    return h.hexdigest()


def run(lib, prob, mech, fdat):
    parts = prob.copy_parts()
    calls = []
    for _ in range(prob.steps):
        for do_move in (1, 0):
            src = prob.new_sources()
            rc, err, _ = lib.update(prob, mech, fdat, parts, src, do_move)
            assert rc == 0, (rc, err.message)
            calls.append(src)
    return parts, calls


def pack(parts, calls):
    out = {}
    for b, p in enumerate(parts):
        for k in ("pos", "rdata", "id"):
            out[f"b{b}_{k}"] = p[k]
    for c, src in enumerate(calls):
        for b, s in enumerate(src):
            flat = s.reshape(-1)
            nz = np.flatnonzero(flat)
            out[f"c{c}_b{b}_idx"] = nz.astype(np.int64)
            out[f"c{c}_b{b}_val"] = flat[nz]
    return out


def unpack_sources(g, prob, ncalls):
    """Dense per-call, per-box source arrays from a golden file."""
    calls = []
    for c in range(ncalls):
        src = prob.new_sources()
        for b, s in enumerate(src):
            s.reshape(-1)[g[f"c{c}_b{b}_idx"]] = g[f"c{c}_b{b}_val"]
        calls.append(src)
    return calls


def main():
    from oracle.pyoracle import Oracle, Reference
    for name, (_, _, pelec) in CASES.items():
        orc = Oracle(libm=True, pelec=pelec)
        prob, _ = problem(name, orc.mech)
        if not Reference.available(prob.nspec, prob.nfuel, pelec=pelec):
            raise SystemExit("the reference build (oracle/_ref) is missing")
        ref = Reference(prob.nspec, prob.nfuel, pelec=pelec)
        mech = orc.mech(prob.species)
        rc, fdat = orc.setup(prob, mech)
        assert rc == 0
        parts, calls = run(ref, prob, mech, fdat)
        out = pack(parts, calls)
        out["input_sha256"] = np.array(input_digest(prob))
        out["ncalls"] = np.array(len(calls))
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        print(name, "calls", len(calls), "droplets", sum(p["id"].size for p in parts))


if __name__ == "__main__":
    main()
