"""Raw-file exchange with the C++ driver (pelemp_b200/pmp_spray_driver).

write_problem(prob, dir): the layout documented in
pelemp_b200/csrc/host/spray_driver.cpp; read_result(prob, dir): the droplets
and summed deposits the driver wrote back.
"""
import ctypes as C
import os

import numpy as np

from . import capi
from .workloads import view_of


def write_problem(prob, d, steps=None):
    os.makedirs(d, exist_ok=True)
    with open(os.path.join(d, "meta.txt"), "w") as f:
        f.write(f"nspec {prob.nspec}\n")
        f.write("species " + " ".join(prob.species) + "\n")
        f.write(f"nfuel {prob.nfuel}\nnboxes {len(prob.boxes)}\n")
        f.write(f"steps {prob.steps if steps is None else steps}\n")
        f.write(f"flow_dt {prob.flow_dt!r}\nstate_ghosts {prob.state_ghosts}\n")
        f.write(f"source_ghosts {prob.source_ghosts}\nspray_cfl_lev {prob.spray_cfl_lev!r}\n")
    for name, obj in (("inputs", prob.inputs()), ("comps", prob.comps()),
                      ("geom", prob.geometry())):
        with open(os.path.join(d, name + ".bin"), "wb") as f:
            f.write(bytes(obj))
    with open(os.path.join(d, "boxes.bin"), "wb") as f:
        f.write(bytes(prob.box_array()))
    sv = (capi.BoxView * len(prob.boxes))()
    rv = (capi.BoxView * len(prob.boxes))()
    srcs = prob.new_sources()
    for b in range(len(prob.boxes)):
        v = view_of(prob.state[b], prob.grown(b, prob.state_ghosts)[0])
        v.p = None
        sv[b] = v
        w = view_of(srcs[b], prob.grown(b, prob.source_ghosts)[0])
        w.p = None
        rv[b] = w
        prob.state[b].astype(np.float64).tofile(os.path.join(d, f"state_{b}.bin"))
        p = prob.parts[b]
        p["pos"].tofile(os.path.join(d, f"pos_{b}.bin"))
        p["rdata"].tofile(os.path.join(d, f"rdata_{b}.bin"))
        p["id"].astype(np.int32).tofile(os.path.join(d, f"id_{b}.bin"))
    with open(os.path.join(d, "state_views.bin"), "wb") as f:
        f.write(bytes(sv))
    with open(os.path.join(d, "source_views.bin"), "wb") as f:
        f.write(bytes(rv))


def read_result(prob, d):
    parts, srcs = [], []
    shapes = [s.shape for s in prob.new_sources()]
    nr = capi.pstate_num(prob.nfuel)
    for b in range(len(prob.boxes)):
        n = prob.parts[b]["id"].shape[0]
        parts.append(dict(
            pos=np.fromfile(os.path.join(d, f"out_pos_{b}.bin")).reshape(3, n),
            rdata=np.fromfile(os.path.join(d, f"out_rdata_{b}.bin")).reshape(nr, n),
            id=np.fromfile(os.path.join(d, f"out_id_{b}.bin"), dtype=np.int32)))
        srcs.append(np.fromfile(os.path.join(d, f"out_src_{b}.bin")).reshape(shapes[b]))
    return parts, srcs
