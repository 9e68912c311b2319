"""Benchmark of the spray particle update (droplet-substeps/s).

Workload (one GPU, per rank): 16M two-component droplets (n-decane/n-heptane)
on a 128^3 mesh of 8 boxes of 64^3, gas [N2, O2, NC10H22, NC7H16, CO2],
dt = 5e-7 s, spray_cfl_lev = 2 (MKD runs 4 sub-cycles).  One step is what a
PeleLMeX time step asks of the spray container: zero the source
(transferSource's setVal), moveKickDrift (4 sub-cycles, moving), moveKick
(1 sub-cycle) -- 5 droplet-substeps per live droplet.  A droplet-substep is
one execution of the sub-cycle body SprayParticles.cpp:357-480.

Arms
* default: the B200 library, inputs resident in HBM, in three forms timed on
  the same initial droplets: plain FP64, mixed (FP32 physics, FP64 state and
  deposits) and learned (surrogate trained first, untimed, on tuples the FP64
  teacher labels from a sample of the workload).  ``value`` is the fastest
  non-FP64 form; ``forms`` lists every form with its speed-up over FP64 and
  its per-droplet error against the FP64 form (bit-identical to the FP64
  oracle) after all steps.  ``e2e``: the headline form's steps through
  pmp_spray_update_host with the mesh state and source in pinned host memory
  (copies inside the timed region).  ``other_workloads`` (N=1, default
  sizes): the figures of configs 3, 4 and 5, each from a run of this script
  in its own process.  ``operations``: the time-step estimate, derived
  fields, source transfer and re-binning on the config-2 workload (device
  time, algorithmic bytes, HBM fraction; their numpy oracle on one core
  beside them).
* --impl reference: PeleMP's own spray physics headers (oracle/_ref, built
  from the reference sources) on the host cores, OpenMP over droplets, on a
  bounded random sample of the same workload.

Multi-GPU: one process per GPU (torchrun); each rank runs its own replica of
the workload (boxes are independent; no collective on the data path), time
is the max over ranks.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

FALLBACK_HBM_GBS = 6650.0


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.file = None

    def start(self):
        try:
            self.file = tempfile.NamedTemporaryFile("w+", delete=False, suffix=".csv")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.file, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": []}
        if self.proc is None:
            return out
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.file.flush()
        self.file.seek(0)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.file.read().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        self.file.close()
        os.unlink(self.file.name)
        if sm:
            out["sm_mhz"] = float(np.median(sm))
            out["sm_max_mhz"] = float(max(smax))
            out["samples"] = len(sm)
        out["reasons"] = sorted(reasons)
        return out


def algorithmic_bytes(n_live, nfuel, nspec, ncells, do_move):
    """Compulsory bytes of one update call: droplet reads/writes + mesh state
    read + source read-modify-write.  R_p = 8(10+F)+8, W_p = 8(8+F) (MKD) or
    8(5+F) (MK); per cell 8(5+NSP) state bytes and 16(5+F) source bytes."""
    rp = 8 * (10 + nfuel) + 8
    wp = 8 * (8 + nfuel) if do_move else 8 * (5 + nfuel)
    return n_live * (rp + wp) + ncells * (8 * (5 + nspec) + 16 * (5 + nfuel))


def reduce_over_ranks(pg, t_ms, count, device="cuda"):
    """Whole-job timing of replicas: the max of the ranks' timed milliseconds
    and the sum of their work (unchanged without a process group)."""
    if not pg:
        return t_ms, count
    import torch
    tt = torch.tensor([t_ms], device=device, dtype=torch.float64)
    pg.all_reduce(tt, op=pg.ReduceOp.MAX)
    nn = torch.tensor([float(count)], device=device, dtype=torch.float64)
    pg.all_reduce(nn, op=pg.ReduceOp.SUM)
    return float(tt.item()), int(nn.item())


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def _reference_lib(nspec, nfuel):
    """The reference's CPU path (oracle/_ref, PeleMP's spray physics headers
    compiled from the reference sources) or, without it, the C oracle."""
    from oracle.pyoracle import Oracle, Reference
    if Reference.available(nspec, nfuel):
        return Reference(nspec, nfuel), "reference", (
            "PeleMP Drag.H/SprayFuelData.H/SprayInterpolation.H/WallFunctions.H compiled from the "
            "reference sources (oracle/_ref), project thermo/transport, OpenMP over droplets with "
            "atomic deposits")
    return Oracle(libm=True), "port", "CPU oracle (C restatement of the reference path, C library math), OpenMP"


def cpu_sample_size(seconds):
    """Droplets of the config-2 workload whose MKD+MK step takes about `seconds`
    of the reference's CPU path on this host (all cores), at most 4M."""
    from pelemp_b200 import workloads as W
    from oracle.pyoracle import Oracle
    cores = os.cpu_count() or 1
    probe = W.config2(n=20_000, steps=1)
    lib, _, _ = _reference_lib(probe.nspec, probe.nfuel)
    orc = Oracle(libm=True)
    mech = orc.mech(probe.species)
    _, fdat = orc.setup(probe, mech)
    src = probe.new_sources()
    parts = probe.copy_parts()
    t0 = time.perf_counter()
    for do_move in (1, 0):
        for a in src:
            a.fill(0.0)
        rc, err, _ = lib.update(probe, mech, fdat, parts, src, do_move, nthreads=cores)
        assert rc == 0, err.message
    dt = time.perf_counter() - t0
    return int(min(4_000_000, max(20_000, 20_000 * seconds / max(dt, 1e-3))))


def time_reference_steps(n, steps, warmup):
    """The reference's CPU path on n droplets of the config-2 workload: warmup
    + steps MKD+MK steps from the same initial droplets, the source arrays
    allocated (and faulted in) before the timed region and zeroed inside it,
    as the GPU step zeroes its sources.  Returns (substeps/s, seconds per
    timed step, cores, kind, description)."""
    from pelemp_b200 import workloads as W
    from oracle.pyoracle import Oracle
    cores = os.cpu_count() or 1
    prob = W.config2(n=n, steps=1)
    lib, kind, desc = _reference_lib(prob.nspec, prob.nfuel)
    orc = Oracle(libm=True)
    mech = orc.mech(prob.species)
    _, fdat = orc.setup(prob, mech)
    src = prob.new_sources()
    for a in src:
        a.fill(1.0)  # fault the pages in outside the timed region
    total_sub, t_total = 0, 0.0
    for step in range(warmup + steps):
        parts = prob.copy_parts()
        t0 = time.perf_counter()
        nsub = 0
        for do_move in (1, 0):
            for a in src:
                a.fill(0.0)
            rc, err, ns = lib.update(prob, mech, fdat, parts, src, do_move, nthreads=cores)
            assert rc == 0, err.message
            nsub += ns
        dt = time.perf_counter() - t0
        if step >= warmup:
            total_sub += nsub
            t_total += dt
    return total_sub / t_total, t_total / max(steps, 1), cores, kind, desc


def run_reference(args, world, rank):
    """PeleMP's spray physics (oracle/_ref) on the host cores, bounded sample."""
    if rank != 0:
        return None
    n = args.cpu_sample or cpu_sample_size(args.cpu_seconds)
    value, s_per_step, cores, kind, desc = time_reference_steps(n, args.steps, args.warmup)
    line = {
        "metric": "droplet-substeps/s", "value": value, "unit": "droplet-substeps/s",
        "impl": "reference", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * s_per_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded config-2 sample)",
        "config": {"workload": "config2 sample: two-fuel droplets on 128^3 (8 boxes of 64^3), "
                               "5 species, dt=5e-7 s, MKD (4 sub-cycles) + MK",
                   "droplets_per_step": n},
        "cpu_baseline": {"value": value, "unit": "droplet-substeps/s", "cores": cores,
                         "kind": kind,
                         "sample": f"{n} droplets of the 16M config-2 workload per step "
                                   f"(the same sample size as the GPU arm's cpu_baseline), "
                                   f"{args.warmup} + {args.steps} steps; {desc}"},
        "e2e": {"value": value, "unit": "droplet-substeps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    return line


def cpu_baseline(args):
    """The reference's CPU path on a bounded sample, for rank 0 at N=1: one
    MKD+MK step (after one untimed step) of the sample the reference arm uses."""
    n = args.cpu_sample or cpu_sample_size(args.cpu_seconds)
    value, s_per_step, cores, kind, desc = time_reference_steps(n, 1, 1)
    return {"value": value, "unit": "droplet-substeps/s", "cores": cores, "kind": kind,
            "sample": (f"{n} droplets of the config-2 workload, one timed MKD+MK step "
                       f"({s_per_step:.1f} s) after one untimed; {desc}")}


WORKLOAD_TEXT = {
    "config2": "config2: {n:.0f}M two-fuel droplets (decane/heptane), 128^3 mesh as 8 boxes of 64^3, "
               "5 gas species, dt=5e-7 s, MKD 4 sub-cycles + MK 1 sub-cycle per step",
    "config4": "config4: {n:.0f}M heptane droplets with config-1 distributions, 256x128x128 mesh as "
               "8 boxes of 64^3, 3 gas species, dt=1e-6 s, MKD + MK (1 sub-cycle each) per step",
    "config5": "config5: {n:.0f}M heptane droplets with config-1 distributions, 256x128x128 mesh as "
               "8 boxes of 64^3, 3 gas species, dt=1e-6 s, MKD + MK (1 sub-cycle each) per step",
    "config3": "config3: {n:.0f}M heptane droplets in 256 boxes of 32^3 (256x256x128 cells) with "
               "capped-Zipf counts, config-1 physics, MKD + MK per step, FP64",
}
FORM_MODE = {"fp64": 0, "mixed": 1, "learned": 2}
# the library's kernels one update call launches (MKD and MK alike):
# FP64: gas records + update; mixed: gas records + small-droplet selection +
# update + FP64 list kernel (side stream); learned: the same + the FP64 kernel
# over the droplets its gate rejected
KERNELS_PER_CALL = {"fp64": 2, "mixed": 4, "learned": 5}
FORM_NAME = {"fp64": "plain FP64", "mixed": "mixed FP32 physics / FP64 state and deposits",
             "learned": "learned surrogate (bf16 MLP on tensor cores) + FP32 physics / FP64 state"}
KERNEL = {"fp64": "spray_update_fp64<5,2,128>", "mixed": "spray_update_mixed<5,2,128,fuel_first>",
          "learned": "spray_update_learned<5,2,128,fuel_first>"}
# DRAM bytes per droplet of one config-2 MKD launch, measured by ncu on a
# 2M-droplet launch of the same kernel at config-2 density (64^3 mesh, 7-8
# droplets per cell; one-launch capture): dram read + write minus the mesh's
# algorithmic bytes (state read once, source read-modify-write), divided by
# the droplets.  The droplet part grows with the droplet count, the mesh part
# does not, so a full launch's traffic is estimated as mesh bytes + droplets
# x this.  The mixed and learned kernels move less than the 184 algorithmic
# bytes per droplet: their gathers read the FP32 gas records (written by a
# separate pass) instead of the FP64 state.
DRAM_BYTES_PER_DROPLET = {"fp64": 175.6, "mixed": 158.3, "learned": 153.6}
# Pipe utilisation of each form's update kernel in the same captures (% of
# the pipe's peak while the SM is active: sm__inst_executed_pipe_*; issue:
# smsp__issue_active), and its measured pipe peaks: the compute side of the
# roofline.  The kernels are bound by instruction issue and latency, not by
# one pipe.
PIPE_PCT = {
    "mixed": {"issue": 60.23, "xu": 39.97, "fma": 23.11, "alu": 23.52, "fp64": 11.94, "lsu": 16.02,
              "tensor": 0.0},
    "fp64": {"issue": 47.17, "xu": 13.48, "fma": 6.19, "alu": 16.31, "fp64": 32.35, "lsu": 9.86,
             "tensor": 0.0},
    "learned": {"issue": 47.10, "xu": 38.67, "fma": 16.86, "alu": 19.74, "fp64": 7.84, "lsu": 10.02,
                "tensor": 5.41},
}


def compute_roofline(form, peaks):
    """The compute side of the roofline of the form's update kernel: the
    measured pipe peaks of this GPU and the kernel's pipe utilisation."""
    out = {"pipes_pct_of_peak": PIPE_PCT.get(form),
           "pipes_source": "ncu capture of the same kernel: one MKD launch of 2M droplets at config-2 density "
                           "(sm__inst_executed_pipe_*.avg.pct_of_peak_sustained_active, "
                           "smsp__issue_active, sm__pipe_tensor_cycles_active), taken before the FP64 "
                           "divisions of the FP32 forms' state update were cut and the mixed form's B_T "
                           "fixed point stopped at its noise floor (the mixed MKD launch is 17 % shorter "
                           "since)"}
    if peaks is not None:
        out["peaks"] = peaks
        out["peaks_source"] = ("pmp_measure_peaks on this GPU: loop kernels of independent DFMA, FFMA and "
                               "ex2.approx, best of three launches")
    return out


def train_surrogate(sp, prob, st_v, src_v, stream, args):
    """Tuples labelled by the plain FP64 teacher along the workload's own
    trajectory: every learn_gap steps (advanced by the FP64 form) for
    learn_gens states, a sample of the droplets (every learn_stride-th, plus 3
    perturbed copies of each); then GPU training, and the initial droplets
    put back.  Returns (seconds, report, tuples)."""
    from pelemp_b200 import capi
    t0 = time.perf_counter()
    sp.set_mode(capi.PMP_MODE_FP64)
    for g in range(args.learn_gens):
        sp.learn_generate(st_v, prob.flow_dt, prob.state_ghosts, True, prob.spray_cfl_lev,
                          sample_stride=args.learn_stride, augment=3, seed=7 + g, stream=stream)
        if g + 1 < args.learn_gens:
            for _ in range(args.learn_gap):
                for do_move in (1, 0):
                    sp.update_particles(st_v, src_v, prob.flow_dt, 0.0, prob.state_ghosts,
                                        prob.source_ghosts, 0, 0, do_move, prob.spray_cfl_lev, stream,
                                        sync=False)
            # re-bin the moved droplets to their boxes (periodic wrap), as the
            # flow solver's step does, so the trajectory can run any length
            sp.sync()
            sp.redistribute(stream)
    sp.sync()
    tuples = sp.learn_count()
    rep = sp.learn_train(epochs=args.learn_epochs, batch=4096, audit_fraction=0.0)
    for b, p in enumerate(prob.parts):
        sp.set_particles(b, p["pos"], p["rdata"], p["id"])
    sp.set_mode(capi.PMP_MODE_LEARNED)
    return time.perf_counter() - t0, rep, tuples


def droplet_errors(pa, pb, prob):
    """Per-droplet relative errors of pa vs pb: temperature, diameter, liquid mass
    (d^3 / sum(Y/rho_l)) and velocity (|du| / max(|u|, 1 m/s))."""
    from pelemp_b200 import workloads as W
    nfuel = prob.nfuel
    rho = np.array([W.LIQUIDS[f]["rho"] for f in prob.fuels])
    e = {"T": [], "dia": [], "mass": [], "vel": []}
    for a, b in zip(pa, pb):
        al = (a["id"] > 0) & (b["id"] > 0)
        ra, rb = a["rdata"][:, al], b["rdata"][:, al]
        e["T"].append(np.abs(ra[3] / rb[3] - 1))
        e["dia"].append(np.abs(ra[4] / rb[4] - 1))

        def mass(r):
            return r[4] ** 3 / np.sum(r[5:5 + nfuel] / rho[:, None], axis=0)
        e["mass"].append(np.abs(mass(ra) / mass(rb) - 1))
        speed = np.maximum(np.sqrt(np.sum(rb[0:3] ** 2, axis=0)), 1.0)
        e["vel"].append(np.sqrt(np.sum((ra[0:3] - rb[0:3]) ** 2, axis=0)) / speed)

    def q(v):
        v = np.concatenate(v)
        return {"rms": float(np.sqrt(np.mean(v ** 2))), "p99_9": float(np.quantile(v, 0.999)),
                "max": float(v.max())}
    out = {k: q(v) for k, v in e.items()}
    out["droplets"] = int(sum(x.size for x in e["T"]))
    return out


def deposit_errors(sa, sb, prob):
    """Per source component (momentum, density, fuel species, energy): the
    largest |sa - sb| over the cells as a fraction of the largest |sb|."""
    c = prob.comps()
    names = {c.momSrcIndx + d: "mom_" + "xyz"[d] for d in range(3)}
    names[c.rhoSrcIndx] = "mass"
    names[c.engSrcIndx] = "energy"
    for f in range(prob.nfuel):
        names[c.specSrcIndx + f] = "species_" + prob.fuels[f]
    out = {}
    for k, name in names.items():
        scale = float(np.max(np.abs(sb[k])))
        out[name] = float(np.max(np.abs(sa[k] - sb[k]))) / scale if scale > 0 else 0.0
    return out


def step_balance(prob, fdat, p0, p1, src, rho_l):
    """Liquid + gas balances of one step of the droplets of one box (p0 -> p1,
    deposits src): mass (gas gain + liquid change) / |liquid change|, and the
    liquid enthalpy change plus the enthalpy the gas receives, over the sum of
    the exchanged magnitudes (the explicit scheme's own energy residual: not
    zero by construction, the FP64 form's value is the reference)."""
    nf = prob.nfuel
    c = prob.comps()
    vol = float(np.prod(prob.dx))
    tau = fdat.dtmod * prob.flow_dt

    def liquid(p):
        Y = p["rdata"][5:5 + nf]
        m = np.pi / 6 * p["rdata"][4] ** 3 / np.sum(Y / np.asarray(rho_l)[:, None], axis=0)
        m = np.where(p["id"] > 0, m, 0.0) * p["rdata"][5 + nf]
        hL = sum(Y[f] * (fdat.cp[f] * (p["rdata"][3] - fdat.ref_T) - fdat.latent[f]) for f in range(nf))
        return float(np.sum(m)), float(np.sum(m * hL))
    m0, h0 = liquid(p0)
    m1, h1 = liquid(p1)
    gas_m = float(np.sum(src[c.rhoSrcIndx])) * vol * tau
    gas_e = float(np.sum(src[c.engSrcIndx])) * vol * tau
    scale_e = float(np.sum(np.abs(src[c.engSrcIndx]))) * vol * tau
    return {"mass": (gas_m + m1 - m0) / abs(m1 - m0), "energy": (gas_e + h1 - h0) / scale_e}


def bench_batched(args, world, rank, local, pg):
    """Config 3: the FP64 form over 256 uneven boxes -- the default launch, the
    autotuned launch (replayed from a CUDA graph) and one launch per box."""
    import torch
    from pelemp_b200 import capi
    from pelemp_b200 import workloads as W
    from pelemp_b200.spray import from_problem, views
    prob = W.config3(total=args.droplets or 16_000_000, seed=rank, steps=args.steps)
    nboxes = len(prob.boxes)
    stream = torch.cuda.current_stream()
    st = [torch.from_numpy(s).cuda() for s in prob.state]
    st_v = views(st, [prob.grown(b, prob.state_ghosts)[0] for b in range(nboxes)])
    src = [torch.zeros(s.shape, dtype=torch.float64, device="cuda") for s in prob.new_sources()]
    src_v = views(src, [prob.grown(b, prob.source_ghosts)[0] for b in range(nboxes)])

    def step(sp, st_handle):
        for s in src:
            s.zero_()
        for do_move in (1, 0):
            sp.update_particles(st_v, src_v, prob.flow_dt, 0.0, prob.state_ghosts, prob.source_ghosts,
                                0, 0, do_move, prob.spray_cfl_lev, st_handle, sync=False)

    def timed(sp, steps, whole_graph=False):
        """Eager steps, or replays of one CUDA graph of a whole step; returns
        (droplet-substeps/s, ms per step)."""
        for _ in range(args.warmup):
            step(sp, stream.cuda_stream)
        sp.sync()
        run = lambda: step(sp, stream.cuda_stream)  # noqa: E731
        g = None
        if whole_graph:
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                step(sp, torch.cuda.current_stream().cuda_stream)
            run = g.replay
        if pg:
            pg.barrier()
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(steps):
            run()
        ev1.record(stream)
        torch.cuda.synchronize()
        sp.sync()
        n = sp.stats().substeps
        del g
        t, n = reduce_over_ranks(pg, ev0.elapsed_time(ev1), n)
        return n / (t * 1e-3), t / steps

    # each phase starts from the initial droplets (no re-binning inside the
    # timed steps: the ghost widths cover the drift of warmup + steps steps)
    sp = from_problem(prob, device=local)
    v_default, ms_default = timed(sp, args.steps)
    sp.close()
    sp = from_problem(prob, device=local)
    v_default_g, ms_default_g = timed(sp, args.steps, whole_graph=True)
    sp.close()
    sp = from_problem(prob, device=local)
    rep = sp.autotune(st_v, src_v, prob.flow_dt, prob.state_ghosts, prob.source_ghosts, 0, 1,
                      prob.spray_cfl_lev, stream=stream.cuda_stream)
    best = rep.best
    sp.close()
    # the tuned shape, each call replaying the library's graph of its device work
    sp = from_problem(prob, device=local)
    sp.set_launch(kind=best.kind, block=best.block, regs=best.regs, chunk=best.chunk,
                  ctas_per_sm=best.ctas_per_sm, use_graph=True)
    v_call_g, ms_call_g = timed(sp, args.steps)
    sp.close()
    # the tuned shape inside one CUDA graph of the whole step (the headline)
    sp = from_problem(prob, device=local)
    sp.set_launch(kind=best.kind, block=best.block, regs=best.regs, chunk=best.chunk,
                  ctas_per_sm=best.ctas_per_sm, use_graph=False)
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    v_tuned, ms_tuned = timed(sp, args.steps, whole_graph=True)
    clocks = sampler.stop()
    sp.close()
    sp = from_problem(prob, device=local)
    sp.set_launch(kind=capi.PMP_LAUNCH_PER_BOX)
    v_box, ms_box = timed(sp, max(2, args.steps // 5))
    if rank == 0:
        line = {
            "metric": "droplet-substeps/s", "value": v_tuned, "unit": "droplet-substeps/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_tuned,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded, numpy PCG64)",
            "config": {"workload": WORKLOAD_TEXT["config3"].format(n=prob.n_droplets / 1e6),
                       "droplets_per_gpu": prob.n_droplets, "boxes": nboxes,
                       "largest_box": int(max(prob.meta["counts"])), "smallest_box": int(min(prob.meta["counts"])),
                       "parallelism": f"replicas x{world}"},
            "launches": {
                "autotuned_step_graph": {"value": v_tuned, "ms_per_step": ms_tuned,
                                         "what": "tuned shape, one CUDA graph of the whole step replayed",
                                         "shape": {"kind": best.kind, "block": best.block, "regs": best.regs,
                                                   "chunk": best.chunk},
                                         "tuner": {"candidates": rep.ncandidates, "best_ms": rep.best_ms,
                                                   "default_ms": rep.default_ms,
                                                   "per_box_ms": rep.per_box_ms}},
                "autotuned_call_graphs": {"value": v_call_g, "ms_per_step": ms_call_g,
                                          "what": "tuned shape, eager steps, each call replaying the "
                                                  "library's graph of its device work"},
                "default_one_launch": {"value": v_default, "ms_per_step": ms_default,
                                       "what": "default shape, eager steps"},
                "default_step_graph": {"value": v_default_g, "ms_per_step": ms_default_g,
                                       "what": "default shape, one CUDA graph of the whole step"},
                "per_box_baseline": {"value": v_box, "ms_per_step": ms_box,
                                     "what": "one launch per box, stream synchronised after each "
                                             "(SprayParticles.cpp:244-248,499)"},
                "speedup_vs_per_box": v_tuned / v_box},
            # the headline (autotuned) run: gas records + update per call
            "gpu_launches": 2 * args.steps * KERNELS_PER_CALL["fp64"],
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    sp.close()
    if pg:
        pg.destroy_process_group()


def pcie_rates(host_in, host_out, stream, reps=3):
    """Host<->device copy rates of the e2e path's pinned arrays, copied with
    no update beside them: host-to-device, device-to-host, and both at once
    on two streams (GB/s per direction, from CUDA events)."""
    import torch
    din = [torch.empty(a.shape, dtype=torch.float64, device="cuda") for a in host_in]
    dout = [torch.zeros(a.shape, dtype=torch.float64, device="cuda") for a in host_out]
    tin = [torch.from_numpy(a) for a in host_in]
    tout = [torch.from_numpy(a) for a in host_out]
    b_in = sum(a.nbytes for a in host_in)
    b_out = sum(a.nbytes for a in host_out)
    s2 = torch.cuda.Stream()

    def run(h2d, d2h):
        torch.cuda.synchronize()
        e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        e[0].record(stream)
        e[2].record(s2)
        for _ in range(reps):
            if h2d:
                with torch.cuda.stream(stream):
                    for d, h in zip(din, tin):
                        d.copy_(h, non_blocking=True)
            if d2h:
                with torch.cuda.stream(s2):
                    for h, d in zip(tout, dout):
                        h.copy_(d, non_blocking=True)
        e[1].record(stream)
        e[3].record(s2)
        torch.cuda.synchronize()
        return e[0].elapsed_time(e[1]) * 1e-3, e[2].elapsed_time(e[3]) * 1e-3

    t_in, _ = run(True, False)
    _, t_out = run(False, True)
    b1, b2 = run(True, True)
    out = {"h2d": reps * b_in / t_in / 1e9, "d2h": reps * b_out / t_out / 1e9,
           "both_h2d": reps * b_in / b1 / 1e9, "both_d2h": reps * b_out / b2 / 1e9}
    del din, dout
    return out


def bench_operations(prob, sp, stream, peak, calls=5, cpu_sample=1_000_000):
    """The operations around the update on the config-2 workload, each timed
    with CUDA events on the stream over `calls` calls after two (the entry
    points that return a value -- the time-step estimate and the re-binning's
    removed count -- include their read-back): algorithmic bytes, GB/s and
    the fraction of the HBM peak; beside each, the numpy oracle of the same
    operation on one host core (the reference's versions are AMReX code that
    does not build here) on a bounded sample, scaled to the workload."""
    import torch
    from pelemp_b200 import workloads as W
    from pelemp_b200.spray import views
    from oracle import mesh_oracle as MO
    nb = len(prob.boxes)
    nf = prob.nfuel
    n = prob.n_droplets

    def timed(fn):
        for _ in range(2):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(calls):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / calls

    def cpu_timed(fn, scale):
        t0 = time.perf_counter()
        fn()
        return (time.perf_counter() - t0) * 1e3 * scale

    def grown_cells(g):
        tot = 0
        for b in range(nb):
            lo, hi = prob.grown(b, g)
            tot += int(np.prod([hi[d] - lo[d] + 1 for d in range(3)]))
        return tot

    out = {}
    cs = stream.cuda_stream
    # est_timestep (SprayParticles.cpp:89-140): velocity and id of every droplet
    ms = timed(lambda: sp.est_timestep(0.5, stream=cs))
    nbytes = n * (3 * 8 + 4)
    sub = [{k: v[..., :cpu_sample // nb] for k, v in p.items()} for p in prob.parts]
    cpu = cpu_timed(lambda: MO.est_timestep(sub, prob.dx, 0.5), n / sum(p["id"].size for p in sub))
    out["est_timestep"] = {"ms": ms, "bytes": nbytes, "cpu_ms": cpu}
    # computeDerivedVars (SprayDerive.cpp:9-155): droplets in, 15 + F fields per cell
    g = 1
    nvar = 15 + nf
    dshapes = []
    for b in range(nb):
        lo, hi = prob.grown(b, g)
        dshapes.append((nvar,) + tuple(hi[d] - lo[d] + 1 for d in (2, 1, 0)))
    dvars = [torch.zeros(s, dtype=torch.float64, device="cuda") for s in dshapes]
    dv = views(dvars, [prob.grown(b, g)[0] for b in range(nb)])
    ms = timed(lambda: sp.compute_derived_vars(dv, 0, True, stream=cs))
    nbytes = n * ((3 + 3 + 1 + 1 + nf + 1 + 1) * 8 + 4) + 2 * grown_cells(g) * nvar * 8
    rho_coef = np.zeros(16)
    for f, name in enumerate(prob.fuels):
        rho_coef[4 * f] = W.LIQUIDS[name]["rho"]
    want = [np.zeros(s) for s in dshapes]
    cpu = cpu_timed(lambda: MO.derive(sub, want, [prob.grown(b, g)[0] for b in range(nb)], 0, nf, True,
                                      rho_coef, prob.plo, prob.dx), n / sum(p["id"].size for p in sub))
    out["derive"] = {"ms": ms, "bytes": nbytes, "cpu_ms": cpu}
    del dvars, dv
    # transferSource + addSpraySrc (SprayParticles.H:250-319): fold the
    # temporary source's ghosts, add it into the flow's source, zero it
    gs, ga = prob.source_ghosts, 1
    tmp = [torch.zeros(s.shape, dtype=torch.float64, device="cuda") for s in prob.new_sources()]
    tv = views(tmp, [prob.grown(b, gs)[0] for b in range(nb)])
    act = []
    for b in range(nb):
        lo, hi = prob.grown(b, ga)
        act.append(torch.zeros((prob.n_state_comp,) + tuple(hi[d] - lo[d] + 1 for d in (2, 1, 0)),
                               dtype=torch.float64, device="cuda"))
    av = views(act, [prob.grown(b, ga)[0] for b in range(nb)])
    ms = timed(lambda: sp.transfer_source(tv, av, gs, ga, stream=cs))
    nsrc = prob.n_src_comp
    nbytes = 2 * grown_cells(gs) * nsrc * 8 + 2 * grown_cells(ga) * nsrc * 8
    periodic = [prob.bndry_lo[d] == 0 for d in range(3)]
    tmp_h = [np.zeros(s.shape) for s in prob.new_sources()]
    act_h = [a.cpu().numpy() for a in act]
    dep = list(sp.spray_data().dep_indx)[:nf]
    cpu = cpu_timed(lambda: MO.transfer_source(tmp_h, [prob.grown(b, gs)[0] for b in range(nb)], act_h,
                                               [prob.grown(b, ga)[0] for b in range(nb)], prob.boxes,
                                               prob.domain_lo, prob.domain_hi, periodic, gs, ga,
                                               comps=prob.comps(), nfuel=nf, dep_indx=dep), 1.0)
    out["transfer_source"] = {"ms": ms, "bytes": nbytes, "cpu_ms": cpu}
    del tmp, act, tv, av
    # re-binning (AMReX Redistribute for this container): every droplet read
    # and written once in its new order
    ms = timed(lambda: sp.redistribute(stream=cs))
    nbytes = 2 * n * ((3 + 10 + nf) * 8 + 4)
    cpu = cpu_timed(lambda: MO.redistribute(sub, prob.boxes, prob.plo, prob.phi, prob.dx, prob.domain_lo,
                                            prob.domain_hi, periodic), n / sum(p["id"].size for p in sub))
    out["redistribute"] = {"ms": ms, "bytes": nbytes, "cpu_ms": cpu}
    for v in out.values():
        v["gbs"] = v["bytes"] / (v["ms"] * 1e-3) / 1e9
        v["frac_hbm"] = v["gbs"] / peak
    out["what"] = ("device time per call (CUDA events on the stream, mean of %d calls after 2); bytes: "
                   "algorithmic (droplet fields read or written once, mesh arrays read / written once); "
                   "cpu_ms: the numpy oracle on one host core, %d droplets (the transfer on the whole "
                   "mesh), scaled to the workload" % (calls, cpu_sample))
    return out


def other_workloads(args):
    """The other workloads' lines, each from its own process (`--workload W
    --steps S --no-cpu --no-e2e`), reduced to their figures: config 3 the
    batched FP64 launches against one launch per box, configs 4 and 5 the
    three forms at 32M / 16M droplets of config 1's distributions."""
    out = {}
    for w in [x for x in args.also.split(",") if x and x != "none"]:
        cmd = [sys.executable, os.path.abspath(__file__), "--workload", w, "--steps", str(args.also_steps),
               "--warmup", "3", "--no-cpu", "--no-e2e", "--also", "none"]
        if w == "config4":
            cmd += ["--learn-stride", "32"]
        t0 = time.perf_counter()
        try:
            r = subprocess.run(cmd, capture_output=True, text=True, timeout=900)
        except subprocess.TimeoutExpired:
            out[w] = {"error": "no line within 900 s"}
            continue
        lines = [x for x in r.stdout.splitlines() if x.startswith("{")]
        if r.returncode != 0 or not lines:
            out[w] = {"error": "exit %d: %s" % (r.returncode, r.stderr.strip().splitlines()[-1:] or "")}
            continue
        d = json.loads(lines[-1])
        o = {"workload": d["config"]["workload"], "value": d["value"], "ms_per_step": d["ms_per_step"],
             "steps": d["steps"], "clocks": d.get("clocks"), "wall_s": round(time.perf_counter() - t0, 1)}
        if "launches" in d:
            o["launches"] = {k: (v if k == "speedup_vs_per_box" else
                                 {"value": v["value"], "ms_per_step": v["ms_per_step"]})
                             for k, v in d["launches"].items()}
        for f, v in d.get("forms", {}).items():
            e = v.get("error_vs_fp64", {})
            o.setdefault("forms", {})[f] = {
                "value": v["value"], "speedup_vs_fp64": v["speedup_vs_fp64"],
                # per quantity (diameter, T_d, velocity, the last step's deposits
                # of mass, energy and species) and the global balances
                "error_vs_fp64": {q: e[q] for q in ("T", "mass", "dia", "vel", "deposits_last_step",
                                                    "mass_balance_last_step", "energy_drift_vs_fp64")
                                  if q in e} or None,
                "train_s": v.get("train", {}).get("seconds"), "tuples": v.get("train", {}).get("tuples"),
                "fallback_frac": v["fallback_frac"], "inner_per_substep": v.get("inner_per_substep")}
        out[w] = o
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--droplets", type=int, default=None,
                    help="droplets per GPU (default: the workload's, 16M; 32M for config4)")
    ap.add_argument("--workload", default="config2", choices=["config2", "config3", "config4", "config5"],
                    help="config2 (default): the headline; config3: batched FP64 launch shapes; "
                         "config4 / config5: config-1 distributions at 32M / 16M droplets")
    ap.add_argument("--mesh", type=int, default=0,
                    help="config2 only: cells per side of a smaller cubic mesh (boxes of half that), "
                         "keeping droplets per cell at a given --droplets (profiling captures)")
    ap.add_argument("--e2e-steps", type=int, default=6)
    ap.add_argument("--e2e-copy-source", action="store_true",
                    help="e2e: copy the host source in and add the deposits to it (default: the "
                         "source is zero on entry, as transferSource leaves it, and is overwritten)")
    ap.add_argument("--eager-steps", type=int, default=2,
                    help="eager steps timed beside the graph replays (the droplets' drift over all "
                         "steps must stay inside the ghost cells)")
    ap.add_argument("--cpu-sample", type=int, default=0,
                    help="droplets per CPU step (0: sized for --cpu-seconds per step)")
    ap.add_argument("--cpu-seconds", type=float, default=8.0)
    ap.add_argument("--no-graph", action="store_true",
                    help="time eager steps only (default: the timed steps replay one CUDA graph of a "
                         "whole step -- source zeroing, MKD and MK -- and eager steps are timed beside)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-ops", action="store_true",
                    help="skip the timing of the operations around the update (config 2)")
    ap.add_argument("--forms", default="fp64,mixed,learned",
                    help="forms to time; the fastest non-FP64 one is the headline value")
    ap.add_argument("--learn-stride", type=int, default=16,
                    help="label every n-th droplet (x4 with the perturbed copies) at each state")
    ap.add_argument("--learn-gens", type=int, default=13,
                    help="states along the trajectory labelled (13 x 16M / 16 x 4 = 52M tuples at 16M droplets)")
    ap.add_argument("--learn-gap", type=int, default=2, help="FP64 steps between labelled states")
    ap.add_argument("--learn-epochs", type=int, default=4)
    ap.add_argument("--also", default="config3,config4,config5",
                    help="after the config-2 line (N=1, default sizes), the other workloads' figures, each "
                         "run in its own process; 'none' skips them")
    ap.add_argument("--also-steps", type=int, default=5)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    world, rank, local = dist_setup()

    if args.impl == "reference":
        line = run_reference(args, world, rank)
        if line is not None:
            print(json.dumps(line), flush=True)
        return

    import torch
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist

    from pelemp_b200 import workloads as W
    from pelemp_b200.spray import from_problem, views

    if args.workload == "config3":
        bench_batched(args, world, rank, local, pg)
        return
    forms = [f for f in args.forms.split(",") if f]
    ndrop = args.droplets or {"config2": 16_000_000, "config4": 32_000_000,
                              "config5": 16_000_000}[args.workload]
    if args.mesh and args.workload == "config2":
        m = args.mesh
        prob = W.config2(n=ndrop, seed=rank, steps=args.steps, ncells=(m, m, m), box=(m // 2, m // 2, m // 2))
    else:
        prob = W.CONFIGS[args.workload](n=ndrop, seed=rank, steps=args.steps)
    nboxes = len(prob.boxes)
    ncells = int(np.prod([prob.domain_hi[d] - prob.domain_lo[d] + 1 for d in range(3)]))
    stream = torch.cuda.current_stream()
    st = [torch.from_numpy(s).cuda() for s in prob.state]
    st_v = views(st, [prob.grown(b, prob.state_ghosts)[0] for b in range(nboxes)])
    src = [torch.zeros(s.shape, dtype=torch.float64, device="cuda") for s in prob.new_sources()]
    src_v = views(src, [prob.grown(b, prob.source_ghosts)[0] for b in range(nboxes)])
    peak, peak_src = measured_peaks()
    graphs = {}
    balance = {}

    def step(sp, st_handle):
        """One step, stream-ordered: zero the sources, MKD, MK (no host wait)."""
        for s in src:
            s.zero_()
        for do_move in (1, 0):
            sp.update_particles(st_v, src_v, prob.flow_dt, 0.0, prob.state_ghosts,
                                prob.source_ghosts, 0, 0, do_move, prob.spray_cfl_lev,
                                st_handle, sync=False)

    def timed_steps(sp, run, steps):
        """Device time of `steps` calls of run() on the stream, max over ranks,
        and the droplet-substeps and fallback count they executed."""
        sp.sync()  # clears the accumulated counters
        if pg:
            pg.barrier()
        torch.cuda.synchronize()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(steps):
            run()
        ev1.record(stream)
        torch.cuda.synchronize()
        sp.sync()
        st_ = sp.stats()
        t_max, sub_total = reduce_over_ranks(pg, ev0.elapsed_time(ev1), st_.substeps)
        return t_max, sub_total, st_.substeps, st_.fallback, st_.inner_steps

    results = {}
    containers = {}
    for form in forms:
        sp = from_problem(prob, device=local, mode=FORM_MODE[form])
        containers[form] = sp
        info = {}
        if form == "learned":
            t_train, rep, ntup = train_surrogate(sp, prob, st_v, src_v, stream.cuda_stream, args)
            info["train"] = {"seconds": t_train, "tuples": rep.tuples, "adam_steps": rep.steps,
                             "val_rel_rms": list(rep.val_rel_rms), "epochs": args.learn_epochs,
                             "baseline_residual_spread": list(rep.base_resid_frac),
                             "sample_stride": args.learn_stride, "states": args.learn_gens,
                             "steps_between_states": args.learn_gap,
                             "what": "tuples labelled by the FP64 teacher along the workload's "
                                     "trajectory (FP64 steps), untimed; the timed steps start from "
                                     "the initial droplets"}
        # warm-up steps; the MKD call of each is waited for, for its kernel time
        # (the library's events around the call's kernels: the roofline's launch)
        mkd_ms = []
        for w in range(args.warmup):
            for s_ in src:
                s_.zero_()
            for do_move in (1, 0):
                sp.update_particles(st_v, src_v, prob.flow_dt, 0.0, prob.state_ghosts,
                                    prob.source_ghosts, 0, 0, do_move, prob.spray_cfl_lev,
                                    stream.cuda_stream, sync=True)
                if do_move and w > 0:
                    mkd_ms.append(sp.stats().kernel_ms)
        # eager steps (a launch per kernel, the host never waits inside)
        t_eager, _, _, _, _ = timed_steps(sp, lambda: step(sp, stream.cuda_stream), args.eager_steps)
        graph = None
        sampler = ClockSampler(local)
        if not args.no_graph:
            # one CUDA graph of a whole step, captured on torch's capture
            # stream (the library's calls are capturable once run outside)
            graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(graph):
                step(sp, torch.cuda.current_stream().cuda_stream)
            sampler.start()
            time.sleep(0.3)
            t_max, sub_total, sub_local, fb, inner = timed_steps(sp, graph.replay, args.steps)
        else:
            sampler.start()
            time.sleep(0.3)
            t_max, sub_total, sub_local, fb, inner = timed_steps(sp, lambda: step(sp, stream.cuda_stream),
                                                          args.steps)
        c = sampler.stop()
        graphs[form] = graph
        # one more step, waited for, on which the balances and deposits are
        # compared (the droplets of box 0; every form takes the same steps)
        sp.sync()
        b0_before = sp.get_particles(0) if rank == 0 else None
        step(sp, stream.cuda_stream)
        sp.sync()
        if rank == 0:
            balance[form] = (b0_before, sp.get_particles(0), src[0].cpu().numpy())
        info.update({"value": sub_total / (t_max * 1e-3), "ms_per_step": t_max / args.steps,
                     "ms_per_step_eager": t_eager / args.eager_steps,
                     "timed": "whole-step CUDA graph replays" if graph is not None else "eager steps",
                     "mkd_launch_ms": float(np.mean(mkd_ms)), "substeps": sub_total,
                     "fallback_frac": fb / max(sub_local, 1), "clocks": c,
                     "inner_per_substep": inner / max(sub_local, 1)})
        results[form] = info

    fast = [f for f in forms if f != "fp64"]
    head = max(fast, key=lambda f: results[f]["value"]) if fast else "fp64"
    value = results[head]["value"]
    t_max = results[head]["ms_per_step"] * args.steps
    clocks = results[head]["clocks"]

    # accuracy of the fast forms against the FP64 form (bit-identical to the FP64
    # oracle): every form advanced the same initial droplets by warmup + steps steps
    accuracy = {}
    if "fp64" in containers and rank == 0:
        ref = [balance["fp64"][1]]
        fd = containers["fp64"].spray_data()
        rho_l = [W.LIQUIDS[f]["rho"] for f in prob.fuels]
        bal = {f: step_balance(prob, fd, balance[f][0], balance[f][1], balance[f][2], rho_l) for f in forms}
        for f in fast:
            accuracy[f] = droplet_errors([balance[f][1]], ref, prob)
            accuracy[f]["deposits_last_step"] = deposit_errors(balance[f][2], balance["fp64"][2], prob)
            accuracy[f]["mass_balance_last_step"] = bal[f]["mass"]
            accuracy[f]["energy_drift_vs_fp64"] = bal[f]["energy"] - bal["fp64"]["energy"]
        accuracy["fp64_balance_last_step"] = bal["fp64"]
        accuracy["steps"] = args.warmup + args.eager_steps + (0 if args.no_graph else args.steps) + 1
        accuracy["what"] = ("box 0's droplets after all steps against the FP64 form (bit-identical to the FP64 "
                            "oracle); deposits and balances of the last step; energy drift: the form's "
                            "(liquid enthalpy change + gas gain) / exchanged enthalpy minus the FP64 form's")

    peaks_c = None
    try:
        from pelemp_b200.spray import measure_peaks
        peaks_c = measure_peaks(local)
    except Exception as e:  # noqa: BLE001 -- reported, not fatal
        print("measure_peaks:", e, file=sys.stderr)
    # roofline of the headline form's MKD launch (algorithmic bytes / launch time)
    mkd_bytes = algorithmic_bytes(prob.n_droplets, prob.nfuel, prob.nspec, ncells, True)
    achieved = mkd_bytes / (results[head]["mkd_launch_ms"] * 1e-3) / 1e9
    traffic = None
    if args.workload == "config2":
        mesh = algorithmic_bytes(0, prob.nfuel, prob.nspec, ncells, True)
        traffic = mesh + prob.n_droplets * DRAM_BYTES_PER_DROPLET[head]

    # ---- e2e: host views through pmp_spray_update_host (headline form) ----
    e2e = None
    if not args.no_e2e:
        sp = containers[head]
        # from the initial droplets again (their drift stays inside the ghost cells)
        for b, p in enumerate(prob.parts):
            sp.set_particles(b, p["pos"], p["rdata"], p["id"])
        st_h = [torch.from_numpy(s).pin_memory().numpy() for s in prob.state]
        src_h = [torch.zeros(s.shape, dtype=torch.float64).pin_memory().numpy()
                 for s in prob.new_sources()]
        st_hv = views(st_h, [prob.grown(b, prob.state_ghosts)[0] for b in range(nboxes)])
        src_hv = views(src_h, [prob.grown(b, prob.source_ghosts)[0] for b in range(nboxes)])
        # the state components the update reads (rho, velocity, T, species: all
        # but rhoH) are copied in for MKD and MK, the source components back;
        # the source is zero on entry to each call, as the reference's
        # transferSource leaves it, so it is not copied in unless asked
        # (--e2e-copy-source: copied in and the deposits added to it)
        sp.set_host_source_in(args.e2e_copy_source)
        used = (5 + prob.nspec) / prob.n_state_comp
        h2d = 2 * used * sum(a.nbytes for a in st_h)
        if args.e2e_copy_source:
            h2d += 2 * sum(a.nbytes for a in src_h)
        d2h = 2 * sum(a.nbytes for a in src_h)

        # with --e2e-copy-source the deposits accumulate in the host source
        # arrays over the timed steps (zeroing them is the caller's host
        # work, and the droplets do not read them)
        def host_step():
            for do_move in (1, 0):
                sp.update_particles_host(st_hv, src_hv, prob.flow_dt, 0.0, prob.state_ghosts,
                                         prob.source_ghosts, 0, 0, do_move, prob.spray_cfl_lev,
                                         stream.cuda_stream, sync=False)

        host_step()
        sp.sync()
        if pg:
            pg.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e_ev0 = torch.cuda.Event(enable_timing=True)
        e_ev1 = torch.cuda.Event(enable_timing=True)
        e_ev0.record(stream)
        for _ in range(args.e2e_steps):
            host_step()
        e_ev1.record(stream)
        torch.cuda.synchronize()
        te = max(e_ev0.elapsed_time(e_ev1), 1e3 * (time.perf_counter() - t0))
        sp.sync()
        te, ns = reduce_over_ranks(pg, te, sp.stats().substeps)
        e2e = {"value": ns / (te * 1e-3), "unit": "droplet-substeps/s",
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
               "steps": args.e2e_steps, "form": head,
               "path": "pmp_spray_update_host: pinned host state/source, H2D+D2H inside, "
                       "copies overlapped with the update in box groups, calls stream-ordered "
                       "(the host waits once, after the last step); host source "
                       + ("copied in, deposits added" if args.e2e_copy_source else
                          "zero on entry (as transferSource leaves it): not copied in, overwritten")}
        # the link the copies cross: the same pinned arrays copied alone, each
        # direction alone and both at once (GB/s per direction)
        e2e["pcie_gbs"] = pcie_rates(st_h, src_h, stream)

    ops = None
    if rank == 0 and world == 1 and args.workload == "config2" and not args.no_ops:
        ops = bench_operations(prob, containers[head], stream, peak)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(args)

    if rank == 0:
        forms_out = {}
        for f in forms:
            r = results[f]
            forms_out[f] = {"value": r["value"], "ms_per_step": r["ms_per_step"],
                            "ms_per_step_eager": r["ms_per_step_eager"], "timed": r["timed"],
                            "mkd_launch_ms": r["mkd_launch_ms"], "fallback_frac": r["fallback_frac"],
                            "inner_per_substep": r["inner_per_substep"],
                            "speedup_vs_fp64": (r["value"] / results["fp64"]["value"]
                                                if "fp64" in results else None)}
            if "train" in r:
                forms_out[f]["train"] = r["train"]
            if f in accuracy:
                forms_out[f]["error_vs_fp64"] = accuracy[f]
        line = {
            "metric": "droplet-substeps/s", "value": value, "unit": "droplet-substeps/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None,
            "dtype": {"fp64": "f64", "mixed": "f32 physics, f64 state/deposits",
                      "learned": "bf16 MLP (f32 accumulate), f32 physics, f64 state/deposits"}[head],
            "data": "synthetic (seeded, numpy PCG64)",
            "config": {"workload": (WORKLOAD_TEXT[args.workload].format(n=prob.n_droplets / 1e6) if not args.mesh
                                    else WORKLOAD_TEXT[args.workload].format(n=prob.n_droplets / 1e6).replace(
                                        "128^3 mesh as 8 boxes of 64^3",
                                        f"{args.mesh}^3 mesh as 8 boxes of {args.mesh // 2}^3")),
                       "droplets_per_gpu": prob.n_droplets, "boxes": nboxes, "form": head,
                       "form_name": FORM_NAME[head],
                       "l2": "inputs larger than L2 (droplet SoA %.1f GB per GPU)" % (
                           prob.n_droplets * 8 * (13 + prob.nfuel) / 1e9),
                       "parallelism": f"replicas x{world}"},
            "forms": forms_out,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "traffic_source": "ncu dram bytes of a 2M-droplet MKD launch of the same kernel at "
                                           "config-2 density, scaled by droplet count (mesh part fixed)"
                         if traffic else None,
                         "kernel": KERNEL[head] + " (MKD launch)",
                         "launch_ms": results[head]["mkd_launch_ms"],
                         "algorithmic_bytes_per_launch": mkd_bytes,
                         "peak_source": f"{peak_src} (MEASURED_PEAKS.json hbm_gbs)"
                         if peak_src == "measured" else "fallback 6650 GB/s",
                         "compute": compute_roofline(head, peaks_c)},
            "e2e": e2e,
            "operations": ops,
            "cpu_baseline": cpu,
            "gpu_launches": 2 * args.steps * KERNELS_PER_CALL[head],
            "clocks": clocks,
            "substeps_per_step": results[head]["substeps"] / args.steps,
        }
    graphs.clear()  # release the graphs before their containers
    for sp in containers.values():
        sp.close()
    if rank == 0:
        if (world == 1 and args.workload == "config2" and not args.mesh and not args.droplets
                and args.also != "none"):
            del st, src, st_v, src_v
            torch.cuda.empty_cache()
            line["other_workloads"] = other_workloads(args)
        print(json.dumps(line), flush=True)
    if pg:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
