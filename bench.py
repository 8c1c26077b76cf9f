#!/usr/bin/env python
"""Throughput of the hotspin hot path on B200: two-temperature model + LLB at 512x512x4.

Workload (the configuration the headline metric is quoted on): 512 x 512 x 4 cells of
4 nm, demag padded to 1024 x 1024 x 8, Ms0 = 8e5 A/m, A = 1.3e-11 J/m, lambda = 0.02,
Tc = 630 K, J = 1/2, Philox thermal field (seed 3), electrons Ce = 700 Te J/m^3K, lattice
Cl = 3e6 J/m^3K, G = 6e17 W/m^3K, ke = 90 W/mK, Gaussian laser 100 fs FWHM, 5e20 W/m^3,
sigma = 400 nm, T0 = 300 K, adaptive Dormand-Prince 4(5) at rtol 1e-5.  One "step" is one
accepted DP45 step of the whole grid; value = cells x accepted steps / device time
(Mcell-steps/s), summed over ranks (independent replicas: the path does not shard).

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]
"""
import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mcell-steps/s (TTM+LLB, DP45 rtol 1e-5) at 512x512x4"
UNIT = "Mcell-steps/s"
MU0 = 4e-7 * math.pi
MUB = 9.27400968202020202e-24


# DRAM bytes (read + write) per launch of each kernel family on this workload, from one ncu
# capture each (dram__bytes_read.sum + dram__bytes_write.sum; stage: the 7 launches of one
# DP45 attempt averaged).
TRAFFIC_PER_LAUNCH = {"stage": 133_196_000, "yz": 56_891_000, "xfwd": 12_633_000, "xinv": 25_285_000}
STAGE_KERNEL_NAME = "k_stagec<5,0,2,NK> (load-first fused RHS + DP45 stage; 7 launches per attempt)"


def workload():
    """Program order: (N0, N1, N2) = (z, y, x)."""
    ms = 8e5
    lex = math.sqrt(2 * 1.3e-11 / (MU0 * ms * ms))
    return dict(size=(4, 512, 512), cellsize=(4e-9, 4e-9, 4e-9), msat0T0=ms, lex=lex,
                gamma_ll=2.211e5 / (1 + 0.02 ** 2), alpha=(0.02, 0.02, 0.02), b_ext=(0.0, 0.0, 0.02),
                demag=True, llb=True, tc=630.0, spin_j=0.5, n_spins=ms / (2 * MUB * 0.5), temperature=300.0,
                thermal=True, seed=3, ttm=True, gamma_e=700.0, c_l=3e6, g_ep=6e17, k_e=90.0, k_l=0.0,
                laser_p0=5e20, laser_t0=2.5e-13, laser_fwhm=1e-13, laser_sigma=400e-9)


def equilibrium_lib(kw, T=300.0):
    """m_e(T) from the product library's FP64 mean-field table."""
    from hotspin_b200 import _lib
    me = ctypes.c_double()
    _lib.check(_lib.load().hsb_mfa_equilibrium(T, kw["tc"], kw["spin_j"], ctypes.byref(me)), "m_e")
    return me.value


def initial_state(kw, me):
    """m = me (= m_e(300 K)) along user x with a seeded 5 degree random tilt; Te = Tl = 300 K."""
    size = kw["size"]
    rng = np.random.default_rng(3)
    th = np.deg2rad(5.0) * rng.random(size)
    ph = 2 * np.pi * rng.random(size)
    m = np.stack([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)])  # around program Z
    return {"m": me * m, "Te": np.full(size, 300.0), "Tl": np.full(size, 300.0)}


def run_config(kw):
    """The workload description both arms print (identical dicts)."""
    ncell = int(np.prod(kw["size"]))
    ws = int((ncell * 4 * (5 * 13 + 12) + 3 * 4 * 513 * 512 * 8 + 31.6e6) / 1e6)
    return {"workload": "TTM+LLB 512x512x4 (demag 1024x1024x8), DP45 rtol 1e-5, thermal field",
            "cells": ncell, "l2": "working set %d MB > 126 MB L2 (no flush needed)" % ws}


def algorithmic_bytes(kw, fused=True):
    """Unique bytes each kernel family must move per launch (inputs once, outputs once)."""
    n0, n1, n2 = kw["size"]
    ncell = n0 * n1 * n2
    L0, L1, L2 = [2 * s if s > 1 else s for s in kw["size"]]
    c2 = L2 // 2 + 1
    spec = 3 * n0 * c2 * n1 * 8                  # X1: complex FP32 after the x pass
    # kernel rows read per kx column: L0/2 + 1 folded z frequencies, or the N0 z-space rows of
    # the direct z convolution (zero-padded z axis of 2 or 4 cells)
    zrows = n0 if L0 in (4, 8) else L0 // 2 + 1
    kern = c2 * (L1 // 2 + 1) * zrows * 6 * 4
    nch = 5 if kw.get("ttm") else 3
    # DP45 attempt with a thermal field: stage 1 + stages 2..6 + stage 7
    stage = 0
    stage += ncell * (nch * 4 + 12 + nch * 4 + nch * 4)               # s1: ys, hd, write k1, y2
    for s in range(2, 7):                                              # ys, hd, y0, k1..k(s-1), write k_s, y(s+1)
        stage += ncell * (nch * 4 + 12 + nch * 4 + nch * 4 * (s - 1) + nch * 4 + nch * 4)
    stage += ncell * (nch * 4 + 12 + nch * 4 + nch * 4 * 6 + nch * 4)  # s7: ys, hd, y0(T), k1..k6, k7
    return {"xfwd": ncell * 12 + spec, "yz": 2 * spec + kern, "xinv": spec + ncell * 12,
            "stage_attempt": stage, "stage_launches": 7, "demag_per_attempt": 6}


def family_roofline(kw, solver, prof_ms):
    """Algorithmic bytes and HBM fraction of each kernel family for one attempt of `solver`
    (`prof_ms`: the attempt's device time per family, summed over its launches)."""
    n0, n1, n2 = kw["size"]
    ncell = n0 * n1 * n2
    L0, L1, L2 = [2 * s if s > 1 else s for s in kw["size"]]
    c2 = L2 // 2 + 1
    spec = 3 * n0 * c2 * n1 * 8
    x2 = 3 * n0 * c2 * L1 * 8                     # multi-pass y-transformed spectrum
    zrows = n0 if L0 in (4, 8) else L0 // 2 + 1   # direct z convolution reads N0 rows
    kern = c2 * (L1 // 2 + 1) * zrows * 6 * 4
    nch = 5 if kw.get("ttm") else 3
    fused = L0 <= 16
    yz = 2 * spec + kern if fused else 2 * spec + 4 * x2 + kern
    if solver == "rk4":
        ndemag = 4
        # s1: y0, H_d, write k-sum, y2; s2, s3: y_s, H_d, y0, k-sum, write k-sum, y_(s+1);
        # s4: y4, H_d, y0, k-sum, write y_new
        stage = ncell * (nch * 4 * (3 + 5 + 5 + 4) + 4 * 12)
    else:
        ndemag = 6
        stage = algorithmic_bytes(kw)["stage_attempt"]
    peak, _ = peaks()
    byt = {"stage": stage, "xfwd": ndemag * (ncell * 12 + spec), "yz": ndemag * yz,
           "xinv": ndemag * (spec + ncell * 12)}
    out = {}
    for k, b in byt.items():
        gbs = b / (prof_ms[k] / 1e3) / 1e9
        out[k] = {"algorithmic_bytes_per_attempt": int(b), "ms_per_attempt": round(prof_ms[k], 4),
                  "achieved_gbs": round(gbs, 1), "frac_of_measured_hbm": round(gbs / peak, 3)}
    return out


class Clocks:
    """nvidia-smi sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                       "--format=csv,noheader,nounits", "-lms", "100"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.p = None
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.p is not None:
            self.p.terminate()
            try:
                out, _ = self.p.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()
                out, _ = self.p.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def cpu_baseline(kw, state):
    """The FP64 oracle (NumPy, all host cores through numpy's own threading) timed on one
    DP45 step of the same workload."""
    from oracle.model import Model, Spec
    from oracle.solvers import Integrator
    spec = Spec(**kw)
    model = Model(spec)
    it = Integrator(model, state, "dp45", 2e-16, rtol=1e-5, mindt=1e-20, maxdt=1e-13)
    t0 = time.perf_counter()
    it.step()
    dtw = time.perf_counter() - t0
    ncell = int(np.prod(kw["size"]))
    base = {"value": ncell * it.step_count / dtw / 1e6, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
            "sample": "1 accepted DP45 step (%d RHS evaluations) of the 512x512x4 workload by the FP64 "
                      "NumPy oracle, %.1f s" % (7 * (1 + it.bad_steps), dtw)}
    return base, accuracy(kw, state, it, model)


def accuracy(kw, state, it, model):
    """The same accepted DP45 step on the device, from the same state, against the FP64
    oracle's (the oracle as checker): max |dm|, relative max |dTe|, relative energy error."""
    from hotspin_b200.sim import Simulation
    with Simulation(**kw, solver="dp45", dt=2e-16, rtol=1e-5, mindt=1e-20, maxdt=1e-13) as sim:
        for k, v in state.items():
            sim.set(k, v)
        sim.step(1)
        st = sim.status()
        m, Te, E = sim.get("m"), sim.get("Te"), sim.energy()
        scale = sum(abs(v) for v in sim.energy_terms().values())
    Eo = model.energy(it.y)
    return {"reference": "FP64 oracle, one accepted DP45 step of the full workload from the same state",
            "same_step": bool(abs(st["t"] - it.t) <= 1e-9 * it.t),
            "max_abs_dm": float(np.abs(m - it.y["m"]).max()),
            "rel_max_abs_dTe": float(np.abs(Te - it.y["Te"]).max() / np.abs(it.y["Te"]).max()),
            "rel_energy_err": float(abs(E - Eo) / abs(Eo)),
            "energy_err_vs_sum_of_abs_terms": float(abs(E - Eo) / scale),
            "note": "the total energy here is a residual of terms ~250x larger (Zeeman vs exchange + demag); "
                    "FP32 state storage bounds its relative accuracy"}


def dist_setup(backend="nccl"):
    """One process per GPU (torchrun environment); replicas only, so the process group carries
    nothing but the barrier and the max-over-ranks of the timings."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    import torch
    if backend == "nccl":
        torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
        pg = dist
    return world, rank, local, pg


def barrier(pg):
    if pg is not None:
        pg.barrier()


def max_over_ranks(pg, v, device="cuda"):
    if pg is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def whole_job_value(world, ncell, steps, ms_max):
    """Mcell-steps/s of all replicas together: every rank advances its own copy of the
    workload, and the job takes as long as the slowest rank."""
    return world * ncell * steps / (ms_max / 1e3) / 1e6


def timed_reps(sim, stream, pg, steps, min_reps, min_s):
    """Repetitions of exactly `steps` steps, each from the same checkpoint (so every repetition
    does the same work: same trajectory, same attempts), each bracketed by a barrier and a
    device synchronisation and timed with CUDA events on the handle's stream; the max over
    ranks of each.  Repeats until at least `min_reps` repetitions and `min_s` seconds of timed
    work, so the clock sampler sees the timed region."""
    import torch
    sim.checkpoint()
    reps = []
    while True:
        sim.restore()
        s0 = sim.status()
        n0 = sim.launch_count()
        barrier(pg)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        sim.step(steps)
        e1.record(stream)
        e1.synchronize()
        torch.cuda.synchronize()
        barrier(pg)
        ms = max_over_ranks(pg, e0.elapsed_time(e1))
        s1 = sim.status()
        reps.append({"ms": ms, "attempts": s1["attempts"] - s0["attempts"], "rejects": s1["rejects"] - s0["rejects"],
                     "t_ps": s1["t"] * 1e12, "launches": sim.launch_count() - n0})
        if len(reps) >= min_reps and sum(r["ms"] for r in reps) >= 1e3 * min_s:
            return reps


def pinned_like(a):
    """A page-locked float64 host copy of `a` (a numpy view of pinned torch memory)."""
    import torch
    t = torch.empty(a.shape, dtype=torch.float64, pin_memory=True)
    v = t.numpy()
    v[...] = a
    return t, v


def run_ours(args):
    import torch
    from hotspin_b200 import _lib
    from hotspin_b200.sim import Simulation
    world, rank, local, pg = dist_setup()
    kw = workload()
    ncell = int(np.prod(kw["size"]))
    st0 = initial_state(kw, equilibrium_lib(kw))
    if args.stage_variant is not None:      # fixed stage-kernel variant (e.g. under a profiler)
        _lib.load().hsb_set_stage_variant(args.stage_variant)
    sim = Simulation(**kw, solver="dp45", dt=2e-16, rtol=1e-5, mindt=1e-20, maxdt=1e-13)
    for k, v in st0.items():
        sim.set(k, v)
    stream = torch.cuda.ExternalStream(sim._lib.hsb_sim_stream(sim._h))
    sim.step(args.warmup)
    with Clocks(local) as clk:
        reps = timed_reps(sim, stream, pg, args.steps, args.min_reps, args.min_timed_s)
    med = sorted(reps, key=lambda r: r["ms"])[len(reps) // 2]
    ms = med["ms"]
    same = all(r["attempts"] == reps[0]["attempts"] and r["t_ps"] == reps[0]["t_ps"] for r in reps)
    value = whole_job_value(world, ncell, args.steps, ms)
    # ---- live per-kernel timing of one attempt (eager launches between CUDA events)
    prof = (ctypes.c_double * 7)()
    _lib.check(sim._lib.hsb_sim_profile(sim._h, 3, prof), "profile")
    cats = {"stage": prof[0], "xfwd": prof[1], "yz": prof[2], "xinv": prof[3], "other": prof[4]}
    ab = algorithmic_bytes(kw)
    per_launch = {"stage": (ab["stage_attempt"], prof[0], ab["stage_launches"]),
                  "yz": (ab["yz"] * ab["demag_per_attempt"], prof[2], ab["demag_per_attempt"]),
                  "xfwd": (ab["xfwd"] * ab["demag_per_attempt"], prof[1], ab["demag_per_attempt"]),
                  "xinv": (ab["xinv"] * ab["demag_per_attempt"], prof[3], ab["demag_per_attempt"])}
    dom = max(per_launch, key=lambda k: per_launch[k][1])
    byt, tms, nlaunch = per_launch[dom]
    peak, kind = peaks()
    achieved = (byt / nlaunch) / ((tms / nlaunch) / 1e3) / 1e9
    traffic = TRAFFIC_PER_LAUNCH.get(dom)
    names = {"stage": STAGE_KERNEL_NAME,
             "yz": "k_yz4<1024,8,1> (y/z FFT + tensor multiply + inverse)",
             "xfwd": "k_xfwd4<512,1> (R2C + transpose)", "xinv": "k_xinv4<512,1> (C2R)"}
    roof = {"bound": "hbm", "kernel": names[dom], "achieved": round(achieved, 1), "peak": peak,
            "peak_kind": kind, "unit": "GB/s", "frac": round(achieved / peak, 4), "traffic": traffic,
            "algorithmic_bytes_per_launch": int(byt / nlaunch),
            "avg_launch_ms": round(tms / nlaunch, 5),
            "attempt_ms_by_family": {k: round(v, 4) for k, v in cats.items()}}
    # ---- end to end through the C-ABI: page-locked FP64 host state uploaded, K step calls each
    # followed by the status read, m read back into page-locked host memory
    keep = [pinned_like(v) for v in st0.values()]
    host_state = dict(zip(st0.keys(), [v for _, v in keep]))
    mt, mout = pinned_like(np.zeros((3,) + tuple(kw["size"])))

    def e2e_run():
        barrier(pg)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        sim.set_time(0.0, 2e-16)
        for k, v in host_state.items():
            sim.set(k, v)
        for _ in range(args.steps):
            sim.step(1)
            sim.status()          # the step's result: t, dt, steps, err, status
        sim.get("m", out=mout)
        torch.cuda.synchronize()
        return max_over_ranks(pg, time.perf_counter() - t0)

    e2e_run()                     # untimed: builds the one-step graph
    e2e_s = statistics.median([e2e_run() for _ in range(3)])
    h2d = sum(v.nbytes for v in host_state.values())
    per_step_d2h = _lib.load().hsb_solver_word_bytes()   # the solver word each step call reads back
    d2h = mout.nbytes + args.steps * per_step_d2h
    e2e = {"value": round(world * ncell * args.steps / e2e_s / 1e6, 3), "unit": UNIT,
           "h2d_bytes_per_step": int(h2d / args.steps), "d2h_bytes_per_step": int(d2h / args.steps),
           "note": "median of 3 runs; per run: page-locked FP64 host state uploaded, K step calls each "
                   "reading the solver block back, m downloaded to page-locked memory"}
    out = {"metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 4), "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
           "parallelism": "replicas" if world > 1 else "single",
           "config": run_config(kw),
           "timing": {"repetitions": len(reps), "statistic": "median repetition",
                      "rep_ms_min": round(min(r["ms"] for r in reps), 4),
                      "rep_ms_max": round(max(r["ms"] for r in reps), 4),
                      "identical_repetitions": same,
                      "each": "exactly K accepted steps from the checkpoint taken after the W warm-up steps"},
           "progress": {"attempts": med["attempts"], "rejected": med["rejects"],
                        "sim_time_ps_at_end": round(med["t_ps"], 4)},
           "roofline": roof, "gpu_launches": int(med["launches"]), "e2e": e2e, "clocks": clk.summary()}
    sim.close()
    if rank == 0:
        if world == 1 and not args.no_cpu_baseline:
            out["cpu_baseline"], out["accuracy"] = cpu_baseline(kw, st0)
        if world == 1 and not args.no_configs:
            out["other_configs"] = other_configs()
        if world == 1 and not args.no_serving:
            out["serving"] = serving(args)
        print(json.dumps(out))
    if pg is not None:
        pg.destroy_process_group()


def other_configs():
    """Device throughput of the other single-simulation workloads (synthetic states): LLB at
    300 K on 256x256x8 cells of 2 nm (FePt-like, Ku 7e6 along z, lambda 0.1, thermal field,
    DP45 rtol 1e-5) and plain LLG on 1024x1024x32 cells of 2 nm (alpha 0.5, RK4 20 fs; demag
    padded to 2048x2048x64 on the multi-pass FFT path)."""
    import ctypes
    import torch
    from hotspin_b200 import _lib
    from hotspin_b200.sim import Simulation
    lib = _lib.load()
    out = {}
    cases = {
        "llb_256x256x8_dp45": (dict(size=(8, 256, 256), cellsize=(2e-9,) * 3, msat0T0=1.1e6,
                                        lex=math.sqrt(2 * 1e-11 / (MU0 * 1.1e6 ** 2)), gamma_ll=2.211e5,
                                        alpha=(0.1,) * 3, ku=7e6, anis_u=(1.0, 0.0, 0.0), demag=True, llb=True,
                                        tc=700.0, spin_j=0.5, n_spins=1.1e6 / (2 * MUB * 0.5), temperature=300.0,
                                        thermal=True, seed=2, solver="dp45", dt=1e-16, rtol=1e-5, mindt=1e-20,
                                        maxdt=1e-12), 100),
        "llg_1024x1024x32_rk4": (dict(size=(32, 1024, 1024), cellsize=(2e-9,) * 3, msat0T0=8e5,
                                          lex=math.sqrt(2 * 1.3e-11 / (MU0 * 8e5 ** 2)),
                                          gamma_ll=2.211e5 / (1 + 0.25), alpha=(0.5,) * 3, demag=True,
                                          normalize=True, solver="rk4", dt=20e-15), 20),
    }
    for name, (kw, nsteps) in cases.items():
        size = kw["size"]
        rng = np.random.default_rng(5)
        if kw.get("llb"):
            me = ctypes.c_double()
            _lib.check(lib.hsb_mfa_equilibrium(300.0, kw["tc"], 0.5, ctypes.byref(me)), "m_e")
            th = np.deg2rad(5.0) * rng.random(size)
            ph = 2 * np.pi * rng.random(size)
            m = me.value * np.stack([np.cos(th), np.sin(th) * np.sin(ph), np.sin(th) * np.cos(ph)])
        else:
            m = rng.normal(size=(3,) + size)
            m /= np.sqrt((m * m).sum(0))
        with Simulation(**kw) as sim:
            sim.set("m", m)
            sim.step(3)
            stream = torch.cuda.ExternalStream(sim._lib.hsb_sim_stream(sim._h))
            s0 = sim.status()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            sim.step(nsteps)
            e1.record(stream)
            e1.synchronize()
            ms = e0.elapsed_time(e1)
            s1 = sim.status()
            prof = (ctypes.c_double * 7)()
            _lib.check(lib.hsb_sim_profile(sim._h, 2, prof), "profile")
        n = int(np.prod(size))
        fam = {"stage": prof[0], "xfwd": prof[1], "yz": prof[2], "xinv": prof[3]}
        out[name] = {"value": round(n * nsteps / (ms / 1e3) / 1e6, 1), "unit": UNIT, "cells": n,
                     "ms_per_step": round(ms / nsteps, 4), "steps": nsteps,
                     "attempts": int(s1["attempts"] - s0["attempts"]),
                     "kernel_roofline": family_roofline(kw, kw["solver"], fam)}
    return out


def serving(args):
    """Continuous-batching serving stream against the sequential plain path (one GPU).

    256 independent LLG/LLB requests (Poisson arrivals at 50/s; square films with sides
    32..512 log-uniform and 1 or 2 layers; cubic cells 2-5 nm; Ms0, damping, temperature,
    field and initial m drawn from seed 4), DP45 at rtol 1e-5 to 50 ps each.  The batched
    loop (hotspin_b200.serve.Server) runs them as they arrive; the plain path runs one
    Simulation per request in arrival order.  Both report p50/p99 time-to-solution and
    throughput over the makespan; every result is compared between the two.
    """
    from hotspin_b200 import serve
    reqs = serve.make_requests(n=args.serving_requests, seed=4, t_end=args.serving_tend)
    warm = serve.make_requests(n=2, seed=99, t_end=2e-14, sides=(32,), layers=(1,))
    w = serve.Server()
    w.run(warm, realtime=False)
    w.close()
    serve.run_sequential(warm)
    srv = serve.Server()
    res = srv.run(reqs, realtime=True)
    nclass = len(srv.classes)
    launches = sum(c.launches for c in srv.classes.values())
    srv.close()
    seq, service, setup = serve.run_sequential(reqs)
    sb, ss = serve.summarize(res, reqs), serve.summarize(seq, reqs)
    dm = max(float(np.abs(res[k].m - seq[k].m).max()) for k in res)
    same = sum(int(res[k].steps == seq[k].steps) for k in res)
    rnd = lambda d: {k: (round(v, 4) if isinstance(v, float) else v) for k, v in d.items()}
    return {"workload": "%d Poisson(50/s) LLG/LLB requests, square films 32..512 x 1..2 layers, cells 2-5 nm, "
                        "DP45 rtol 1e-5 to %g ps, seed 4" % (len(reqs), args.serving_tend * 1e12),
            "batched": rnd(sb), "sequential_plain": rnd(ss),
            "throughput_ratio": round(sb["req_per_s"] / ss["req_per_s"], 3),
            "p50_ratio": round(ss["p50_s"] / sb["p50_s"], 3), "p99_ratio": round(ss["p99_s"] / sb["p99_s"], 3),
            "max_abs_dm_batched_vs_plain": dm, "same_step_counts": "%d/%d" % (same, len(res)),
            "size_classes": nclass, "class_graph_launches": launches,
            "plain_setup_share": round(sum(setup.values()) / sum(service.values()), 4)}


def profile_sim():
    """The bench simulation: 2 steps, then 2 attempts with every launch group between CUDA
    events (the workload the stage and launch-list captures run)."""
    import ctypes
    from hotspin_b200.sim import Simulation
    kw = workload()
    st0 = initial_state(kw, equilibrium_lib(kw))
    s = Simulation(**kw, solver="dp45", dt=2e-16, rtol=1e-5, mindt=1e-20, maxdt=1e-13)
    for k, v in st0.items():
        s.set(k, v)
    s.step(2)
    out = (ctypes.c_double * 7)()
    s._lib.hsb_sim_profile(s._h, 2, out)
    print("attempt ms: stage %.4f x-fwd %.4f y-z %.4f x-inv %.4f other %.4f launches %d" % tuple(out[:6]))
    s.close()


def profile_demag(size):
    """One demag plan of `size` (4 nm cells, open) and 3 + 10 convolutions of a random field."""
    import ctypes
    import torch
    from hotspin_b200 import _lib
    from hotspin_b200.sim import demag_plan
    plan = demag_plan(size, (4e-9,) * 3, (0, 0, 0))
    lib = _lib.load()
    m = torch.randn((3,) + tuple(size), device="cuda", dtype=torch.float32)
    H = torch.empty_like(m)
    for _ in range(3):
        _lib.check(lib.hsb_demag_field(plan, ctypes.c_void_p(m.data_ptr()), None, 8e5,
                                       ctypes.c_void_p(H.data_ptr()), None), "hsb_demag_field")
    ms = (ctypes.c_double * 3)()
    _lib.check(lib.hsb_demag_profile(plan, ctypes.c_void_p(m.data_ptr()), None, 8e5, ctypes.c_void_p(H.data_ptr()),
                                     None, 10, ms), "hsb_demag_profile")
    torch.cuda.synchronize()
    print("demag", tuple(size), "ms x-fwd / y-z / x-inv", [round(x, 5) for x in ms])
    lib.hsb_demag_plan_destroy(plan)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-serving", action="store_true", help="skip the batched-serving comparison")
    ap.add_argument("--no-configs", action="store_true", help="skip the LLB 256x256x8 and LLG 1024x1024x32 throughput lines")
    ap.add_argument("--stage-variant", type=int, default=None, choices=[0, 1, 2, 4],
                    help="run this stage-kernel variant instead of the one timed at creation")
    ap.add_argument("--min-reps", type=int, default=5, help="timed repetitions of the K steps (at least)")
    ap.add_argument("--min-timed-s", type=float, default=1.0, help="seconds of timed work (at least)")
    ap.add_argument("--profile", choices=["sim", "demag"], default=None,
                    help="profiling workload: 'sim' = 2 steps + 2 profiled attempts of the bench "
                         "simulation, 'demag' = one plan at --size and 3 + 10 convolutions")
    ap.add_argument("--size", type=int, nargs=3, default=(4, 512, 512), help="demag profile grid (N0 N1 N2)")
    ap.add_argument("--serving-requests", type=int, default=256)
    ap.add_argument("--serving-tend", type=float, default=50e-12)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.profile == "sim":
        profile_sim()
        return
    if args.profile == "demag":
        profile_demag(tuple(args.size))
        return
    if args.impl == "reference":
        from oracle.replay import bench_reference
        bench_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
