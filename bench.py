#!/usr/bin/env python3
"""Benchmark: KMC steps/s of the STZ-KMC + Lippmann-Schwinger step on B200,
chosen form vs plain form.

One step = one thermal KMC event of one replica's run_simulation
(kmc_solver.hpp:783-938): sweep of every (voxel, mode) barrier and rate, event
selection, flip with its catalog/barrier redraw, and the warm-started FP64 LS
re-solve; cascades and the end-of-interval mixed-BC solves that fall inside
the timed region are part of the work, as in the reference.

Workload (the heterogeneous 2D case): ``hetero2d_256`` at seeds 0-3, four
independent replicas (2D 256x256 plane strain, seeded synthetic lognormal
modulus field, CoV 0.10, correlation 4 voxels, M = 18 modes per voxel).

* ``value`` -- the chosen form: the four replicas advanced together by the
  batched, device-resident kernel (mgk_batch_run), K thermal events each;
  CUDA-event time of the launch.  ``e2e``: the same call (the same events)
  timed by the wall clock through the public API, its host<->device copies
  and the replicas' macroscopic results read back included.
* ``plain`` -- the drop-in form (mgk_kmc_run, one replica at a time, host RNG
  replay), K events of seed 0, CUDA-event time of the run; its ``e2e``
  through the public API with every step's copies.
* ``ensemble`` (unless --no-ensemble) -- the 64-replica mixed ensemble (16 each
  of 2D 64^2, 128^2, 512^2, 16 3D of 32^3 / 48^3 / 96^3) in one launch for a
  fixed device time, against the plain form's per-replica rates.
* ``cpu_baseline`` / --impl reference -- the reference's own CPU code
  (oracle/_ref/ref_driver, compiled from the reference sources), one process
  per replica run concurrently, on a bounded sample of the same workload.

Every step reads the whole working set (~40 MB per replica, under the 126 MB
L2), so no L2 flush is done between steps (noted in config).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

N > 1 (launched with torch.distributed.run): replicas only -- every rank runs
its own four replicas (seeds 4*rank .. 4*rank+3); the process group only times
(barrier, max over ranks) and sums events.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

WORKLOAD = "hetero2d_256"
METRIC = "KMC steps/s, chosen vs plain on 1 B200 at 1e-8 rel err; p50/p99 step latency"
UNIT = "KMC steps/s"
# algorithmic bytes of one FP64 LS iteration per voxel: read eps, eps_p, write eps
# (3 x S words), lam and mu (2 words), half spectrum written once and read once
# (S complex words / 2 each way); S = 3 in 2D, 6 in 3D
BYTES_LS = {2: 8 * (3 * 3 + 2) + 2 * 3 * 16 // 2, 3: 8 * (3 * 6 + 2) + 2 * 6 * 16 // 2}


def peaks():
    p = os.path.join(HERE, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    def __init__(self, index: int = 0):
        self.index = index
        self.proc = None
        self.lines = []
        self._t = None

    def start(self):
        cmd = ["nvidia-smi", "-i", str(self.index), "--query-gpu=clocks.sm,clocks.max.sm,power.draw,"
               "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
               "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap,utilization.gpu",
               "--format=csv,noheader,nounits", "-lms", "200"]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self._t = threading.Thread(target=self._read, daemon=True)
        self._t.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self._t:
            self._t.join(timeout=2)
        return summarize_clocks(self.lines)


def summarize_clocks(lines):
    """Clock summary of nvidia-smi sample lines (clocks.sm, clocks.max.sm,
    power.draw, four event reasons, utilization.gpu): the median SM clock
    under load (samples with the GPU at least half busy; the window also holds
    host-side gaps, where an idle GPU lowers its clock), the median over all
    samples, the largest max clock, and every event reason seen active."""
    sm, busy, mx, reasons = [], [], [], set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    for ln in lines:
        parts = [x.strip() for x in ln.split(",")]
        if len(parts) < 7:
            continue
        try:
            f = float(parts[0])
            m = float(parts[1])
        except ValueError:
            continue
        sm.append(f)
        mx.append(m)
        try:
            if len(parts) > 7 and float(parts[7]) >= 50.0:
                busy.append(f)
        except ValueError:
            pass
        for n, v in zip(names, parts[3:7]):
            if v.lower() == "active":
                reasons.add(n)
    load = busy if busy else sm
    return {"sm_mhz": float(np.median(load)) if load else None, "sm_max_mhz": max(mx) if mx else None,
            "reasons": sorted(reasons), "samples": len(sm), "samples_under_load": len(busy),
            "sm_mhz_all_samples": float(np.median(sm)) if sm else None,
            "what": "median SM clock over samples with utilization >= 50 % (all samples if none)"}


def _traffic(key: str):
    """A DRAM-traffic figure (dram__bytes_read.sum + dram__bytes_write.sum of
    one ncu capture, scaled to the unit named by the key) from
    profiles/traffic.json, written beside the ncu summaries it comes from."""
    p = os.path.join(HERE, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        return json.load(f).get(key)


def traffic_from_profiles(workload: str, iterations_per_launch: float):
    """DRAM bytes of one plain-form LS launch: the captured launch's bytes per
    LS iteration (ncu, ls_kernel on the workload's grid) times the launches'
    mean iteration count."""
    t = _traffic("ls_kernel/%s/bytes_per_iteration" % workload)
    return t * iterations_per_launch if t is not None else None


def batch_traffic_from_profiles(workload: str, events: float):
    """DRAM bytes of a batch_kernel launch of `events` thermal events: the
    captured launch's bytes per thermal event (the same four replicas) times
    the events, traffic growing with the events (each is a sweep and its LS
    iterations).  None without the figure."""
    t = _traffic("batch_kernel/%sx4/bytes_per_event" % workload)
    return t * events if t is not None else None


def host_cpu():
    """CPU model and whether it runs the AVX2/FMA build of the reference."""
    model, flags = "unknown", set()
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name") and model == "unknown":
                    model = line.split(":", 1)[1].strip()
                elif line.startswith("flags") and not flags:
                    flags = set(line.split(":", 1)[1].split())
    except OSError:
        pass
    return model, {"avx2", "fma", "bmi2"} <= flags


def run_reference(cfg_paths, n_events: int, timeout: float = 900.0):
    """Time the reference's own CPU path (the unmodified reference headers
    driven by oracle/_ref/ref_driver kmc_trace; its -O3 AVX2 build
    ref_driver_o3 where the host runs it): the first n_events thermal events of
    every workload in cfg_paths, one process each, all at once; setup
    excluded.  Returns the aggregate rate (events of all processes / the
    slowest process's loop time)."""
    model, v3 = host_cpu()
    drv = os.path.join(HERE, "oracle", "_ref", "ref_driver_o3")
    build = "-O3 -march=x86-64-v3"
    if not (v3 and os.path.exists(drv)):
        drv = os.path.join(HERE, "oracle", "_ref", "ref_driver")
        build = "-O2 -ffp-contract=off"
    if not os.path.exists(drv):
        return None, "oracle/_ref/ref_driver not built"
    dirs = [tempfile.mkdtemp(prefix="mgk_ref_") for _ in cfg_paths]
    procs = [subprocess.Popen([drv, "kmc_trace", c, d, "1000000", str(n_events)], stdout=subprocess.DEVNULL,
                              stderr=subprocess.PIPE, text=True) for c, d in zip(cfg_paths, dirs)]
    t_end = time.time() + timeout
    errs = []
    for p in procs:
        try:
            _, err = p.communicate(timeout=max(1.0, t_end - time.time()))
        except subprocess.TimeoutExpired:
            p.kill()
            p.communicate()
            errs.append("reference sample exceeded %.0f s" % timeout)
            continue
        if p.returncode != 0:
            errs.append("ref_driver failed: " + (err or "")[-300:])
    if errs:
        return None, errs[0]
    nev, secs = 0, 0.0
    for d in dirs:
        vals = open(os.path.join(d, "timing.txt")).read().split()
        nev += int(float(vals[1]))
        secs = max(secs, float(vals[2]))
    return {"events": nev, "seconds": secs, "value": nev / secs if secs > 0 else 0.0, "processes": len(cfg_paths),
            "cpu": model, "binary": os.path.basename(drv), "build": build}, None


def reduce_over_ranks(dist, seconds: float, events: float, device=None):
    """Max of the per-rank times, sum of the per-rank events (replicas)."""
    if dist is None:
        return seconds, events
    import torch
    t = torch.tensor([seconds], dtype=torch.float64, device=device)
    e = torch.tensor([events], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(e, op=dist.ReduceOp.SUM)
    return float(t.item()), float(e.item())


def sweep_bytes(cfg):
    """Algorithmic bytes of one sweep: per mode Q0 and the catalog read, Q
    written; per voxel the symmetric stress inputs (strain, plastic strain,
    lam, mu) and the softening state read."""
    D = cfg.dim
    S = 3 if D == 2 else 6
    C = 6 if (D == 3 and cfg.use_3d_barriers) else 2
    return cfg.n_voxels * (cfg.M * 8 * (2 + C) + 8 * (2 * S + 2 + 3))


T_START = time.time()


def progress(msg):
    print("[bench %7.1fs] %s" % (time.time() - T_START, msg), file=sys.stderr, flush=True)


def percentile(x, q):
    return float(np.percentile(x, q)) if len(x) else None


def ensemble_block(G, workloads, workdir, seconds, plain_events):
    """The 64-replica mixed ensemble in one launch for a `seconds` window of
    device time, and the plain form's rate per size class (plain_events
    events on one replica of each class, one after another)."""
    from mgkmc_cpp_b200.workloads import ENSEMBLE
    t0 = time.time()
    reps = workloads.ensemble(os.path.join(workdir, "ens"), ENSEMBLE)
    cfgs = [c for _, _, c in reps]
    b = G.KmcBatch(cfgs)
    t_setup = time.time() - t0
    progress("ensemble: %d replicas set up in %.1f s" % (len(cfgs), t_setup))
    b.set_time_limit(min(seconds, 5.0))
    b.run(10 ** 9)  # warm-up
    progress("ensemble: warm-up done")
    # timed: once every replica is past the window each stops at its next decision; the
    # launch ends when the last one does (its overshoot is counted as time)
    b.set_time_limit(seconds)
    ms = b.run(10 ** 9)
    progress("ensemble: timed run %.1f s" % (ms / 1e3))
    st = [b.stats(r) for r in range(len(cfgs))]
    events = sum(x["events"] for x in st)
    vox_iters = sum(x["ls_iters"] * c.n_voxels for x, c in zip(st, cfgs))
    lat = np.concatenate([x["event_us"] for x in st if len(x["event_us"])]) if events else np.zeros(0)
    classes = {}
    rep_rate = []
    for name, x in zip(ENSEMBLE, st):
        k = classes.setdefault(name, {"replicas": 0, "events": 0, "ctas": int(x["ctas"])})
        k["replicas"] += 1
        k["events"] += int(x["events"])
        rep_rate.append((name, x["events"] / (ms / 1e3) if ms > 0 else 0.0))
    b.close()
    # plain form, replica by replica: per-class rate on the class's first replica
    kw = dict(enable_console_log=False, enable_summary_log=False, enable_global_log=False)
    plain_time = 0.0
    for name, k in classes.items():
        c = cfgs[ENSEMBLE.index(name)]
        sim = G.from_config(c, output_dir=os.path.join(workdir, "ens_plain"))
        sim.run_simulation(10 ** 6, c.step_size, c.driving, c.targets, c.mixed_tol_pa, 50, max_events=3, **kw)
        sim.set_profiling(True)
        e0 = sim.stats["thermal_events"]
        sim.run_simulation(10 ** 6, c.step_size, c.driving, c.targets, c.mixed_tol_pa, 50, max_events=plain_events,
                           **kw)
        ev = sim.stats["thermal_events"] - e0
        rate = ev / (sim.profile()["run_ms"] / 1e3) if ev else 0.0
        k["plain_steps_per_s"] = rate
        progress("ensemble: plain %s %.1f steps/s" % (name, rate))
        if rate > 0:
            plain_time += k["events"] / rate
        del sim
    chosen = events / (ms / 1e3) if ms > 0 else 0.0
    plain = events / plain_time if plain_time > 0 else None
    # per class: the class's events per second in the batch against the plain
    # form's per-replica rate (what running the class's replicas one after
    # another would give); makespan: the time for every replica to advance
    # 20 events, in the batch (its slowest replica) and replica by replica
    for k in classes.values():
        k["batch_steps_per_s"] = k["events"] / (ms / 1e3) if ms > 0 else 0.0
        p = k.get("plain_steps_per_s") or 0.0
        k["speedup_vs_plain"] = k["batch_steps_per_s"] / p if p > 0 else None
    K = 20
    mk_batch = max((K / r for _, r in rep_rate if r > 0), default=None)
    mk_plain = sum(K / classes[n]["plain_steps_per_s"] for n, _ in rep_rate
                   if classes[n].get("plain_steps_per_s"))
    makespan = {"events_per_replica": K, "batch_s": mk_batch, "plain_replica_by_replica_s": mk_plain,
                "speedup": (mk_plain / mk_batch) if mk_batch else None}
    return {"replicas": len(cfgs), "composition": "16x2D 64^2, 16x2D 128^2, 16x2D 512^2, 5x3D 32^3, 5x3D 48^3, "
                                                "6x3D 96^3 (M 18 in 2D, 100 in 3D)",
            "device_seconds": ms / 1e3, "events": int(events), "value": chosen, "unit": UNIT,
            "ls_voxel_iterations_per_s": vox_iters / (ms / 1e3) if ms > 0 else None,
            "plain_replica_by_replica": plain, "speedup_vs_plain": (chosen / plain) if plain else None,
            "latency_us": {"p50": percentile(lat, 50), "p99": percentile(lat, 99)},
            "per_class": classes, "makespan": makespan, "setup_seconds": t_setup}


# algorithmic bytes of one LS iteration per voxel with an FP32 spectrum: the
# FP64 real-space traffic and S complex FP32 words written and read once
BYTES_LS_FP32 = {2: 8 * (3 * 3 + 2) + 2 * 3 * 8 // 2, 3: 8 * (3 * 6 + 2) + 2 * 6 * 8 // 2}


def precision_block(G, cases=(((512, 512), 11), ((64, 64, 64), 12)), solves=3):
    """The precision form of the LS solve: FP64 against FP32-refined (FP32
    spectrum and FFTs to a relative change of 1e-6, then FP64 iterations), on
    a lognormal modulus field (CoV 0.1), cold starts at the reference's
    tolerance (1e-6) timed on the device, and the two fields compared after
    both are solved to 1e-11."""
    from mgkmc_cpp_b200 import fields
    out = {}
    for dims, seed in cases:
        D = len(dims)
        N = int(np.prod(dims))
        E = fields.lognormal_modulus(dims, 90e9, 0.10, 4.0 if D == 2 else 3.0, seed).reshape(-1)
        nu = np.full(N, 0.36)
        eb = np.zeros((D, D))
        eb[0, 0], eb[1, 1], eb[0, 1], eb[1, 0] = 1e-3, -4e-4, 2e-4, 2e-4
        row, fields_at = {}, {}
        for prec in ("fp64", "fp32_refined"):
            s = G.LsSolver(dims, E, nu, precision=prec)
            s.solve(eb, tol=1e-6)
            ms, its = [], []
            for _ in range(solves):
                r = s.solve(eb, tol=1e-6)
                ms.append(s.last_solve_ms())
                its.append(r[4])
            fields_at[prec] = s.solve(eb, tol=1e-11, max_iter=1000)[0]
            s.close()
            t = float(np.median(ms))
            it = float(np.median(its))
            per_voxel = BYTES_LS[D] if prec == "fp64" else BYTES_LS_FP32[D]
            row[prec] = {"ms_per_solve": t, "iterations": it, "ls_voxel_iterations_per_s": N * it / (t / 1e3),
                         "achieved_gbs": per_voxel * N * it / (t / 1e3) / 1e9}
        e64, e32 = fields_at["fp64"], fields_at["fp32_refined"]
        row["field_rel_l2_fp32_refined_vs_fp64_at_tol_1e-11"] = float(np.linalg.norm(e32 - e64) / np.linalg.norm(e64))
        row["speedup"] = row["fp64"]["ms_per_solve"] / row["fp32_refined"]["ms_per_solve"]
        out["x".join(map(str, dims))] = row
        progress("precision: %s fp64 %.3f ms, fp32-refined %.3f ms" % (dims, row["fp64"]["ms_per_solve"],
                                                                       row["fp32_refined"]["ms_per_solve"]))
    return out


def kmc_precision_block(G, workloads, workdir, events=100, seed=0, workload="hetero2d_256"):
    """The chosen form's LS re-solves in FP32-refined arithmetic against FP64:
    the same replica (one seed of the benchmark workload) advanced `events`
    thermal events in the batched kernel in each arithmetic, both with the
    LS re-solves converged to a relative change of 1e-10 (the benchmark
    description's tolerance; at the reference's 1e-6 both stop ~1e-7 from
    the fixed point, along different paths).  Reports the
    flip-sequence agreement (the fraction of events whose selected mode is
    the same as in the FP64 run, up to the first difference and over the
    whole run), the strain field's relative L2 difference after the run, the
    device time of each and their LS iteration counts."""
    import dataclasses
    _, cfg = workloads.write_workload(workload, os.path.join(workdir, "prec"), seed=seed)
    out = {}
    res = {}
    for prec in ("fp64", "fp32_refined"):
        c = dataclasses.replace(cfg, ls_precision=prec, ls_tol=1e-10)
        b = G.KmcBatch([c])
        b.run(3)  # warm-up (its own, identical in both arithmetics up to rounding)
        ms = b.run(events)
        st = b.stats(0)
        res[prec] = (st["selected"], b.field(0, "eps_field"), ms, st)
        out[prec] = {"device_ms": ms, "events": int(st["events"]), "ls_iterations": int(st["ls_iters"]),
                     "steps_per_s": st["events"] / (ms / 1e3) if ms > 0 else None}
        b.close()
    s64, e64 = res["fp64"][0], res["fp64"][1]
    s32, e32 = res["fp32_refined"][0], res["fp32_refined"][1]
    n = min(len(s64), len(s32))
    same = s64[:n] == s32[:n]
    first = int(np.argmin(same)) if not same.all() else n
    out.update({"workload": workload, "seed": seed, "events_compared": n, "identical_prefix": first,
                "flip_agreement": float(same.mean()) if n else None,
                "field_rel_l2_vs_fp64": float(np.linalg.norm(e32 - e64) / np.linalg.norm(e64)),
                "speedup": out["fp64"]["device_ms"] / out["fp32_refined"]["device_ms"]
                if out["fp32_refined"]["device_ms"] > 0 else None})
    progress("kmc precision: agreement %s, field %.2e, speedup %.2f" % (out["flip_agreement"],
                                                                          out["field_rel_l2_vs_fp64"], out["speedup"]))
    return out


def cfg2_block(G, workloads, workdir, events=10):
    """The benchmark's config 2 physics (workload bl_cfg2_64: 3D 64^3, lognormal
    E CoV 0.15, 100 Fibonacci-plane shears of gamma0 0.1 along the local
    resolved shear stress, per-voxel dF N(1.0, 0.1) eV clipped to [0.6, 1.4],
    z tension): thermal events per second of the plain and the batched form."""
    _, cfg = workloads.write_workload("bl_cfg2_64", os.path.join(workdir, "cfg2"), seed=0)
    kw = dict(enable_console_log=False, enable_summary_log=False, enable_global_log=False)
    sim = G.from_config(cfg, output_dir=None)
    sim.run_simulation(10 ** 6, cfg.step_size, cfg.driving, cfg.targets, cfg.mixed_tol_pa, 50, max_events=2, **kw)
    sim.set_profiling(True)
    e0 = sim.stats["thermal_events"]
    sim.run_simulation(10 ** 6, cfg.step_size, cfg.driving, cfg.targets, cfg.mixed_tol_pa, 50, max_events=events, **kw)
    ev = sim.stats["thermal_events"] - e0
    plain = ev / (sim.profile()["run_ms"] / 1e3) if ev else None
    del sim
    b = G.KmcBatch([cfg])
    b.run(2)
    ms = b.run(events)
    st = b.stats(0)
    b.close()
    out = {"workload": "bl_cfg2_64", "modes": cfg.n_voxels * cfg.M, "plain_steps_per_s": plain,
           "batched_steps_per_s": st["events"] / (ms / 1e3) if ms > 0 else None, "batched_events": int(st["events"]),
           "ls_iterations_per_step": st["ls_iters"] / max(st["events"], 1)}
    progress("cfg2: plain %s, batched %s steps/s" % (plain, out["batched_steps_per_s"]))
    return out


def ls_sweep_block(G, grids, iters=20, reps=5):
    """The FP64 LS iteration alone: for each grid (a seeded lognormal modulus
    field, CoV 0.1), cold solves of 2 and 2 + iters fixed iterations (tol 0),
    the difference of their median device times over `iters`; algorithmic
    bytes 136 B (2D) / 256 B (3D) per voxel-iteration; the measured pass plan."""
    from mgkmc_cpp_b200 import fields
    out = {}
    for dims in grids:
        D, N = len(dims), int(np.prod(dims))
        E = fields.lognormal_modulus(dims, 90e9, 0.10, 4.0 if D == 2 else 3.0, 3).reshape(-1)
        s = G.LsSolver(dims, E, np.full(N, 0.36))
        eb = np.zeros((D, D))
        eb[0, 0], eb[1, 1] = 1e-3, -4e-4
        s.solve(eb, max_iter=5, tol=0.0)
        t = {}
        for it in (2, 2 + iters):
            ms = []
            for _ in range(reps):
                s.solve(eb, max_iter=it, tol=0.0)
                ms.append(s.last_solve_ms())
            t[it] = float(np.median(ms))
        per = (t[2 + iters] - t[2]) / iters
        row = {"us_per_iteration": per * 1e3, "achieved_gbs": BYTES_LS[D] * N / (per * 1e-3) / 1e9, "plan": s.plan()}
        s.close()
        out["x".join(map(str, dims))] = row
        progress("ls: %s %.2f us/iteration" % (dims, per * 1e3))
    return out


def serve_block(G, workloads, workdir, n_jobs, flips, sizes, slice_seconds=0.05, plain_events=20, max_seconds=None,
                build_threads=4):
    """The serving loop on a Poisson request stream (20 jobs/s, seed 7): jobs
    are admitted as they arrive (wall clock) and as memory allows, every
    active job advances in shared batched launches of slice_seconds of device
    time, finished jobs retire.  Returns throughput, per-step latency and job
    completion latency."""
    jobs = workloads.serve_jobs(os.path.join(workdir, "serve"), n_jobs, flips=flips, sizes=sizes)
    # a job without a thermal event for 5 s of device time is in an avalanche
    # that never ends (the reference would run it forever): retired as stalled
    # jobs after the first of their grid shape are built on host threads
    # while the GPU runs the active ones (their initial draws follow the
    # reference's sequential random stream on the host)
    srv = G.Server(slice_seconds=slice_seconds, stall_seconds=5.0, build_threads=build_threads)
    for arrival, cfg, target in jobs:
        srv.submit(cfg, target, arrival=arrival)
    t0 = time.perf_counter()
    dev_ms = 0.0
    capped = False
    while not srv.idle():
        now = time.perf_counter() - t0
        if max_seconds is not None and now > max_seconds:
            capped = True  # the window ends: report what finished and what ran
            break
        if not srv.active and srv.queue and srv.queue[0]["arrival"] > now:
            time.sleep(min(0.05, srv.queue[0]["arrival"] - now))
            continue
        dev_ms += srv.step(now)
        if srv.launches % 20 == 0:
            progress("serving: %d launches, %d active, %d queued, %d done" % (srv.launches, len(srv.active),
                                                                                len(srv.queue), len(srv.done)))
    wall = time.perf_counter() - t0
    srv.close()
    done = list(srv.done.values())
    events_unfinished = sum(j["events"] for j in srv.active)
    events = sum(j["events"] for j in done)
    stalled = [j for j in done if j["stalled"]]
    terminated = [j for j in done if not j["stalled"] and j["events"] < j["target"]]
    comp = [j["finished"] - j["arrival"] for j in done]
    lat = np.array(srv.step_latency_us)
    # the plain form on the same job stream: each size class's rate on its
    # first job that reached its target (plain_events events after 3 of
    # warm-up; a stalled job's avalanche would never end a plain run), every
    # job's events at its class's rate, one job after another
    kw = dict(enable_console_log=False, enable_summary_log=False, enable_global_log=False)
    rates = {}
    for j in sorted(done, key=lambda x: x["id"]):
        cfg = j["cfg"]
        key = (cfg.dim, cfg.nx)
        if key in rates or j["stalled"] or j["events"] < plain_events + 3:
            continue
        sim = G.from_config(cfg, output_dir=None)
        sim.run_simulation(10 ** 6, cfg.step_size, cfg.driving, cfg.targets, cfg.mixed_tol_pa, 50, max_events=3, **kw)
        sim.set_profiling(True)
        e0 = sim.stats["thermal_events"]
        sim.run_simulation(10 ** 6, cfg.step_size, cfg.driving, cfg.targets, cfg.mixed_tol_pa, 50,
                           max_events=plain_events, **kw)
        ev = sim.stats["thermal_events"] - e0
        rates[key] = ev / (sim.profile()["run_ms"] / 1e3) if ev else 0.0
        del sim
    served = done + list(srv.active)
    plain_events_s = sum(j["events"] / rates[(j["cfg"].dim, j["cfg"].nx)] for j in served
                         if rates.get((j["cfg"].dim, j["cfg"].nx)))
    # a stalled job's avalanche never ends a plain run either: run job by job,
    # the plain form needs the same detector and spends the same window on it
    stall_budget = srv.stall_seconds * len(stalled)
    plain_s = plain_events_s + stall_budget
    ev_all = events + events_unfinished
    return {"jobs": len(done), "arrivals": "Poisson 20 jobs/s, seed 7", "flips_per_job": list(flips),
            "sizes": ["%s %d" % x for x in sizes], "slice_seconds": slice_seconds, "events": int(events),
            "wall_seconds": wall, "device_seconds": dev_ms / 1e3, "launches": srv.launches,
            "build_threads": build_threads, "jobs_built_on_threads": srv.built_on_pool,
            "host_seconds": {k: round(v, 2) for k, v in srv.host_seconds.items()},
            "stalled_jobs": len(stalled), "stalled_why": "no thermal event for %.0f s of device time (an avalanche "
                                                        "whose cascade batches never settle)" % srv.stall_seconds,
            "terminated_jobs": len(terminated),
            "value": (events + events_unfinished) / wall if wall > 0 else None, "unit": UNIT,
            "window_capped": capped, "jobs_unfinished": len(srv.active) + len(srv.queue),
            "events_in_unfinished_jobs": int(events_unfinished),
            "plain_job_by_job_seconds": plain_s, "plain_stall_budget_seconds": stall_budget,
            "plain_what": "every job's events at its size class's plain-form rate, one job after another, plus "
                          "the stall window for each stalled job (a plain run leaves a never-ending avalanche only "
                          "by the same detector)",
            "plain_steps_per_s": ev_all / plain_s if plain_s > 0 else None,
            "speedup_vs_plain": plain_s / wall if plain_s > 0 and wall > 0 else None,
            "speedup_vs_plain_without_stall_budget": plain_events_s / wall if plain_events_s > 0 and wall > 0 else None,
            "plain_rates_by_class": {"%dD %d" % k: v for k, v in rates.items()},
            "step_latency_us": {"p50": percentile(lat, 50), "p99": percentile(lat, 99)},
            "job_completion_s": {"p50": percentile(comp, 50), "p99": percentile(comp, 99)}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000, help="thermal events per replica in the timed region")
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default=WORKLOAD)
    ap.add_argument("--replicas", type=int, default=4)
    ap.add_argument("--cpu-events", type=int, default=40, help="events per replica in the bounded CPU-baseline sample")
    ap.add_argument("--ref-events", type=int, default=150, help="events per replica timed by --impl reference")
    ap.add_argument("--no-ensemble", action="store_true", help="skip the 64-replica ensemble block")
    ap.add_argument("--no-precision", action="store_true", help="skip the FP64 / FP32-refined LS block")
    ap.add_argument("--ls-sweep", nargs="+", default=None, metavar="NXxNY[xNZ]",
                    help="run only the FP64 LS iteration microbenchmark on these grids and print its JSON")
    ap.add_argument("--only-precision", action="store_true",
                    help="run only the FP64 / FP32-refined LS block and print its JSON (profiling the LS kernels)")
    ap.add_argument("--ensemble-seconds", type=float, default=40.0)
    ap.add_argument("--ensemble-plan", default="throughput", choices=["throughput", "balanced"],
                    help="how the ensemble's batch spreads CTAs over the replicas (mgk_set_batch_plan)")
    ap.add_argument("--serve-jobs", type=int, default=40, help="jobs of the serving block (0: skip)")
    ap.add_argument("--serve-flips", type=int, nargs=2, default=[50, 500])
    ap.add_argument("--serve-seconds", type=float, default=None, help="wall-time cap of the serving block")
    ap.add_argument("--serve-plan", default="throughput", choices=["throughput", "balanced"])
    ap.add_argument("--serve-full-sizes", action="store_true",
                    help="serve the full size set (2D 32^2..512^2, 3D 32^3, 64^3); default 2D 32^2..256^2, 3D 32^3")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    from mgkmc_cpp_b200 import workloads

    workdir = tempfile.mkdtemp(prefix="mgk_bench_")
    seeds = [args.replicas * rank + i for i in range(args.replicas)]
    made = [workloads.write_workload(args.workload, workdir, seed=sd) for sd in seeds]
    cfg_paths = [m[0] for m in made]
    cfgs = [m[1] for m in made]
    cfg = cfgs[0]
    base_cfg = {"workload": args.workload, "replicas": args.replicas, "seeds": seeds,
                "grid": [cfg.nx, cfg.ny] + ([cfg.nz] if cfg.dim == 3 else []), "M": cfg.M,
                "modes_per_replica": cfg.n_voxels * cfg.M, "temperature_K": cfg.temperature,
                "step": "one thermal KMC event of one replica", "steps_are": "thermal events per replica",
                "form": "chosen: batched device-resident kernel, fp64, the reference's RNG stream continued on the GPU",
                "l2": "working set < L2 (126 MB) per replica; no flush between steps",
                "parallelism": "replicas" if args.gpus > 1 else "single GPU, %d replicas" % args.replicas}

    if args.impl == "reference":
        if rank != 0:
            return 0
        res, err = run_reference(cfg_paths, max(3, min(args.steps, args.ref_events)))
        if res is None:
            print(json.dumps({"impl": "reference", "unavailable": err}))
            return 0
        sample = ("first %d thermal events of each of %d replicas of %s (seeds %s), one process per replica run "
                  "concurrently: the reference's KmcSimulation2D/3D methods driven through run_simulation's control "
                  "flow, each single-threaded by construction" % (res["events"] // len(cfg_paths), len(cfg_paths),
                                                                   args.workload, seeds))
        line = {"impl": "reference", "metric": METRIC, "value": res["value"], "unit": UNIT, "n_gpus": args.gpus,
                "steps": res["events"] // len(cfg_paths), "warmup": 0,
                "ms_per_step": 1e3 * res["seconds"] * len(cfg_paths) / max(res["events"], 1),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded lognormal modulus fields)", "config": base_cfg,
                "cpu_baseline": {"value": res["value"], "unit": UNIT, "cores": len(cfg_paths), "kind": "reference",
                                 "sample": sample, "cpu": res["cpu"], "binary": res["binary"], "build": res["build"]},
                "e2e": {"value": res["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return 0

    # ------------------------------------------------------------------ b200 arm
    import mgkmc_cpp_b200 as G

    if args.only_precision:
        print(json.dumps({"precision": precision_block(G)}))
        return 0
    if args.ls_sweep:
        grids = [tuple(int(x) for x in g.lower().split("x")) for g in args.ls_sweep]
        print(json.dumps({"ls_sweep": ls_sweep_block(G, grids)}))
        return 0

    dist, dev = None, None
    if world > 1:
        import torch
        import torch.distributed as tdist
        from datetime import timedelta

        torch.cuda.set_device(local_rank)
        dev = "cuda"
        tdist.init_process_group("nccl", timeout=timedelta(seconds=300))
        dist = tdist

    def barrier():
        if dist is not None:
            import torch
            torch.cuda.synchronize()
            dist.barrier()

    # chosen form: all replicas in one device-resident launch
    progress("chosen form: %d replicas" % len(cfgs))
    # clocks sampled from before the batch is built (nvidia-smi takes ~0.5 s to
    # start) to the end of the plain form's timed run
    clocks = ClockSampler(local_rank)
    clocks.start()
    batch = G.KmcBatch(cfgs)
    batch.run(args.warmup)
    barrier()
    # one public call: its launch is timed on the device (value) and the
    # whole call -- control blocks and generator states to the device, the
    # launch, counters, states, selections and event times back -- plus every
    # replica's macroscopic result read back, by the wall clock (e2e): the
    # same events for both
    t0 = time.perf_counter()
    ms = batch.run(args.steps)
    macros = [batch.macro(r) for r in range(len(cfgs))]
    barrier()
    t_e2e = time.perf_counter() - t0
    st = [batch.stats(r) for r in range(len(cfgs))]
    ev = sum(x["events"] for x in st)
    t_chosen, ev_all = reduce_over_ranks(dist, ms / 1e3, ev, dev)
    value = ev_all / t_chosen if t_chosen > 0 else 0.0
    lat = np.concatenate([x["event_us"] for x in st])
    iters = sum(x["ls_iters"] for x in st)
    sweeps = sum(x["sweeps"] for x in st)
    h2d = sum(x["h2d_bytes"] for x in st)
    d2h = sum(x["d2h_bytes"] for x in st) + sum(m.nbytes for m in macros)
    t_e2e, ev2_all = reduce_over_ranks(dist, t_e2e, ev, dev)
    ev2 = ev
    e2e_value = ev2_all / t_e2e if t_e2e > 0 else 0.0
    batch.close()

    # plain form: the drop-in engine, one replica (seed of this rank's first replica)
    progress("plain form")
    sim = G.from_config(cfg, output_dir=os.path.join(workdir, "out"))
    kw = dict(enable_console_log=False, enable_summary_log=False, enable_global_log=False)

    def segment(n):
        sim.run_simulation(10 ** 6, cfg.step_size, cfg.driving, cfg.targets, cfg.mixed_tol_pa, 50, max_events=n, **kw)

    segment(args.warmup)
    sim.set_profiling(True)
    p0 = sim.stats
    barrier()
    # the same segment timed on the device (its launches' CUDA events) and by
    # the wall clock through the public API (host RNG draws and every step's
    # copies included)
    t0 = time.perf_counter()
    segment(args.steps)
    barrier()
    tp_e2e = time.perf_counter() - t0
    prof = sim.profile()
    p1 = sim.stats
    clk = clocks.stop()
    pev = p1["thermal_events"] - p0["thermal_events"]
    t_plain, pev_all = reduce_over_ranks(dist, prof["run_ms"] / 1e3, pev, dev)
    plain_value = pev_all / t_plain if t_plain > 0 else 0.0
    tp_e2e, pev2 = reduce_over_ranks(dist, tp_e2e, pev, dev)
    plain_e2e = pev2 / tp_e2e if tp_e2e > 0 else 0.0
    sim.set_profiling(False)
    # the pass plan the LS autotuner picks for this grid (standalone solver)
    try:
        grid = (cfg.nx, cfg.ny) if cfg.dim == 2 else (cfg.nx, cfg.ny, cfg.nz)
        ls_plan = G.LsSolver(grid, cfg.E, cfg.nu).plan()
    except Exception as e:  # reported, not fatal
        ls_plan = {"error": str(e)[-200:]}
    del sim

    ens = None
    progress("ensemble")
    if not args.no_ensemble and rank == 0:
        try:
            G.set_batch_plan(args.ensemble_plan)
            ens = ensemble_block(G, workloads, workdir, args.ensemble_seconds, 20)
            ens["plan"] = args.ensemble_plan
            G.set_batch_plan("throughput")
        except Exception as e:  # reported, never silently dropped
            ens = {"error": str(e)[-300:]}
            progress("ensemble failed: " + ens["error"])
    prec = kprec = c2 = None
    if rank == 0 and not args.no_precision:
        try:
            prec = precision_block(G)
        except Exception as e:
            prec = {"error": str(e)[-300:]}
        try:
            kprec = kmc_precision_block(G, workloads, workdir)
        except Exception as e:
            kprec = {"error": str(e)[-300:]}
            progress("kmc precision failed: " + kprec["error"])
        try:
            c2 = cfg2_block(G, workloads, workdir)
        except Exception as e:
            c2 = {"error": str(e)[-300:]}
            progress("cfg2 failed: " + c2["error"])
    srv = None
    progress("serving")
    if args.serve_jobs > 0 and rank == 0:
        sizes = workloads.SERVE_SIZES if args.serve_full_sizes else [x for x in workloads.SERVE_SIZES
                                                                     if x in (("2d", 32), ("2d", 64), ("2d", 128),
                                                                              ("2d", 256), ("3d", 32))]
        try:
            G.set_batch_plan(args.serve_plan)
            srv = serve_block(G, workloads, workdir, args.serve_jobs, tuple(args.serve_flips), sizes,
                              max_seconds=args.serve_seconds)
            srv["plan"] = args.serve_plan
            G.set_batch_plan("throughput")
        except Exception as e:
            srv = {"error": str(e)[-300:]}
            progress("serving failed: " + srv["error"])
    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return 0
    peak, peak_kind = peaks()
    # roofline of the chosen form's kernel: algorithmic bytes of its sweeps
    # and LS iterations over the launch's CUDA-event time
    alg_bytes = sweeps * sweep_bytes(cfg) + iters * BYTES_LS[cfg.dim] * cfg.n_voxels
    achieved = alg_bytes / (ms / 1e3) / 1e9 if ms > 0 else 0.0
    n_launch = max(prof["ls_launches"], 1)
    avg_ms = prof["ls_ms"] / n_launch
    ls_bytes = BYTES_LS[cfg.dim] * cfg.n_voxels * prof["ls_iterations"] / n_launch
    ls_achieved = ls_bytes / (avg_ms * 1e-3) / 1e9 if avg_ms > 0 else 0.0
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t_chosen / max(ev, 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded lognormal modulus fields)",
            "config": dict(base_cfg, ls_iterations_per_step=iters / max(ev, 1), sweeps_per_step=sweeps / max(ev, 1),
                           ls_plan=ls_plan,
                           ctas_per_replica=[int(x["ctas"]) for x in st],
                           phase_ms={k[3:]: round(sum(x[k] for x in st) / len(st), 3) for k in st[0] if k.startswith("ms_")}),
            "latency_us": {"p50": percentile(lat, 50), "p99": percentile(lat, 99),
                           "what": "device time between consecutive thermal events of a replica"},
            "ls_voxel_iterations_per_s": iters * cfg.n_voxels / (ms / 1e3) if ms > 0 else None,
            "roofline": {"kernel": "batch_kernel (one persistent launch: every replica's sweeps, selections, flips, "
                                   "redraws and LS solves)", "bound": "hbm", "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind,
                         "traffic": batch_traffic_from_profiles(args.workload, ev),
                         "traffic_note": "ncu DRAM bytes per thermal event of a captured launch of the same four "
                                         "replicas (profiles/traffic.json), times this launch's events",
                         "alg_bytes_per_launch": alg_bytes, "avg_launch_ms": ms},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d / max(ev2, 1),
                    "d2h_bytes_per_step": d2h / max(ev2, 1)},
            "gpu_launches": 1,
            "plain": {"value": plain_value, "unit": UNIT, "what": "drop-in form (mgk_kmc_run), replica by replica",
                      "chosen_speedup": value / plain_value if plain_value > 0 else None,
                      "latency_us": {"p50": percentile(prof["event_us"], 50), "p99": percentile(prof["event_us"], 99)},
                      "e2e": {"value": plain_e2e, "unit": UNIT,
                              "h2d_bytes_per_step": 8 * (1 + cfg.M * ((6 if (cfg.dim == 3 and cfg.use_3d_barriers) else 2) + 1)),
                              "d2h_bytes_per_step": 56 + 112 + 4},
                      "gpu_launches": int(p1["launches"] - p0["launches"]),
                      "roofline": {"kernel": "ls_kernel (one persistent launch per LS solve)", "bound": "hbm",
                                   "achieved": ls_achieved, "peak": peak, "unit": "GB/s", "frac": ls_achieved / peak,
                                   "traffic": traffic_from_profiles(args.workload,
                                                                    prof["ls_iterations"] / n_launch),
                                   "alg_bytes_per_launch": ls_bytes,
                                   "avg_launch_ms": avg_ms}},
            "clocks": clk}
    if ens is not None:
        line["ensemble"] = ens
    if srv is not None:
        line["serving"] = srv
    if prec is not None:
        line["precision"] = prec
    if kprec is not None:
        line["kmc_precision"] = kprec
    if c2 is not None:
        line["cfg2"] = c2
    if args.gpus == 1:
        progress("cpu baseline")
        res, err = run_reference(cfg_paths, args.cpu_events)
        if res is not None:
            line["cpu_baseline"] = {"value": res["value"], "unit": UNIT, "cores": len(cfg_paths), "kind": "reference",
                                    "cpu": res["cpu"], "binary": res["binary"], "build": res["build"],
                                    "sample": "first %d thermal events of each replica of the same workload, one "
                                              "reference process (oracle/_ref/ref_driver) per replica run "
                                              "concurrently, setup excluded" % args.cpu_events}
        else:
            line["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": len(cfg_paths), "kind": "reference",
                                    "sample": err}
    print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
