#!/usr/bin/env python3
"""Benchmark: KMC steps/s of the STZ-KMC + Lippmann-Schwinger step on B200.

One step = one thermal KMC event of run_simulation (kmc_solver.hpp:783-938):
sweep of every (voxel, mode) barrier and rate, event selection, flip with its
catalog/barrier redraw, and the warm-started FP64 LS re-solve; cascades and the
end-of-interval mixed-BC solves that fall inside the timed segment are part of
the work, as in the reference.  Default workload ``hetero2d_256`` (2D 256x256
plane strain, seeded synthetic lognormal modulus field, CoV 0.10, correlation 4
voxels, M = 18 modes per voxel), the single-replica heterogeneous case.  Its
working set (~40 MB) is smaller than L2 and every step reads all of it; no L2
flush between steps (noted in config).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

N > 1 (launched with torch.distributed.run): independent replicas, one per
GPU, each with its own seed; no data-path collective ("replicas only"), the
process group only times (barrier, max over ranks) and sums events.
--impl reference times the reference's own CPU implementation (the reference
sources compiled by oracle/Makefile into oracle/_ref/ref_driver) on the same
workload (bounded sample), rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import re
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
               "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
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
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for n, v in zip(names, parts[3:7]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def traffic_from_profiles(workload: str):
    """DRAM bytes per LS launch from the committed ncu summary, if present."""
    p = os.path.join(HERE, "profiles", "ls_kernel_%s.md" % workload)
    if not os.path.exists(p):
        return None
    m = re.search(r"traffic_bytes_per_launch:\s*([0-9.eE+]+)", open(p).read())
    return float(m.group(1)) if m else None


def run_reference(cfg_path: str, n_events: int, timeout: float = 900.0):
    """Time the reference's own CPU path (oracle/_ref/ref_driver kmc_trace):
    the first n_events thermal events of the workload, setup excluded."""
    drv = os.path.join(HERE, "oracle", "_ref", "ref_driver")
    if not os.path.exists(drv):
        return None, "oracle/_ref/ref_driver not built"
    with tempfile.TemporaryDirectory() as d:
        try:
            r = subprocess.run([drv, "kmc_trace", cfg_path, d, "1000000", str(n_events)], capture_output=True, text=True,
                               timeout=timeout)
        except subprocess.TimeoutExpired:
            return None, "reference sample exceeded %.0f s" % timeout
        if r.returncode != 0:
            return None, "ref_driver failed: " + r.stderr[-300:]
        vals = open(os.path.join(d, "timing.txt")).read().split()
    nev, loop_s = int(float(vals[1])), float(vals[2])
    return {"events": nev, "seconds": loop_s, "value": nev / loop_s if loop_s > 0 else 0.0}, None


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


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default=WORKLOAD)
    ap.add_argument("--cpu-events", type=int, default=40, help="events in the bounded CPU-baseline sample")
    ap.add_argument("--ref-events", type=int, default=150, help="events timed by --impl reference (bounded sample)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    from mgkmc_cpp_b200 import workloads

    workdir = tempfile.mkdtemp(prefix="mgk_bench_")
    cfg_path, cfg = workloads.write_workload(args.workload, workdir, seed=rank)
    base_cfg = {"workload": args.workload, "grid": [cfg.nx, cfg.ny] + ([cfg.nz] if cfg.dim == 3 else []), "M": cfg.M,
                "modes": cfg.n_voxels * cfg.M, "temperature_K": cfg.temperature, "step": "one thermal KMC event",
                "form": "plain (fp64, host RNG replay of the reference's draws)",
                "l2": "working set < L2 (126 MB); no flush between steps",
                "parallelism": "replicas" if args.gpus > 1 else "single"}

    if args.impl == "reference":
        if rank != 0:
            return 0
        res, err = run_reference(cfg_path, max(3, min(args.steps, args.ref_events)))
        if res is None:
            print(json.dumps({"impl": "reference", "unavailable": err}))
            return 0
        sample = ("first %d thermal events of %s: the reference's KmcSimulation2D/3D methods driven through "
                  "run_simulation's control flow, single-threaded by construction" % (res["events"], args.workload))
        line = {"impl": "reference", "metric": METRIC, "value": res["value"], "unit": UNIT, "n_gpus": args.gpus,
                "steps": res["events"], "warmup": 0, "ms_per_step": 1e3 * res["seconds"] / max(res["events"], 1),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded lognormal modulus field)", "config": base_cfg,
                "cpu_baseline": {"value": res["value"], "unit": UNIT, "cores": 1, "kind": "reference", "sample": sample},
                "e2e": {"value": res["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return 0

    # ------------------------------------------------------------------ b200 arm
    import mgkmc_cpp_b200 as G

    dist, dev = None, None
    if world > 1:
        import torch
        import torch.distributed as tdist
        from datetime import timedelta

        torch.cuda.set_device(local_rank)
        dev = "cuda"
        tdist.init_process_group("nccl", timeout=timedelta(seconds=300))
        dist = tdist

    sim = G.from_config(cfg, output_dir=os.path.join(workdir, "out"))
    kw = dict(enable_console_log=False, enable_summary_log=False, enable_global_log=False)

    def segment(n):
        sim.run_simulation(10 ** 6, cfg.step_size, cfg.driving, cfg.targets, cfg.mixed_tol_pa, 50, max_events=n, **kw)

    def barrier():
        if dist is not None:
            import torch
            torch.cuda.synchronize()
            dist.barrier()

    segment(args.warmup)
    # timed region: device-resident state, CUDA-event timing on the engine stream
    sim.set_profiling(True)
    st0 = sim.stats
    clocks = ClockSampler(local_rank)
    clocks.start()
    barrier()
    segment(args.steps)
    barrier()
    clk = clocks.stop()
    prof = sim.profile()
    st1 = sim.stats
    events = st1["thermal_events"] - st0["thermal_events"]
    t_run, events_all = reduce_over_ranks(dist, prof["run_ms"] / 1e3, events, dev)
    value = events_all / t_run if t_run > 0 else 0.0
    lat = prof["event_us"]
    # e2e: the public API call under the host clock.  Every step copies its
    # inputs (target u2*total and the M redraw records, pinned) host->device and
    # reads its result (rate total, selection, LS macro tensors) device->host.
    sim.set_profiling(False)
    barrier()
    t0 = time.perf_counter()
    segment(args.steps)
    barrier()
    t_e2e = time.perf_counter() - t0
    st2 = sim.stats
    t_e2e, ev_e2e = reduce_over_ranks(dist, t_e2e, st2["thermal_events"] - st1["thermal_events"], dev)
    e2e_value = ev_e2e / t_e2e if t_e2e > 0 else 0.0
    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return 0
    peak, peak_kind = peaks()
    n_launch = max(prof["ls_launches"], 1)
    avg_ms = prof["ls_ms"] / n_launch
    alg_bytes = BYTES_LS[cfg.dim] * cfg.n_voxels * prof["ls_iterations"] / n_launch
    achieved = alg_bytes / (avg_ms * 1e-3) / 1e9 if avg_ms > 0 else 0.0
    C = 6 if (cfg.dim == 3 and cfg.use_3d_barriers) else 2
    kernel_ms = {"ls_kernel": prof["ls_ms"], "sweep_kernel": prof["sweep_ms"], "select_flip_kernel": prof["select_ms"],
                 "timed_region": prof["run_ms"]}
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": int(events_all),
            "warmup": args.warmup, "ms_per_step": 1e3 * t_run / max(events, 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded lognormal modulus field)",
            "config": dict(base_cfg, ls_iterations_per_step=prof["ls_iterations"] / max(events, 1), kernel_ms=kernel_ms,
                           cascades=st1["cascades"] - st0["cascades"]),
            "latency_us": {"p50": float(np.percentile(lat, 50)) if len(lat) else None,
                           "p99": float(np.percentile(lat, 99)) if len(lat) else None},
            "roofline": {"kernel": "ls_kernel (one persistent launch per LS solve)", "bound": "hbm",
                         "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_source": peak_kind, "traffic": traffic_from_profiles(args.workload),
                         "alg_bytes_per_launch": alg_bytes, "avg_launch_ms": avg_ms},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 8 * (1 + cfg.M * (C + 1)),
                    "d2h_bytes_per_step": 56 + 112 + 4},
            "gpu_launches": int(st1["launches"] - st0["launches"]),
            "clocks": clk}
    if args.gpus == 1:
        res, err = run_reference(cfg_path, args.cpu_events)
        if res is not None:
            line["cpu_baseline"] = {"value": res["value"], "unit": UNIT, "cores": 1, "kind": "reference",
                                    "sample": "first %d thermal events of the same workload, reference code "
                                              "(oracle/_ref/ref_driver), setup excluded" % res["events"]}
        else:
            line["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": 1, "kind": "reference", "sample": err}
    print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
