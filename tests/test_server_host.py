"""The request loop's host logic (Server) on the CPU, with stand-ins for the
device-side simulation and batch: admission gated by the memory budget, the
first job of a grid shape built between launches and the others on host
threads, jobs joining the batch when their build is done, retirement at the
target or after stall_seconds without an event, and close()."""
import threading
import time

import numpy as np
import pytest

import mgkmc_cpp_b200 as G
from mgkmc_cpp_b200 import workloads


class FakeSim:
    def __init__(self, cfg, stall=False):
        self.cfg, self.stall, self.events, self.closed = cfg, stall, 0, False
        self.thread = threading.current_thread().name

    @property
    def eps_field(self):
        return np.zeros(3)

    def macro(self):
        return np.zeros(4)

    def close(self):
        self.closed = True


class FakeBatch:
    """Advances every simulation by up to 7 events a launch (none for a
    stalling one); a launch takes 1000 ms of device time."""
    built = 0

    def __init__(self, sims=None):
        FakeBatch.built += 1
        self.sims, self.cfgs, self.limit = list(sims), None, None

    def set_time_limit(self, s):
        self.limit = s

    def run(self, max_events, budgets=None):
        self._ev = [0 if s.stall else min(7, b) for s, b in zip(self.sims, budgets)]
        return 1000.0

    def stats(self, r):
        s, n = self.sims[r], self._ev[r]
        sel = np.arange(s.events, s.events + n, dtype=np.int64)
        s.events += n
        return {"events": n, "selected": sel, "event_us": np.ones(n), "terminated": 0}

    def close(self):
        pass


@pytest.fixture
def fakes(monkeypatch):
    stalling = set()

    def from_config(cfg, output_dir=None):
        time.sleep(0.01)  # a build takes a while
        return FakeSim(cfg, stall=id(cfg) in stalling)

    monkeypatch.setattr(G, "from_config", from_config)
    monkeypatch.setattr(G, "KmcBatch", FakeBatch)
    monkeypatch.setattr(G, "current_device", lambda: 0)
    monkeypatch.setattr(G, "_build_on", lambda dev, cfg: from_config(cfg))
    monkeypatch.setattr(G, "device_memory", lambda: (1 << 40, 1 << 40))
    return stalling


def cfgs(tmp_path, names):
    return [workloads.write_workload(n, str(tmp_path / str(i)), seed=i)[1] for i, n in enumerate(names)]


def test_first_job_of_a_shape_built_between_launches_others_on_threads(fakes, tmp_path):
    cs = cfgs(tmp_path, ["ens2d_64", "ens2d_128", "ens2d_64", "ens2d_128", "ens2d_64", "ens2d_64"])
    srv = G.Server(slice_seconds=0.05, build_threads=2, hbm_budget=1 << 40)
    ids = [srv.submit(c, 30) for c in cs]
    srv.step()
    # the first 64^2 and the first 128^2 job were built in this thread and run
    # in the first launch; the other four were handed to the pool
    assert srv.built_on_pool == 4
    first = {j["id"] for j in srv.active}
    assert first <= {ids[0], ids[1]} and ids[0] in first
    while not srv.idle():
        srv.step()
    srv.close()
    for j in ids:
        job = srv.done[j]
        assert job["events"] == 30 and not job["stalled"]
        assert np.array_equal(job["selected"], np.arange(30))  # each job's own events, in order
    assert srv.committed == 0
    assert set(srv.host_seconds) == {"build_wait", "rebuild", "readback", "retire"}


def test_admission_gated_by_the_budget(fakes, tmp_path):
    cs = cfgs(tmp_path, ["ens2d_64"] * 3)
    need = G.job_device_bytes(cs[0])
    srv = G.Server(slice_seconds=0.05, build_threads=2, hbm_budget=int(1.5 * need))
    for c in cs:
        srv.submit(c, 14)
    launches_with_two = 0
    while not srv.idle():
        srv.step()
        assert srv.committed <= srv.budget
        launches_with_two += len(srv.active) + len(srv.building) > 1
    srv.close()
    assert launches_with_two == 0
    assert len(srv.done) == 3 and srv.launches == 6  # two launches of 7 events per job, one job at a time


def test_stalled_job_retired_and_arrivals_respected(fakes, tmp_path):
    cs = cfgs(tmp_path, ["ens2d_64", "ens2d_64", "ens2d_64"])
    fakes.add(id(cs[1]))  # this one never gets a thermal event
    srv = G.Server(slice_seconds=0.05, build_threads=1, hbm_budget=1 << 40, stall_seconds=3.0)
    a = srv.submit(cs[0], 21, arrival=0.0)
    b = srv.submit(cs[1], 21, arrival=0.0)
    c = srv.submit(cs[2], 21, arrival=5.0)
    now = 0.0
    while not srv.idle():
        srv.step(now)
        if now < 5.0:  # not admitted before its arrival
            assert c not in srv.done and all(j["id"] != c for j in srv.active + srv.building)
        now += 1.0
    srv.close()
    assert srv.done[a]["events"] == 21 and not srv.done[a]["stalled"]
    assert srv.done[b]["stalled"] and srv.done[b]["events"] == 0
    assert srv.done[c]["admitted"] >= 5.0


def test_close_releases_jobs_still_building(fakes, tmp_path):
    cs = cfgs(tmp_path, ["ens2d_64"] * 4)
    srv = G.Server(slice_seconds=0.05, build_threads=2, hbm_budget=1 << 40)
    for c in cs:
        srv.submit(c, 1000)
    srv.step()
    sims_before = [j.get("sim") for j in srv.active]
    srv.close()
    assert srv.building == [] and srv._pool is None
    assert all(s.closed for s in sims_before if s is not None)
    assert all("sim" not in j for j in srv.active)


def test_bench_serving_block_bookkeeping(fakes, monkeypatch, tmp_path):
    """bench.py's serving block on the stand-ins: events, stalled jobs, and the
    plain comparison (every job's events at its class's plain rate, plus the
    stall window for each stalled job, which a plain run needs as well)."""
    import bench

    def plain_sim(cfg, output_dir=None):
        s = FakeSim(cfg)
        s.stats = {"thermal_events": 0}
        s.t0 = 0

        def run_simulation(*a, max_events=0, **k):
            s.stats["thermal_events"] += max_events

        def set_profiling(on):
            s.t0 = s.stats["thermal_events"]

        s.run_simulation, s.set_profiling = run_simulation, set_profiling
        s.profile = lambda: {"run_ms": 0.5 * (s.stats["thermal_events"] - s.t0)}  # 2000 steps/s
        return s

    made = []
    real_serve_jobs = workloads.serve_jobs

    def serve_jobs(*a, **k):
        jobs = real_serve_jobs(*a, **k)
        made.extend(jobs)
        fakes.add(id(jobs[2][1]))  # the third job never gets a thermal event
        return jobs

    monkeypatch.setattr(workloads, "serve_jobs", serve_jobs)
    srv_from_config = G.from_config
    # the serving loop builds with the stand-in above; the plain measurement afterwards
    # uses plain_sim (from_config is looked up at each call)
    calls = {"n": 0}

    def from_config(cfg, output_dir=None):
        calls["n"] += 1
        return srv_from_config(cfg) if calls["n"] <= len(made) else plain_sim(cfg)

    monkeypatch.setattr(G, "from_config", from_config)
    monkeypatch.setattr(G, "_build_on", lambda dev, cfg: from_config(cfg))
    out = bench.serve_block(G, workloads, str(tmp_path), 6, (30, 40), [("2d", 32)], slice_seconds=0.05,
                            plain_events=20, build_threads=2)
    targets = [t for _, _, t in made]
    assert out["jobs"] == 6 and out["stalled_jobs"] == 1 and out["terminated_jobs"] == 0
    assert out["events"] == sum(targets) - targets[2]
    assert out["plain_stall_budget_seconds"] == 5.0
    assert out["plain_job_by_job_seconds"] == pytest.approx(out["events"] / 2000.0 + 5.0)
    assert out["speedup_vs_plain"] > out["speedup_vs_plain_without_stall_budget"]
