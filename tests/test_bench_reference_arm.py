"""bench.py's reference arm on the CPU: the reference's own code
(oracle/_ref/ref_driver), one process per replica, prints one JSON line with
the contract's keys (or an `unavailable` line when the reference binaries
were not built)."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_json_line():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "3",
                        "--warmup", "3", "--ref-events", "3"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    if "unavailable" in line:
        return
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "dtype", "config", "cpu_baseline", "e2e"):
        assert k in line, k
    assert line["value"] > 0 and line["cpu_baseline"]["kind"] == "reference" and line["cpu_baseline"]["cores"] == 4
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0


def test_roofline_traffic_from_committed_profiles():
    """The roofline's DRAM traffic comes from profiles/traffic.json, beside the
    committed ncu summaries: the LS kernel's bytes per iteration scaled by a
    launch's iterations, and the batch kernel's bytes per event scaled by the
    events of the timed launch."""
    sys.path.insert(0, ROOT)
    import bench
    ls = bench.traffic_from_profiles("hetero2d_256", 10.0)
    assert ls is not None and ls > 0
    assert bench.traffic_from_profiles("hetero2d_256", 20.0) == 2 * ls
    per_event = bench.batch_traffic_from_profiles("hetero2d_256", 1)
    assert per_event is not None and 1e6 < per_event < 1e9
    assert bench.batch_traffic_from_profiles("hetero2d_256", 4000) == 4000 * per_event
    assert bench.batch_traffic_from_profiles("no_such_workload", 4000) is None
