"""The linear-elastic simulation (main.cpp's simulation_type "linear_elastic")
against the reference executable's own logs (tests/golden/le*.npz, written by
oracle/_ref/mgkmc_ref from the reference sources).

The global log (every step's macroscopic strain and stress, fixed 6-decimal
text) and the Step / Eps / Sig columns of the summary log must match the
reference's line for line and column for column: identical text except for
components that are zero up to rounding noise (there the sign of a printed
zero may differ), every number within one unit of its last printed digit.
The macro values returned are checked against the log text too."""
import os

import numpy as np
import pytest

from helpers import golden

pytestmark = pytest.mark.gpu

LE_CASES = ["le2d_16x12_hetero", "le2d_12x10_stress_xy", "le3d_8x6x4_hetero"]


def summary_columns(text):
    rows = []
    for line in text.splitlines()[2:]:
        f = line.split()
        if len(f) == 6:
            rows.append(" ".join(f[3:]))
    return "\n".join(rows)


def same_text(ours, ref):
    """Same lines, same columns, same text in every column but for the
    components that are zero up to rounding noise: there the last printed
    digit or the sign of a zero may differ, so numbers are held to one unit of
    the sixth decimal."""
    a, b = ours.splitlines(), ref.splitlines()
    assert len(a) == len(b)
    for la, lb in zip(a, b):
        if la == lb:
            continue
        fa, fb = la.split(), lb.split()
        assert len(fa) == len(fb) and fa[0] == fb[0], (la, lb)
        for x, y in zip(fa[1:], fb[1:]):
            assert abs(float(x) - float(y)) <= 1.01e-6, (la, lb)
        assert len(la) == len(lb) or abs(len(la) - len(lb)) <= la.count("-") + lb.count("-"), (la, lb)


@pytest.mark.parametrize("name", LE_CASES)
def test_linear_elastic_matches_reference_logs(name, tmp_path):
    import mgkmc_cpp_b200 as G
    from mgkmc_cpp_b200.workloads import load_config
    G._lib.require_device()
    g = golden(name)
    np.save(tmp_path / "E.npy", g["E_gpa"])
    out = tmp_path / "out"
    cfg = load_config(str(g["yaml"]).replace("$E", str(tmp_path / "E.npy")).replace("$OUT", str(out)))
    em, sm, iters = G.linear_elastic_run(cfg, str(out))
    glog = open(os.path.join(out, "global_log.txt")).read()
    same_text(glog, str(g["global_log"]))
    same_text(summary_columns(open(os.path.join(out, "summary_log.txt")).read()), str(g["summary"]))
    assert em.shape[0] == cfg.n_steps + 1 and iters > 0
    # the returned values are the logged ones
    rows = [l.split() for l in glog.splitlines()[2:]]
    D = cfg.dim
    cols = [(0, 0), (1, 1), (0, 1)] if D == 2 else [(0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2)]
    for s, r in enumerate(rows):
        for c, (i, j) in enumerate(cols):
            assert abs(float(r[1 + c]) - em[s, i, j]) <= 5e-7
            assert abs(float(r[1 + len(cols) + c]) - sm[s, i, j] / 1e9) <= 5e-7


def test_run_config_dispatches_linear_elastic(tmp_path):
    import mgkmc_cpp_b200 as G
    G._lib.require_device()
    g = golden("le2d_16x12_hetero")
    np.save(tmp_path / "E.npy", g["E_gpa"])
    out = tmp_path / "cli"
    cfgp = tmp_path / "cfg.yaml"
    cfgp.write_text(str(g["yaml"]).replace("$E", str(tmp_path / "E.npy")).replace("$OUT", str(out)))
    from mgkmc_cpp_b200.__main__ import main
    assert main([str(cfgp)]) == 0
    same_text(open(out / "global_log.txt").read(), str(g["global_log"]))
