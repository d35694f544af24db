"""Shared helpers for the test suite (fixture loading, comparisons)."""
import os
import tempfile

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def rel(a, b):
    a, b = np.ravel(a), np.ravel(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def kmc_config_from_golden(g):
    """SimConfig of a golden KMC case (writes its modulus field to a temp file)."""
    from mgkmc_cpp_b200.config import SimConfig, YAMLConfig
    y = str(g["yaml"])
    if "E_gpa" in g:
        d = tempfile.mkdtemp()
        p = os.path.join(d, "E.npy")
        np.save(p, g["E_gpa"])
        y = y.replace("$E", p)
    return SimConfig.from_yaml(YAMLConfig.loads(y)), y


KMC_CASES = ["kmc2d_12_nosoft", "kmc2d_8_soft_neigh", "kmc2d_8_kmcmode", "kmc2d_10_hetero_stress", "kmc2d_8_noredraw",
             "kmc2d_8_mixexp", "kmc3d_6x6x4_soft", "kmc3d_5x4x3_b3dir"]
LS_CASES = ["ls2d_16_fixed3", "ls2d_16_conv", "ls2d_12x10_stress_warm", "ls2d_9x7_odd", "ls2d_32_homog",
            "ls2d_48x30_fixed2", "ls3d_8_fixed2", "ls3d_6x4x5_conv", "ls3d_8x8x1_conv", "ls3d_12x6x10_conv"]
KMC_RUN = {"kmc2d_12_nosoft": (25, 300), "kmc2d_8_soft_neigh": (25, 300), "kmc2d_8_kmcmode": (25, 300),
           "kmc2d_10_hetero_stress": (25, 300), "kmc2d_8_noredraw": (25, 300), "kmc2d_8_mixexp": (25, 300),
           "kmc3d_6x6x4_soft": (25, 300), "kmc3d_5x4x3_b3dir": (25, 300)}


def compare_trace(tr, ref, tol=1e-9, eps_floor=0.0, sig_floor=0.0):
    """Kinds, selected indices and counters must be identical; the continuous
    columns (total rate, wait, clock, macro tensors) within `tol` relative to
    each column's scale.  A macro tensor is a mean over the field, whose
    rounding noise scales with the field's own magnitude: eps_floor and
    sig_floor (the fields' RMS) put a floor under the tensors' scales, for
    runs whose mean strain is still far below the local strains."""
    assert tr.shape == ref.shape, (tr.shape, ref.shape)
    kind = ref[:, 0]
    assert np.array_equal(tr[:, 0], kind)
    ev = kind != 2  # column 1 of an interval-end row is the u1 draw (float)
    assert np.array_equal(tr[ev, 1], ref[ev, 1])
    assert np.array_equal(tr[:, 2], ref[:, 2])
    DD = (ref.shape[1] - 6) // 2
    scale = np.abs(ref[:, 3:]).max(axis=0) + 1e-300
    # tensor columns share one scale per tensor (components that are zero in
    # exact arithmetic carry only rounding noise)
    scale[3:3 + DD] = max(scale[3:3 + DD].max(), eps_floor)
    scale[3 + DD:] = max(scale[3 + DD:].max(), sig_floor)
    err = np.abs(tr[:, 3:] - ref[:, 3:]) / scale
    assert err.max() <= tol, (err.max(), np.unravel_index(np.argmax(err), err.shape))
    assert np.allclose(tr[~ev, 1], ref[~ev, 1], rtol=0, atol=0)


def _close_token(a, b):
    """Two printed numbers agree to one unit of the last printed digit
    (fixed notation) or 2e-6 relative (exponent notation); other tokens must
    be equal."""
    if a == b:
        return True
    try:
        x, y = float(a), float(b)
    except ValueError:
        return False
    if "e" in b.lower():
        return abs(x - y) <= 2e-6 * max(abs(y), 1e-300)
    dec = len(b.split(".")[1]) if "." in b else 0
    return abs(x - y) <= 1.01 * 10.0 ** (-dec)


def same_log(ours, ref, skip_prefix=2):
    """Logs with the same lines and columns; numbers within one unit of their
    last printed digit (components that are zero up to rounding noise may
    print as -0.000 on one side).  The first skip_prefix tokens of lines that
    start with a date (timestamp and elapsed seconds) and the run-time
    trailer lines are not compared."""
    import re
    a = [l for l in ours.splitlines() if not l.startswith(("Simulation Finish", "Total Duration"))]
    b = [l for l in ref.splitlines() if not l.startswith(("Simulation Finish", "Total Duration"))]
    assert len(a) == len(b), (len(a), len(b))
    for la, lb in zip(a, b):
        if la == lb:
            continue
        fa, fb = la.split(), lb.split()
        if re.match(r"\d{4}-\d\d-\d\d", lb):
            fa, fb = fa[skip_prefix + 1:], fb[skip_prefix + 1:]
        assert len(fa) == len(fb), (la, lb)
        for x, y in zip(fa, fb):
            assert _close_token(x, y), (x, y, la, lb)
