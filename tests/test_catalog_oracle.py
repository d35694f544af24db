"""The oracle's restatement of the catalog and per-voxel barrier extensions
(catalog.type even / fibonacci, barriers.per_voxel; no counterpart in the
reference), checked on the CPU against their definitions:

* even: mode m of M is (gamma0/2)(s n + n s) with s = (cos t, sin t),
  n = (-sin t, cos t), t = m pi / M, identical in every voxel and never
  redrawn;
* fibonacci (3D): every mode's work sigma : eps0 = gamma0 |tau| >= 0, so a
  mode's barrier Q = Q0 - W never exceeds Q0 without softening; the plastic
  strain of a flip is a shear of magnitude gamma0 (Frobenius norm
  gamma0 / sqrt 2);
* per-voxel barriers: one value for all M modes of a voxel;
* with the extensions off the oracle is the reference (tests/test_oracle_pins.py).
"""
import numpy as np

import oracle as O
from test_gpu_catalog import CASES, MAXEV, NSTEPS, config


def test_even_catalog_is_the_fixed_shears():
    cfg = config("even2d_voxel")
    ok = O.OracleKmc(cfg)
    M, N = cfg.M, cfg.n_voxels
    t = np.arange(M) * np.pi / M
    h = 0.5 * cfg.gamma0
    want = np.stack([-h * np.sin(2 * t), h * np.cos(2 * t), h * np.cos(2 * t), h * np.sin(2 * t)], axis=1)
    cat0 = ok.get("catalog").reshape(N, M, 4)
    assert np.allclose(cat0, want[None], rtol=0, atol=1e-17)
    ok.run(NSTEPS, MAXEV)
    assert np.array_equal(ok.get("catalog").reshape(N, M, 4), cat0)  # never redrawn


def test_per_voxel_barriers_are_shared_by_the_modes():
    for name in ("even2d_voxel", "random2d_voxel", "fib3d_voxel"):
        cfg = config(name)
        ok = O.OracleKmc(cfg)
        ok.run(NSTEPS, 50)
        Q0 = ok.get("Q0").reshape(cfg.n_voxels, cfg.M)
        assert np.array_equal(Q0, np.repeat(Q0[:, :1], cfg.M, axis=1)), name
        assert Q0.min() >= 0.6 and Q0.max() <= 1.4


def test_fibonacci_modes_do_positive_work_and_have_magnitude_gamma0():
    cfg = config("fib3d_mode")
    ok = O.OracleKmc(cfg)
    tr = ok.run(NSTEPS, MAXEV)
    assert ok.get("catalog").size == 0  # no stored catalog
    # Q of the last sweep against Q0, on voxels that never flipped (a flipped
    # voxel's barriers may have been redrawn after that sweep)
    prev = ok.get("prev_dir").reshape(cfg.n_voxels, 3, 3)
    flipped = np.abs(prev).sum(axis=(1, 2)) > 0
    Q = ok.get("Q").reshape(cfg.n_voxels, cfg.M)[~flipped]
    Q0 = ok.get("Q0").reshape(cfg.n_voxels, cfg.M)[~flipped]
    assert np.all(Q <= Q0 + 1e-15)  # W = 0.5 V gamma0 |tau| >= 0, no softening
    assert np.any(Q < Q0 - 1e-6)
    # every flipped voxel's last mode is a shear: deviatoric, norm gamma0 / sqrt 2
    assert (tr[:, 0] == 0).sum() > 50 and flipped.sum() >= 10
    p = prev[flipped]
    assert np.allclose(np.trace(p, axis1=1, axis2=2), 0.0, atol=1e-15)
    assert np.allclose(np.linalg.norm(p, axis=(1, 2)), cfg.gamma0 / np.sqrt(2.0), rtol=1e-12)
    assert np.allclose(p, p.transpose(0, 2, 1), atol=0)


def test_extension_cases_are_known():
    assert len(CASES) >= 6
