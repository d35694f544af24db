#!/usr/bin/env python3
"""Golden fixtures at the benchmark configurations, written by the reference.

Every number comes from oracle/_ref/ref_driver kmc_trace: the unmodified
mgkmc_cpp headers (KmcSimulation2D/3D, run_cascade, elastic_run ...) driven
through run_simulation's control flow.  The inputs are the named workloads of
mgkmc_cpp_b200.workloads (the reference's YAML keys plus a seeded synthetic
lognormal modulus field in its .npy format), so a test regenerates the same
inputs with write_workload and checks them against the checksums stored here.

The fields of these grids are megabytes each, so a fixture keeps:
  trace        one row per event (kind, selected mode, counters, clock, macro)
  E_sum, E_sq  checksums of the modulus field the reference ran on
  sub          voxel indices: an even stride over the grid plus every voxel
               that flipped
  eps_sub, sig_sub, epsp_sub   the final full tensors at those voxels
  eps_sq, sig_sq               sum of squares of the whole final fields
  flip_vox, cat_flip, Q0_flip  catalog and barriers of every mode of every
                               flipped voxel (they pin the random stream)
  macro        the final macroscopic state

    python tests/golden/make_golden_configs.py [name ...]
"""
from __future__ import annotations

import os
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle as O  # noqa: E402
from mgkmc_cpp_b200 import workloads  # noqa: E402

# fixture name -> (workload, seed, thermal events)
CASES = {
    "cfg0_homog2d_32": ("homog2d_32", 0, 2000),
    "cfg1_hetero2d_256_s0": ("hetero2d_256", 0, 100),
    "cfg1_hetero2d_256_s1": ("hetero2d_256", 1, 100),
    "cfg1_hetero2d_256_s2": ("hetero2d_256", 2, 100),
    "cfg1_hetero2d_256_s3": ("hetero2d_256", 3, 100),
    "cfg2_hetero3d_64": ("hetero3d_64", 0, 20),
    "ens2d_512_s32": ("ens2d_512", 32, 20),
    "ens3d_96_s58": ("ens3d_96", 58, 20),
}
N_SUB = 1024


def compact(res, cfg, E):
    D = cfg.dim
    N = cfg.n_voxels
    M = cfg.M
    tr = res["trace"]
    kind = tr[:, 0].astype(int)
    # selected modes of thermal events (kind 0); cascades flip many modes per
    # row, recorded through the plastic strain of the voxels they touched
    sel = tr[kind == 0, 1].astype(np.int64)
    epsp = res["epsp"].reshape(N, D * D)
    touched = np.nonzero(np.any(epsp != 0.0, axis=1))[0]
    flip_vox = np.unique(np.concatenate([sel // M, touched]))
    stride = max(1, N // N_SUB)
    sub = np.unique(np.concatenate([np.arange(0, N, stride), flip_vox]))
    eps = res["eps"].reshape(N, D * D)
    sig = res["sig"].reshape(N, D * D)
    cat = res["catalog"].reshape(N, M, -1)
    Q0 = res["Q0"].reshape(N, M)
    return dict(trace=tr, E_sum=float(np.sum(E)), E_sq=float(np.sum(E * E)), sub=sub, eps_sub=eps[sub],
                sig_sub=sig[sub], epsp_sub=epsp[sub], eps_sq=float(np.sum(eps * eps)), sig_sq=float(np.sum(sig * sig)),
                flip_vox=flip_vox, cat_flip=cat[flip_vox], Q0_flip=Q0[flip_vox], macro=res["macro"])


def make(name, rd):
    wl, seed, nev = CASES[name]
    d = tempfile.mkdtemp(prefix="mgk_golden_")
    path, cfg = workloads.write_workload(wl, d, seed=seed)
    with open(path) as f:
        text = f.read()
    t0 = time.time()
    res = rd.kmc(text, "kmc_trace", nsteps=10 ** 6, maxev=nev)
    dt = time.time() - t0
    E = np.asarray(cfg.E, dtype=np.float64).reshape(-1)
    out = compact(res, cfg, E)
    out.update(workload=np.array(wl), seed=seed, events=nev)
    tmp = os.path.join(HERE, name + ".tmp.npz")
    np.savez_compressed(tmp, **out)
    os.replace(tmp, os.path.join(HERE, name + ".npz"))  # never a half-written fixture
    kinds = np.bincount(res["trace"][:, 0].astype(int), minlength=4)
    print("wrote %s: %d rows (kinds %s), %d flipped voxels, reference %.1f s" % (name, len(res["trace"]), kinds,
                                                                                  len(out["flip_vox"]), dt), flush=True)


def main(names):
    rd = O.RefDriver()
    for n in names or list(CASES):
        make(n, rd)


if __name__ == "__main__":
    main(sys.argv[1:])
