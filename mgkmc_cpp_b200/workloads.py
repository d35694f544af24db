"""Named benchmark / parity workloads, written in the reference's own input
format (YAML keys of main.cpp and a ``.npy`` modulus field).

No public dataset is involved: the heterogeneous cases use seeded synthetic
lognormal modulus fields (``fields.lognormal_modulus``) with the shapes,
correlation lengths and coefficients of variation of the benchmark cases.

* ``homog2d_32``  -- 2D plane strain 32x32, E = 90 GPa, nu = 0.36, M = 18,
  gamma0 = 0.1, barriers N(1.0, 0) (every Q0 = 1.0 eV), T = 300 K,
  nu0 = 1e13 /s, strain rate 0.1 /s, sigma_yy = sigma_xy = 0, seed 0.
* ``hetero2d_256`` -- 2D plane strain 256x256, lognormal E (mean 90 GPa,
  CoV 0.10, correlation length 4 voxels), nu = 0.36, M = 18, Q0 per
  (voxel, mode) from the reference's default barrier generator (N(2.0, 0.6)
  eV, cut off below 0.1 eV), otherwise as above.
* ``hetero2d_256_dF1`` -- the same with Q0 ~ N(1.0, 0.1) clipped to
  [0.6, 1.4] eV per (voxel, mode).  In the reference's model this enters a
  sustained avalanche after about 1100 thermal events at seed 0 (the cascade
  loop never settles), in the reference and in this build alike.
* ``hetero2d_64``  -- 64x64 with the N(1.0, 0.1) barriers (parity-test size).
* ``hetero3d_64``  -- 3D 64^3, lognormal E (CoV 0.15, correlation 3), M = 100
  random deviatoric 3D modes (system.3d_barriers), z tension, gamma0 = 0.03
  (at 0.1 the reference's own run of this case enters an avalanche before its
  20th thermal event: over 10 CPU-minutes inside it; see the ensemble note).
* ``hetero3d_16``  -- the 3D case at 16^3 with M = 20 (parity-test size).
* ``ens2d_64``, ``ens2d_128``, ``ens2d_512``, ``ens3d_32``, ``ens3d_48``,
  ``ens3d_96`` -- replicas of the batched ensemble: lognormal E whose CoV is
  drawn uniformly from [0.05, 0.2] by the replica's seed (correlation length 4
  voxels in 2D, 3 in 3D), the reference's default barriers, M = 18 in 2D and
  M = 100 random deviatoric modes in 3D with gamma0 = 0.03 (the reference's
  3D catalog draws magnitudes gamma0 * sqrt(-2 ln u), mean 1.25 gamma0, and
  the flip work scales with gamma0^2: at gamma0 = 0.1 the first cascade of a
  32^3 replica never settles (312k flips in 118 batches within 30 s); at 0.05
  two of six 96^3 replicas enter a system-spanning avalanche within ~40
  events -- ~900k flips per cascade batch, LS solves at their 200-iteration
  cap).  ``ensemble()`` lists the 64-replica
  mix: 16 each of 2D 64^2, 128^2, 512^2 and 16 3D replicas (5 of 32^3, 5 of
  48^3, 6 of 96^3), seeds 0..63.
"""
from __future__ import annotations

import os
from typing import Tuple

import numpy as np

from . import fields
from .config import SimConfig, YAMLConfig

_BASE = """
seed: {seed}
simulation_type: "kmc"
system:
  dimensionality: "{dim}"
  plane_mode: "plane_strain"
  nx: {nx}
  ny: {ny}
  nz: {nz}
  pixel: 1.0
  M: {M}
  gamma0: {gamma0}
  3d_barriers: {b3}
material:
  E:
{Eblock}
  nu:
    mode: "constant"
    value: 0.36
catalog:
  type: "{cat}"
loading:
  eps_target: {eps_target}
  step_size: 1e-4
boundary_conditions:
  driving_component: "{drive}"
  mixed_targets:
{targets}
  mixed_tol: 1.0
barriers:
  type: "gaussian"
  per_voxel: {pv}
  kwargs:
    mean: {bmean}
    std: {bstd}
    min_cutoff: {bmin}
    max_cutoff: {bmax}
physics:
  enable_softening: false
dynamics:
  instability_mode: "cascade"
  temperature: 300
  nu0: 1e13
  physical_strain_rate: 0.1
output:
  enable_console: false
"""

# barrier distributions: the reference's BarrierGenerator defaults
# (gaussian, mean 2.0 eV, std 0.6, min cutoff 0.1, main.cpp:283-286) and the
# N(1.0, 0.1) eV clipped to [0.6, 1.4] distribution of the heterogeneous cases
_B_REF = dict(bmean="2.0", bstd="0.6", bmin="0.1", bmax="-1.0")
_B_DF1 = dict(bmean="1.0", bstd="0.1", bmin="0.6", bmax="1.4")
_T2 = dict(drive="xx", targets="    yy: 0.0\n    xy: 0.0")
_T3 = dict(drive="zz", targets="    xx: 0.0\n    yy: 0.0")

WORKLOADS = {
    "homog2d_32": dict(dim="2d", nx=32, ny=32, nz=1, M=18, b3="false", hetero=None, **_T2, bmean="1.0", bstd="0.0",
                       bmin="0.6", bmax="1.4"),
    "hetero2d_256": dict(dim="2d", nx=256, ny=256, nz=1, M=18, b3="false", hetero=(0.10, 4.0), **_T2, **_B_REF),
    "hetero2d_256_dF1": dict(dim="2d", nx=256, ny=256, nz=1, M=18, b3="false", hetero=(0.10, 4.0), **_T2, **_B_DF1),
    "hetero2d_64": dict(dim="2d", nx=64, ny=64, nz=1, M=18, b3="false", hetero=(0.10, 4.0), **_T2, **_B_DF1),
    "hetero3d_64": dict(dim="3d", nx=64, ny=64, nz=64, M=100, b3="true", hetero=(0.15, 3.0), **_T3, **_B_REF,
                        gamma0=0.03),
    "hetero3d_16": dict(dim="3d", nx=16, ny=16, nz=16, M=20, b3="true", hetero=(0.15, 3.0), **_T3, **_B_DF1),
}
for _n in (64, 128, 512):
    WORKLOADS["ens2d_%d" % _n] = dict(dim="2d", nx=_n, ny=_n, nz=1, M=18, b3="false", hetero=("draw", 4.0), **_T2,
                                      **_B_REF)
for _n in (32, 48, 96):
    WORKLOADS["ens3d_%d" % _n] = dict(dim="3d", nx=_n, ny=_n, nz=_n, M=100, b3="true", hetero=("draw", 3.0), **_T3,
                                      **_B_REF, gamma0=0.03)

# The benchmark description's own physics, through the catalog and per-voxel
# barrier extensions (catalog.type, barriers.per_voxel; no counterpart in the
# reference, whose random catalog these replace):
#   bl_cfg0_32   2D 32^2 homogeneous, 18 shears evenly spaced in [0, pi),
#                dF = 1.0 eV in every voxel (per voxel, sd 0)
#   bl_cfg1_256  2D 256^2 lognormal E (CoV 0.1, correlation 4), 18 even
#                shears, dF per voxel N(1.0, 0.1) eV clipped to [0.6, 1.4]
#   bl_cfg2_64   3D 64^3 lognormal E (CoV 0.15, correlation 3), 100 Fibonacci
#                plane normals sheared along their largest resolved shear
#                stress, gamma0 0.1, dF per voxel as above, z tension to 3 %
_BL = dict(pv="true", **_B_DF1)
WORKLOADS["bl_cfg0_32"] = dict(dim="2d", nx=32, ny=32, nz=1, M=18, b3="false", hetero=None, **_T2, cat="even",
                               pv="true", bmean="1.0", bstd="0.0", bmin="0.6", bmax="1.4")
WORKLOADS["bl_cfg1_256"] = dict(dim="2d", nx=256, ny=256, nz=1, M=18, b3="false", hetero=(0.10, 4.0), **_T2, cat="even",
                                **_BL)
WORKLOADS["bl_cfg2_64"] = dict(dim="3d", nx=64, ny=64, nz=64, M=100, b3="false", hetero=(0.15, 3.0), **_T3,
                               cat="fibonacci", eps_target=0.03, **_BL)

ENSEMBLE = ["ens2d_64"] * 16 + ["ens2d_128"] * 16 + ["ens2d_512"] * 16 + ["ens3d_32"] * 5 + ["ens3d_48"] * 5 + \
    ["ens3d_96"] * 6


SERVE_SIZES = [("2d", 32), ("2d", 64), ("2d", 128), ("2d", 256), ("2d", 512), ("3d", 32), ("3d", 64)]


def serve_jobs(directory: str, n_jobs: int, rate: float = 20.0, seed: int = 7, flips=(500, 5000), sizes=None):
    """The request stream of the serving case: Poisson arrivals (``rate``
    jobs/s), each job's grid drawn uniformly from ``sizes`` (default 2D 32^2 ..
    512^2 powers of two, 3D 32^3, 64^3), its own lognormal E field (CoV
    uniform in [0.05, 0.2]) and seed, the reference's default barriers, and a
    target of ``flips`` thermal events (uniform).  Returns a list of
    (arrival_s, config, target_flips)."""
    sizes = SERVE_SIZES if sizes is None else sizes
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for j in range(n_jobs):
        t += rng.exponential(1.0 / rate)
        dim, n = sizes[int(rng.integers(len(sizes)))]
        name = "ens%s_%d" % (dim, n)
        if name not in WORKLOADS:
            base = WORKLOADS["ens2d_64" if dim == "2d" else "ens3d_32"]
            WORKLOADS[name] = dict(base, nx=n, ny=n, nz=n if dim == "3d" else 1)
        target = int(rng.integers(flips[0], flips[1] + 1))
        out.append((t, write_workload(name, directory, seed=10000 + j)[1], target))
    return out


def ensemble_cov(seed: int) -> float:
    """CoV of an ensemble replica's modulus field: uniform in [0.05, 0.2]."""
    return float(np.random.default_rng(1000 + seed).uniform(0.05, 0.2))


def ensemble(directory: str, names=None):
    """(name, seed, config) of every ensemble replica; seed = position in the list."""
    names = ENSEMBLE if names is None else names
    return [(n, s, write_workload(n, directory, seed=s)[1]) for s, n in enumerate(names)]


def write_workload(name: str, directory: str, seed: int = 0) -> Tuple[str, SimConfig]:
    """Writes <directory>/<name>_s<seed>.yaml (+ its E .npy) and returns (yaml_path, config)."""
    w = WORKLOADS[name]
    os.makedirs(directory, exist_ok=True)
    if w["hetero"] is None:
        eblock = '    mode: "constant"\n    value: 90'
    else:
        cov, corr = w["hetero"]
        if cov == "draw":
            cov = ensemble_cov(seed)
        shape = (w["nx"], w["ny"], w["nz"]) if w["dim"] == "3d" else (w["nx"], w["ny"])
        E = fields.lognormal_modulus(shape, 90e9, cov, corr, seed)
        epath = os.path.join(directory, "E_%s_s%d.npy" % (name, seed))
        np.save(epath, E)
        eblock = '    mode: "file"\n    parameters:\n      path: "%s"' % epath
    fmt = {k: v for k, v in w.items() if k != "hetero"}
    fmt.setdefault("gamma0", 0.1)
    fmt.setdefault("cat", "random")
    fmt.setdefault("pv", "false")
    fmt.setdefault("eps_target", 0.05)
    text = _BASE.format(seed=seed, Eblock=eblock, **fmt)
    path = os.path.join(directory, "%s_s%d.yaml" % (name, seed))
    with open(path, "w") as f:
        f.write(text)
    return path, SimConfig.from_yaml(path)


def load_config(text: str) -> SimConfig:
    return SimConfig.from_yaml(YAMLConfig.loads(text))
