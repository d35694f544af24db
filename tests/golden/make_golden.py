#!/usr/bin/env python3
"""Regenerates the golden fixtures in tests/golden/ from the reference itself.

Every output comes from oracle/_ref/ref_driver, i.e. the unmodified mgkmc_cpp
headers compiled by oracle/Makefile (run `make -C oracle` where the reference
sources are present).  Inputs are seeded synthetic fields and small configs in
the reference's YAML key surface; nothing is copied from the reference tree.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle as O  # noqa: E402

# ------------------------------------------------------------------ LS cases
LS_CASES = [
    # name, dims, plane_mode, pixel, max_iter, tol, hetero, epsp, warm
    ("ls2d_16_fixed3", (16, 16), "plane_strain", 1.0, 3, 0.0, True, True, False),
    ("ls2d_16_conv", (16, 16), "plane_strain", 1.0, 200, 1e-6, True, True, False),
    ("ls2d_12x10_stress_warm", (12, 10), "plane_stress", 0.5, 200, 1e-6, True, False, True),
    ("ls2d_9x7_odd", (9, 7), "plane_strain", 1.0, 200, 1e-6, True, True, False),
    ("ls2d_32_homog", (32, 32), "plane_strain", 1.0, 200, 1e-6, False, False, False),
    ("ls2d_48x30_fixed2", (48, 30), "plane_strain", 1.0, 2, 0.0, True, True, True),
    ("ls3d_8_fixed2", (8, 8, 8), "", 1.0, 2, 0.0, True, True, False),
    ("ls3d_6x4x5_conv", (6, 4, 5), "", 0.7, 200, 1e-6, True, True, True),
    ("ls3d_8x8x1_conv", (8, 8, 1), "", 1.0, 200, 1e-6, True, False, False),
    ("ls3d_12x6x10_conv", (12, 6, 10), "", 1.0, 200, 1e-6, True, True, False),
]


def ls_inputs(name, dims, hetero, with_epsp, warm):
    rng = np.random.default_rng(sum(map(ord, name)))
    D = len(dims)
    N = int(np.prod(dims))
    E = 90e9 * (1 + 0.2 * rng.standard_normal(N)) if hetero else np.full(N, 90e9)
    nu = np.full(N, 0.36) if hetero else np.full(N, 0.3)
    eb = 1e-3 * rng.standard_normal((D, D))
    epsp = None
    if with_epsp:
        epsp = 0.01 * rng.standard_normal((N, D, D))
        epsp = epsp + epsp.transpose(0, 2, 1)
    eps0 = 1e-3 * rng.standard_normal((N, D, D)) if warm else None
    return E, nu, eb, epsp, eps0


# ------------------------------------------------------------------ KMC cases
KMC_YAML = """
seed: {seed}
system:
  dimensionality: "{dim}"
  plane_mode: "{plane}"
  nx: {nx}
  ny: {ny}
  nz: {nz}
  pixel: {pixel}
  M: {M}
  gamma0: 0.1
  3d_barriers: {b3}
material:
  E:
{Eblock}
  nu:
    mode: "constant"
    value: 0.36
loading:
  eps_target: 0.05
  step_size: 1e-3
boundary_conditions:
  driving_component: "{drive}"
  mixed_targets:
{targets}
  mixed_tol: 1.0
barriers:
  type: "{btype}"
  kwargs:
    mean: 1.0
    std: 0.1
    min_cutoff: 0.6
    max_cutoff: 1.4
    loc: 0.7
    scale: 0.2
    epsilon: 0.3
    ratio: 0.5
physics:
  enable_softening: {soft}
  softening_scheme: "{scheme}"
  neighbor_softening_fraction: {neigh}
  jp: 1.0
  jt: 3.0
  softening_cap: 0.5
  q_act_temp: 0.6
  redraw_directions: {rdir}
  redraw_barriers: {rbar}
dynamics:
  instability_mode: "{mode}"
  temperature: 300
  nu0: 1e13
  physical_strain_rate: 0.1
"""

_K = dict(seed=3, dim="2d", plane="plane_strain", nx=12, ny=12, nz=1, pixel=1.0, M=6, b3="false", hetero=False,
          drive="xx", targets="    yy: 0.0\n    xy: 0.0", btype="gaussian", soft="false", scheme="isotropic", neigh=0.0,
          rdir="true", rbar="true", mode="cascade", nsteps=25, maxev=300)

KMC_CASES = {
    "kmc2d_12_nosoft": dict(),
    "kmc2d_8_soft_neigh": dict(nx=8, ny=8, M=5, soft="true", neigh=0.1),
    "kmc2d_8_kmcmode": dict(nx=8, ny=8, M=4, soft="true", neigh=0.1, mode="kmc"),
    "kmc2d_10_hetero_stress": dict(nx=10, ny=10, M=4, plane="plane_stress", hetero=True, btype="modified_rayleigh",
                                   soft="true", scheme="directional", pixel=0.8, seed=5),
    "kmc2d_8_noredraw": dict(nx=8, ny=6, M=3, rdir="false", rbar="false", btype="rayleigh", drive="xy",
                             targets="    xx: 0.0\n    yy: 0.0", seed=11),
    "kmc2d_8_mixexp": dict(nx=8, ny=8, M=4, btype="modified_rayleigh_with_exponential", rbar="false", seed=13),
    "kmc3d_6x6x4_soft": dict(dim="3d", nx=6, ny=6, nz=4, M=4, soft="true", neigh=0.1),
    "kmc3d_5x4x3_b3dir": dict(dim="3d", nx=5, ny=4, nz=3, M=3, b3="true", soft="true", scheme="directional",
                              drive="zz", targets="    xx: 0.0\n    yy: 0.0", hetero=True, seed=7),
}


def kmc_yaml(name, epath=None):
    k = dict(_K)
    k.update(KMC_CASES[name])
    if k["hetero"]:
        eblock = '    mode: "file"\n    parameters:\n      path: "%s"' % (epath or "$E")
    else:
        eblock = '    mode: "constant"\n    value: 90'
    return KMC_YAML.format(Eblock=eblock, **k), k


def kmc_field(name):
    k = dict(_K)
    k.update(KMC_CASES[name])
    if not k["hetero"]:
        return None
    shape = (k["nx"], k["ny"], k["nz"]) if k["dim"] == "3d" else (k["nx"], k["ny"])
    rng = np.random.default_rng(sum(map(ord, name)))
    return 90.0 * np.exp(0.15 * rng.standard_normal(shape))  # GPa; the reader converts to Pa


def main():
    rd = O.RefDriver()
    # RNG draws
    with tempfile.TemporaryDirectory() as d:
        subprocess.run([rd.path, "draws", "7", "200", d + "/x.npy"], check=True)
        np.savez_compressed(os.path.join(HERE, "draws_seed7.npz"), draws=np.load(d + "/x.npy"))
    # LS
    for (name, dims, pm, pixel, it, tol, het, wep, warm) in LS_CASES:
        E, nu, eb, epsp, eps0 = ls_inputs(name, dims, het, wep, warm)
        D = len(dims)
        N = int(np.prod(dims))
        eps, sig, em, sm, _ = rd.ls(dims, E, nu, eb, eps0=None if eps0 is None else eps0.reshape(N, D * D),
                                    epsp=None if epsp is None else epsp.reshape(N, D * D),
                                    plane_mode=pm or "plane_strain", pixel=pixel, max_iter=it, tol=tol)
        arrs = dict(dims=np.array(dims), E=E, nu=nu, eps_bar=eb, pixel=pixel, max_iter=it, tol=tol,
                    plane_stress=int(pm == "plane_stress"), eps=eps, sig=sig, eps_macro=em, sig_macro=sm)
        if epsp is not None:
            arrs["epsp"] = epsp.reshape(N, D * D)
        if eps0 is not None:
            arrs["eps0"] = eps0.reshape(N, D * D)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrs)
        print("wrote", name)
    # KMC traces
    for name in KMC_CASES:
        y, k = kmc_yaml(name, "$DIR/E.npy")
        Ef = kmc_field(name)
        files = {"E.npy": Ef} if Ef is not None else {}
        res = rd.kmc(y, "kmc_trace", nsteps=k["nsteps"], maxev=k["maxev"], files=files)
        arrs = {f: res[f] for f in ("trace", "eps", "sig", "epsp", "catalog", "Q0", "soft", "prev_dir", "macro", "last_t")}
        arrs["yaml"] = np.array(kmc_yaml(name, "$E")[0])
        if Ef is not None:
            arrs["E_gpa"] = Ef
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrs)
        print("wrote", name, "rows", len(res["trace"]), "kinds", np.bincount(res["trace"][:, 0].astype(int)))


# linear-elastic runs of the reference executable (main.cpp's
# simulation_type "linear_elastic"): its global log (fixed 6-decimal text) and
# the Step / Eps / Sig columns of its summary log are the fixture
LE_CASES = {
    "le2d_16x12_hetero": dict(dim="2d", nx=16, ny=12, nz=1, pm="plane_strain", drive="xx",
                              targets="    yy: 0.0\n    xy: 0.0", eps_target="0.002", step="1e-4", field=True),
    "le2d_12x10_stress_xy": dict(dim="2d", nx=12, ny=10, nz=1, pm="plane_stress", drive="xy",
                                 targets="    xx: 0.0\n    yy: 0.05", eps_target="0.001", step="1e-4", field=True),
    "le3d_8x6x4_hetero": dict(dim="3d", nx=8, ny=6, nz=4, pm="plane_strain", drive="zz",
                              targets="    xx: 0.0\n    yy: 0.0", eps_target="0.0008", step="1e-4", field=True),
}


def le_yaml(name, epath, outdir):
    c = LE_CASES[name]
    return f"""seed: 1
simulation_type: "linear_elastic"
system:
  dimensionality: "{c['dim']}"
  plane_mode: "{c['pm']}"
  nx: {c['nx']}
  ny: {c['ny']}
  nz: {c['nz']}
  pixel: 1.0
material:
  E:
    mode: "file"
    parameters:
      path: "{epath}"
  nu:
    mode: "constant"
    value: 0.33
loading:
  eps_target: {c['eps_target']}
  step_size: {c['step']}
boundary_conditions:
  driving_component: "{c['drive']}"
  mixed_targets:
{c['targets']}
  mixed_tol: 1.0
output:
  directory: "{outdir}"
  enable_console: false
  enable_summary_log: true
  enable_global_log: true
  vtk_interval: "none"
"""


def le_field(name):
    c = LE_CASES[name]
    shape = (c["nx"], c["ny"], c["nz"]) if c["dim"] == "3d" else (c["nx"], c["ny"])
    rng = np.random.default_rng(sum(map(ord, name)))
    return rng.uniform(60.0, 120.0, shape)


def summary_columns(text):
    """Step, Eps and Sig columns of a summary log (timestamp and elapsed dropped)."""
    rows = []
    for line in text.splitlines()[2:]:
        f = line.split()
        if len(f) == 6:
            rows.append(" ".join(f[3:]))
    return "\n".join(rows)


def main_le():
    exe = os.path.abspath(os.path.join(HERE, "..", "..", "oracle", "_ref", "mgkmc_ref"))
    for name in LE_CASES:
        Ef = le_field(name)
        with tempfile.TemporaryDirectory() as d:
            np.save(os.path.join(d, "E.npy"), Ef)
            out = os.path.join(d, "out")
            with open(os.path.join(d, "cfg.yaml"), "w") as f:
                f.write(le_yaml(name, os.path.join(d, "E.npy"), out))
            subprocess.run([exe, os.path.join(d, "cfg.yaml")], check=True, capture_output=True, cwd=d, timeout=600)
            glog = open(os.path.join(out, "global_log.txt")).read()
            summ = summary_columns(open(os.path.join(out, "summary_log.txt")).read())
        np.savez_compressed(os.path.join(HERE, name + ".npz"), yaml=np.array(le_yaml(name, "$E", "$OUT")), E_gpa=Ef,
                            global_log=np.array(glog), summary=np.array(summ))
        print("wrote", name, glog.count("\n"), "global-log lines")


# fast patching (kmc_solver.hpp:276-332, 866-913): the reference's own
# run_simulation (ref_driver kmc_run) over a short loading with thermal
# events, cascades and periodic full solves; its final state and summary log
FP_YAML = """seed: {seed}
system:
  dimensionality: "{dim}"
  plane_mode: "plane_strain"
  nx: {nx}
  ny: {ny}
  nz: {nz}
  pixel: 1.0
  M: {M}
  gamma0: {g0}
  3d_barriers: {b3}
material:
  E:
    mode: "constant"
    value: 90
  nu:
    mode: "constant"
    value: 0.36
loading:
  eps_target: 2e-5
  step_size: 1e-6
boundary_conditions:
  driving_component: "{drive}"
  mixed_targets:
{targets}
  mixed_tol: 1.0
barriers:
  type: "gaussian"
  kwargs:
    mean: 2.0
    std: 0.6
    min_cutoff: 0.1
physics:
  enable_softening: true
  softening_scheme: "isotropic"
  jp: 1.0
  jt: 3.0
  softening_cap: 0.5
dynamics:
  instability_mode: "cascade"
  temperature: 300
  nu0: 1e13
  physical_strain_rate: 0.1
  fast_patching:
    enabled: true
    patch_radius: {R}
    sync_interval: {sync}
"""
FP_CASES = {
    "fp2d_16": dict(seed=5, dim="2d", nx=16, ny=16, nz=1, M=6, g0=0.1, b3="false", drive="xx",
                    targets="    yy: 0.0\n    xy: 0.0", R=3, sync=4, nsteps=20),
    "fp3d_8x8x6": dict(seed=9, dim="3d", nx=8, ny=8, nz=6, M=8, g0=0.05, b3="true", drive="zz",
                       targets="    xx: 0.0\n    yy: 0.0", R=2, sync=3, nsteps=20),
}


def main_fp():
    rd = O.RefDriver()
    for name, c in FP_CASES.items():
        y = FP_YAML.format(**c)
        res = rd.kmc(y, "kmc_run", nsteps=c["nsteps"])
        arrs = {f: res[f] for f in ("eps", "sig", "epsp", "catalog", "Q0", "soft", "macro")}
        arrs["yaml"] = np.array(y)
        arrs["summary"] = np.array(res["summary"])
        arrs["nsteps"] = np.array(c["nsteps"])
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrs)
        print("wrote", name, res["summary"].count("KMC"), "KMC rows,", res["summary"].count("CASCADE"), "cascade rows")


# generate_correlated_field_cpp (material_generator.hpp:130-258), the
# reference's own output for main.cpp's "generated" material mode
GRF_CASES = {
    "grf2d_32x24": dict(nx=32, ny=24, nz=1, is3d=0, mean=70.0, std=7.0, corr=4.0, has_min=1, cmin=55.0, has_max=0,
                        cmax=0.0, seed=11),
    "grf3d_12x10x8": dict(nx=12, ny=10, nz=8, is3d=1, mean=90.0, std=9.0, corr=3.0, has_min=0, cmin=0.0, has_max=1,
                          cmax=100.0, seed=5),
}


def main_grf():
    rd = O.RefDriver()
    for name, c in GRF_CASES.items():
        with tempfile.TemporaryDirectory() as d:
            out = os.path.join(d, "f.npy")
            args = [c[k] for k in ("nx", "ny", "nz", "is3d", "mean", "std", "corr", "has_min", "cmin", "has_max", "cmax",
                                   "seed")]
            subprocess.run([rd.path, "grf"] + [repr(a) if isinstance(a, float) else str(a) for a in args] + [out],
                           check=True, capture_output=True)
            f = np.load(out)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), field=f, **{k: np.array(v) for k, v in c.items()})
        print("wrote", name, f.shape, float(f.mean()), float(f.std()))


if __name__ == "__main__":
    if "--grf" in sys.argv:
        main_grf()
    elif "--le" in sys.argv:
        main_le()
    elif "--fp" in sys.argv:
        main_fp()
    else:
        main()
        main_le()
        main_fp()
        main_grf()
