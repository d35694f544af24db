"""The catalog and per-voxel barrier extensions (catalog.type even /
fibonacci, barriers.per_voxel; no counterpart in the reference) on the GPU,
plain and batched forms, against the oracle's restatement of them
(oracle/mgk_oracle.c), which defines them.

Bar: event kinds, selected modes and cascade sizes identical; the trace's
continuous columns within 1e-9 of each column's scale; strain field within
1e-10; barriers identical in the plain form (the same host draws) and within
1e-13 in the batched form (device log/exp); plastic strain identical for the
stored (even) catalog in the plain form, within 1e-12 where the modes are
computed from the local stress (fibonacci) or on the device."""
import numpy as np
import pytest

import oracle as O
from helpers import compare_trace, rel

pytestmark = pytest.mark.gpu

YAML = """
seed: {seed}
system:
  dimensionality: "{dim}"
  plane_mode: "plane_strain"
  nx: {nx}
  ny: {ny}
  nz: {nz}
  pixel: 1.0
  M: {M}
  gamma0: {gamma0}
catalog:
  type: "{cat}"
material:
  E:
    mode: "constant"
    value: 90
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
  type: "gaussian"
  per_voxel: {pv}
  kwargs:
    mean: 1.0
    std: 0.1
    min_cutoff: 0.6
    max_cutoff: 1.4
physics:
  enable_softening: {soft}
  softening_scheme: "{scheme}"
  jp: 1.0
  jt: 3.0
  softening_cap: 0.5
  redraw_directions: {rdir}
  redraw_barriers: {rbar}
dynamics:
  instability_mode: "cascade"
  temperature: 300
  nu0: 1e13
  physical_strain_rate: 0.1
"""
_T2 = "    yy: 0.0\n    xy: 0.0"
_T3 = "    xx: 0.0\n    yy: 0.0"
_BASE = dict(seed=3, dim="2d", nx=12, ny=12, nz=1, M=6, gamma0=0.1, cat="even", drive="xx", targets=_T2, pv="true",
             soft="false", scheme="isotropic", rdir="true", rbar="true")
CASES = {
    "even2d_voxel": dict(),
    "even2d_mode": dict(pv="false", seed=5),
    "even2d_noredraw": dict(rdir="false", rbar="false", seed=7, soft="true", scheme="directional"),
    "random2d_voxel": dict(cat="random", M=4, nx=10, ny=10, seed=9),
    "random2d_voxel_dironly": dict(cat="random", M=4, nx=10, ny=10, rbar="false", seed=11),
    "even3d_mode": dict(dim="3d", nx=6, ny=6, nz=4, M=4, pv="false", drive="xx", targets="    yy: 0.0\n    zz: 0.0",
                        seed=13),
    "fib3d_voxel": dict(dim="3d", nx=8, ny=8, nz=8, M=10, cat="fibonacci", drive="zz", targets=_T3, seed=15,
                        soft="true", scheme="directional"),
    "fib3d_mode": dict(dim="3d", nx=6, ny=8, nz=5, M=7, cat="fibonacci", pv="false", drive="zz", targets=_T3,
                       seed=17),
}
NSTEPS, MAXEV = 20, 200


def config(name):
    from mgkmc_cpp_b200.workloads import load_config
    k = dict(_BASE)
    k.update(CASES[name])
    return load_config(YAML.format(**k))


@pytest.fixture(scope="module")
def G():
    import mgkmc_cpp_b200 as G
    G._lib.require_device()
    return G


@pytest.mark.parametrize("name", list(CASES))
def test_extension_plain_and_batched_against_oracle(G, name, tmp_path):
    cfg = config(name)
    ok = O.OracleKmc(cfg)
    ref = ok.run(NSTEPS, MAXEV)
    assert (ref[:, 0] == 0).sum() > 10  # the case exercises thermal events
    sim = G.from_config(cfg, output_dir=str(tmp_path))
    tr = sim.run_simulation(NSTEPS, cfg.step_size, cfg.driving, cfg.targets, cfg.mixed_tol_pa, 50,
                            enable_console_log=False, enable_summary_log=False, enable_global_log=False,
                            max_events=MAXEV, trace=True)
    compare_trace(tr, ref, tol=1e-9)
    stored = cfg.catalog_type != "fibonacci"
    assert np.array_equal(sim.Q0, ok.get("Q0"))
    if stored:
        assert np.array_equal(sim.catalog.reshape(-1), ok.get("catalog"))
        assert np.array_equal(sim.eps_plastic.reshape(-1), ok.get("epsp"))
    else:
        assert sim.catalog.size == 0
        assert rel(sim.eps_plastic, ok.get("epsp")) < 1e-12
    assert rel(sim.eps_field, ok.get("eps")) < 1e-10
    if cfg.barrier_per_voxel:  # one barrier per voxel
        Q0 = sim.Q0.reshape(cfg.n_voxels, cfg.M)
        assert np.array_equal(Q0, np.repeat(Q0[:, :1], cfg.M, axis=1))
    # batched form: the same run on the device-resident kernel
    b = G.KmcBatch([cfg])
    b.run(MAXEV, n_global_steps=NSTEPS)
    st = b.stats(0)
    sel_ref = ref[ref[:, 0] == 0, 1].astype(np.int64)
    assert np.array_equal(st["selected"], sel_ref)
    assert np.allclose(b.field(0, "Q0"), ok.get("Q0"), rtol=1e-13, atol=0)
    assert rel(b.field(0, "eps_plastic"), ok.get("epsp")) < 1e-12
    assert rel(b.field(0, "eps_field"), ok.get("eps")) < 1e-10
    b.close()


def test_fibonacci_needs_3d():
    from mgkmc_cpp_b200.workloads import load_config
    k = dict(_BASE)
    k.update(cat="fibonacci")
    with pytest.raises(ValueError, match="3D"):
        load_config(YAML.format(**k))
