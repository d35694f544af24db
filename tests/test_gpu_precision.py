"""The FP32-refined LS solve (FP32 spectrum and FFTs, then FP64 iterations)
against the FP64 solve and the reference's golden fields: the refinement
reaches the FP64 fixed point, so at a tight tolerance the fields agree within
1e-8 relative L2 (the benchmark description's bar; observed far below), and
at the reference's tolerance (1e-6) both sit within the same distance of
the converged solution."""
import numpy as np
import pytest

from helpers import golden, rel

pytestmark = pytest.mark.gpu


def _case(name):
    g = golden(name)
    dims = tuple(int(d) for d in g["dims"])
    return g, dims


@pytest.mark.parametrize("name", ["ls2d_32_homog", "ls2d_16_conv", "ls3d_12x6x10_conv", "ls2d_48x30_fixed2"])
def test_fp32_refined_matches_fp64(name):
    import mgkmc_cpp_b200 as G
    G._lib.require_device()
    g, dims = _case(name)
    rng = np.random.default_rng(3)
    N = int(np.prod(dims))
    E = 90e9 * np.exp(0.2 * rng.standard_normal(N))
    nu = np.full(N, 0.33)
    D = len(dims)
    eb = np.zeros((D, D))
    eb[0, 0] = 1e-3
    eb[1, 1] = -4e-4
    eb[0, 1] = eb[1, 0] = 2e-4
    out = {}
    for prec in ("fp64", "fp32_refined"):
        s = G.LsSolver(dims, E, nu, precision=prec)
        out[prec] = s.solve(eb, max_iter=400, tol=1e-12)
        s.close()
    e64, s64, _, sm64, it64 = out["fp64"]
    e32, s32, _, sm32, it32 = out["fp32_refined"]
    assert rel(e32, e64) < 1e-8 and rel(s32, s64) < 1e-8
    assert np.max(np.abs(sm32 - sm64)) <= 1e-8 * np.max(np.abs(sm64))


def test_fp32_refined_against_reference_golden():
    """The golden converged case (reference at tol 1e-6): the refined solve at
    the same tolerance is as close to it as the FP64 solve is."""
    import mgkmc_cpp_b200 as G
    G._lib.require_device()
    g, dims = _case("ls2d_16_conv")
    res = {}
    for prec in ("fp64", "fp32_refined"):
        s = G.LsSolver(dims, g["E"], g["nu"], precision=prec,
                       plane_mode="plane_stress" if int(g["plane_stress"]) else "plane_strain", pixel=float(g["pixel"]))
        res[prec] = s.solve(g["eps_bar"], max_iter=int(g["max_iter"]), tol=float(g["tol"]),
                            eps_plastic=g["epsp"] if "epsp" in g else None)
        s.close()
    d64 = rel(res["fp64"][0], g["eps"])
    d32 = rel(res["fp32_refined"][0], g["eps"])
    assert d64 < 1e-10
    assert d32 < 1e-6


@pytest.mark.parametrize("workload", ["ens2d_64", "ens3d_32"])
def test_kmc_fp32_refined_flips_and_fields_match_fp64(workload, tmp_path):
    """The chosen arithmetic in both KMC forms: every re-solve FP32-refined
    (ls.precision fp32_refined) against the FP64 run (which the reference
    pins), both converged to 1e-10: the same flips, fields within 1e-8.
    (Workloads with the reference's default barriers: the N(1.0, 0.1) ones can
    enter avalanches that never end a plain-form run.)"""
    import dataclasses
    import mgkmc_cpp_b200 as G
    from mgkmc_cpp_b200 import workloads
    G._lib.require_device()
    _, cfg = workloads.write_workload(workload, str(tmp_path), seed=2)
    nev = 120 if cfg.dim == 2 else 30
    runs = {}
    for prec in ("fp64", "fp32_refined"):
        c = dataclasses.replace(cfg, ls_precision=prec, ls_tol=1e-10)
        sim = G.from_config(c, output_dir=str(tmp_path))
        tr = sim.run_simulation(10 ** 6, c.step_size, c.driving, c.targets, c.mixed_tol_pa, 50,
                                enable_console_log=False, enable_summary_log=False, enable_global_log=False,
                                max_events=nev, trace=True)
        b = G.KmcBatch([c])
        b.run(nev)
        runs[prec] = (tr[tr[:, 0] == 0, 1].astype(np.int64), sim.eps_field, b.stats(0)["selected"],
                      b.field(0, "eps_field"))
        b.close()
    sel64, eps64, bsel64, beps64 = runs["fp64"]
    sel32, eps32, bsel32, beps32 = runs["fp32_refined"]
    assert len(sel64) == nev and np.array_equal(sel32, sel64)
    assert np.array_equal(bsel32, sel64) and np.array_equal(bsel64, sel64)
    assert rel(eps32, eps64) < 1e-8
    assert rel(beps32, eps64) < 1e-8
