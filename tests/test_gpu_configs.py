"""Parity at the benchmark configurations, both forms, against traces written
by the reference itself (tests/golden/make_golden_configs.py):

* cfg0_homog2d_32       2D 32^2 homogeneous, M = 18, seed 0, 2000 thermal events
* cfg1_hetero2d_256_s*  2D 256^2 lognormal E (CoV 0.1), M = 18, seeds 0-3, 100 events
                        (the benchmark's four-replica launch in the batched form)
* cfg2_hetero3d_64      3D 64^3 lognormal E (CoV 0.15), M = 100 random 3D modes
                        (gamma0 0.03), 20 events
* ens2d_512_s32, ens3d_96_s58   one 512^2 and one 96^3 replica of the ensemble, 20 events

Bar, as in the small golden cases: event kinds, selected modes and cascade
sizes identical; the trace's continuous columns within 1e-9 of each column's
scale; strain and stress within 1e-10 relative (at a strided voxel subsample
plus every flipped voxel, and the whole fields' sums of squares); plastic
strain, catalog and barriers of every flipped voxel identical in the plain
form (host RNG, same draws) and within 1e-13 in the batched form (device
log/exp).  The inputs are regenerated from the named workloads and checked
against the checksums the reference ran on."""
import os

import numpy as np
import pytest

from helpers import GOLDEN, compare_trace, golden, rel

pytestmark = pytest.mark.gpu

CFG1 = ["cfg1_hetero2d_256_s%d" % s for s in range(4)]
SINGLE = ["cfg0_homog2d_32", "cfg2_hetero3d_64", "ens2d_512_s32", "ens3d_96_s58"]
SINGLE = [n for n in SINGLE if os.path.exists(os.path.join(GOLDEN, n + ".npz"))]


@pytest.fixture(scope="module")
def G():
    import mgkmc_cpp_b200 as G
    G._lib.require_device()
    return G


def inputs(g, tmp_path):
    from mgkmc_cpp_b200 import workloads
    _, cfg = workloads.write_workload(str(g["workload"]), str(tmp_path), seed=int(g["seed"]))
    E = np.asarray(cfg.E, dtype=np.float64).reshape(-1)
    assert abs(E.sum() - float(g["E_sum"])) <= 1e-13 * abs(float(g["E_sum"]))
    assert abs((E * E).sum() - float(g["E_sq"])) <= 1e-13 * abs(float(g["E_sq"]))
    return cfg


def clock_rtol(cfg):
    """The simulation clock is a sum of waits -ln(u1)/R; the reference sums the
    NM rates of R left to right in FP64, an error that grows like sqrt(NM)
    ulps (about 6e-12 at 96^3 x 100 modes), against this build's nearly exact
    double-double sum."""
    return max(1e-12, 2e-15 * np.sqrt(cfg.n_voxels * cfg.M))


def check_fields(g, cfg, eps, sig, epsp, cat, Q0, exact):
    D, M = cfg.dim, cfg.M
    N = cfg.n_voxels
    eps, sig, epsp = eps.reshape(N, D * D), sig.reshape(N, D * D), epsp.reshape(N, D * D)
    sub = g["sub"]
    assert rel(eps[sub], g["eps_sub"]) < 1e-10
    assert rel(sig[sub], g["sig_sub"]) < 1e-10
    assert abs((eps * eps).sum() - float(g["eps_sq"])) <= 1e-10 * float(g["eps_sq"])
    assert abs((sig * sig).sum() - float(g["sig_sq"])) <= 1e-10 * float(g["sig_sq"])
    fv = g["flip_vox"]
    # the voxels carrying plastic strain are the same as in the reference run
    # (the subsample holds every flipped voxel, so the reference's set is there)
    ref_epsp_fv = g["epsp_sub"][np.searchsorted(sub, fv)]
    ref_plastic = fv[np.any(ref_epsp_fv != 0.0, axis=1)]
    assert np.array_equal(np.nonzero(np.any(epsp != 0.0, axis=1))[0], ref_plastic)
    cat_f = cat.reshape(N, M, -1)[fv]
    Q0_f = Q0.reshape(N, M)[fv]
    ref_cat = g["cat_flip"].reshape(len(fv), M, -1)
    if exact:
        assert np.array_equal(epsp[sub], g["epsp_sub"])
        assert np.array_equal(cat_f, ref_cat)
        assert np.array_equal(Q0_f, g["Q0_flip"])
    else:
        assert rel(epsp[sub], g["epsp_sub"]) < 1e-13
        assert np.allclose(cat_f, ref_cat, rtol=1e-13, atol=1e-300)
        assert np.allclose(Q0_f, g["Q0_flip"], rtol=1e-13, atol=0)


def run_plain(G, cfg, nev, tmp_path):
    sim = G.from_config(cfg, output_dir=str(tmp_path))
    tr = sim.run_simulation(10 ** 6, cfg.step_size, cfg.driving, cfg.targets, cfg.mixed_tol_pa, 50,
                            enable_console_log=False, enable_summary_log=False, enable_global_log=False,
                            max_kmc_steps_pct=cfg.max_kmc_steps_pct, max_events=nev, trace=True)
    return sim, tr


@pytest.mark.parametrize("name", SINGLE + CFG1)
def test_plain_form_at_config(G, name, tmp_path):
    g = golden(name)
    cfg = inputs(g, tmp_path)
    sim, tr = run_plain(G, cfg, int(g["events"]), tmp_path)
    N = cfg.n_voxels
    compare_trace(tr, g["trace"], tol=1e-9, eps_floor=np.sqrt(float(g["eps_sq"]) / N),
                  sig_floor=np.sqrt(float(g["sig_sq"]) / N))
    check_fields(g, cfg, sim.eps_field, sim.sig_field, sim.eps_plastic, sim.catalog, sim.Q0, exact=True)
    D = cfg.dim
    m = sim.macro()
    assert abs(m[2 * D * D] - g["macro"][-1]) <= clock_rtol(cfg) * abs(g["macro"][-1])  # simulation clock


def check_batch_replica(b, r, g, cfg):
    st = b.stats(r)
    tr = g["trace"]
    ref_sel = tr[tr[:, 0] == 0, 1].astype(np.int64)
    assert st["events"] == len(ref_sel)
    assert np.array_equal(st["selected"], ref_sel)
    casc = tr[tr[:, 0] == 1]
    assert st["cascade_flips"] == casc[:, 2].sum()
    check_fields(g, cfg, b.field(r, "eps_field"), b.field(r, "sig_field"), b.field(r, "eps_plastic"),
                 b.field(r, "catalog"), b.field(r, "Q0"), exact=False)
    D = cfg.dim
    m = b.macro(r)
    assert abs(m[2 * D * D] - g["macro"][-1]) <= clock_rtol(cfg) * abs(g["macro"][-1])


@pytest.mark.parametrize("name", SINGLE)
def test_batched_form_at_config(G, name, tmp_path):
    g = golden(name)
    cfg = inputs(g, tmp_path)
    b = G.KmcBatch([cfg])
    b.set_time_limit(600.0)
    b.run(int(g["events"]))
    assert not b.time_limited
    check_batch_replica(b, 0, g, cfg)
    b.close()


def test_batched_form_cfg1_four_replicas(G, tmp_path):
    """The benchmark's launch: seeds 0-3 of the 256^2 case together."""
    gs = [golden(n) for n in CFG1]
    cfgs = [inputs(g, tmp_path / str(i)) for i, g in enumerate(gs)]
    b = G.KmcBatch(cfgs)
    b.set_time_limit(600.0)
    b.run(100)
    assert not b.time_limited
    for r, (g, cfg) in enumerate(zip(gs, cfgs)):
        check_batch_replica(b, r, g, cfg)
    b.close()
