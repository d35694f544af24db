"""Batched, device-resident KMC (mgk_batch_*) against the reference's own
traces and against the plain engine.

The batch kernel continues each replica's std::mt19937 stream on the device,
so with the same seed it must select the same modes as the reference: the
selected-mode sequence is compared index for index with the golden traces
(written by the reference), the strain and stress fields within 1e-10
relative L2.  The catalog and barrier redraws run the reference's
distributions on the device, whose log/exp may differ from glibc's by an ulp,
so the catalog, the barriers and the plastic strain accumulated from the
catalog are held to 1e-13 relative."""
import numpy as np
import pytest

from helpers import KMC_CASES, KMC_RUN, golden, kmc_config_from_golden, rel

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def G():
    import mgkmc_cpp_b200 as G
    G._lib.require_device()
    return G


def events_of(trace):
    return trace[trace[:, 0] == 0, 1].astype(np.int64)


def check_against_golden(b, r, g, cfg):
    st = b.stats(r)
    ref_sel = events_of(g["trace"])
    assert st["events"] == len(ref_sel)
    assert np.array_equal(st["selected"], ref_sel)
    assert rel(b.field(r, "eps_plastic"), g["epsp"]) < 1e-13
    assert rel(b.field(r, "eps_field"), g["eps"]) < 1e-10
    assert rel(b.field(r, "sig_field"), g["sig"]) < 1e-10
    assert np.allclose(b.field(r, "catalog").reshape(-1), g["catalog"].reshape(-1), rtol=1e-13, atol=1e-300)
    assert np.allclose(b.field(r, "Q0"), g["Q0"].reshape(-1), rtol=1e-13, atol=0)
    D = cfg.dim
    m = b.macro(r)
    assert abs(m[2 * D * D] - g["macro"][-1]) <= 1e-12 * abs(g["macro"][-1])  # simulation clock


def test_batch_mixed_golden(G):
    """All golden cases (2D and 3D, two- and six-component catalogs) in one launch."""
    gs = [golden(n) for n in KMC_CASES]
    cfgs = [kmc_config_from_golden(g)[0] for g in gs]
    nsteps = {KMC_RUN[n][0] for n in KMC_CASES}
    maxev = {KMC_RUN[n][1] for n in KMC_CASES}
    assert len(nsteps) == 1 and len(maxev) == 1
    b = G.KmcBatch(cfgs)
    b.run(maxev.pop(), n_global_steps=nsteps.pop())
    assert not b.time_limited
    for r, (g, cfg) in enumerate(zip(gs, cfgs)):
        check_against_golden(b, r, g, cfg)
        assert b.stats(r)["fallbacks"] == 0


@pytest.mark.parametrize("name", ["kmc2d_8_soft_neigh", "kmc3d_6x6x4_soft"])
def test_batch_single_golden(G, name):
    g = golden(name)
    cfg, _ = kmc_config_from_golden(g)
    nsteps, maxev = KMC_RUN[name]
    b = G.KmcBatch([cfg])
    b.run(maxev, n_global_steps=nsteps)
    check_against_golden(b, 0, g, cfg)


def test_batch_continuation(G):
    """Two runs of 120 + 180 events equal one run of 300: the interval clock,
    macro state and device random stream are handed back and forth exactly."""
    name = "kmc2d_12_nosoft"
    g = golden(name)
    cfg, _ = kmc_config_from_golden(g)
    nsteps, maxev = KMC_RUN[name]
    b = G.KmcBatch([cfg])
    b.run(120, n_global_steps=nsteps)
    s1 = b.stats(0)["selected"]
    b.run(maxev - 120, n_global_steps=nsteps)
    s2 = b.stats(0)["selected"]
    assert np.array_equal(np.concatenate([s1, s2]), events_of(g["trace"]))
    assert rel(b.field(0, "eps_plastic"), g["epsp"]) < 1e-13
    assert rel(b.field(0, "eps_field"), g["eps"]) < 1e-10


def test_batch_same_alone_and_in_mix(G, tmp_path):
    """A replica's result does not depend on what else shares the launch: the
    flips are identical; the fields agree to rounding (alone, the replica
    gets more CTAs, which changes the order of the LS norm partial sums)."""
    from mgkmc_cpp_b200 import workloads
    cfgs = []
    for name, seed in [("ens2d_64", 3), ("ens2d_128", 1), ("hetero3d_16", 1), ("ens2d_64", 4)]:
        cfgs.append(workloads.write_workload(name, str(tmp_path), seed=seed)[1])
    mix = G.KmcBatch(cfgs)
    mix.run(60)
    assert not mix.time_limited
    alone = G.KmcBatch([cfgs[2]])
    alone.run(60)
    assert np.array_equal(mix.stats(2)["selected"], alone.stats(0)["selected"])
    assert mix.stats(2)["events"] == 60
    assert np.array_equal(mix.field(2, "eps_plastic"), alone.field(0, "eps_plastic"))
    assert rel(mix.field(2, "eps_field"), alone.field(0, "eps_field")) < 1e-12
    D = cfgs[2].dim
    ma, mb = mix.macro(2), alone.macro(0)
    for blk in (slice(0, D * D), slice(D * D, 2 * D * D)):  # eps_macro, sig_macro: to each tensor's scale
        assert np.abs(ma[blk] - mb[blk]).max() <= 1e-12 * np.abs(mb[blk]).max() + 1e-300
    assert np.allclose(ma[2 * D * D:], mb[2 * D * D:], rtol=1e-12, atol=0)


def test_batch_matches_plain_engine(G, tmp_path):
    from mgkmc_cpp_b200 import workloads
    _, cfg = workloads.write_workload("ens2d_128", str(tmp_path), seed=5)
    sim = G.from_config(cfg, output_dir=str(tmp_path))
    tr = sim.run_simulation(10 ** 6, cfg.step_size, cfg.driving, cfg.targets, cfg.mixed_tol_pa, 50,
                            enable_console_log=False, enable_summary_log=False, enable_global_log=False,
                            max_events=200, trace=True)
    b = G.KmcBatch([cfg])
    b.run(200)
    assert np.array_equal(b.stats(0)["selected"], events_of(tr))
    assert rel(b.field(0, "eps_plastic"), sim.eps_plastic) < 1e-13
    assert rel(b.field(0, "eps_field"), sim.eps_field) < 1e-10


def test_batch_time_limit(G, tmp_path):
    """An event budget the run cannot reach within its time limit: the run
    stops at the limit with MGK_TIME_LIMIT and the replica can still be read."""
    from mgkmc_cpp_b200 import workloads
    _, cfg = workloads.write_workload("hetero2d_64", str(tmp_path), seed=0)
    b = G.KmcBatch([cfg])
    b.set_time_limit(0.5)
    ms = b.run(10 ** 9)
    assert b.time_limited
    assert b.stats(0)["terminated"] == 2
    assert 400 < ms < 10000
    assert np.isfinite(b.field(0, "eps_field")).all()


def test_batch_time_limit_mixed_sizes(G, tmp_path):
    """A mixed batch under a short time limit: every replica stops on the time
    limit (a replica past it keeps working until all are), the small one has
    been taking events through the limit, and the state stays readable."""
    from mgkmc_cpp_b200 import workloads
    _, small = workloads.write_workload("ens2d_64", str(tmp_path / "s"), seed=0)
    _, big = workloads.write_workload("ens2d_512", str(tmp_path / "b"), seed=32)
    b = G.KmcBatch([small, big])
    b.set_time_limit(0.2)
    ms = b.run(10 ** 9)
    assert b.time_limited and ms >= 200.0
    st_s, st_b = b.stats(0), b.stats(1)
    assert st_s["terminated"] == 2 and st_b["terminated"] == 2
    assert st_s["events"] > 0 and st_s["event_us"].sum() / 1e3 > 0.8 * 200.0
    assert np.isfinite(b.field(0, "eps_field")).all() and np.isfinite(b.field(1, "eps_field")).all()


def test_generator_handed_between_batched_and_plain_runs(G, tmp_path):
    """Between batched runs the generator stays in the device layout and is
    handed back to the plain form only when that form draws again: split
    batched runs select what one run selects, and a plain run after them
    continues the same stream as a plain run after plain runs of the same
    events."""
    from mgkmc_cpp_b200 import workloads
    cfg = workloads.write_workload("ens2d_64", str(tmp_path), seed=3)[1]
    kw = dict(enable_console_log=False, enable_summary_log=False, enable_global_log=False)

    def plain(sim, nev):
        tr = sim.run_simulation(10 ** 6, cfg.step_size, cfg.driving, cfg.targets, cfg.mixed_tol_pa, 50,
                                max_events=nev, trace=True, **kw)
        return events_of(tr)

    a = G.from_config(cfg, output_dir=None)
    ba = G.KmcBatch(sims=[a])
    ba.run(40)
    sel_a = ba.stats(0)["selected"]
    ba.close()
    b = G.from_config(cfg, output_dir=None)
    parts = []
    for nev in (15, 25):  # two batches over the same simulation, one run each
        bb = G.KmcBatch(sims=[b])
        bb.run(nev)
        parts.append(bb.stats(0)["selected"])
        bb.close()
    assert np.array_equal(np.concatenate(parts), sel_a)
    e = G.from_config(cfg, output_dir=None)
    assert np.array_equal(plain(e, 40), sel_a)
    after_e = plain(e, 10)
    assert len(after_e) == 10
    assert np.array_equal(plain(a, 10), after_e)
    assert np.array_equal(plain(b, 10), after_e)
