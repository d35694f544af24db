"""The serving loop (Server): continuous batching of KMC jobs.

A job's result must be the same alone and in the mix: jobs that arrive while
others are on the GPU are admitted between launches, their launches are
shared, and each job still selects exactly the modes it selects alone (its
random stream and interval clock are its own); its fields agree to rounding
(the LS partial sums are split over a different number of CTAs)."""
import numpy as np
import pytest

from helpers import rel

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def G():
    import mgkmc_cpp_b200 as G
    G._lib.require_device()
    return G


def _cfg(name, seed, tmp_path):
    from mgkmc_cpp_b200 import workloads
    return workloads.write_workload(name, str(tmp_path), seed=seed)[1]


def test_served_job_same_alone_and_in_mix(G, tmp_path):
    a = _cfg("ens2d_64", 3, tmp_path)
    # reference trajectory: one uninterrupted batched run
    ref = G.KmcBatch([a])
    ref.run(120)
    ref_sel = ref.stats(0)["selected"]
    ref_eps = ref.field(0, "eps_field")
    ref.close()
    # alone, in slices of 40 events (three launches)
    srv = G.Server(slice_events=40)
    ja = srv.submit(a, 120)
    while not srv.idle():
        srv.step()
    alone = srv.done[ja]
    assert np.array_equal(alone["selected"], ref_sel)
    assert rel(alone["eps_field"], ref_eps) < 1e-12
    assert srv.launches == 3
    # in a mix: other jobs already running when it arrives, others arriving after it
    srv = G.Server(slice_events=40)
    jb = srv.submit(_cfg("ens2d_128", 1, tmp_path), 200, arrival=0.0)
    ja = srv.submit(a, 120, arrival=1.0)
    jc = srv.submit(_cfg("hetero3d_16", 1, tmp_path), 60, arrival=2.0)
    jd = srv.submit(_cfg("ens2d_64", 9, tmp_path), 30, arrival=2.0)
    now, active_seen = 0.0, []
    while not srv.idle():
        srv.step(now)
        active_seen.append(len(srv.active))
        now += 1.0
    mixed = srv.done[ja]
    assert np.array_equal(mixed["selected"], ref_sel)
    assert rel(mixed["eps_field"], ref_eps) < 1e-12
    assert {jb, jc, jd} <= set(srv.done)
    for j in (jb, jc, jd):
        assert srv.done[j]["events"] == srv.done[j]["target"]
    assert max(active_seen) >= 3  # the launches were shared
    assert len(srv.step_latency_us) == sum(srv.done[j]["events"] for j in srv.done)


def test_time_sliced_serving_same_as_alone(G, tmp_path):
    """Time slices (the default): every job stops at its first decision past
    the slice's device time; the flips are still exactly the job's own."""
    cfgs = [_cfg("ens2d_64", 3, tmp_path), _cfg("ens2d_128", 1, tmp_path), _cfg("hetero3d_16", 1, tmp_path)]
    targets = [150, 80, 40]
    refs = []
    for c, t in zip(cfgs, targets):
        b = G.KmcBatch([c])
        b.run(t)
        refs.append(b.stats(0)["selected"])
        b.close()
    srv = G.Server(slice_seconds=0.002)
    ids = [srv.submit(c, t, arrival=float(i)) for i, (c, t) in enumerate(zip(cfgs, targets))]
    now = 0.0
    while not srv.idle():
        srv.step(now)
        now += 1.0
    assert srv.launches > 3
    for jid, ref in zip(ids, refs):
        assert np.array_equal(srv.done[jid]["selected"], ref)


def test_admission_gated_by_free_memory(G, tmp_path):
    """With an HBM budget that holds one job, jobs run one at a time."""
    cfgs = [_cfg("ens2d_64", s, tmp_path) for s in range(3)]
    need = G.job_device_bytes(cfgs[0])
    srv = G.Server(slice_events=20, hbm_budget=int(1.5 * need))
    for c in cfgs:
        srv.submit(c, 20)
    while not srv.idle():
        srv.step()
        assert srv.committed <= srv.budget
    assert len(srv.done) == 3
    assert srv.launches == 3


def test_jobs_built_on_the_pool_same_as_alone(G, tmp_path):
    """build_threads > 0: jobs after the first of their grid shape are built
    on host threads while the others run, and join the batch when ready; each
    still selects exactly its own modes."""
    seeds = [3, 4, 5, 6, 7, 8]
    cfgs = [_cfg("ens2d_64" if s % 2 else "ens2d_128", s, tmp_path) for s in seeds]
    targets = [60, 40, 50, 30, 45, 35]
    refs = []
    for c, t in zip(cfgs, targets):
        b = G.KmcBatch([c])
        b.run(t)
        refs.append(b.stats(0)["selected"])
        b.close()
    srv = G.Server(slice_seconds=0.002, build_threads=2)
    ids = [srv.submit(c, t) for c, t in zip(cfgs, targets)]
    while not srv.idle():
        srv.step()
    srv.close()
    assert srv.built_on_pool == 4  # every job after the first of its grid shape
    for jid, ref in zip(ids, refs):
        assert np.array_equal(srv.done[jid]["selected"], ref)
    assert srv.committed == 0
    assert set(srv.host_seconds) == {"build_wait", "rebuild", "readback", "retire"}
