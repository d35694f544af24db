"""KMC engine on the GPU against the reference (golden traces produced by the
reference itself) and the oracle.

Bar: event kinds, selected (voxel, mode) indices and cascade sizes identical;
catalog, barriers and plastic strain bit-identical (same host RNG draws, same
flips); strain field within 1e-10 relative L2; accumulated macro columns of the
trace within 1e-9 of each column's scale."""
import numpy as np
import pytest

import oracle as O
from helpers import KMC_CASES, KMC_RUN, compare_trace, golden, kmc_config_from_golden, rel

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def G():
    import mgkmc_cpp_b200 as G
    G._lib.require_device()
    return G


def run(G, cfg, nsteps, maxev, tmp_path):
    sim = G.from_config(cfg, output_dir=str(tmp_path))
    tr = sim.run_simulation(nsteps, cfg.step_size, cfg.driving, cfg.targets, cfg.mixed_tol_pa, 50,
                            enable_console_log=False, enable_summary_log=False, enable_global_log=False,
                            max_kmc_steps_pct=cfg.max_kmc_steps_pct, max_events=maxev, trace=True)
    return sim, tr


@pytest.mark.parametrize("name", KMC_CASES)
def test_kmc_trace_golden(G, name, tmp_path):
    g = golden(name)
    cfg, _ = kmc_config_from_golden(g)
    nsteps, maxev = KMC_RUN[name]
    sim, tr = run(G, cfg, nsteps, maxev, tmp_path)
    compare_trace(tr, g["trace"], tol=1e-9)
    D = cfg.dim
    assert np.array_equal(sim.catalog.reshape(-1), g["catalog"].reshape(-1))
    assert np.array_equal(sim.Q0, g["Q0"].reshape(-1))
    assert np.array_equal(sim.eps_plastic.reshape(-1), g["epsp"].reshape(-1))
    assert rel(sim.eps_field, g["eps"]) < 1e-10
    assert rel(sim.sig_field, g["sig"]) < 1e-10
    assert np.allclose(sim.soft_prop.reshape(-1), g["soft"].reshape(-1), rtol=1e-12, atol=1e-300)
    assert np.array_equal(sim.prev_strain_dir.reshape(-1), g["prev_dir"].reshape(-1))
    lt_ref, lt = g["last_t"].reshape(-1), sim.last_event_time
    fin = np.isfinite(lt_ref)
    assert np.array_equal(np.isfinite(lt), fin) and np.allclose(lt[fin], lt_ref[fin], rtol=1e-12, atol=0)
    m = sim.macro()
    assert abs(m[2 * D * D] - g["macro"][-1]) <= 1e-12 * abs(g["macro"][-1])  # simulation clock


@pytest.mark.parametrize("name", ["hetero2d_64", "hetero3d_16"])
def test_kmc_workloads_against_oracle(G, name, tmp_path):
    from mgkmc_cpp_b200 import workloads
    _, cfg = workloads.write_workload(name, str(tmp_path), seed=1)
    nev = 150 if cfg.dim == 2 else 60
    ok = O.OracleKmc(cfg)
    ref = ok.run(10 ** 6, nev)
    sim, tr = run(G, cfg, 10 ** 6, nev, tmp_path)
    compare_trace(tr, ref, tol=1e-9)
    assert np.array_equal(sim.eps_plastic.reshape(-1), ok.get("epsp"))
    assert rel(sim.eps_field, ok.get("eps")) < 1e-10


def test_kmc_deterministic(G, tmp_path):
    g = golden("kmc2d_8_soft_neigh")
    cfg, _ = kmc_config_from_golden(g)
    _, t1 = run(G, cfg, 25, 300, tmp_path)
    _, t2 = run(G, cfg, 25, 300, tmp_path)
    assert np.array_equal(t1, t2)


def test_kmc_logs_and_vtu(G, tmp_path):
    g = golden("kmc2d_12_nosoft")
    cfg, _ = kmc_config_from_golden(g)
    sim = G.from_config(cfg, output_dir=str(tmp_path))
    sim.run_simulation(2, cfg.step_size, cfg.driving, cfg.targets, cfg.mixed_tol_pa, 50, enable_console_log=False,
                       vtk_interval="1", max_events=50)
    summ = (tmp_path / "summary_log.txt").read_text().splitlines()
    assert summ[0].startswith("Timestamp") and set(summ[1]) == {"-"}
    assert any(" KMC " in l for l in summ[2:])
    glob_ = (tmp_path / "global_log.txt").read_text().splitlines()
    assert glob_[0].split()[0] == "GlobalStep" and len(glob_[1].split()) == 18
    vtus = sorted(p.name for p in tmp_path.glob("*.vtu"))
    assert "vtk_step_000000.vtu" in vtus
    txt = (tmp_path / vtus[0]).read_text()
    assert 'NumberOfPoints="338" NumberOfCells="144"' in txt and "eps_plastic_vm" in txt and "g_t" in txt


def test_kmc_bad_args(G):
    with pytest.raises(G.MgkError, match="BAD_SHAPE"):
        G.KmcSimulation2D(4, 4, 2, 0.1, np.full(16, 90e9), np.full(16, 0.3), fast_patching_enabled=True,
                          sync_interval=0)
    with pytest.raises(ValueError):
        G.KmcSimulation2D(4, 4, 2, 0.1, np.full(15, 90e9), np.full(16, 0.3))
