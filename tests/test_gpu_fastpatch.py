"""Fast patching (kmc_solver.hpp:276-332 / :1256-1331 precomputed stress
kernels; :866-913 / :1877-1939 stencil updates after thermal flips, :525-560
after cascade flips; a full LS solve every sync_interval flips) against the
reference's own run_simulation (golden fp*.npz, written by ref_driver kmc_run
from the reference sources): the summary log row for row (event types,
counters, strain and stress to their printed digits), the random draws
(catalog and barriers bit-identical: same flips, same host stream), the
plastic strain, and the strain and kept stress fields within 1e-10."""
import numpy as np
import pytest

from helpers import golden, rel, same_log

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["fp2d_16", "fp3d_8x8x6"])
def test_fast_patching_matches_reference(name, tmp_path):
    import mgkmc_cpp_b200 as G
    from mgkmc_cpp_b200.workloads import load_config
    G._lib.require_device()
    g = golden(name)
    cfg = load_config(str(g["yaml"]))
    assert cfg.fast_patching
    sim = G.from_config(cfg, output_dir=str(tmp_path))
    sim.run_simulation(int(g["nsteps"]), cfg.step_size, cfg.driving, cfg.targets, cfg.mixed_tol_pa, 50,
                       enable_console_log=False, enable_summary_log=True, enable_global_log=False,
                       max_kmc_steps_pct=cfg.max_kmc_steps_pct)
    same_log(open(tmp_path / "summary_log.txt").read(), str(g["summary"]))
    assert np.array_equal(sim.catalog.reshape(-1), g["catalog"].reshape(-1))
    assert np.array_equal(sim.Q0, g["Q0"].reshape(-1))
    assert rel(sim.eps_plastic, g["epsp"]) < 1e-13
    assert rel(sim.eps_field, g["eps"]) < 1e-10
    assert rel(sim.sig_field, g["sig"]) < 1e-10
    D = cfg.dim
    assert abs(sim.macro()[2 * D * D] - g["macro"][-1]) <= 1e-12 * abs(g["macro"][-1])


def test_fast_patching_rejected_by_the_batched_form(tmp_path):
    import mgkmc_cpp_b200 as G
    from mgkmc_cpp_b200.workloads import load_config
    G._lib.require_device()
    cfg = load_config(str(golden("fp2d_16")["yaml"]))
    with pytest.raises(G.MgkError) as e:
        G.KmcBatch([cfg])
    assert e.value.status == 7  # MGK_UNSUPPORTED
