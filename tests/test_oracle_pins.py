"""The oracle (C restatement, oracle/mgk_oracle.c) pinned against the reference.

Golden fixtures were produced by the reference itself (tests/golden/make_golden.py
runs oracle/_ref/ref_driver); when the compiled reference is present the pins
are also checked live on fresh inputs."""
import os

import numpy as np
import pytest

import oracle as O
from helpers import KMC_CASES, KMC_RUN, LS_CASES, compare_trace, golden, kmc_config_from_golden, rel

HAVE_REF = os.path.exists(os.path.join(O.REF_DIR, "ref_driver"))


def test_rng_draws_bit_exact():
    g = golden("draws_seed7")["draws"]
    mine = O.draws(7, len(g))
    assert np.array_equal(mine, g)


@pytest.mark.parametrize("name", LS_CASES)
def test_ls_matches_reference(name):
    g = golden(name)
    dims = tuple(int(x) for x in g["dims"])
    eps, sig, me, ms, it = O.ls_solve(dims, g["E"], g["nu"], g["eps_bar"], eps0=g.get("eps0"), epsp=g.get("epsp"),
                                      plane_stress=bool(g["plane_stress"]), pixel=float(g["pixel"]),
                                      max_iter=int(g["max_iter"]), tol=float(g["tol"]))
    assert rel(eps, g["eps"]) < 1e-13
    assert rel(sig, g["sig"]) < 1e-13
    assert rel(ms, g["sig_macro"]) < 1e-12


def test_homogeneous_closed_form():
    # uniform strain, sigma = C : eps_bar (plane strain Hooke), one LS iteration
    g = golden("ls2d_32_homog")
    E, nu = float(g["E"][0]), float(g["nu"][0])
    mu = E / (2 * (1 + nu))
    lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    eb = g["eps_bar"]
    sig = 2 * mu * eb + lam * np.trace(eb) * np.eye(2)
    assert np.allclose(g["eps"].reshape(-1, 2, 2), eb[None], rtol=0, atol=1e-17)
    assert np.allclose(g["sig_macro"].reshape(2, 2), sig, rtol=1e-12, atol=0)


@pytest.mark.parametrize("name", KMC_CASES)
def test_kmc_trace_matches_reference(name):
    g = golden(name)
    cfg, _ = kmc_config_from_golden(g)
    sim = O.OracleKmc(cfg)
    nsteps, maxev = KMC_RUN[name]
    tr = sim.run(nsteps, maxev)
    compare_trace(tr, g["trace"], tol=1e-9)
    assert np.array_equal(sim.get("catalog"), g["catalog"].reshape(-1))
    assert np.array_equal(sim.get("Q0"), g["Q0"].reshape(-1))
    assert np.array_equal(sim.get("epsp"), g["epsp"].reshape(-1))
    assert rel(sim.get("eps"), g["eps"]) < 1e-13
    assert np.allclose(sim.get("soft"), g["soft"].reshape(-1), rtol=1e-14, atol=1e-300)


@pytest.mark.skipif(not HAVE_REF, reason="compiled reference (oracle/_ref) not present")
@pytest.mark.parametrize("dims", [(20, 14), (7, 6, 5)])
def test_ls_live_against_reference(dims):
    rng = np.random.default_rng(42)
    D, N = len(dims), int(np.prod(dims))
    E = 70e9 * np.exp(0.3 * rng.standard_normal(N))
    nu = 0.25 + 0.1 * rng.random(N)
    eb = 1e-3 * rng.standard_normal((D, D))
    ep = 1e-2 * rng.standard_normal((N, D, D))
    r = O.RefDriver().ls(dims, E, nu, eb, epsp=(ep + ep.transpose(0, 2, 1)).reshape(N, -1), max_iter=200, tol=1e-8)
    o = O.ls_solve(dims, E, nu, eb, epsp=(ep + ep.transpose(0, 2, 1)).reshape(N, -1), max_iter=200, tol=1e-8)
    assert rel(o[0], r[0]) < 1e-12
