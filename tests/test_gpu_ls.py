"""LS solver on the GPU (C ABI) against the reference's spectral_solver_2d/3d.

Tolerance: fields within 1e-12 relative L2 of the reference (FP64 on both
sides, different FFT rounding); iteration counts identical."""
import ctypes

import numpy as np
import pytest

import oracle as O
from helpers import LS_CASES, golden, rel

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def G():
    import mgkmc_cpp_b200 as G
    G._lib.require_device()
    return G


@pytest.mark.parametrize("name", LS_CASES)
def test_ls_golden(G, name):
    g = golden(name)
    dims = tuple(int(x) for x in g["dims"])
    D = len(dims)
    s = G.LsSolver(dims, g["E"], g["nu"], "plane_stress" if int(g["plane_stress"]) else "plane_strain", float(g["pixel"]))
    eps, sig, em, sm, it = s.solve(g["eps_bar"], g.get("eps0"), g.get("epsp"), int(g["max_iter"]), float(g["tol"]))
    assert rel(eps, g["eps"]) < 1e-12
    assert rel(sig, g["sig"]) < 1e-12
    assert rel(em, g["eps_macro"]) < 1e-12
    assert rel(sm, g["sig_macro"]) < 1e-12
    o = O.ls_solve(dims, g["E"], g["nu"], g["eps_bar"], eps0=g.get("eps0"), epsp=g.get("epsp"),
                   plane_stress=bool(g["plane_stress"]), pixel=float(g["pixel"]), max_iter=int(g["max_iter"]),
                   tol=float(g["tol"]))
    assert it == o[4]


@pytest.mark.parametrize("dims", [(64, 64), (128, 96), (256, 256), (50, 36), (16, 16, 16), (24, 20, 18), (32, 32, 1)])
def test_ls_oracle_sizes(G, dims):
    rng = np.random.default_rng(sum(dims))
    D, N = len(dims), int(np.prod(dims))
    E = 90e9 * np.exp(0.15 * rng.standard_normal(N))
    nu = np.full(N, 0.36)
    eb = 1e-3 * rng.standard_normal((D, D))
    ep = 1e-2 * rng.standard_normal((N, D, D))
    ep = ep + ep.transpose(0, 2, 1)
    s = G.LsSolver(dims, E, nu)
    for it, tol in ((2, 0.0), (200, 1e-6)):
        g = s.solve(eb, None, ep, it, tol)
        o = O.ls_solve(dims, E, nu, eb, epsp=ep.reshape(N, -1), max_iter=it, tol=tol)
        assert rel(g[0], o[0]) < 1e-12
        assert rel(g[1], o[1]) < 1e-12
        assert g[4] == o[4]


def test_ls_warm_restart_is_one_iteration(G):
    rng = np.random.default_rng(3)
    N = 64 * 48
    E = 90e9 * np.exp(0.1 * rng.standard_normal(N))
    s = G.LsSolver((64, 48), E, np.full(N, 0.36))
    eb = np.array([[1e-3, 0.0], [0.0, -2e-4]])
    e1 = s.solve(eb, None, None, 200, 1e-8)
    e2 = s.solve(eb, e1[0], None, 200, 1e-8)
    assert e2[4] == 1 and rel(e2[0], e1[0]) < 1e-8


def test_ls_bad_arguments(G):
    L = G._lib.lib()
    h = ctypes.c_void_p()
    E = np.ones(4)
    assert L.mgk_ls_create(ctypes.byref(h), 4, 2, 2, 1, 0, 1.0, G._lib.dptr(E), G._lib.dptr(E)) == 2  # MGK_BAD_SHAPE
    assert L.mgk_ls_create(ctypes.byref(h), 2, 0, 2, 1, 0, 1.0, G._lib.dptr(E), G._lib.dptr(E)) == 2
    assert L.mgk_ls_create(ctypes.byref(h), 2, 2, 2, 1, 0, 1.0, None, None) == 6  # MGK_BAD_ARG
    # a length with a prime factor > 13 is refused, not mis-transformed
    E17 = np.full(17 * 4, 90e9)
    assert L.mgk_ls_create(ctypes.byref(h), 2, 17, 4, 1, 0, 1.0, G._lib.dptr(E17), G._lib.dptr(E17 * 0 + 0.3)) == 2


def test_ls_not_converged_status(G):
    rng = np.random.default_rng(5)
    N = 32 * 32
    E = 90e9 * np.exp(0.5 * rng.standard_normal(N))
    s = G.LsSolver((32, 32), E, np.full(N, 0.3))
    L = G._lib.lib()
    eps = np.zeros((N, 4))
    eb = np.array([1e-3, 0, 0, 0.0])
    it = ctypes.c_int(0)
    st = L.mgk_ls_solve(s._h, G._lib.dptr(eb), None, G._lib.dptr(eps), 0, None, None, 3, 1e-12, ctypes.byref(it))
    assert st == 1 and it.value == 3  # MGK_LS_NOT_CONVERGED, fields still written
    assert np.abs(eps).max() > 0
