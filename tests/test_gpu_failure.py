"""Device-side failure detection of the persistent LS launch.

Every barrier wait inside the launch is bounded by device time.  The test
injects a failure from the host: one CTA of the next solve leaves before its
first barrier, as if it had died.  The other CTAs' waits then run out after
the wait limit (set to 1 ms here), every CTA returns without trapping, and the
call reports MGK_DEVICE_TIMEOUT.  The handle stays usable afterwards: with the
injection off, the same handle solves again and matches a fresh solver.
Nothing traps, faults or waits without a bound."""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def G():
    import mgkmc_cpp_b200 as G
    G._lib.require_device()
    return G


def _case(dims, seed):
    rng = np.random.default_rng(seed)
    N = int(np.prod(dims))
    E = 90e9 * np.exp(0.1 * rng.standard_normal(N))
    nu = np.full(N, 0.36)
    D = len(dims)
    eb = np.zeros((D, D))
    eb[0, 0], eb[1, 1] = 1e-3, -3e-4
    return E, nu, eb


@pytest.mark.parametrize("dims", [(64, 48), (16, 12, 10)])
def test_absent_cta_times_out_and_handle_recovers(G, dims):
    E, nu, eb = _case(dims, 5)
    s = G.LsSolver(dims, E, nu)
    s.set_wait_limit(1e-3)
    s.inject_absent_cta(0)
    t0 = time.perf_counter()
    with pytest.raises(G.MgkError, match="DEVICE_TIMEOUT"):
        s.solve(eb, max_iter=50, tol=1e-10)
    assert time.perf_counter() - t0 < 10.0  # returned after bounded waits
    s.inject_absent_cta(-1)
    eps, sig, em, sm, it = s.solve(eb, max_iter=200, tol=1e-10)
    s.close()
    f = G.LsSolver(dims, E, nu)
    eps_f, sig_f, em_f, sm_f, it_f = f.solve(eb, max_iter=200, tol=1e-10)
    f.close()
    assert it == it_f
    assert np.array_equal(eps, eps_f) and np.array_equal(sig, sig_f)


def test_wait_limit_arguments(G):
    E, nu, eb = _case((8, 8), 1)
    s = G.LsSolver((8, 8), E, nu)
    with pytest.raises(G.MgkError, match="BAD_ARG"):
        s.set_wait_limit(-1.0)
    with pytest.raises(G.MgkError, match="BAD_ARG"):
        s.inject_absent_cta(10 ** 6)
    s.set_wait_limit(0.0)  # back to the default bound
    s.solve(eb)
    s.close()
