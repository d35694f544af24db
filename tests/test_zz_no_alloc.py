"""mgk_ls_solve_noalloc: the LS solve for callers that may not allocate device
memory (their host application owns the GPU's memory pool, or their loop cannot
afford the device-wide synchronisation of cudaMalloc/cudaFree).

The test hands the entry point device buffers it allocated itself (through
torch), calls it twice in a row on different problems, and checks every output
against the allocating entry point mgk_ls_solve with the LS parity tolerance
(1e-12 relative L2).  It also checks that a grid too large for the static
scratch array is refused.  This file is collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel(a, b):
    a, b = np.ravel(a), np.ravel(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="module")
def env():
    import torch
    import mgkmc_cpp_b200 as G
    G._lib.require_device()
    L = G._lib.lib()
    dp = C.POINTER(C.c_double)
    L.mgk_ls_solve_noalloc.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_void_p, C.c_void_p,
                                       dp, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, dp, C.c_int, C.c_double,
                                       C.POINTER(C.c_int), C.c_void_p]
    L.mgk_ls_solve_noalloc.restype = C.c_int
    L.mgk_noalloc_last_error.restype = C.c_char_p
    return torch, G, L


def case(dims, seed, warm, plastic):
    rng = np.random.default_rng(seed)
    D, N = len(dims), int(np.prod(dims))
    E = 90e9 * np.exp(0.15 * rng.standard_normal(N))
    nu = 0.3 + 0.05 * rng.random(N)
    eb = 1e-3 * rng.standard_normal((D, D))
    epsp = None
    if plastic:
        epsp = 1e-2 * rng.standard_normal((N, D, D))
        epsp = epsp + epsp.transpose(0, 2, 1)
    eps0 = 1e-3 * rng.standard_normal((N, D, D)) if warm else None
    return E, nu, eb, epsp, eps0


def solve_noalloc(env, dims, E, nu, eb, epsp, eps0, plane_stress, max_iter, tol):
    torch, G, L = env
    D, N = len(dims), int(np.prod(dims))
    dev = "cuda"
    tE = torch.tensor(E, dtype=torch.float64, device=dev)
    tnu = torch.tensor(nu, dtype=torch.float64, device=dev)
    teps = torch.tensor(eps0.reshape(N, D * D) if eps0 is not None else np.zeros((N, D * D)), dtype=torch.float64,
                        device=dev)
    tep = torch.tensor(epsp.reshape(N, D * D), dtype=torch.float64, device=dev) if epsp is not None else None
    tsig = torch.zeros((N, D * D), dtype=torch.float64, device=dev)
    ebh = np.ascontiguousarray(eb, dtype=np.float64).reshape(-1)
    mac = np.zeros(2 * D * D)
    it = C.c_int(0)
    torch.cuda.synchronize()
    st = L.mgk_ls_solve_noalloc(D, dims[0], dims[1], dims[2] if D == 3 else 1, int(plane_stress), 1.0, tE.data_ptr(),
                                tnu.data_ptr(), G._lib.dptr(ebh), tep.data_ptr() if tep is not None else None,
                                teps.data_ptr(), int(eps0 is not None), tsig.data_ptr(), G._lib.dptr(mac), max_iter, tol,
                                C.byref(it), None)
    assert st in (0, 1), L.mgk_noalloc_last_error()
    return teps.cpu().numpy(), tsig.cpu().numpy(), mac, it.value, st


def solve_alloc(env, dims, E, nu, eb, epsp, eps0, plane_stress, max_iter, tol):
    torch, G, L = env
    s = G.LsSolver(dims, E, nu, "plane_stress" if plane_stress else "plane_strain", 1.0)
    eps, sig, em, sm, it = s.solve(eb, eps0, epsp, max_iter, tol)
    s.close()
    D = len(dims)
    return eps.reshape(-1, D * D), sig.reshape(-1, D * D), np.concatenate([em.ravel(), sm.ravel()]), it


CASES = [((64, 48), 11, True, True, False, 200, 1e-8),   # 2D, warm start, plastic strain
         ((20, 16, 12), 12, False, True, False, 200, 1e-8),  # 3D, cold start
         ((50, 30), 13, True, False, True, 3, 0.0)]        # 2D plane stress, fixed 3 iterations


def test_noalloc_matches_allocating_solver_twice_in_a_row(env):
    for dims, seed, warm, plastic, ps, mi, tol in CASES:
        args = case(dims, seed, warm, plastic)
        n_eps, n_sig, n_mac, n_it, _ = solve_noalloc(env, dims, *args, ps, mi, tol)
        a_eps, a_sig, a_mac, a_it = solve_alloc(env, dims, *args, ps, mi, tol)
        assert n_it == a_it
        assert rel(n_eps, a_eps) < 1e-12
        assert rel(n_sig, a_sig) < 1e-12
        assert rel(n_mac, a_mac) < 1e-12
    # the first case once more: the shared scratch keeps the previous call's
    # contents, which must not leak into this result
    dims, seed, warm, plastic, ps, mi, tol = CASES[0]
    args = case(dims, seed, warm, plastic)
    again = solve_noalloc(env, dims, *args, ps, mi, tol)
    ref = solve_alloc(env, dims, *args, ps, mi, tol)
    assert again[3] == ref[3] and rel(again[0], ref[0]) < 1e-12 and rel(again[1], ref[1]) < 1e-12


def _noalloc_status(env, dims, plastic):
    torch, G, L = env
    D, N = len(dims), int(np.prod(dims))
    t = torch.full((N,), 90e9, dtype=torch.float64, device="cuda")
    nu = torch.full((N,), 0.3, dtype=torch.float64, device="cuda")
    e = torch.zeros((N, D * D), dtype=torch.float64, device="cuda")
    ep = torch.zeros((N, D * D), dtype=torch.float64, device="cuda") if plastic else None
    eb = np.zeros(D * D)
    eb[0] = 1e-3
    it = C.c_int(0)
    st = L.mgk_ls_solve_noalloc(D, dims[0], dims[1], dims[2] if D == 3 else 1, 0, 1.0, t.data_ptr(), nu.data_ptr(),
                                G._lib.dptr(eb), ep.data_ptr() if ep is not None else None, e.data_ptr(), 0, None, None,
                                5, 1e-6, C.byref(it), None)
    torch.cuda.synchronize()
    return st


def test_noalloc_refuses_grids_beyond_its_static_scratch(env):
    torch, G, L = env
    # 16 MiB of scratch: just below the limit, 2D with a plastic strain and 3D
    assert _noalloc_status(env, (432, 432), True) in (0, 1)
    assert _noalloc_status(env, (45, 45, 45), True) in (0, 1)
    # just above it, and far above it
    for dims, plastic in (((448, 432), True), ((48, 48, 48), True), ((512, 512), False)):
        assert _noalloc_status(env, dims, plastic) == 2  # MGK_BAD_SHAPE
        assert b"static limit" in L.mgk_noalloc_last_error()


def test_noalloc_leaves_other_solvers_launchable(env):
    # the kernel's dynamic shared-memory limit is process-wide: a no-alloc
    # call on a small grid must not lower it below what a live solver of a
    # larger grid planned for
    torch, G, L = env
    big = (384, 512)  # row pass of 512-point lines: above the 48 KiB default limit
    E, nu, eb, epsp, eps0 = case(big, 21, False, False)
    s = G.LsSolver(big, E, nu, "plane_strain", 1.0)
    ref = s.solve(eb, None, None, 200, 1e-8)
    small = (12, 10)
    solve_noalloc(env, small, *case(small, 22, False, False), False, 50, 1e-8)
    again = s.solve(eb, None, None, 200, 1e-8)
    s.close()
    assert again[4] == ref[4] and rel(again[0], ref[0]) < 1e-12
