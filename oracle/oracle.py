"""TEST INFRASTRUCTURE ONLY -- Python access to the oracle.

Two checkers live here, both CPU-only and never imported by the product:

* ``Oracle*`` wrap ``_ref/liboracle.so``, the plain-C restatement of the
  reference algorithm (mgk_oracle.c).
* ``RefDriver`` runs ``_ref/ref_driver``, the unmodified reference headers
  compiled by oracle/Makefile, through temporary directories of ``.npy`` files.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference arm
may use this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import tempfile
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
_lib = None


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(REF_DIR, "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError("oracle not built: run `make -C oracle`")
        _lib = C.CDLL(path)
        dp = C.POINTER(C.c_double)
        _lib.oracle_draws.argtypes = [C.c_int, C.c_int, dp]
        _lib.oracle_ls_solve.argtypes = [C.c_int, C.POINTER(C.c_int), C.c_int, C.c_double, dp, dp, dp, dp, C.c_int, dp,
                                         C.c_int, C.c_double, dp, dp, dp]
        _lib.oracle_ls_solve.restype = C.c_int
        _lib.oracle_kmc_create.argtypes = [C.c_void_p, dp, dp]
        _lib.oracle_kmc_create.restype = C.c_void_p
        _lib.oracle_kmc_destroy.argtypes = [C.c_void_p]
        _lib.oracle_kmc_run.argtypes = [C.c_void_p, C.c_int, C.c_long, dp, C.c_long]
        _lib.oracle_kmc_run.restype = C.c_long
        _lib.oracle_kmc_get.argtypes = [C.c_void_p, C.c_int, dp]
        _lib.oracle_kmc_get.restype = C.c_long
        _lib.oracle_kmc_macro.argtypes = [C.c_void_p, dp]
        _lib.oracle_sizeof_params.restype = C.c_long
        assert _lib.oracle_sizeof_params() == C.sizeof(KmcParams), "kmc_params layout mismatch"
    return _lib


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class BarrierC(C.Structure):
    _fields_ = [("type", C.c_int), ("mean", C.c_double), ("std_val", C.c_double), ("min_cutoff", C.c_double),
                ("max_cutoff", C.c_double), ("loc", C.c_double), ("scale", C.c_double), ("epsilon", C.c_double),
                ("ratio", C.c_double)]


class KmcParams(C.Structure):
    _fields_ = [("dim", C.c_int), ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("M", C.c_int),
                ("plane_stress", C.c_int), ("seed", C.c_int), ("gamma0", C.c_double), ("pixel", C.c_double),
                ("bar", BarrierC), ("directional", C.c_int), ("softening_cap", C.c_double), ("jp", C.c_double),
                ("jt", C.c_double), ("neighbor_fraction", C.c_double), ("q_act_temp", C.c_double),
                ("temperature", C.c_double), ("strain_rate", C.c_double), ("stability_threshold", C.c_double),
                ("nu0", C.c_double), ("instability_kmc", C.c_int), ("scale_rate_by_volume", C.c_int),
                ("redraw_directions", C.c_int), ("redraw_barriers", C.c_int), ("use_3d_barriers", C.c_int),
                ("step_size", C.c_double), ("mixed_tol", C.c_double), ("max_kmc_steps_pct", C.c_double),
                ("comp_i", C.c_int), ("comp_j", C.c_int), ("n_targets", C.c_int), ("target_i", C.c_int * 9),
                ("target_j", C.c_int * 9), ("target_v", C.c_double * 9), ("catalog_type", C.c_int),
                ("barrier_per_voxel", C.c_int)]


CATALOG_TYPES = {"random": 0, "even": 1, "fibonacci": 2}


def params_from_config(cfg) -> KmcParams:
    from mgkmc_cpp_b200.config import BARRIER_TYPES
    p = KmcParams()
    p.dim, p.nx, p.ny, p.nz, p.M = cfg.dim, cfg.nx, cfg.ny, cfg.nz if cfg.dim == 3 else 1, cfg.M
    p.plane_stress = 1 if cfg.plane_mode == "plane_stress" else 0
    p.seed, p.gamma0, p.pixel = cfg.seed, cfg.gamma0, cfg.pixel
    b = cfg.barrier
    p.bar = BarrierC(BARRIER_TYPES.get(b.type, -1), b.mean, b.std, b.min_cutoff, b.max_cutoff, b.loc, b.scale, b.epsilon,
                     b.ratio)
    p.directional = 1 if cfg.softening_scheme == "directional" else 0
    p.softening_cap, p.jp, p.jt = cfg.softening_cap, cfg.jp, cfg.jt
    p.neighbor_fraction, p.q_act_temp = cfg.neighbor_softening_fraction, cfg.q_act_temp
    p.temperature, p.strain_rate, p.stability_threshold, p.nu0 = cfg.temperature, cfg.strain_rate, cfg.stability_threshold, cfg.nu0
    p.instability_kmc = 1 if cfg.instability_mode == "kmc" else 0
    p.scale_rate_by_volume, p.redraw_directions = int(cfg.scale_rate_by_volume), int(cfg.redraw_directions)
    p.redraw_barriers, p.use_3d_barriers = int(cfg.redraw_barriers), int(cfg.use_3d_barriers)
    p.step_size, p.mixed_tol, p.max_kmc_steps_pct = cfg.step_size, cfg.mixed_tol_pa, cfg.max_kmc_steps_pct
    p.comp_i, p.comp_j = cfg.driving
    p.catalog_type = CATALOG_TYPES[cfg.catalog_type]
    p.barrier_per_voxel = int(cfg.barrier_per_voxel)
    tg = sorted(cfg.targets.items())
    p.n_targets = len(tg)
    for k, ((i, j), v) in enumerate(tg):
        p.target_i[k], p.target_j[k], p.target_v[k] = i, j, v
    return p


def draws(seed: int, n: int) -> np.ndarray:
    out = np.zeros((n, 4))
    lib().oracle_draws(seed, n, _dp(out))
    return out


def ls_solve(dims, E, nu, eps_bar, eps0=None, epsp=None, plane_stress=False, pixel=1.0, max_iter=200, tol=1e-6):
    """spectral_solver_2d/3d restated; tensors (N, D*D) row-major.  Returns
    (eps, sig, macro_eps(D*D), macro_sig(D*D), iterations)."""
    D = len(dims)
    N = int(np.prod(dims))
    eps = np.ascontiguousarray(np.array(eps0, dtype=np.float64).reshape(N, D * D)) if eps0 is not None else np.zeros((N, D * D))
    sig = np.zeros((N, D * D))
    me, ms = np.zeros(D * D), np.zeros(D * D)
    E = np.ascontiguousarray(E, dtype=np.float64).reshape(-1)
    nu = np.ascontiguousarray(nu, dtype=np.float64).reshape(-1)
    eb = np.ascontiguousarray(eps_bar, dtype=np.float64).reshape(-1)
    ep = None if epsp is None else np.ascontiguousarray(epsp, dtype=np.float64).reshape(N, D * D)
    d = (C.c_int * 3)(*(list(dims) + [1] * (3 - D)))
    it = lib().oracle_ls_solve(D, d, int(plane_stress), pixel, _dp(E), _dp(nu), _dp(eb), _dp(eps), int(eps0 is not None),
                               _dp(ep) if ep is not None else None, max_iter, tol, _dp(sig), _dp(me), _dp(ms))
    return eps, sig, me, ms, it


FIELDS = {"eps": 0, "sig": 1, "epsp": 2, "soft": 3, "last_t": 4, "Q": 5, "Q0": 6, "catalog": 7, "prev_dir": 8}


class OracleKmc:
    """KmcSimulation2D/3D restated in C (construction + run_simulation)."""

    def __init__(self, cfg):
        self.cfg = cfg
        self.p = params_from_config(cfg)
        self.D = cfg.dim
        E = np.ascontiguousarray(cfg.E, dtype=np.float64)
        nu = np.ascontiguousarray(cfg.nu, dtype=np.float64)
        self.h = lib().oracle_kmc_create(C.byref(self.p), _dp(E), _dp(nu))
        if not self.h:
            raise ValueError("the oracle refused the configuration (fibonacci catalogs need 3D)")

    def __del__(self):
        if getattr(self, "h", None):
            lib().oracle_kmc_destroy(self.h)
            self.h = None

    def run(self, nsteps: int, maxev: int = 1 << 60, cap: int = 1 << 20) -> np.ndarray:
        w = 6 + 2 * self.D * self.D
        buf = np.zeros((cap, w))
        n = lib().oracle_kmc_run(self.h, nsteps, maxev, _dp(buf), cap)
        return buf[:min(n, cap)].copy()

    def get(self, name: str) -> np.ndarray:
        f = FIELDS[name]
        n = lib().oracle_kmc_get(self.h, f, None)
        out = np.zeros(n)
        lib().oracle_kmc_get(self.h, f, _dp(out))
        return out

    def macro(self) -> np.ndarray:
        out = np.zeros(2 * self.D * self.D + 3)
        lib().oracle_kmc_macro(self.h, _dp(out))
        return out


class RefDriver:
    """The reference itself (oracle/_ref/ref_driver), run as a subprocess."""

    def __init__(self, path: Optional[str] = None):
        self.path = path or os.path.join(REF_DIR, "ref_driver")
        if not os.path.exists(self.path):
            raise RuntimeError("reference harness not built: run `make -C oracle` where the reference sources exist")

    def _run(self, args, timeout=3600):
        r = subprocess.run([self.path] + [str(a) for a in args], capture_output=True, text=True, timeout=timeout)
        if r.returncode != 0:
            raise RuntimeError("ref_driver failed: %s\n%s" % (r.stderr[-2000:], r.stdout[-2000:]))
        return r

    def ls(self, dims, E, nu, eps_bar, eps0=None, epsp=None, plane_mode="plane_strain", pixel=1.0, max_iter=200, tol=1e-6):
        D = len(dims)
        N = int(np.prod(dims))
        with tempfile.TemporaryDirectory() as d:
            np.save(os.path.join(d, "E.npy"), np.asarray(E, dtype=np.float64).reshape(-1))
            np.save(os.path.join(d, "nu.npy"), np.asarray(nu, dtype=np.float64).reshape(-1))
            if eps0 is not None:
                np.save(os.path.join(d, "eps0.npy"), np.asarray(eps0, dtype=np.float64).reshape(N, D * D))
            if epsp is not None:
                np.save(os.path.join(d, "epsp.npy"), np.asarray(epsp, dtype=np.float64).reshape(N, D * D))
            eb = " ".join(repr(float(x)) for x in np.asarray(eps_bar, dtype=np.float64).reshape(-1))
            with open(os.path.join(d, "params.txt"), "w") as f:
                if D == 2:
                    f.write(f"{dims[0]} {dims[1]} {plane_mode} {pixel!r} {max_iter} {tol!r} {eb}\n")
                else:
                    f.write(f"{dims[0]} {dims[1]} {dims[2]} {pixel!r} {max_iter} {tol!r} {eb}\n")
            self._run(["ls2d" if D == 2 else "ls3d", d])
            eps = np.load(os.path.join(d, "out_eps.npy"))
            sig = np.load(os.path.join(d, "out_sig.npy"))
            mac = np.load(os.path.join(d, "out_macro.npy"))
        DD = D * D
        return eps, sig, mac[:DD], mac[DD:2 * DD], float(mac[2 * DD])

    def kmc(self, yaml_text: str, mode: str, nsteps: int = 1, maxev: Optional[int] = None, files=None):
        """mode: 'kmc_trace' | 'kmc_run' | 'kmc_init'.  Returns dict of arrays."""
        with tempfile.TemporaryDirectory() as d:
            for name, arr in (files or {}).items():
                np.save(os.path.join(d, name), arr)
            yaml_text = yaml_text.replace("$DIR", d)
            cfgp = os.path.join(d, "cfg.yaml")
            with open(cfgp, "w") as f:
                f.write(yaml_text)
            out = os.path.join(d, "out")
            os.makedirs(out)
            args = [mode, cfgp, out, nsteps]
            if maxev is not None:
                args.append(maxev)
            self._run(args)
            res = {}
            for fn in os.listdir(out):
                if fn.endswith(".npy"):
                    res[fn[:-4]] = np.load(os.path.join(out, fn))
            tp = os.path.join(out, "timing.txt")
            if os.path.exists(tp):
                res["timing"] = np.array([float(x) for x in open(tp).read().split()])
            sp = os.path.join(out, "summary_log.txt")
            if os.path.exists(sp):
                res["summary"] = open(sp).read()
        return res
