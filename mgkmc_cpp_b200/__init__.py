"""mgkmc_cpp_b200 -- B200-native STZ kinetic Monte Carlo + FFT Lippmann-Schwinger solver.

Python mirror of the reference's solver surface (mgkmc_cpp: kmc_solver.hpp,
linear_elastic_solver.hpp), backed by CUDA kernels for sm_100a in
libmgkmc_b200.so through its C ABI (include/mgkmc_b200.h):

* ``spectral_solver_2d`` / ``spectral_solver_3d`` -- same arguments and results
  as linear_elastic_solver.hpp:146-160 / :431-444 (``Gamma`` is accepted and
  ignored: the Green operator is evaluated on the device from ``pixel``);
  ``LsSolver`` keeps the fields resident for repeated solves.
* ``KmcSimulation2D`` / ``KmcSimulation3D`` -- constructor arguments of
  kmc_solver.hpp:165-182 / :1142-1158, ``run_simulation`` (:721-729),
  ``elastic_run`` and the public fields as numpy arrays.
* ``BarrierGenerator`` -- kmc_solver.hpp:24-33.

Tensors are numpy arrays of shape (N, D, D) in the reference's voxel order.
"""
from __future__ import annotations

import dataclasses
import os
import time
from typing import Dict, Optional, Tuple

import numpy as np

from . import _lib
from ._lib import MgkError

__all__ = ["BarrierGenerator", "LsSolver", "spectral_solver_2d", "spectral_solver_3d", "KmcSimulation2D",
           "KmcSimulation3D", "KmcBatch", "Server", "from_config", "linear_elastic_run", "run_config",
           "MgkError"]

_BAR = {"gaussian": 0, "rayleigh": 1, "modified_rayleigh": 2, "modified_rayleigh_with_exponential": 3}


@dataclasses.dataclass
class BarrierGenerator:
    type: str = "gaussian"
    mean: float = 2.0
    std_val: float = 0.6
    min_cutoff: float = 0.1
    max_cutoff: float = -1.0
    loc: float = 1.0
    scale: float = 0.5
    epsilon: float = 0.1
    ratio: float = 0.8


def _as_tensors(a, N: int, D: int) -> np.ndarray:
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float64)).reshape(N, D * D)
    return a


class LsSolver:
    """Device-resident Lippmann-Schwinger solver for one grid and modulus field."""

    def __init__(self, dims, E, nu, plane_mode: str = "plane_strain", pixel: float = 1.0, precision: str = "fp64"):
        """precision: "fp64" (the reference's arithmetic) or "fp32_refined" (FP32
        spectrum and FFTs to a relative change of 1e-6, then FP64 iterations)."""
        L = _lib.lib()
        _lib.require_device()
        self.dims = tuple(int(d) for d in dims)
        self.D = len(self.dims)
        if self.D not in (2, 3):
            raise ValueError("dims must have 2 or 3 entries")
        self.N = int(np.prod(self.dims))
        self._E = np.ascontiguousarray(E, dtype=np.float64).reshape(-1)
        self._nu = np.ascontiguousarray(nu, dtype=np.float64).reshape(-1)
        if self._E.size != self.N or self._nu.size != self.N:
            raise ValueError("E and nu need one value per voxel")
        h = _lib.C.c_void_p()
        nz = self.dims[2] if self.D == 3 else 1
        _lib.check(L.mgk_ls_create(_lib.C.byref(h), self.D, self.dims[0], self.dims[1], nz,
                                   1 if plane_mode == "plane_stress" else 0, float(pixel), _lib.dptr(self._E),
                                   _lib.dptr(self._nu)))
        self._h = h
        if precision not in ("fp64", "fp32_refined"):
            raise ValueError("precision must be 'fp64' or 'fp32_refined'")
        _lib.check(L.mgk_ls_set_precision(h, 1 if precision == "fp32_refined" else 0))

    def plan(self) -> dict:
        """The pass plan of this solver's launches (measured at creation)."""
        out = (_lib.C.c_int * 4)()
        _lib.check(_lib.lib().mgk_ls_plan(self._h, out))
        return {"rows_per_chunk": out[0], "cols_per_tile": out[1], "fft": "warp" if out[2] == 0 else "cta",
                "ctas": out[3]}

    def set_wait_limit(self, seconds: float):
        """Bound of every device-side barrier wait of the solver (0: 120 s)."""
        _lib.check(_lib.lib().mgk_ls_set_wait_limit(self._h, float(seconds)))

    def inject_absent_cta(self, cta: int):
        """Failure-detection tests: CTA ``cta`` of the next solves leaves before
        its first barrier (-1: off)."""
        _lib.check(_lib.lib().mgk_ls_inject_absent_cta(self._h, int(cta)))

    def last_solve_ms(self) -> float:
        """Device time of the last solve's kernels (no host copies)."""
        ms = np.zeros(1)
        _lib.check(_lib.lib().mgk_ls_last_solve_ms(self._h, _lib.dptr(ms)))
        return float(ms[0])

    def solve(self, eps_bar, eps=None, eps_plastic=None, max_iter: int = 200, tol: float = 1e-6):
        """Returns (eps, sig, eps_macro, sig_macro, iterations); ``eps`` given = warm start."""
        D, N = self.D, self.N
        eb = np.ascontiguousarray(eps_bar, dtype=np.float64).reshape(D * D)
        warm = eps is not None and np.asarray(eps).size == N * D * D
        e = _as_tensors(eps, N, D).copy() if warm else np.zeros((N, D * D))
        ep = _as_tensors(eps_plastic, N, D) if eps_plastic is not None and np.asarray(eps_plastic).size else None
        sig = np.zeros((N, D * D))
        mac = np.zeros(2 * D * D)
        it = _lib.C.c_int(0)
        _lib.check(_lib.lib().mgk_ls_solve(self._h, _lib.dptr(eb), _lib.dptr(ep), _lib.dptr(e), int(warm), _lib.dptr(sig),
                                           _lib.dptr(mac), int(max_iter), float(tol), _lib.C.byref(it)), allow=(1,))
        return (e.reshape(N, D, D), sig.reshape(N, D, D), mac[:D * D].reshape(D, D), mac[D * D:].reshape(D, D), it.value)

    def close(self):
        if getattr(self, "_h", None):
            _lib.lib().mgk_ls_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def spectral_solver_2d(nx, ny, E, nu, eps_bar, plane_mode="plane_strain", Gamma=None, eps=None, max_iter=200, tol=1e-6,
                       verbose=False, eps_plastic=None, pixel=1.0):
    """linear_elastic_solver.hpp:146-309.  Returns (eps, sig, eps_macro, sig_macro)."""
    s = LsSolver((nx, ny), E, nu, plane_mode, pixel)
    try:
        e, sg, em, sm, _ = s.solve(eps_bar, eps, eps_plastic, max_iter, tol)
    finally:
        s.close()
    return e, sg, em, sm


def spectral_solver_3d(nx, ny, nz, E, nu, eps_bar, Gamma=None, eps=None, max_iter=200, tol=1e-6, verbose=False,
                       eps_plastic=None, pixel=1.0):
    """linear_elastic_solver.hpp:431-593.  Returns (eps, sig, eps_macro, sig_macro)."""
    s = LsSolver((nx, ny, nz), E, nu, "plane_strain", pixel)
    try:
        e, sg, em, sm, _ = s.solve(eps_bar, eps, eps_plastic, max_iter, tol)
    finally:
        s.close()
    return e, sg, em, sm


_FIELDS = {"eps_field": 0, "sig_field": 1, "eps_plastic": 2, "soft_prop": 3, "last_event_time": 4, "Q": 5, "Q0": 6,
           "catalog": 7, "prev_strain_dir": 8, "E_field": 9, "nu_field": 10}


class _KmcBase:
    D = 2

    def _create(self, nx, ny, nz, M, gamma0, E_field, nu_field, pixel, barrier_gen, softening_scheme, softening_cap, jp,
                jt, neighbor_softening_fraction, q_act_temp, output_dir, temperature, strain_rate, stability_threshold,
                nu0, plane_mode, fast_patching_enabled, patch_radius, sync_interval, instability_mode, cascade_timing,
                scale_rate_by_volume, redraw_directions, redraw_barriers, use_3d_barriers, seed, ls_tol, ls_max_iter,
                catalog_type="random", barrier_per_voxel=False, ls_precision="fp64"):
        L = _lib.lib()
        _lib.require_device()
        self.nx, self.ny, self.nz, self.M = nx, ny, nz, M
        self.N = nx * ny * nz
        self.output_dir = output_dir
        bg = barrier_gen or BarrierGenerator()
        if bg.type not in _BAR:
            raise ValueError("unknown barrier type %r" % bg.type)
        p = _lib.KmcParamsC()
        p.dim, p.nx, p.ny, p.nz, p.M = self.D, nx, ny, nz, M
        p.plane_stress = 1 if plane_mode == "plane_stress" else 0
        p.seed, p.gamma0, p.pixel = int(seed), float(gamma0), float(pixel)
        p.barrier_type = _BAR[bg.type]
        p.bar_mean, p.bar_std, p.bar_min_cutoff, p.bar_max_cutoff = bg.mean, bg.std_val, bg.min_cutoff, bg.max_cutoff
        p.bar_loc, p.bar_scale, p.bar_epsilon, p.bar_ratio = bg.loc, bg.scale, bg.epsilon, bg.ratio
        p.directional = 1 if softening_scheme == "directional" else 0
        p.softening_cap, p.jp, p.jt = softening_cap, jp, jt
        p.neighbor_fraction, p.q_act_temp = neighbor_softening_fraction, q_act_temp
        p.temperature, p.strain_rate, p.stability_threshold, p.nu0 = temperature, strain_rate, stability_threshold, nu0
        p.instability_kmc = 1 if instability_mode == "kmc" else 0
        p.scale_rate_by_volume = int(bool(scale_rate_by_volume))
        p.redraw_directions, p.redraw_barriers = int(bool(redraw_directions)), int(bool(redraw_barriers))
        p.use_3d_barriers = int(bool(use_3d_barriers))
        p.fast_patching, p.patch_radius, p.sync_interval = int(bool(fast_patching_enabled)), patch_radius, sync_interval
        p.ls_tol, p.ls_max_iter = float(ls_tol), int(ls_max_iter)
        if catalog_type not in ("random", "even", "fibonacci") or ls_precision not in ("fp64", "fp32_refined"):
            raise ValueError("catalog_type: random | even | fibonacci; ls_precision: fp64 | fp32_refined")
        p.catalog_type = {"random": 0, "even": 1, "fibonacci": 2}[catalog_type]
        p.barrier_per_voxel = int(bool(barrier_per_voxel))
        p.ls_precision = 1 if ls_precision == "fp32_refined" else 0
        self._params = p
        E = np.ascontiguousarray(E_field, dtype=np.float64).reshape(-1)
        nu = np.ascontiguousarray(nu_field, dtype=np.float64).reshape(-1)
        if E.size != self.N or nu.size != self.N:
            raise ValueError("E_field and nu_field need one value per voxel")
        h = _lib.C.c_void_p()
        _lib.check(L.mgk_kmc_create(_lib.C.byref(h), _lib.C.byref(p), _lib.dptr(E), _lib.dptr(nu)))
        self._h = h

    def run_simulation(self, n_global_steps, step_size, component, stress_targets: Dict[Tuple[int, int], float],
                       mixed_tol=1e-4, mixed_max_iter=50, checkpoint_interval="none", checkpoint_path="checkpoint",
                       vtk_interval="none", vtk_elastic_only=True, track_cascades=False, enable_console_log=True,
                       summary_filename="summary_log.txt", enable_summary_log=True, enable_global_log=True,
                       max_kmc_steps_pct=0.3, max_events=0, trace=False, trace_cap=1 << 20, max_cascade_batches=0):
        """kmc_solver.hpp:721-1037.  Returns the event trace (rows of
        [kind, a, b, total_rate, t_wait, time, eps_macro, sig_macro]) when
        ``trace`` is true, else None.  Raises MgkError on failure; the
        instability-limit stop (MGK_TERMINATED) returns normally."""
        rp = _lib.RunParamsC()
        rp.n_global_steps, rp.step_size = int(n_global_steps), float(step_size)
        rp.comp_i, rp.comp_j = int(component[0]), int(component[1])
        tg = sorted(stress_targets.items())
        rp.n_targets = len(tg)
        for k, ((i, j), v) in enumerate(tg):
            rp.target_i[k], rp.target_j[k], rp.target_v[k] = i, j, v
        rp.mixed_tol, rp.mixed_max_iter, rp.max_kmc_steps_pct = mixed_tol, int(mixed_max_iter), max_kmc_steps_pct
        rp.max_events = int(max_events or 0)
        rp.max_cascade_batches = int(max_cascade_batches or 0)
        out = self.output_dir if (enable_summary_log or enable_global_log or vtk_interval != "none") else None
        if out:
            os.makedirs(out, exist_ok=True)
        rp.output_dir = out.encode() if out else None
        rp.summary_filename = summary_filename.encode()
        rp.enable_summary_log, rp.enable_global_log = int(bool(enable_summary_log)), int(bool(enable_global_log))
        rp.enable_console, rp.vtk_interval, rp.vtk_elastic_only = int(bool(enable_console_log)), vtk_interval.encode(), int(vtk_elastic_only)
        w = 6 + 2 * self.D * self.D
        buf = np.zeros((trace_cap, w)) if trace else None
        rows = _lib.C.c_longlong(0)
        self.last_status = _lib.check(_lib.lib().mgk_kmc_run(self._h, _lib.C.byref(rp), _lib.dptr(buf),
                                                             trace_cap if trace else 0, _lib.C.byref(rows)), allow=(8,))
        if trace:
            return buf[:min(rows.value, trace_cap)].copy()
        return None

    def elastic_run(self):
        _lib.check(_lib.lib().mgk_kmc_elastic_run(self._h))

    def _field(self, name):
        f = _FIELDS[name]
        n = _lib.C.c_longlong(0)
        _lib.check(_lib.lib().mgk_kmc_get_field(self._h, f, None, _lib.C.byref(n)))
        out = np.zeros(n.value)
        _lib.check(_lib.lib().mgk_kmc_get_field(self._h, f, _lib.dptr(out), None))
        D = self.D
        if name in ("eps_field", "sig_field", "eps_plastic", "prev_strain_dir", "catalog"):
            return out.reshape(-1, D, D)
        if name == "soft_prop":
            return out.reshape(-1, 2)
        return out

    def __getattr__(self, name):
        if name in _FIELDS:
            return self._field(name)
        raise AttributeError(name)

    def macro(self) -> np.ndarray:
        out = np.zeros(2 * self.D * self.D + 10)
        _lib.check(_lib.lib().mgk_kmc_get_macro(self._h, _lib.dptr(out), out.size))
        return out

    @property
    def eps_macro(self):
        return self.macro()[:self.D * self.D].reshape(self.D, self.D)

    @property
    def sig_macro(self):
        DD = self.D * self.D
        return self.macro()[DD:2 * DD].reshape(self.D, self.D)

    @property
    def time(self):
        return float(self.macro()[2 * self.D * self.D])

    @property
    def stats(self) -> dict:
        m = self.macro()[2 * self.D * self.D + 1:]
        keys = ["thermal_events", "cascades", "ls_solves", "ls_iters", "elastic_steps", "min_margin", "syncs", "launches"]
        return {k: float(v) for k, v in zip(keys, m)}

    def set_profiling(self, on: bool = True):
        _lib.check(_lib.lib().mgk_kmc_set_profiling(self._h, int(bool(on))))

    def profile(self, max_latencies: int = 1 << 20) -> dict:
        out = np.zeros(10)
        lat = np.zeros(max_latencies)
        _lib.check(_lib.lib().mgk_kmc_get_profile(self._h, _lib.dptr(out), _lib.dptr(lat), max_latencies))
        keys = ["ls_ms", "ls_launches", "ls_iterations", "sweep_ms", "sweeps", "select_ms", "selects", "run_ms",
                "events_timed"]
        d = {k: float(v) for k, v in zip(keys, out)}
        d["event_us"] = lat[:int(min(out[8], max_latencies))].copy()
        return d

    def close(self):
        if getattr(self, "_h", None):
            _lib.lib().mgk_kmc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class KmcSimulation2D(_KmcBase):
    """kmc_solver.hpp:98-1038."""
    D = 2

    def __init__(self, nx, ny, M, gamma0, E_field, nu_field, pixel=1.0, barrier_gen=None, softening_scheme="isotropic",
                 softening_cap=2.0, jp=10.0, jt=30.0, neighbor_softening_fraction=0.0, q_act_temp=0.37,
                 output_dir="output", temperature=0.0, strain_rate=1.0, stability_threshold=0.0, nu0=1e13,
                 plane_mode="plane_strain", fast_patching_enabled=False, patch_radius=5, sync_interval=100,
                 instability_mode="cascade", cascade_timing="none", scale_rate_by_volume=True, redraw_directions=True,
                 redraw_barriers=True, seed=42, ls_tol=1e-6, ls_max_iter=200, **ext):
        """The reference constructor's arguments; ``ext`` takes the extensions
        with no counterpart in the reference: catalog_type ("random" |
        "even"), barrier_per_voxel, ls_precision ("fp64" | "fp32_refined")."""
        self._create(nx, ny, 1, M, gamma0, E_field, nu_field, pixel, barrier_gen, softening_scheme, softening_cap, jp, jt,
                     neighbor_softening_fraction, q_act_temp, output_dir, temperature, strain_rate, stability_threshold,
                     nu0, plane_mode, fast_patching_enabled, patch_radius, sync_interval, instability_mode,
                     cascade_timing, scale_rate_by_volume, redraw_directions, redraw_barriers, False, seed, ls_tol,
                     ls_max_iter, **ext)


class KmcSimulation3D(_KmcBase):
    """kmc_solver.hpp:1040-2063."""
    D = 3

    def __init__(self, nx, ny, nz, M, gamma0, E_field, nu_field, pixel=1.0, barrier_gen=None,
                 softening_scheme="isotropic", softening_cap=2.0, jp=10.0, jt=30.0, neighbor_softening_fraction=0.0,
                 q_act_temp=0.37, output_dir="output", temperature=0.0, strain_rate=1.0, stability_threshold=0.0,
                 nu0=1e13, fast_patching_enabled=False, patch_radius=5, sync_interval=100, instability_mode="cascade",
                 cascade_timing="none", scale_rate_by_volume=True, redraw_directions=True, redraw_barriers=True,
                 use_3d_barriers=False, seed=42, ls_tol=1e-6, ls_max_iter=200, **ext):
        """The reference constructor's arguments; ``ext`` takes the extensions
        with no counterpart in the reference: catalog_type ("random" | "even"
        | "fibonacci"), barrier_per_voxel, ls_precision ("fp64" |
        "fp32_refined")."""
        self._create(nx, ny, nz, M, gamma0, E_field, nu_field, pixel, barrier_gen, softening_scheme, softening_cap, jp,
                     jt, neighbor_softening_fraction, q_act_temp, output_dir, temperature, strain_rate,
                     stability_threshold, nu0, "plane_strain", fast_patching_enabled, patch_radius, sync_interval,
                     instability_mode, cascade_timing, scale_rate_by_volume, redraw_directions, redraw_barriers,
                     use_3d_barriers, seed, ls_tol, ls_max_iter, **ext)


def from_config(cfg, output_dir: Optional[str] = None):
    """Construct the simulation main.cpp:379-403 would build from a SimConfig."""
    b = cfg.barrier
    bg = BarrierGenerator(b.type, b.mean, b.std, b.min_cutoff, b.max_cutoff, b.loc, b.scale, b.epsilon, b.ratio)
    kw = dict(pixel=cfg.pixel, barrier_gen=bg, softening_scheme=cfg.softening_scheme, softening_cap=cfg.softening_cap,
              jp=cfg.jp, jt=cfg.jt, neighbor_softening_fraction=cfg.neighbor_softening_fraction,
              q_act_temp=cfg.q_act_temp, output_dir=output_dir or cfg.output_directory, temperature=cfg.temperature,
              strain_rate=cfg.strain_rate, stability_threshold=cfg.stability_threshold, nu0=cfg.nu0,
              fast_patching_enabled=cfg.fast_patching, patch_radius=cfg.patch_radius,
              sync_interval=cfg.sync_interval, instability_mode=cfg.instability_mode,
              cascade_timing=cfg.cascade_timing, scale_rate_by_volume=cfg.scale_rate_by_volume,
              redraw_directions=cfg.redraw_directions, redraw_barriers=cfg.redraw_barriers, seed=cfg.seed,
              ls_tol=cfg.ls_tol, ls_max_iter=cfg.ls_max_iter, catalog_type=cfg.catalog_type,
              barrier_per_voxel=cfg.barrier_per_voxel, ls_precision=cfg.ls_precision)
    if cfg.dim == 3:
        sim = KmcSimulation3D(cfg.nx, cfg.ny, cfg.nz, cfg.M, cfg.gamma0, cfg.E, cfg.nu,
                              use_3d_barriers=cfg.use_3d_barriers, **kw)
    else:
        sim = KmcSimulation2D(cfg.nx, cfg.ny, cfg.M, cfg.gamma0, cfg.E, cfg.nu, plane_mode=cfg.plane_mode, **kw)
    sim._cfg = cfg
    return sim


def linear_elastic_run(cfg, output_dir: Optional[str] = None, write_files: bool = True, max_iter_macro: int = 20,
                       max_iter_ls: int = 200, tol_ls: float = 1e-6):
    """simulation_type "linear_elastic" of main.cpp:418-869 on the GPU: the
    proportional-loading schedule with the mixed stress/strain loop, its logs
    and VTU files (in output_dir, default the config's output.directory).
    Returns (eps_macro, sig_macro, ls_iterations): arrays of shape
    (n_steps + 1, D, D)."""
    L = _lib.lib()
    _lib.require_device()
    D = cfg.dim
    p = _lib.LeParamsC()
    p.dim, p.nx, p.ny, p.nz = D, cfg.nx, cfg.ny, cfg.nz if D == 3 else 1
    p.plane_stress = 1 if cfg.plane_mode == "plane_stress" else 0
    p.pixel, p.eps_target, p.step_size = float(cfg.pixel), float(cfg.eps_target), float(cfg.step_size)
    p.drive_i, p.drive_j = cfg.driving
    tg = sorted(cfg.targets.items())
    p.n_targets = len(tg)
    for k, ((i, j), v) in enumerate(tg):
        p.target_i[k], p.target_j[k], p.target_v[k] = i, j, v
    p.mixed_tol = float(cfg.mixed_tol_pa)
    p.max_iter_macro, p.max_iter_ls, p.tol_ls = int(max_iter_macro), int(max_iter_ls), float(tol_ls)
    out = output_dir or cfg.output_directory
    if write_files:
        os.makedirs(out, exist_ok=True)
        p.output_dir = out.encode()
    else:
        p.output_dir = None
    p.summary_filename = cfg.summary_filename.encode()
    p.enable_summary_log, p.enable_global_log = int(cfg.enable_summary_log), int(cfg.enable_global_log)
    p.enable_console = int(cfg.enable_console)
    p.vtk_interval = str(cfg.vtk_interval).encode()
    n_steps = cfg.n_steps
    E = np.ascontiguousarray(cfg.E, dtype=np.float64).reshape(-1)
    nu = np.ascontiguousarray(cfg.nu, dtype=np.float64).reshape(-1)
    mac = np.zeros((n_steps + 1) * 2 * D * D)
    it = _lib.C.c_int(0)
    _lib.check(L.mgk_le_run(_lib.C.byref(p), _lib.dptr(E), _lib.dptr(nu), _lib.dptr(mac), _lib.C.byref(it)))
    mac = mac.reshape(n_steps + 1, 2, D, D)
    return mac[:, 0], mac[:, 1], int(it.value)


def run_config(path_or_cfg, output_dir: Optional[str] = None):
    """What the reference executable does with a config file (main.cpp:25-416):
    a KMC run (run_simulation with the config's schedule) or the
    linear-elastic simulation."""
    from .config import SimConfig
    cfg = path_or_cfg if not isinstance(path_or_cfg, str) else SimConfig.from_yaml(path_or_cfg)
    out = output_dir or cfg.output_directory
    os.makedirs(out, exist_ok=True)
    if cfg.simulation_type == "linear_elastic":
        return linear_elastic_run(cfg, out)
    sim = from_config(cfg, output_dir=out)
    sim.run_simulation(cfg.n_steps, cfg.step_size, cfg.driving, cfg.targets, cfg.mixed_tol_pa, 50,
                       enable_console_log=cfg.enable_console, summary_filename=cfg.summary_filename,
                       enable_summary_log=cfg.enable_summary_log, enable_global_log=cfg.enable_global_log,
                       vtk_interval=cfg.vtk_interval, vtk_elastic_only=cfg.vtk_elastic_only,
                       max_kmc_steps_pct=cfg.max_kmc_steps_pct)
    return sim


def correlated_field_gpu(shape, mean: float, std: float, corr: float, seed: int, clip_min=None, clip_max=None):
    """generate_correlated_field_cpp (material_generator.hpp:130-258) on the
    GPU; same arguments as fields.correlated_field."""
    shape = tuple(int(s) for s in shape)
    dim = len(shape)
    nx, ny = shape[0], shape[1]
    nz = shape[2] if dim == 3 else 1
    out = np.zeros(int(np.prod(shape)))
    _lib.check(_lib.lib().mgk_correlated_field(dim, nx, ny, nz, float(mean), float(std), float(corr),
                                               int(clip_min is not None), float(clip_min or 0.0),
                                               int(clip_max is not None), float(clip_max or 0.0), int(seed),
                                               _lib.dptr(out)))
    return out.reshape(shape)


def device_memory():
    """(free, total) bytes of the current device."""
    f, t = _lib.C.c_ulonglong(0), _lib.C.c_ulonglong(0)
    _lib.check(_lib.lib().mgk_device_memory(_lib.C.byref(f), _lib.C.byref(t)))
    return int(f.value), int(t.value)


def job_device_bytes(cfg) -> int:
    """Device memory of one simulation: per mode Q0, Q and the catalog; per
    voxel the strain, plastic strain, stress inputs, spectrum, softening and
    KMC bookkeeping (FP64)."""
    D = cfg.dim
    S = 3 if D == 2 else 6
    C = 6 if (D == 3 and cfg.use_3d_barriers) else 2
    N = cfg.n_voxels
    return int(N * cfg.M * 8 * (2 + C) + N * 8 * (4 * S + 2 + 2 + 2 * S + 2 + 1 + C) + (64 << 10))


def _shape_key(cfg):
    return (cfg.dim, cfg.nx, cfg.ny, cfg.nz if cfg.dim == 3 else 1, cfg.plane_mode)


def current_device() -> int:
    """The calling thread's CUDA device (mgk_get_device)."""
    d = _lib.C.c_int(0)
    _lib.check(_lib.lib().mgk_get_device(_lib.C.byref(d)))
    return d.value


def _build_on(device: int, cfg):
    # a pool thread starts on device 0: adopt the submitting thread's device
    _lib.check(_lib.lib().mgk_set_device(int(device)))
    return from_config(cfg, output_dir=None)


class Server:
    """Continuous batching of KMC jobs on one GPU (the serving loop).

    ``submit(cfg, flips)`` queues a job (a simulation that must reach
    ``flips`` thermal events).  Each ``step()`` admits queued jobs, in
    arrival order, while the active set is below ``max_active`` and the job's
    device memory (``job_device_bytes``) fits: the active jobs' memory plus
    the new job's stays within ``hbm_budget`` (default: the device's free
    memory when the server starts, less ``reserve_bytes``), and the device
    has that much free right now.  Admitted jobs keep their fields and random
    stream resident on the device.  The step then advances every active job
    in one batched launch for ``slice_seconds`` of device time (or by
    ``slice_events`` events each, when given) and retires the jobs that
    reached their target (or made no progress for ``stall_seconds``).  A job's trajectory does not depend on
    what shares its launches: its random stream and interval clock are its
    own.

    With ``build_threads`` > 0 an admitted job's simulation is built on a
    thread pool while the active jobs keep running (its initial catalog and
    barriers are drawn on the host from the reference's sequential random
    stream: seconds for a large 3D grid); it joins the batch at the first
    step after its build finished.  Its memory counts against the budget from
    admission."""

    def __init__(self, max_active=64, slice_events=None, slice_seconds=0.05, reserve_bytes=8 << 30, hbm_budget=None,
                 stall_seconds=30.0, build_threads=0):
        self.max_active, self.reserve = int(max_active), int(reserve_bytes)
        self.slice_events = None if slice_events is None else int(slice_events)
        self.slice_seconds = float(slice_seconds)
        self.budget = int(hbm_budget) if hbm_budget is not None else device_memory()[0] - self.reserve
        self.committed = 0
        self.stall_seconds = float(stall_seconds)
        self._batch, self._batch_ids = None, None
        self.queue, self.active, self.done = [], [], {}
        self.building = []  # admitted jobs whose simulation is being built
        self._shapes = set()  # grid shapes built so far
        self.built_on_pool = 0
        self._pool = None
        if int(build_threads) > 0:
            from concurrent.futures import ThreadPoolExecutor
            self._pool = ThreadPoolExecutor(int(build_threads), thread_name_prefix="mgk-build")
        self._next = 0
        self.launches = 0
        self.step_latency_us = []
        self.host_seconds = {"build_wait": 0.0, "rebuild": 0.0, "readback": 0.0, "retire": 0.0}

    def submit(self, cfg, flips: int, arrival: float = 0.0) -> int:
        jid = self._next
        self._next += 1
        self.queue.append({"id": jid, "cfg": cfg, "target": int(flips), "events": 0, "selected": [],
                           "arrival": float(arrival), "admitted": None, "finished": None, "latency_us": [],
                           "idle_s": 0.0, "stalled": False})
        return jid

    def _admit(self, now: float):
        while (self.queue and len(self.active) + len(self.building) < self.max_active
               and self.queue[0]["arrival"] <= now):
            job = self.queue[0]
            need = job_device_bytes(job["cfg"])
            # the device check also covers builds still allocating
            if self.committed + need > self.budget or need > device_memory()[0] - self._building_bytes():
                break
            self.queue.pop(0)
            job["bytes"] = need
            self.committed += need
            job["admitted"] = now
            shape = _shape_key(job["cfg"])
            if self._pool is None or shape not in self._shapes:
                # the first job of a grid shape is built between launches: its
                # LS solver measures pass plans (LsSolver::tune, cached per
                # shape), which needs the GPU to itself
                job["sim"] = from_config(job["cfg"], output_dir=None)
                self._shapes.add(shape)
                self.active.append(job)
            else:
                job["build"] = self._pool.submit(_build_on, current_device(), job["cfg"])
                self.building.append(job)
                self.built_on_pool += 1

    def _building_bytes(self) -> int:
        return sum(j["bytes"] for j in self.building)

    def _join_built(self):
        """Moves finished builds to the active set (in admission order); when
        nothing is active, waits for the first build instead of idling."""
        if not self.building:
            return
        if not self.active:
            t0 = time.perf_counter()
            self.building[0]["build"].result()
            self.host_seconds["build_wait"] += time.perf_counter() - t0
        keep = []
        for job in self.building:
            if job["build"].done():
                job["sim"] = job.pop("build").result()  # a failed build raises here
                self.active.append(job)
            else:
                keep.append(job)
        self.building = keep

    def step(self, now: float = 0.0) -> float:
        """One slice; returns the launch's device milliseconds (0 if idle)."""
        self._admit(now)
        self._join_built()
        if not self.active:
            return 0.0
        ids = [j["id"] for j in self.active]
        if ids != self._batch_ids:  # the active set changed: a new batch (CTA plan) over the resident jobs
            t0 = time.perf_counter()
            if self._batch is not None:
                self._batch.close()
            self._batch = KmcBatch(sims=[j["sim"] for j in self.active])
            self._batch.cfgs = [j["cfg"] for j in self.active]
            self._batch_ids = ids
            self.host_seconds["rebuild"] += time.perf_counter() - t0
        b = self._batch
        # a slice is a device-time budget (every job stops at its first
        # decision past it, so a large job never holds the small ones back),
        # or a fixed number of events per job when slice_events is set
        if self.slice_events is None:
            b.set_time_limit(self.slice_seconds)
            budgets = [j["target"] - j["events"] for j in self.active]
        else:
            b.set_time_limit(60.0)
            budgets = [min(self.slice_events, j["target"] - j["events"]) for j in self.active]
        t0 = time.perf_counter()
        ms = b.run(max(budgets), budgets=budgets)
        self.host_seconds["readback"] += max(0.0, time.perf_counter() - t0 - ms / 1e3)
        self.launches += 1
        t0 = time.perf_counter()
        keep = []
        for r, job in enumerate(self.active):
            st = b.stats(r)
            job["events"] += int(st["events"])
            job["selected"].append(st["selected"])
            job["latency_us"].extend(st["event_us"].tolist())
            self.step_latency_us.extend(st["event_us"].tolist())
            # a job without a thermal event for stall_seconds of device time
            # (an avalanche whose cascade batches never settle -- the
            # reference would run it forever) is retired as stalled
            job["idle_s"] = job["idle_s"] + ms / 1e3 if st["events"] == 0 else 0.0
            job["stalled"] = job["idle_s"] >= self.stall_seconds
            if job["events"] >= job["target"] or st["terminated"] == 1 or job["stalled"]:
                job["finished"] = now
                job["selected"] = np.concatenate(job["selected"]) if job["selected"] else np.zeros(0, np.int64)
                job["eps_field"] = job["sim"].eps_field
                job["macro"] = job["sim"].macro()
                job["sim"].close()
                del job["sim"]
                self.committed -= job["bytes"]
                self.done[job["id"]] = job
            else:
                keep.append(job)
        if len(keep) != len(self.active):
            b.close()
            self._batch, self._batch_ids = None, None
        self.active = keep
        self.host_seconds["retire"] += time.perf_counter() - t0
        return ms

    def idle(self) -> bool:
        return not self.queue and not self.active and not self.building

    def close(self):
        """Waits for builds in flight and releases the batch and the pool (the
        simulations of unfinished jobs are closed)."""
        if self._pool is not None:
            self._pool.shutdown(wait=True)
            self._pool = None
        for job in self.building:
            job["sim"] = job.pop("build").result()
            self.active.append(job)
        self.building = []
        if self._batch is not None:
            self._batch.close()
            self._batch, self._batch_ids = None, None
        for job in self.active:
            if "sim" in job:
                job["sim"].close()
                del job["sim"]


def kmc_params_from_config(cfg) -> "_lib.KmcParamsC":
    """mgk_kmc_params for a SimConfig (the values main.cpp:278-317 passes)."""
    b = cfg.barrier
    if b.type not in _BAR:
        raise ValueError("unknown barrier type %r" % b.type)
    p = _lib.KmcParamsC()
    p.dim, p.nx, p.ny, p.nz, p.M = cfg.dim, cfg.nx, cfg.ny, cfg.nz if cfg.dim == 3 else 1, cfg.M
    p.plane_stress = 1 if cfg.plane_mode == "plane_stress" else 0
    p.seed, p.gamma0, p.pixel = int(cfg.seed), float(cfg.gamma0), float(cfg.pixel)
    p.barrier_type = _BAR[b.type]
    p.bar_mean, p.bar_std, p.bar_min_cutoff, p.bar_max_cutoff = b.mean, b.std, b.min_cutoff, b.max_cutoff
    p.bar_loc, p.bar_scale, p.bar_epsilon, p.bar_ratio = b.loc, b.scale, b.epsilon, b.ratio
    p.directional = 1 if cfg.softening_scheme == "directional" else 0
    p.softening_cap, p.jp, p.jt = cfg.softening_cap, cfg.jp, cfg.jt
    p.neighbor_fraction, p.q_act_temp = cfg.neighbor_softening_fraction, cfg.q_act_temp
    p.temperature, p.strain_rate, p.stability_threshold, p.nu0 = (cfg.temperature, cfg.strain_rate,
                                                                   cfg.stability_threshold, cfg.nu0)
    p.instability_kmc = 1 if cfg.instability_mode == "kmc" else 0
    p.scale_rate_by_volume = int(bool(cfg.scale_rate_by_volume))
    p.redraw_directions, p.redraw_barriers = int(bool(cfg.redraw_directions)), int(bool(cfg.redraw_barriers))
    p.use_3d_barriers = int(bool(cfg.use_3d_barriers))
    p.fast_patching, p.patch_radius, p.sync_interval = int(bool(cfg.fast_patching)), cfg.patch_radius, cfg.sync_interval
    p.ls_tol, p.ls_max_iter = float(cfg.ls_tol), int(cfg.ls_max_iter)
    p.catalog_type = {"random": 0, "even": 1, "fibonacci": 2}[cfg.catalog_type]
    p.barrier_per_voxel = int(cfg.barrier_per_voxel)
    p.ls_precision = 1 if cfg.ls_precision == "fp32_refined" else 0
    return p


def run_params_from_config(cfg, n_global_steps=None, max_cascade_batches=0) -> "_lib.RunParamsC":
    rp = _lib.RunParamsC()
    rp.n_global_steps = int(cfg.n_steps if n_global_steps is None else n_global_steps)
    rp.step_size = float(cfg.step_size)
    rp.comp_i, rp.comp_j = cfg.driving
    tg = sorted(cfg.targets.items())
    rp.n_targets = len(tg)
    for k, ((i, j), v) in enumerate(tg):
        rp.target_i[k], rp.target_j[k], rp.target_v[k] = i, j, v
    rp.mixed_tol, rp.mixed_max_iter, rp.max_kmc_steps_pct = cfg.mixed_tol_pa, 50, cfg.max_kmc_steps_pct
    rp.max_events = 0
    rp.output_dir = None
    rp.summary_filename = b"summary_log.txt"
    rp.vtk_interval = b"none"
    rp.vtk_elastic_only = 1
    rp.max_cascade_batches = int(max_cascade_batches)
    return rp


def set_batch_plan(objective: str):
    """How batches built from now on spread their CTAs: "throughput" (default)
    or "balanced" (see mgk_set_batch_plan)."""
    _lib.check(_lib.lib().mgk_set_batch_plan({"throughput": 0, "balanced": 1}[objective]))


class KmcBatch:
    """Replicas advanced together by one device-resident kernel (mgk_batch_*):
    no host round trip per event; the reference's random stream continued on
    the device.  ``configs`` is a list of SimConfig."""

    def __init__(self, configs=None, sims=None):
        """``configs``: SimConfigs, one new simulation each (owned).  ``sims``:
        existing simulations (KmcSimulation2D/3D from ``from_config``) to
        advance in place; they keep their state after the batch is gone."""
        L = _lib.lib()
        _lib.require_device()
        if sims is not None:
            self.sims = list(sims)
            self.cfgs = [getattr(x, "_cfg", None) for x in self.sims]
            n = len(self.sims)
            hs = (_lib.C.c_void_p * n)(*[x._h.value for x in self.sims])
            h = _lib.C.c_void_p()
            _lib.check(L.mgk_batch_create_from(_lib.C.byref(h), n, hs))
            self._h = h
            return
        self.sims = None
        self.cfgs = list(configs)
        n = len(self.cfgs)
        self._params = (_lib.KmcParamsC * n)(*[kmc_params_from_config(c) for c in self.cfgs])
        self._E = [np.ascontiguousarray(c.E, dtype=np.float64).reshape(-1) for c in self.cfgs]
        self._nu = [np.ascontiguousarray(c.nu, dtype=np.float64).reshape(-1) for c in self.cfgs]
        dp = _lib.C.POINTER(_lib.C.c_double)
        Ep = (dp * n)(*[_lib.dptr(a) for a in self._E])
        np_ = (dp * n)(*[_lib.dptr(a) for a in self._nu])
        h = _lib.C.c_void_p()
        _lib.check(L.mgk_batch_create(_lib.C.byref(h), n, self._params, Ep, np_))
        self._h = h

    def set_time_limit(self, seconds: float):
        """Wall-time bound of one run call (default 60 s): once every replica
        has run past it (or finished), each stops at its next decision."""
        _lib.check(_lib.lib().mgk_batch_set_time_limit(self._h, float(seconds)))

    def run(self, max_events: int, n_global_steps=10 ** 6, max_cascade_batches=0, budgets=None) -> float:
        """Advance every replica by up to max_events thermal events (budgets:
        one count per replica instead); returns
        the kernel time in milliseconds.  A run that reaches the time limit
        returns normally with ``self.time_limited`` set."""
        n = len(self.cfgs)
        key = (int(n_global_steps), int(max_cascade_batches), tuple(id(c) for c in self.cfgs))
        cache = getattr(self, "_rps", None)
        if cache is None or cache[0] != key:  # the run parameters, built once per batch and kind of call
            rps = (_lib.RunParamsC * n)(*[run_params_from_config(c, n_global_steps, max_cascade_batches)
                                          for c in self.cfgs])
            self._rps = (key, rps)
        rps = self._rps[1]
        for r in range(n):
            rps[r].max_events = int(budgets[r]) if budgets is not None else 0
        ms = np.zeros(1)
        st = _lib.lib().mgk_batch_run(self._h, rps, int(max_events), _lib.dptr(ms))
        self.time_limited = st == 9
        if st not in (0, 9):
            _lib.check(st)
        return float(ms[0])

    def stats(self, r: int) -> dict:
        L = _lib.lib()
        out = np.zeros(19)
        ln = _lib.C.c_longlong(0)
        _lib.check(L.mgk_batch_stats(self._h, r, _lib.dptr(out), None, 0, _lib.C.byref(ln)))  # counters, log length
        keys = ["events", "cascades", "cascade_flips", "ls_solves", "ls_iters", "elastic_steps", "fallbacks",
                "min_margin", "terminated", "ctas", "ms_sweep", "ms_decide", "ms_event_solve", "ms_cascade_flips",
                "ms_cascade_solve", "ms_interval_end", "sweeps", "h2d_bytes", "d2h_bytes"]
        d = {k: float(v) for k, v in zip(keys, out)}
        n = ln.value
        if n:
            sel = np.empty(n, dtype=np.int32)
            _lib.check(L.mgk_batch_stats(self._h, r, _lib.dptr(out), sel.ctypes.data_as(_lib.C.POINTER(_lib.C.c_int)),
                                         n, _lib.C.byref(ln)))
            d["selected"] = sel.astype(np.int64)
        else:
            d["selected"] = np.zeros(0, dtype=np.int64)
        # one event time per logged thermal event (the same count as the log)
        cap = min(int(d["events"]), 1 << 16)
        us = np.empty(cap)
        _lib.check(L.mgk_batch_event_times(self._h, r, _lib.dptr(us) if cap else None, cap, _lib.C.byref(ln)))
        d["event_us"] = us[:min(ln.value, cap)]
        return d

    def field(self, r: int, name: str) -> np.ndarray:
        f = _FIELDS[name]
        n = _lib.C.c_longlong(0)
        _lib.check(_lib.lib().mgk_batch_get_field(self._h, r, f, None, _lib.C.byref(n)))
        out = np.zeros(n.value)
        _lib.check(_lib.lib().mgk_batch_get_field(self._h, r, f, _lib.dptr(out), None))
        D = self.cfgs[r].dim
        if name in ("eps_field", "sig_field", "eps_plastic", "prev_strain_dir", "catalog"):
            return out.reshape(-1, D, D)
        return out

    def macro(self, r: int) -> np.ndarray:
        D = self.cfgs[r].dim
        out = np.zeros(2 * D * D + 10)
        _lib.check(_lib.lib().mgk_batch_get_macro(self._h, r, _lib.dptr(out), out.size))
        return out

    def close(self):
        if getattr(self, "_h", None):
            _lib.lib().mgk_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
