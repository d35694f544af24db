"""Configuration surface of mgkmc_cpp, restated for the B200 build.

``YAMLConfig`` follows the reference's flat dotted-key parser
(yaml_parser.hpp:13-155): ``#`` starts a comment anywhere on a line, nesting is
by indentation, leaves are stripped of one pair of quotes, there are no lists.
``SimConfig.from_yaml`` reads the keys and defaults of main.cpp:40-377,
including the GPa -> Pa auto-conversion (main.cpp:61-64, 96-99, 349-351) and the
driving-component / mixed-target parsing (main.cpp:319-375).  Keys the reference
never reads are ignored, as there.  New keys of this build live under new names
(``ls.tol``, ``ls.max_iter``, ``ls.precision``, ``run.max_flips``) and default
to the reference's hard-coded values.  Two keys select extensions with no counterpart in the
reference (defaults: the reference's behaviour):

* ``catalog.type``: ``random`` (the reference's modes, kmc_solver.hpp:231-238,
  :1042-1074), ``even`` (M shears in the x-y plane with slip directions evenly
  spaced in [0, pi), magnitude gamma0, never redrawn) or ``fibonacci`` (3D: M
  plane normals on a Fibonacci lattice of the upper hemisphere, each sheared
  by gamma0 along its largest resolved shear stress, recomputed from the
  local stress whenever it is used);
* ``barriers.per_voxel``: one barrier per voxel shared by its M modes (drawn
  before the voxel's modes, and redrawn as one value after a flip).
"""
from __future__ import annotations

import dataclasses
import os
from typing import Dict, List, Optional, Tuple

import numpy as np

from . import npy


class YAMLConfig:
    """Flat dotted-key view of a YAML file (yaml_parser.hpp:37-92)."""

    def __init__(self, data: Optional[Dict[str, str]] = None):
        self.data: Dict[str, str] = dict(data or {})

    @staticmethod
    def _strip_quotes(s: str) -> str:
        s = s.strip(" \t\r\n")
        if len(s) >= 2 and ((s[0] == '"' and s[-1] == '"') or (s[0] == "'" and s[-1] == "'")):
            return s[1:-1]
        return s

    @classmethod
    def loads(cls, text: str) -> "YAMLConfig":
        data: Dict[str, str] = {}
        hier: List[Tuple[int, str]] = []
        for line in text.splitlines():
            h = line.find("#")
            if h >= 0:
                line = line[:h]
            indent = 0
            while indent < len(line) and line[indent] in " \t":
                indent += 1
            cleaned = line.strip(" \t\r\n")
            if not cleaned:
                continue
            c = cleaned.find(":")
            if c < 0:
                continue
            key = cleaned[:c].strip(" \t\r\n")
            val = cleaned[c + 1:].strip(" \t\r\n")
            while hier and hier[-1][0] >= indent:
                hier.pop()
            prefix = "".join(k + "." for _, k in hier)
            if not val:
                hier.append((indent, key))
            else:
                data[prefix + key] = cls._strip_quotes(val)
        return cls(data)

    @classmethod
    def load(cls, path: str) -> "YAMLConfig":
        with open(path, "r") as f:
            return cls.loads(f.read())

    def get_string(self, key: str, default: str = "") -> str:
        return self.data.get(key, default)

    def get_int(self, key: str, default: int = 0) -> int:
        v = self.data.get(key)
        if v is None:
            return default
        try:
            return _stoi(v)
        except ValueError:
            return default

    def get_double(self, key: str, default: float = 0.0) -> float:
        v = self.data.get(key)
        if v is None:
            return default
        try:
            return _stod(v)
        except ValueError:
            return default

    def get_bool(self, key: str, default: bool = False) -> bool:
        v = self.data.get(key)
        if v is None:
            return default
        v = v.lower()
        if v in ("true", "yes", "1"):
            return True
        if v in ("false", "no", "0"):
            return False
        return default

    def get_dict(self, prefix: str) -> Dict[str, float]:
        out: Dict[str, float] = {}
        p = prefix + "."
        for k, v in self.data.items():
            if k.startswith(p):
                try:
                    out[k[len(p):]] = _stod(v)
                except ValueError:
                    pass
        return out


def _stoi(s: str) -> int:
    """std::stoi: leading whitespace, optional sign, digits; trailing junk ignored."""
    s = s.lstrip()
    i = 0
    if i < len(s) and s[i] in "+-":
        i += 1
    j = i
    while j < len(s) and s[j].isdigit():
        j += 1
    if j == i:
        raise ValueError(s)
    return int(s[:j])


def _stod(s: str) -> float:
    """std::stod: longest valid floating-point prefix (strtod semantics)."""
    s = s.lstrip()
    best = None
    for end in range(len(s), 0, -1):
        try:
            best = float(s[:end])
            break
        except ValueError:
            continue
    if best is None:
        raise ValueError(s)
    return best


COMP_2D = {"xx": (0, 0), "yy": (1, 1), "xy": (0, 1), "yx": (1, 0)}
COMP_3D = {"xx": (0, 0), "yy": (1, 1), "zz": (2, 2), "xy": (0, 1), "yx": (1, 0),
           "xz": (0, 2), "zx": (2, 0), "yz": (1, 2), "zy": (2, 1)}

BARRIER_TYPES = {"gaussian": 0, "rayleigh": 1, "modified_rayleigh": 2, "modified_rayleigh_with_exponential": 3}


@dataclasses.dataclass
class BarrierParams:
    """BarrierGenerator fields and defaults (kmc_solver.hpp:24-33, main.cpp:281-290)."""
    type: str = "gaussian"
    mean: float = 2.0
    std: float = 0.6
    min_cutoff: float = 0.1
    max_cutoff: float = -1.0
    loc: float = 1.0
    scale: float = 0.5
    epsilon: float = 0.1
    ratio: float = 0.8


@dataclasses.dataclass
class SimConfig:
    """Everything main.cpp reads for a KMC or linear-elastic run."""
    simulation_type: str = "kmc"
    dim: int = 2
    plane_mode: str = "plane_strain"
    nx: int = 32
    ny: int = 32
    nz: int = 1
    pixel: float = 1.0
    E: Optional[np.ndarray] = None
    nu: Optional[np.ndarray] = None
    M: int = 20
    gamma0: float = 0.14
    seed: int = 42
    use_3d_barriers: bool = False
    barrier: BarrierParams = dataclasses.field(default_factory=BarrierParams)
    softening_scheme: str = "isotropic"
    softening_cap: float = 2.0
    jp: float = 10.0
    jt: float = 30.0
    neighbor_softening_fraction: float = 0.0
    q_act_temp: float = 0.37
    redraw_barriers: bool = True
    redraw_directions: bool = True
    stability_threshold: float = 0.0
    instability_mode: str = "cascade"
    cascade_timing: str = "none"
    scale_rate_by_volume: bool = True
    nu0: float = 1e13
    strain_rate: float = 1.0
    temperature: float = 0.0
    fast_patching: bool = False
    patch_radius: int = 5
    sync_interval: int = 100
    eps_target: float = 0.05
    step_size: float = 1e-4
    driving: Tuple[int, int] = (0, 0)
    driving_name: str = "xx"
    targets: Dict[Tuple[int, int], float] = dataclasses.field(default_factory=dict)
    mixed_tol_pa: float = 1e6
    max_kmc_steps_pct: float = 0.3
    # new keys of this build (defaults = the reference's hard-coded values)
    ls_tol: float = 1e-6
    ls_max_iter: int = 200
    max_flips: int = -1
    catalog_type: str = "random"
    barrier_per_voxel: bool = False
    ls_precision: str = "fp64"
    output_directory: str = "simulation_results"
    summary_filename: str = "summary_log.txt"
    enable_console: bool = True
    enable_summary_log: bool = True
    enable_global_log: bool = True
    vtk_interval: str = "none"
    vtk_elastic_only: bool = True

    @property
    def n_voxels(self) -> int:
        return self.nx * self.ny * (self.nz if self.dim == 3 else 1)

    @property
    def n_steps(self) -> int:
        """main.cpp:273 n_steps = round(eps_target / step_size)."""
        return int(np.round(self.eps_target / self.step_size))

    @classmethod
    def from_yaml(cls, path_or_cfg, base_dir: Optional[str] = None) -> "SimConfig":
        c = path_or_cfg if isinstance(path_or_cfg, YAMLConfig) else YAMLConfig.load(path_or_cfg)
        if base_dir is None and not isinstance(path_or_cfg, YAMLConfig):
            base_dir = os.path.dirname(os.path.abspath(path_or_cfg))
        s = cls()
        s.simulation_type = c.get_string("simulation_type", "kmc")
        s.dim = 3 if c.get_string("system.dimensionality", "2d").lower() == "3d" else 2
        s.plane_mode = c.get_string("system.plane_mode", "plane_strain")
        s.nx = c.get_int("system.nx", 32)
        s.ny = c.get_int("system.ny", 32)
        s.nz = c.get_int("system.nz", 32) if s.dim == 3 else 1
        s.pixel = c.get_double("system.pixel", 1.0)
        N = s.n_voxels
        shape = (s.nx, s.ny, s.nz) if s.dim == 3 else (s.nx, s.ny)
        s.seed = c.get_int("seed", 42)
        s.E = _field(c, "E", 70.0, N, shape, s.seed, True, base_dir)
        s.nu = _field(c, "nu", 0.3, N, shape, s.seed + 1, False, base_dir)
        s.output_directory = c.get_string("output.directory", "simulation_results")
        s.summary_filename = c.get_string("output.summary_filename", "summary_log.txt")
        s.enable_console = c.get_bool("output.enable_console", True)
        s.enable_summary_log = c.get_bool("output.enable_summary_log", True)
        s.enable_global_log = c.get_bool("output.enable_global_log", True)
        s.vtk_interval = c.get_string("output.vtk_interval", "none").lower()
        s.vtk_elastic_only = c.get_bool("output.vtk_elastic_only", True)
        s.eps_target = c.get_double("loading.eps_target", 0.05)
        s.step_size = c.get_double("loading.step_size", 1e-4)
        s.mixed_tol_pa = c.get_double("boundary_conditions.mixed_tol", 1.0) * 1e6
        b = s.barrier
        b.type = c.get_string("barriers.type", "gaussian")
        b.mean = c.get_double("barriers.kwargs.mean", 2.0)
        b.std = c.get_double("barriers.kwargs.std", 0.6)
        b.min_cutoff = c.get_double("barriers.kwargs.min_cutoff", 0.1)
        b.max_cutoff = c.get_double("barriers.kwargs.max_cutoff", -1.0)
        b.loc = c.get_double("barriers.kwargs.loc", 1.0)
        b.scale = c.get_double("barriers.kwargs.scale", 0.5)
        b.epsilon = c.get_double("barriers.kwargs.epsilon", 0.1)
        b.ratio = c.get_double("barriers.kwargs.ratio", 0.8)
        soft = c.get_bool("physics.enable_softening", True)
        s.softening_scheme = c.get_string("physics.softening_scheme", "isotropic")
        s.softening_cap = c.get_double("physics.softening_cap", 2.0) if soft else 0.0
        s.jp = c.get_double("physics.jp", 10.0) if soft else 0.0
        s.jt = c.get_double("physics.jt", 30.0) if soft else 0.0
        s.neighbor_softening_fraction = c.get_double("physics.neighbor_softening_fraction", 0.0) if soft else 0.0
        s.q_act_temp = c.get_double("physics.q_act_temp", 0.37)
        s.redraw_barriers = c.get_bool("physics.redraw_barriers", True)
        s.redraw_directions = c.get_bool("physics.redraw_directions", True)
        s.stability_threshold = c.get_double("physics.stability_threshold", 0.0)
        s.instability_mode = c.get_string("dynamics.instability_mode", "cascade")
        s.cascade_timing = c.get_string("dynamics.cascade_timing", "none")
        s.scale_rate_by_volume = c.get_bool("dynamics.scale_rate_by_volume", True)
        s.nu0 = c.get_double("dynamics.nu0", 1e13)
        s.strain_rate = c.get_double("dynamics.physical_strain_rate", 1.0)
        s.temperature = c.get_double("dynamics.temperature", 0.0)
        s.fast_patching = c.get_bool("dynamics.fast_patching.enabled", False)
        s.patch_radius = c.get_int("dynamics.fast_patching.patch_radius", 5)
        s.sync_interval = c.get_int("dynamics.fast_patching.sync_interval", 100)
        s.M = c.get_int("system.M", 20)
        s.gamma0 = c.get_double("system.gamma0", 0.14)
        s.use_3d_barriers = c.get_bool("system.3d_barriers", False)
        s.max_kmc_steps_pct = c.get_double("detection.max_kmc_steps_pct", 0.3)
        table = COMP_3D if s.dim == 3 else COMP_2D
        s.driving_name = c.get_string("boundary_conditions.driving_component", "xx")
        s.driving = table.get(s.driving_name, (0, 0))
        for k, v in sorted(c.get_dict("boundary_conditions.mixed_targets").items()):
            if k not in table:
                continue
            s.targets[table[k]] = v * 1e9 if v < 1e6 else v
        s.ls_tol = c.get_double("ls.tol", 1e-6)
        s.ls_max_iter = c.get_int("ls.max_iter", 200)
        s.max_flips = c.get_int("run.max_flips", -1)
        s.catalog_type = c.get_string("catalog.type", "random").lower()
        if s.catalog_type not in ("random", "even", "fibonacci"):
            raise ValueError("catalog.type must be random, even or fibonacci")
        if s.catalog_type == "fibonacci" and s.dim != 3:
            raise ValueError("catalog.type fibonacci needs a 3D system")
        s.barrier_per_voxel = c.get_bool("barriers.per_voxel", False)
        s.ls_precision = c.get_string("ls.precision", "fp64").lower()
        if s.ls_precision not in ("fp64", "fp32_refined"):
            raise ValueError("ls.precision must be fp64 or fp32_refined")
        return s


def _field(c: YAMLConfig, name: str, default: float, N: int, shape, seed: int, is_modulus: bool,
           base_dir: Optional[str]) -> np.ndarray:
    """Material field per main.cpp:56-220 (constant | file | generated)."""
    mode = c.get_string(f"material.{name}.mode", "constant").lower()
    if mode == "constant":
        v = c.get_double(f"material.{name}.value", default)
        if is_modulus and v < 1e6:
            v *= 1e9
        return np.full(N, v, dtype=np.float64)
    if mode == "file":
        path = c.get_string(f"material.{name}.parameters.path", "")
        if not path:
            raise ValueError(f"material.{name}.mode is 'file' but material.{name}.parameters.path is empty or missing")
        if base_dir and not os.path.isabs(path) and not os.path.exists(path):
            path = os.path.join(base_dir, path)
        arr, shp = npy.read_npy_double(path)
        if tuple(shp) != tuple(shape):
            raise ValueError("Loaded npy shape does not match grid shape.")
        arr = np.asarray(arr, dtype=np.float64).reshape(-1)
        if is_modulus and arr.mean() < 1e6:
            arr = arr * 1e9
        return arr
    if mode == "generated":
        from . import fields
        val = c.get_double(f"material.{name}.value", default)
        mean = c.get_double(f"material.{name}.parameters.mean", val)
        std = c.get_double(f"material.{name}.parameters.std", 0.0)
        corr = c.get_double(f"material.{name}.parameters.corr", 10.0)
        cmin = c.get_string(f"material.{name}.parameters.clip_min", "")
        cmax = c.get_string(f"material.{name}.parameters.clip_max", "")
        arr = fields.correlated_field(shape, mean, std, corr, seed,
                                      clip_min=_stod(cmin) if cmin else None,
                                      clip_max=_stod(cmax) if cmax else None).reshape(-1)
        if is_modulus and arr.mean() < 1e6:
            arr = arr * 1e9
        return arr
    raise ValueError(f"Unsupported material {name} mode: {mode}")
