"""Config surface: yaml_parser.hpp semantics and main.cpp's key reading."""
import os

import numpy as np
import pytest

from mgkmc_cpp_b200.config import SimConfig, YAMLConfig, _stod, _stoi

# the reference source tree, when the environment names one (its example configs)
REF = os.environ.get("MGK_REFERENCE_DIR", "")


def test_yaml_flat_keys_comments_quotes():
    c = YAMLConfig.loads("""
seed: 7   # inline comment
system:
  dimensionality: "3D"
  nx: 16
  pixel: 0.7
material:
  E:
    mode: 'file'
    parameters:
      path: "a#b.npy"
boundary_conditions:
  mixed_targets:
    yy: 0.0
    xy: 1.5e-1
  mixed_tol: 2.0
""")
    assert c.get_int("seed") == 7
    assert c.get_string("system.dimensionality") == "3D"
    assert c.get_double("system.pixel") == 0.7
    assert c.get_string("material.E.mode") == "file"
    # '#' starts a comment anywhere, even inside quotes (yaml_parser.hpp:49-52)
    assert c.get_string("material.E.parameters.path") == '"a'
    assert c.get_dict("boundary_conditions.mixed_targets") == {"yy": 0.0, "xy": 0.15}
    assert c.get_double("missing", 3.5) == 3.5


def test_getters_follow_std_conversions():
    assert _stoi("  42abc") == 42
    assert _stod("1e-4 trailing") == 1e-4
    c = YAMLConfig({"a": "yes", "b": "0", "c": "maybe", "d": "12.7"})
    assert c.get_bool("a") is True and c.get_bool("b") is False and c.get_bool("c", True) is True
    assert c.get_int("d") == 12


def test_defaults_and_units():
    s = SimConfig.from_yaml(YAMLConfig.loads("""
system:
  nx: 4
  ny: 3
material:
  E:
    mode: "constant"
    value: 70
physics:
  enable_softening: false
boundary_conditions:
  driving_component: "xy"
  mixed_targets:
    yy: 0.5
    zz: 1.0
"""))
    assert s.dim == 2 and s.nz == 1 and s.n_voxels == 12
    assert np.all(s.E == 70e9)          # GPa auto-converted (main.cpp:61-64)
    assert np.all(s.nu == 0.3)
    assert s.M == 20 and s.gamma0 == 0.14 and s.seed == 42
    assert s.softening_cap == 0.0 and s.jp == 0.0 and s.jt == 0.0
    assert s.driving == (0, 1)
    assert s.targets == {(1, 1): 0.5e9}  # zz ignored in 2D (main.cpp:360-367)
    assert s.n_steps == 500
    assert s.ls_tol == 1e-6 and s.ls_max_iter == 200


def test_npy_modulus_file(tmp_path):
    E = np.arange(12, dtype=np.float32).reshape(4, 3) + 50
    p = tmp_path / "E.npy"
    np.save(p, E)
    s = SimConfig.from_yaml(YAMLConfig.loads(f"""
system:
  nx: 4
  ny: 3
material:
  E:
    mode: "file"
    parameters:
      path: "{p}"
"""))
    assert np.array_equal(s.E, (E.reshape(-1).astype(np.float64)) * 1e9)
    with pytest.raises(ValueError, match="shape does not match"):
        SimConfig.from_yaml(YAMLConfig.loads(f"""
system:
  nx: 3
  ny: 4
material:
  E:
    mode: "file"
    parameters:
      path: "{p}"
"""))


@pytest.mark.skipif(not REF or not os.path.isdir(REF), reason="MGK_REFERENCE_DIR not set to the reference tree")
def test_reference_example_configs_parse():
    n = 0
    for root, _, files in os.walk(os.path.join(REF, "examples")):
        for f in files:
            if f.endswith(".yaml") and "Damask" not in root:
                c = YAMLConfig.load(os.path.join(root, f))
                assert c.get_string("system.dimensionality", "2d").lower() in ("2d", "3d")
                n += 1
    assert n >= 6
