"""`.npy` reader rules (material_generator.hpp:23-116) and the field generator."""
import struct

import numpy as np
import pytest

from mgkmc_cpp_b200 import fields, npy


def _write_v2(path, arr):
    hdr = "{'descr': '<f8', 'fortran_order': False, 'shape': %s, }" % (tuple(arr.shape),)
    hdr += " " * ((64 - (12 + len(hdr) + 1) % 64) % 64) + "\n"
    with open(path, "wb") as f:
        f.write(b"\x93NUMPY\x02\x00" + struct.pack("<I", len(hdr)) + hdr.encode() + arr.astype("<f8").tobytes())


def test_read_v1_v2_f4_f8(tmp_path):
    a = np.random.default_rng(0).standard_normal((5, 4))
    np.save(tmp_path / "a.npy", a)
    np.save(tmp_path / "b.npy", a.astype(np.float32))
    _write_v2(tmp_path / "c.npy", a)
    for name, want in (("a", a), ("b", a.astype(np.float32).astype(np.float64)), ("c", a)):
        d, shp = npy.read_npy_double(str(tmp_path / (name + ".npy")))
        assert shp == [5, 4]
        assert np.array_equal(d, want.reshape(-1))


def test_read_errors(tmp_path):
    (tmp_path / "bad.npy").write_bytes(b"NOTNPY")
    with pytest.raises(ValueError, match="magic"):
        npy.read_npy_double(str(tmp_path / "bad.npy"))
    np.save(tmp_path / "i.npy", np.arange(3))
    with pytest.raises(ValueError, match="Unsupported dtype"):
        npy.read_npy_double(str(tmp_path / "i.npy"))
    with pytest.raises(ValueError, match="Failed to open"):
        npy.read_npy_double(str(tmp_path / "missing.npy"))


def test_lognormal_field_statistics():
    E = fields.lognormal_modulus((128, 128), 90e9, 0.10, 4.0, seed=0)
    assert abs(E.mean() / 90e9 - 1) < 0.01
    assert abs(E.std() / E.mean() - 0.10) < 0.01
    assert np.all(E > 0)
    # deterministic per seed
    assert np.array_equal(E, fields.lognormal_modulus((128, 128), 90e9, 0.10, 4.0, seed=0))


def test_box_muller_stream_is_std_mt19937():
    # first draw of std::mt19937(5): u1, u2 from the first two 32-bit outputs
    bg = np.random.MT19937(0)
    bg._legacy_seeding(5)
    r = bg.random_raw(2).astype(np.float64) / 4294967296.0
    want = np.sqrt(-2 * np.log(r[0])) * np.cos(2 * np.pi * r[1])
    assert fields.box_muller_normals(1, 5)[0] == want


def test_correlated_field_matches_reference():
    """fields.correlated_field against generate_correlated_field_cpp itself
    (golden grf*.npz from the reference sources): same MT19937 stream and
    Box-Muller draws, an FFT of another library, so within 1e-12."""
    from helpers import golden
    from mgkmc_cpp_b200 import fields
    for name in ("grf2d_32x24", "grf3d_12x10x8"):
        g = golden(name)
        shape = (int(g["nx"]), int(g["ny"])) + ((int(g["nz"]),) if int(g["is3d"]) else ())
        f = fields.correlated_field(shape, float(g["mean"]), float(g["std"]), float(g["corr"]), int(g["seed"]),
                                    clip_min=float(g["cmin"]) if int(g["has_min"]) else None,
                                    clip_max=float(g["cmax"]) if int(g["has_max"]) else None)
        ref = g["field"].reshape(shape)
        assert np.max(np.abs(f - ref)) <= 1e-12 * np.max(np.abs(ref)), name
