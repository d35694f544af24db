"""The correlated-field generator on the GPU (mgk_correlated_field) against
generate_correlated_field_cpp itself (golden grf*.npz written by the
reference's sources): the same MT19937 stream and Box-Muller draws (device
log/cos within an ulp of glibc's), FFTs of another library, so the fields
agree within 1e-12 of their scale; and against the host restatement on a
larger 3D grid."""
import numpy as np
import pytest

from helpers import golden

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["grf2d_32x24", "grf3d_12x10x8"])
def test_gpu_field_matches_reference(name):
    import mgkmc_cpp_b200 as G
    G._lib.require_device()
    g = golden(name)
    shape = (int(g["nx"]), int(g["ny"])) + ((int(g["nz"]),) if int(g["is3d"]) else ())
    f = G.correlated_field_gpu(shape, float(g["mean"]), float(g["std"]), float(g["corr"]), int(g["seed"]),
                               clip_min=float(g["cmin"]) if int(g["has_min"]) else None,
                               clip_max=float(g["cmax"]) if int(g["has_max"]) else None)
    ref = g["field"].reshape(shape)
    assert np.max(np.abs(f - ref)) <= 1e-12 * np.max(np.abs(ref))


def test_gpu_field_large_matches_host():
    import mgkmc_cpp_b200 as G
    from mgkmc_cpp_b200 import fields
    G._lib.require_device()
    shape = (40, 36, 30)
    f = G.correlated_field_gpu(shape, 90.0, 9.0, 3.0, 21)
    h = fields.correlated_field(shape, 90.0, 9.0, 3.0, 21)
    assert np.max(np.abs(f - h)) <= 1e-11 * np.max(np.abs(h))
