"""The oracle's depth-camera ingestion against the reference's own kernels (golden fixture
tests/golden/range_image.npz, from RGBDloader and computeNormals built for the host by
oracle/ref_build.py): the point cloud, radii, vertex records and normals, bit for bit, on
exactly the pixels the reference writes (its index bound (width - 1) (height - 1))."""
import numpy as np

from conftest import golden
from oracle import cpu


def _same(a, b):
    written = ~np.isnan(b)
    assert np.array_equal(~np.isnan(a), written)
    assert np.array_equal(a[written].view(np.uint32), b[written].view(np.uint32))


def test_cloud_and_normals_equal_reference():
    z = golden("range_image")
    h, w = z["depth"].shape
    out = cpu.range_image_cloud(z["depth"], z["camera16"], float(z["radius"]))
    for k in ("pos4", "radii", "vao5"):
        _same(out[k], z[k])
    _same(cpu.range_image_normals(out["pos4"], w, h), z["norm4"])
    # the fixture covers holes (zero depth -> z = -1000) and the skipped last pixels
    assert (z["depth"] == 0).sum() > 50
    assert np.isnan(z["radii"]).sum() == w + h - 2


def test_normals_are_unit_length():
    z = golden("range_image")
    n = z["norm4"]
    ok = ~np.isnan(n[:, 0])
    length = np.linalg.norm(n[ok, :3].astype(np.float64), axis=1)
    assert np.abs(length - 1).max() < 1e-6
