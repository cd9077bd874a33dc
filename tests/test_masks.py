"""Body rasterisation against the reference's own masks (pycfd/geometry/obstacles.py:87-367).

Fixtures ``golden/shapes.npz`` (a 12-point star polygon, a rectangle and a
bitmap silhouette, plain and inverted at 3x3 subsamples, on a 200x120 mesh of
1.6 x 1) and ``golden/masks.npz`` (the 2048x1024 cylinder of the wake
benchmark) were made by running the reference.  The fraction and the mask
must agree bit for bit, on the host and on the GPU.
"""

import numpy as np
import pytest

import cases
from pycfd_b200.mesh import StructuredMesh
from pycfd_b200 import obstacles as ob


def _mesh():
    m = cases.SHAPE_MESH
    return StructuredMesh(m["nx"], m["ny"], m["lx"], m["ly"])


def _check(o, frac, mask):
    assert np.array_equal(o.fraction, frac)
    assert np.array_equal(o.mask, mask)


def _all(device, g):
    mesh = _mesh()
    pg = ob.polygon_mask(mesh, g["star"], device=device)
    _check(pg, g["poly_frac"], g["poly_mask"])
    assert pg.characteristic_length == float(g["poly_len"])
    _check(ob.rectangle_mask(mesh, (0.31, 0.22), (0.93, 0.61), device=device), g["rect_frac"], g["rect_mask"])
    im = ob.mask_from_image(mesh, g["image"], threshold=0.5, device=device)
    _check(im, g["img_frac"], g["img_mask"])
    assert im.characteristic_length == float(g["img_len"])
    _check(ob.mask_from_image(mesh, g["image"], threshold=0.5, invert=True, subsamples=3, device=device),
           g["img_inv_frac"], g["img_inv_mask"])


def test_host_rasterisers_match_reference(golden):
    _all("cpu", golden("shapes.npz"))


def test_polygon_file_and_transform(tmp_path):
    p = tmp_path / "tri.csv"
    p.write_text("# a triangle\n0, 0\n1 0\n0.5, 1\n0,0\n")
    v = ob.load_polygon(p)
    assert v.shape == (3, 2)
    t = ob.transform_polygon(v, scale=2.0, center=(5.0, 5.0), rotate_deg=90.0)
    assert np.allclose(t.mean(axis=0), (5.0, 5.0))
    with pytest.raises(ValueError):
        ob.polygon_mask(_mesh(), v + 10.0, device="cpu")


@pytest.mark.gpu
def test_gpu_rasterisers_match_reference(golden):
    pytest.importorskip("torch")
    _all("cuda", golden("shapes.npz"))


@pytest.mark.gpu
def test_gpu_cylinder_mask_2048x1024(golden):
    pytest.importorskip("torch")
    g = golden("masks.npz")
    big = StructuredMesh(2048, 1024, 2.0, 1.0)
    o = ob.circle_mask(big, (0.5, 0.5), 0.05, device="cuda")
    assert int(o.mask.sum()) == int(g["big_count"])
    assert np.array_equal(np.packbits(o.mask.ravel()), g["big_bits"])
    host = ob.circle_mask(big, (0.5, 0.5), 0.05, device="cpu")
    assert np.array_equal(o.fraction, host.fraction)
