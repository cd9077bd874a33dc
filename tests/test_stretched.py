"""Stretched meshes on the host: widths, faces and metrics, the packed metric block
the device reads, the stretched Poisson operator and the refusals
(``pycfd/core/mesh.py:122-311``, ``pycfd/core/pressure.py:193-207``,
``pycfd/core/solver.py:209-230``), against vectors the reference generated."""

import numpy as np
import pytest

import cases
from pycfd_b200.config import BCKind, BCSpec, SimulationConfig
from pycfd_b200.hierarchy import assemble
from pycfd_b200.mesh import MeshMetrics, NonUniformMeshError, StructuredMesh, geometric_widths


@pytest.mark.parametrize("k", range(len(cases.STRETCH_MESHES)))
def test_widths_faces_and_metrics_match_reference(golden, k):
    g = golden("stretched.npz")
    mesh = StructuredMesh(*cases.STRETCH_MESHES[k])
    assert not mesh.is_uniform
    m = mesh.metrics
    for mine, key in ((mesh.dx_cells, "dx"), (mesh.dy_cells, "dy"), (mesh.xf, "xf"), (mesh.yf, "yf"),
                      (np.ravel(m.hxu), "hxu"), (np.ravel(m.hyv), "hyv"), (np.ravel(m.wx_corner), "wx"),
                      (np.ravel(m.wy_corner), "wy")):
        ref = g[f"m{k}_{key}"]
        if ref.size == 1:                       # a uniform axis keeps scalar metrics
            assert np.all(mine == ref.item()), key
        else:
            assert np.array_equal(np.broadcast_to(mine, ref.shape), ref), key


def test_geometric_widths_sum_and_shape():
    for n in (7, 8):
        for mode in ("low", "walls", "centre"):
            w = geometric_widths(2.0, n, 1.1, mode)
            assert w.shape == (n,) and abs(w.sum() - 2.0) < 1e-14
            if mode == "walls":
                assert w[0] == w.min()
            if mode == "centre":
                assert w[n // 2] == w.min()
    assert np.all(geometric_widths(1.0, 5, 1.0) == 0.2)


def test_device_block_layout():
    """The packed block in the order pcfd::Metrics reads it (csrc/common.cuh)."""
    mesh = StructuredMesh(*cases.STRETCH_MESHES[1])
    nx, ny = mesh.shape
    blk = mesh.metrics.device_block()
    assert blk.size == 5 * nx + 5 * ny + 11
    m = mesh.metrics
    off = dict(hx=0, hy=nx, hxu=nx + ny, hyv=2 * nx + ny + 1, hx_ext=2 * nx + 2 * ny + 2,
               hy_ext=3 * nx + 2 * ny + 4, wx=3 * nx + 3 * ny + 6, wy=4 * nx + 3 * ny + 7)
    ln = dict(hx=nx, hy=ny, hxu=nx + 1, hyv=ny + 1, hx_ext=nx + 2, hy_ext=ny + 2, wx=nx + 1, wy=ny + 1)
    for key, src in (("hx", m.hx), ("hy", m.hy), ("hxu", m.hxu), ("hyv", m.hyv), ("hx_ext", m.hx_ext),
                     ("hy_ext", m.hy_ext), ("wx", m.wx_corner), ("wy", m.wy_corner)):
        assert np.array_equal(blk[off[key]:off[key] + ln[key]], np.ravel(src)), key
    vbar = float(m.cell_areas.mean())
    assert blk[-1] == vbar
    assert np.array_equal(blk[4 * nx + 4 * ny + 8:5 * nx + 4 * ny + 9], np.ravel(m.hxu) * vbar)
    assert np.array_equal(blk[5 * nx + 4 * ny + 9:5 * nx + 5 * ny + 10], np.ravel(m.hyv) * vbar)


def test_stretched_poisson_operator_matches_reference(golden):
    g = golden("stretched.npz")
    mesh = StructuredMesh(*cases.STRETCH_MESHES[0])
    nx, ny = mesh.shape
    op = assemble(nx, ny, mesh.metrics.min_hx, mesh.metrics.min_hy, False, False, g["poisson_solid"],
                  {"right": 0.3}, (mesh.dx_cells, mesh.dy_cells))
    A = op.A.tocsr()
    A.sort_indices()
    assert np.array_equal(A.indptr, g["poisson_A_indptr"])
    assert np.array_equal(A.indices, g["poisson_A_indices"])
    assert np.array_equal(A.data, g["poisson_A_data"])
    assert np.array_equal(op.bc_rhs, g["poisson_bc"])
    assert np.array_equal(op.row_scale, g["poisson_row_scale"])


def test_uniform_mesh_keeps_scalar_metrics():
    mesh = StructuredMesh(16, 8, 2.0, 1.0)
    m = mesh.metrics
    assert mesh.is_uniform and m.hx == mesh.dx and m.hyv == mesh.dy and m.wx_corner == 0.5
    assert isinstance(m, MeshMetrics) and m.min_hx == mesh.dx


def test_uniform_spacing_refused_on_a_stretched_mesh():
    mesh = StructuredMesh(16, 16, stretch_y=1.1)
    assert mesh.stretched_y and not mesh.stretched_x
    with pytest.raises(NonUniformMeshError):
        mesh.dy
