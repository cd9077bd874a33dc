"""The identities the batched engine's stencil transfers rest on (CPU).

With ``stencil_transfer`` the batch forms the level-0 <-> level-1 transfers from
the fine cells' flags instead of the stored matrices: the prolongation as
(I - W A) T x_1 and the fused restriction as T^T (I - A W)^2 b, T the 0/1 map of
each solvable cell (i, j) to aggregate (i // 2, j // 2).  That holds when level 1
of the hierarchy is the 2 x 2 aggregation, which the host recognises by its shape;
these tests check both identities on the hierarchy builder's own matrices for
odd and even sizes, periodic axes, masks and Dirichlet walls, and that an
anisotropic grid (semi-coarsened) is not taken for one.
"""

import numpy as np
import pytest
import scipy.sparse as sp

from pycfd_b200.hierarchy import assemble, build_hierarchy, fused_restriction


def _aggregation(nx, ny, solvable):
    ncy = -(-ny // 2)
    ii, jj = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    agg = ((ii // 2) * ncy + jj // 2).ravel()
    rows = np.flatnonzero(solvable)
    return sp.csr_matrix((np.ones(rows.size), (rows, agg[rows])), shape=(nx * ny, -(-nx // 2) * ncy))


def _disk(nx, ny, ci, cj, rad):
    ii, jj = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    return (ii - ci) ** 2 + (jj - cj) ** 2 < rad * rad


STRUCTURES = [
    dict(nx=24, ny=24, px=False, py=False),
    dict(nx=25, ny=37, px=False, py=False),
    dict(nx=33, ny=31, px=True, py=True),
    dict(nx=29, ny=30, px=False, py=True),
    dict(nx=61, ny=10, px=True, py=True),
    dict(nx=47, ny=33, px=False, py=False, solid=(15, 16, 5), dirichlet={"right": 0.0}),
    dict(nx=47, ny=33, px=False, py=True, solid=(20, 10, 4), dirichlet={"left": 0.0, "right": 0.0}),
]


@pytest.mark.parametrize("k", range(len(STRUCTURES)))
def test_level_one_transfers_are_the_aggregation_stencils(k):
    s = STRUCTURES[k]
    nx, ny = s["nx"], s["ny"]
    solid = _disk(nx, ny, *s["solid"]) if "solid" in s else None
    op = assemble(nx, ny, 0.03, 0.03, s["px"], s["py"], solid, s.get("dirichlet"))
    levels, _ = build_hierarchy(op)
    assert tuple(levels[1].shape) == (-(-nx // 2), -(-ny // 2))
    A = op.A.tocsr()
    W = sp.diags(levels[0].weighted_dinv)
    I = sp.identity(nx * ny, format="csr")
    T = _aggregation(nx, ny, op.fluid)
    P = (I - W @ A) @ T
    scale = abs(levels[1].P).max()
    assert abs(levels[1].P - P).max() <= 1e-14 * scale
    M = T.T @ (I - A @ W) @ (I - A @ W)
    Mh = fused_restriction(levels, 1)
    assert abs(Mh - M).max() <= 1e-13 * abs(Mh).max()
    # W: the damped inverse diagonal on solvable cells, the weight itself elsewhere
    d = A.diagonal()
    w0 = levels[0].weight
    np.testing.assert_allclose(levels[0].weighted_dinv, np.where(op.fluid, w0 / d, w0), rtol=1e-15)


def test_anisotropic_grid_is_not_a_two_by_two_aggregation():
    op = assemble(32, 32, 1.0 / 32, 1.0 / 80, False, False)
    levels, _ = build_hierarchy(op)
    assert tuple(levels[1].shape) != (16, 16)
