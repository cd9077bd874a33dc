"""Face solid flags bit for bit against the reference (pycfd/core/solver.py:62-79, :235-296).

The fixture ``golden/faces.npz`` holds the reference's own ``u_upd``/``v_upd`` ranges,
``u_face_solid``/``v_face_solid`` and per-body ``u_face_body``/``v_face_body`` for four
layouts: a body across the periodic x seam, a body across the periodic y seam, a body
touching a pressure outlet beside a second body, and three bodies against walls.
"""

import ctypes as C

import numpy as np
import pytest

import cases
from pycfd_b200.config import BCKind, BCSpec, SimulationConfig


def _config(name):
    case = cases.FACE_CASES[name]
    return cases.to_config({**dict(dt=1e-3, t_end=1.0, adaptive_dt=False, name=name), **case["cfg"]},
                           SimulationConfig, BCSpec, BCKind)


def _periodic(cfg):
    k = {w: BCKind(cfg.boundary_config[w].kind) for w in cases.WALLS}
    return k["left"] is BCKind.PERIODIC, k["bottom"] is BCKind.PERIODIC


@pytest.mark.parametrize("name", sorted(cases.FACE_CASES))
def test_host_face_masks_match_reference(golden, name):
    from pycfd_b200.solver import face_solid_mask
    g = golden("faces.npz")
    cfg = _config(name)
    bodies = cases.face_bodies(cases.FACE_CASES[name], cfg.nx, cfg.ny)
    solid = np.logical_or.reduce(bodies)
    px, py = _periodic(cfg)
    u_lo, u_hi, v_lo, v_hi = (int(x) for x in g[f"{name}_upd"])
    assert np.array_equal(face_solid_mask(solid, u_lo, u_hi, 0, px), g[f"{name}_u_face_solid"])
    assert np.array_equal(face_solid_mask(solid, v_lo, v_hi, 1, py), g[f"{name}_v_face_solid"])
    if f"{name}_u_face_body" in g:
        for k, b in enumerate(bodies):
            assert np.array_equal(face_solid_mask(b, u_lo, u_hi, 0, px), g[f"{name}_u_face_body"][k])
            assert np.array_equal(face_solid_mask(b, v_lo, v_hi, 1, py), g[f"{name}_v_face_body"][k])


def _device_faces(s):
    from pycfd_b200 import _lib
    L = _lib.load()
    nu, nv, nb = C.c_int(), C.c_int(), C.c_int()
    MB = _lib.MAX_BODIES + 1
    bu, bv, lohi = (np.zeros(MB, np.int32), np.zeros(MB, np.int32), np.zeros(4, np.int32))
    _lib.check(L.pycfd_face_lists(s._h, None, 0, None, 0, C.byref(nu), C.byref(nv), None, None,
                                  None, None))
    fu, fv = np.zeros(max(nu.value, 1), np.int32), np.zeros(max(nv.value, 1), np.int32)
    _lib.check(L.pycfd_face_lists(s._h, _lib.ptr(fu), nu.value, _lib.ptr(fv), nv.value,
                                  C.byref(nu), C.byref(nv), _lib.ptr(bu), _lib.ptr(bv),
                                  C.byref(nb), _lib.ptr(lohi)))
    return fu[:nu.value], fv[:nv.value], bu, bv, nb.value, lohi


def _as_mask(idx, shape, lo, axis, rng):
    """Linear face indices of a ghosted array -> boolean mask over [lo, hi) x rows 1..n."""
    W = shape[1]
    i, j = idx // W, idx % W
    out = np.zeros(rng, dtype=bool)
    if axis == 0:
        out[i - lo, j - 1] = True
    else:
        out[i - 1, j - lo] = True
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(cases.FACE_CASES))
def test_device_face_lists_match_reference(golden, name):
    pytest.importorskip("torch")
    from pycfd_b200.solver import ProjectionSolver
    g = golden("faces.npz")
    cfg = _config(name)
    nx, ny = cfg.nx, cfg.ny
    bodies = cases.face_bodies(cases.FACE_CASES[name], nx, ny)
    solid = np.logical_or.reduce(bodies)
    s = ProjectionSolver(cfg, obstacle=solid, bodies=bodies if len(bodies) > 1 else None)
    fu, fv, bu, bv, nb, lohi = _device_faces(s)
    assert lohi.tolist() == [int(x) for x in g[f"{name}_upd"]]
    u_lo, u_hi, v_lo, v_hi = lohi.tolist()
    ushape, vshape = (nx + 3, ny + 2), (nx + 2, ny + 3)
    urng, vrng = (u_hi - u_lo, ny), (nx, v_hi - v_lo)
    # every face listed once, and the union is the reference's flag array bit for bit
    assert len(np.unique(fu)) == len(fu) and len(np.unique(fv)) == len(fv)
    assert np.array_equal(_as_mask(fu, ushape, u_lo, 0, urng), g[f"{name}_u_face_solid"])
    assert np.array_equal(_as_mask(fv, vshape, v_lo, 1, vrng), g[f"{name}_v_face_solid"])
    if len(bodies) > 1:
        assert nb == len(bodies)
        for k in range(nb):
            mu = _as_mask(fu[bu[k]:bu[k + 1]], ushape, u_lo, 0, urng)
            mv = _as_mask(fv[bv[k]:bv[k + 1]], vshape, v_lo, 1, vrng)
            assert np.array_equal(mu, g[f"{name}_u_face_body"][k]), k
            assert np.array_equal(mv, g[f"{name}_v_face_body"][k]), k
    else:
        assert nb == 0
