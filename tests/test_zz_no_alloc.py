"""The allocation-free field reduction, through the C ABI (needs a B200).

``pycfd_reduce_fields_noalloc`` is for callers that cannot allocate device
memory when they need the reductions: a host whose own allocator owns the
device, or a loop that cannot take the device-wide synchronisation a
cudaMalloc/cudaFree pair may impose.  Its scratch is a static device array
instead.  This file is collected last so that a run stopping at the first
failure has run every other test first; it also passes alone in a fresh
process.
"""

import ctypes as C

import numpy as np
import pytest

import cases
from pycfd_b200.config import BCKind, BCSpec, SimulationConfig

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

FIELDS = ("max_u", "max_v", "max_du", "max_dv", "max_div", "kinetic_energy", "max_vorticity",
          "finite")


def _existing(L, s, f, prev):
    from pycfd_b200 import _lib
    a = _lib.FieldStats()
    _lib.check(L.pycfd_reduce_fields(s._h, _lib.ptr(f.u), _lib.ptr(f.v),
                                     _lib.ptr(f.p) if f.p is not None else None,
                                     _lib.ptr(prev.u) if prev is not None else None,
                                     _lib.ptr(prev.v) if prev is not None else None, C.byref(a), None))
    return a


def _noalloc(L, s, f, prev, solid_dev, with_p=True):
    from pycfd_b200 import _lib
    b = _lib.FieldStats()
    nx, ny = s.mesh.shape
    _lib.check(L.pycfd_reduce_fields_noalloc(
        _lib.ptr(f.u), _lib.ptr(f.v), _lib.ptr(f.p) if with_p else None,
        _lib.ptr(prev.u) if prev is not None else None,
        _lib.ptr(prev.v) if prev is not None else None,
        _lib.ptr(solid_dev) if solid_dev is not None else None,
        nx, ny, s.mesh.dx, s.mesh.dy, C.byref(b), None))
    return b


def _same(a, b, tag):
    for k in FIELDS:
        x, y = getattr(a, k), getattr(b, k)
        assert x == pytest.approx(y, rel=1e-12, abs=1e-300), (tag, k)


def test_noalloc_reduction_matches_existing_entry_point_twice():
    from pycfd_b200 import _lib
    from pycfd_b200.mesh import StructuredMesh
    from pycfd_b200.obstacles import circle_mask
    from pycfd_b200.solver import ProjectionSolver
    L = _lib.load()
    cfg = cases.to_config(cases.cylinder_cfg(96, 48), SimulationConfig, BCSpec, BCKind)
    ob = circle_mask(StructuredMesh.from_config(cfg), (0.5, 0.5), 0.1)
    s = ProjectionSolver(cfg, obstacle=ob.mask)
    solid_dev = torch.as_tensor(ob.mask.astype(np.uint8), device="cuda")
    f = s.initialize(*cases.cylinder_init(96, 48))
    for call in range(2):                     # two calls in a row on fresh states
        prev = f.copy()
        f = s.step(f, 2e-3)
        a = _existing(L, s, f, prev)
        b = _noalloc(L, s, f, prev, solid_dev)
        _same(a, b, call)
        assert b.finite == 1 and b.max_u > 0.5 and b.kinetic_energy > 0.0


def test_noalloc_reduction_wide_grid_without_optional_inputs():
    """nx near the limit (more blocks than the solver-backed reduction launches), no
    pressure, no previous state and no solid mask; device memory is unchanged by the calls."""
    from pycfd_b200 import _lib
    from pycfd_b200.solver import ProjectionSolver
    L = _lib.load()
    nx = 4093
    walls = {w: BCSpec(BCKind.NO_SLIP) for w in ("left", "right", "bottom")}
    walls["top"] = BCSpec(BCKind.MOVING_WALL, velocity=1.0)
    cfg = SimulationConfig(nx=nx, ny=6, lx=float(nx) / 6.0, ly=1.0, re=100.0,
                           pressure_solver="mgcg", poisson_tol=1e-8, boundary_config=walls, name="wide")
    s = ProjectionSolver(cfg)
    f1 = s.step(s.initialize(), 1e-3)
    f2 = s.step(f1, 1e-3)
    _noalloc(L, s, f1, None, None, with_p=False)            # first call: scratch look-up
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for call, f in enumerate((f1, f2)):
        a = _existing(L, s, f, None)
        b = _noalloc(L, s, f, None, None, with_p=False)
        _same(a, b, call)
        assert b.max_u > 0.0 and b.max_du == 0.0 and b.finite == 1   # six rows: the lid has barely diffused in
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0            # the calls allocated nothing


def test_noalloc_reduction_refuses_oversized_grid():
    from pycfd_b200 import _lib
    L = _lib.load()
    u = torch.zeros(8, dtype=torch.float64, device="cuda")
    out = _lib.FieldStats()
    for nx in (4094, 5000, 2**31 - 2):
        with pytest.raises(ValueError, match="nx <="):
            _lib.check(L.pycfd_reduce_fields_noalloc(_lib.ptr(u), _lib.ptr(u), None, None, None, None,
                                                     nx, 8, 1.0, 1.0, C.byref(out), None))
