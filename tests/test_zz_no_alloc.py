"""The allocation-free field reduction, through the C ABI (needs a B200).

``pycfd_reduce_fields_noalloc`` is for callers that cannot allocate device
memory when they need the reductions (their own allocator owns the device, or
they cannot take cudaMalloc's implicit synchronisation, or they are recording a
stream capture); its scratch is a static device array instead.  This file is
collected last so that a run stopping at the first failure has run every other
test first; it also passes alone in a fresh process.
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


def _pair(L, s, f, prev, solid_dev):
    """(existing entry point, allocation-free entry point) on the same inputs."""
    from pycfd_b200 import _lib
    a = _lib.FieldStats()
    _lib.check(L.pycfd_reduce_fields(s._h, _lib.ptr(f.u), _lib.ptr(f.v), _lib.ptr(f.p),
                                     _lib.ptr(prev.u), _lib.ptr(prev.v), C.byref(a), None))
    b = _lib.FieldStats()
    nx, ny = s.mesh.shape
    _lib.check(L.pycfd_reduce_fields_noalloc(_lib.ptr(f.u), _lib.ptr(f.v), _lib.ptr(f.p),
                                             _lib.ptr(prev.u), _lib.ptr(prev.v), _lib.ptr(solid_dev),
                                             nx, ny, s.mesh.dx, s.mesh.dy, C.byref(b), None))
    return a, b


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
        a, b = _pair(L, s, f, prev, solid_dev)
        for k in FIELDS:
            x, y = getattr(a, k), getattr(b, k)
            assert x == pytest.approx(y, rel=1e-12, abs=1e-300), (call, k)
        assert b.finite == 1 and b.max_u > 0.5 and b.kinetic_energy > 0.0


def test_noalloc_reduction_refuses_oversized_grid():
    from pycfd_b200 import _lib
    L = _lib.load()
    u = torch.zeros(8, dtype=torch.float64, device="cuda")
    out = _lib.FieldStats()
    with pytest.raises(ValueError, match="nx <="):
        _lib.check(L.pycfd_reduce_fields_noalloc(_lib.ptr(u), _lib.ptr(u), None, None, None, None,
                                                 5000, 8, 1.0, 1.0, C.byref(out), None))
