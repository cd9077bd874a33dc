"""Host-side operators that restructure the V-cycle (no GPU needed).

The dense tail M_t must be the linear map of the V-cycle at and below level t, and the
fused restriction M_l must be R_l (I - A W) -- the first sweep from zero on level l-1
followed by the restriction of its residual (pycfd/core/multigrid.py:430-474).  Both are
checked here against the cycle run step by step on random right-hand sides.
"""

import math

import numpy as np
import pytest

from pycfd_b200.hierarchy import (TAIL_MAX_ROWS, assemble, build_hierarchy, fused_restriction,
                                  tail_level, tail_operator)


def _hierarchy(n, periodic):
    h = (2 * math.pi if periodic else 1.0) / n
    op = assemble(n, n, h, h, periodic, periodic)
    return build_hierarchy(op)


def _cycle(levels, cinv, l, b, sweeps):
    """The V-cycle from zero at level l >= 1, as the device runs it."""
    lv = levels[l]
    W, A = lv.weighted_dinv, lv.A
    x = W * b
    for _ in range(1, sweeps):
        x = x + W * (b - A @ x)
    res = b - A @ x
    nxt = levels[l + 1]
    bc = nxt.P.T @ res
    xc = cinv @ bc if l + 1 == len(levels) - 1 else _cycle(levels, cinv, l + 1, bc, sweeps)
    x = x + nxt.P @ xc
    for _ in range(sweeps):
        x = x + W * (b - A @ x)
    return x


@pytest.mark.parametrize("n,periodic,sweeps", [(64, True, 1), (64, False, 1), (128, False, 2)])
def test_tail_operator_is_the_cycle_below_its_level(n, periodic, sweeps):
    levels, cinv = _hierarchy(n, periodic)
    t = tail_level(levels)
    assert 1 <= t < len(levels) - 1 and levels[t].n <= TAIL_MAX_ROWS
    M = tail_operator(levels, cinv, t, sweeps)
    assert M.shape == (levels[t].n, levels[t].n)
    rng = np.random.default_rng(0)
    for _ in range(3):
        b = rng.standard_normal(levels[t].n)
        ref = _cycle(levels, cinv, t, b, sweeps)
        assert np.abs(M @ b - ref).max() <= 1e-12 * np.abs(ref).max()
    # the symmetric V-cycle gives a symmetric operator
    assert np.abs(M - M.T).max() <= 1e-10 * np.abs(M).max()


@pytest.mark.parametrize("periodic", [True, False])
def test_fused_restriction_is_sweep_then_restriction(periodic):
    levels, _ = _hierarchy(64, periodic)
    rng = np.random.default_rng(1)
    for l in range(1, len(levels) - 1):
        M = fused_restriction(levels, l)
        f = levels[l - 1]
        b = rng.standard_normal(f.n)
        x = f.weighted_dinv * b
        ref = levels[l].P.T @ (b - f.A @ x)
        assert M.shape == (levels[l].n, f.n)
        assert np.abs(M @ b - ref).max() <= 1e-12 * np.abs(ref).max()


def test_tail_level_rule():
    levels, _ = _hierarchy(128, False)
    sizes = [lv.n for lv in levels]
    t = tail_level(levels)
    assert t == next(l for l in range(1, len(levels) - 1) if sizes[l] <= TAIL_MAX_ROWS)
    # a byte bound moves the tail down to a level whose operator fits it
    tb = tail_level(levels, ratio=4.0)
    assert tb == 0 or (tb >= t and sizes[tb] ** 2 <= 4.0 * sizes[0])
    # a grid with no level above the coarsest gets no tail
    small, _ = _hierarchy(8, True)
    assert tail_level(small) == 0


@pytest.mark.parametrize("tail,ratio,fused,sweeps", [(True, None, True, 1), (True, 4.0, True, 1),
                                                     (True, None, False, 1), (True, None, True, 2),
                                                     (False, None, True, 1)])
def test_solver_descriptor_carries_the_cycle_options(tail, ratio, fused, sweeps):
    """The options reach the native descriptor: the tail level and its operator, and the
    fused restrictions onto levels 1..tail (one sweep per level only)."""
    import cases
    from pycfd_b200.config import BCKind, BCSpec, PressureSolver, SimulationConfig
    from pycfd_b200.mesh import StructuredMesh
    from pycfd_b200.solver import BoundaryInfo, GpuOptions, native_desc
    from pycfd_b200.hierarchy import hierarchy_for
    cfg = cases.to_config(dict(nx=128, ny=128, re=100.0, pressure_solver="mgcg", mg_sweeps=sweeps,
                               boundary_config=cases.bcs(top=("moving_wall", 1.0))),
                          SimulationConfig, BCSpec, BCKind)
    mesh = StructuredMesh.from_config(cfg)
    bnd = BoundaryInfo(cfg.boundary_config, mesh)
    solid = np.zeros(mesh.shape, bool)
    _, (levels, cinv) = hierarchy_for(cfg.nx, cfg.ny, mesh.dx, mesh.dy, False, False, None, {})
    opts = GpuOptions(coarse_tail=tail, tail_ratio=ratio, fused_restriction=fused)
    d, keep = native_desc(cfg, mesh, bnd, solid, False, (), PressureSolver.MGCG, opts, levels, cinv)
    expect = tail_level(levels, ratio) if tail else 0
    assert d.tail_level == expect
    assert bool(d.tail_operator) == (expect > 0)
    for l in range(1, d.n_levels):
        has_m = bool(d.levels[l].m_indptr)
        assert has_m == (expect > 0 and fused and sweeps == 1 and l <= expect), l
