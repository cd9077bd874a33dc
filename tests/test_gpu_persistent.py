"""Whole CG / MG-PCG solves as one cooperative launch (needs a B200).

The persistent kernel runs the same per-row arithmetic as the one-kernel-per-
phase form; only the CTA partition of the dot products differs, so the two
agree to rounding (the iterates of a CG solve amplify a last-bit difference in
a dot product only mildly: 1e-9 relative after several steps at tol 1e-12).
The persistent form is itself deterministic: a recorded step equals the eager
one bit for bit, and two runs give the same bits.
"""

import numpy as np
import pytest

import cases
from pycfd_b200.config import BCKind, BCSpec, SimulationConfig

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

FAMILIES = {
    "cavity": cases.bcs(top=("moving_wall", 1.0)),
    "doubly periodic": cases.PER,
    "inlet/outlet": cases.bcs(left=("inlet", 1.0), right=("outlet",)),
    "pressure outlet": cases.bcs(left=("inlet", 1.0), right=("pressure_outlet",)),
}


def _cfg(d, **kw):
    return cases.to_config(d, SimulationConfig, BCSpec, BCKind, **kw)


def _run(cfg, persistent, steps, solid=None, graphs=True, dt=2e-3, u0=1.0):
    from pycfd_b200.solver import GpuOptions, ProjectionSolver
    s = ProjectionSolver(cfg, obstacle=solid, options=GpuOptions(persistent_solve=persistent, graphs=graphs))
    f = s.initialize(u0)
    its = []
    for _ in range(steps):
        f = s.advance(f, dt)
        its.append(s.last_stats.total_iterations)
    return f.numpy(), its, s


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("solver", ["cg", "mgcg"])
@pytest.mark.parametrize("label", list(FAMILIES))
def test_persistent_matches_phase_kernels(label, solver):
    cfg = _cfg(dict(nx=48, ny=40, lx=1.2, ly=1.0, re=200.0, pressure_solver=solver, poisson_tol=1e-12,
                    boundary_config=FAMILIES[label]))
    a, ia, sa = _run(cfg, True, 6)
    b, ib, sb = _run(cfg, False, 6)
    assert sa._persistent and not sb._persistent
    for x, y in zip(a, b):
        assert _rel(x, y) < 1e-9, label
    assert all(abs(p - q) <= 3 for p, q in zip(ia, ib)), (ia, ib)


@pytest.mark.parametrize("n,sweeps", [(8, 1), (64, 1), (64, 2), (256, 1)])
def test_persistent_hierarchy_depths(n, sweeps):
    """Single-level (8x8: the dense coarsest only), 4 and 6 levels, two sweeps."""
    cfg = _cfg(dict(nx=n, ny=n, lx=2 * np.pi, ly=2 * np.pi, re=1000.0, pressure_solver="mgcg",
                    poisson_tol=1e-12, mg_sweeps=sweeps, boundary_config=cases.PER))
    rng = np.random.default_rng(3)
    u0 = rng.standard_normal((n + 1, n))
    from pycfd_b200.solver import GpuOptions, ProjectionSolver
    out = []
    for persistent in (True, False):
        s = ProjectionSolver(cfg, options=GpuOptions(persistent_solve=persistent))
        f = s.initialize(u0)
        for _ in range(4):
            f = s.advance(f, 1e-3)
        out.append(f.numpy())
        assert s.last_stats.status == 0 and s.last_stats.converged
    for x, y in zip(*out):
        assert _rel(x, y) < 1e-9


def test_persistent_with_obstacle_and_forces():
    from pycfd_b200.mesh import StructuredMesh
    from pycfd_b200.obstacles import circle_mask
    cfg = _cfg(dict(nx=96, ny=48, lx=2.0, ly=1.0, re=100.0, pressure_solver="mgcg", poisson_tol=1e-12,
                    boundary_config=cases.bcs(left=("inlet", 1.0), right=("outlet",), top=("symmetry",),
                                              bottom=("symmetry",))))
    ob = circle_mask(StructuredMesh.from_config(cfg), (0.5, 0.5), 0.1)
    a, _, sa = _run(cfg, True, 8, solid=ob.mask)
    b, _, sb = _run(cfg, False, 8, solid=ob.mask)
    for x, y in zip(a, b):
        assert _rel(x, y) < 1e-9
    assert sa.body_force_reaction[0] == pytest.approx(sb.body_force_reaction[0], rel=1e-9)


def test_persistent_recorded_equals_eager_and_is_deterministic():
    cfg = _cfg(dict(nx=64, ny=64, re=400.0, pressure_solver="mgcg", poisson_tol=1e-11,
                    boundary_config=cases.bcs(top=("moving_wall", 1.0))))
    rec1, i1, _ = _run(cfg, True, 5, graphs=True, u0=0.0)
    rec2, i2, _ = _run(cfg, True, 5, graphs=True, u0=0.0)
    eag, i3, _ = _run(cfg, True, 5, graphs=False, u0=0.0)
    for x, y, z in zip(rec1, rec2, eag):
        assert np.array_equal(x, y) and np.array_equal(x, z)
    assert i1 == i2 == i3


def test_persistent_solve_is_one_launch():
    """A recorded MG-PCG step: the launches no longer grow with the iterations."""
    from pycfd_b200 import _lib
    cfg = _cfg(dict(nx=128, ny=128, lx=2 * np.pi, ly=2 * np.pi, re=1000.0, pressure_solver="mgcg",
                    poisson_tol=1e-10, boundary_config=cases.PER))
    L = _lib.load()
    from pycfd_b200.solver import GpuOptions, ProjectionSolver
    s = ProjectionSolver(cfg, options=GpuOptions(graphs=False, persistent_solve=True))
    f = s.initialize(np.random.default_rng(1).standard_normal((129, 128)))
    torch.cuda.synchronize()
    n0 = L.pycfd_launch_count()
    f = s.advance(f, 1e-3)
    torch.cuda.synchronize()
    n = L.pycfd_launch_count() - n0
    assert s.last_stats.total_iterations > 3
    assert n < 40, n    # 3 substeps x (stencils + one solve launch)


@pytest.mark.parametrize("persistent", [False, True])
@pytest.mark.parametrize("n,sweeps", [(64, 1), (256, 1), (256, 2)])
def test_dense_tail_matches_level_by_level(n, sweeps, persistent):
    """The V-cycle closed by the dense operator of its tail (levels of at most 2048
    rows down to the coarsest), with and without the fused restrictions above it,
    against the level-by-level cycle."""
    from pycfd_b200.hierarchy import tail_level
    from pycfd_b200.solver import GpuOptions, ProjectionSolver
    cfg = _cfg(dict(nx=n, ny=n, re=400.0, pressure_solver="mgcg", poisson_tol=1e-12, mg_sweeps=sweeps,
                    boundary_config=cases.bcs(top=("moving_wall", 1.0))))
    out, its = [], []
    for tail, fused in ((True, True), (True, False), (False, False)):
        s = ProjectionSolver(cfg, options=GpuOptions(coarse_tail=tail, fused_restriction=fused,
                                                     persistent_solve=persistent))
        f = s.initialize()
        k = []
        for _ in range(5):
            f = s.advance(f, 2e-3)
            k.append(s.last_stats.total_iterations)
        out.append(f.numpy())
        its.append(k)
    assert tail_level(s._levels) > 0
    for k in (0, 1):
        for x, y in zip(out[k], out[2]):
            assert _rel(x, y) < 1e-9
        assert all(abs(p - q) <= 2 for p, q in zip(its[k], its[2])), its


def test_barrier_wait_limit_ends_the_solve_and_the_solver_stays_usable():
    """A grid-barrier wait that runs out (limit set to 1 ns, so the first CTA that has
    to wait gives up) ends the persistent solve with status -6 -- reported as a
    RuntimeError, no fault, no hang -- and the next solve with the default limit
    is correct."""
    from pycfd_b200.solver import GpuOptions, ProjectionSolver
    cfg = _cfg(dict(nx=64, ny=64, re=100.0, pressure_solver="mgcg", poisson_tol=1e-12,
                    boundary_config=FAMILIES["cavity"]))
    s = ProjectionSolver(cfg, options=GpuOptions(persistent_solve=True, graphs=False))
    assert s._persistent
    rng = np.random.default_rng(3)
    rhs = rng.standard_normal((64, 64))
    rhs -= rhs.mean()
    ref = s.pressure_solver.solve(rhs).cpu().numpy()
    s.set_wait_limit(1e-9)
    with pytest.raises(RuntimeError, match="grid barrier"):
        s.pressure_solver.solve(rhs)
    assert s.last_stats.status == -6
    s.set_wait_limit(2.0)
    again = s.pressure_solver.solve(rhs).cpu().numpy()
    assert s.last_stats.status == 0
    assert _rel(again, ref) < 1e-12
