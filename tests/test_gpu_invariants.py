"""Invariants, determinism and failure modes of the GPU path (needs a B200).

Ports of the reference's own algebraic checks (pycfd/tests/test_solver.py:42-197):
divergence-free to round-off after every step for five boundary families,
exact zeros on masked faces and in quiescent flow, exact preservation of
uniform periodic flow, Taylor-Green energy decay; plus bitwise run-to-run
determinism and loud failures mapped onto the reference's exception types.
"""

import numpy as np
import pytest

import cases
from pycfd_b200.config import BCKind, BCSpec, SimulationConfig

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

DIVERGENCE_TOL = 1.0e-11


def _cfg(d, **kw):
    return cases.to_config(d, SimulationConfig, BCSpec, BCKind, **kw)


def _solver(cfg, solid=None, **kw):
    from pycfd_b200.solver import ProjectionSolver
    return ProjectionSolver(cfg, obstacle=solid, **kw)


FAMILIES = {
    "cavity": cases.bcs(top=("moving_wall", 1.0)),
    "doubly periodic": cases.PER,
    "channel": cases.bcs(left=("periodic",), right=("periodic",)),
    "inlet/outlet": cases.bcs(left=("inlet", 1.0), right=("outlet",)),
    "symmetry": cases.bcs(top=("symmetry",), bottom=("symmetry",), left=("inlet", 1.0),
                          right=("outlet",)),
}


@pytest.mark.parametrize("solver", ["cg", "mgcg", "multigrid"])
@pytest.mark.parametrize("label", list(FAMILIES))
def test_divergence_free_after_every_step(label, solver):
    cfg = _cfg(dict(nx=16, ny=16, re=50.0, dt=1e-3, pressure_solver=solver,
                    poisson_tol=1e-13, boundary_config=FAMILIES[label]))
    s = _solver(cfg)
    rng = np.random.default_rng(0)
    f = s.initialize(0.1 * rng.standard_normal((17, 16)), 0.1 * rng.standard_normal((16, 17)))
    assert s.max_divergence(f) < DIVERGENCE_TOL
    for _ in range(6):
        f = s.step(f, 1e-3)
        assert s.max_divergence(f) < DIVERGENCE_TOL, label


def test_obstacle_faces_exactly_zero_and_divergence_free():
    from pycfd_b200.obstacles import circle_mask
    from pycfd_b200.mesh import StructuredMesh
    cfg = _cfg(dict(nx=40, ny=40, lx=2.0, ly=2.0, re=50.0, pressure_solver="mgcg",
                    poisson_tol=1e-13, boundary_config=cases.bcs(top=("moving_wall", 1.0))))
    ob = circle_mask(StructuredMesh.from_config(cfg), (1.0, 1.0), 0.3)
    s = _solver(cfg, ob.mask)
    f = s.initialize()
    for _ in range(8):
        f = s.step(f, 2e-3)
    u, v, _ = f.numpy()
    assert np.all(u[s.u_upd][s.u_face_solid] == 0.0)
    assert np.all(v[s.v_upd][s.v_face_solid] == 0.0)
    assert s.max_divergence(f) < DIVERGENCE_TOL


def test_quiescent_flow_stays_exactly_zero():
    cfg = _cfg(dict(nx=16, ny=16, re=100.0, pressure_solver="mgcg", boundary_config=cases.bcs()))
    s = _solver(cfg)
    f = s.initialize()
    for _ in range(20):
        f = s.step(f, 1e-3)
    u, v, p = f.numpy()
    assert np.abs(u).max() == 0.0 and np.abs(v).max() == 0.0


def test_uniform_periodic_flow_preserved():
    cfg = _cfg(dict(nx=16, ny=16, re=100.0, pressure_solver="cg", boundary_config=cases.PER))
    s = _solver(cfg)
    f = s.initialize(u_init=2.0, v_init=-1.0)
    for _ in range(10):
        f = s.step(f, 1e-3)
    u, v, _ = f.numpy()
    assert np.abs(u[1:18, 1:17] - 2.0).max() < 1e-13
    assert np.abs(v[1:17, 1:18] + 1.0).max() < 1e-13


def test_taylor_green_energy_decay():
    from pycfd_b200.timestepper import TimeStepper
    nu, t_end, n = 0.1, 0.4, 48
    cfg = _cfg(dict(nx=n, ny=n, lx=2 * np.pi, ly=2 * np.pi, re=1.0 / nu, dt=0.2 * 2 * np.pi / n,
                    t_end=t_end, adaptive_dt=False, pressure_solver="mgcg",
                    boundary_config=cases.PER))
    s = _solver(cfg)
    xf, xc = cases.axis(2 * np.pi, n)
    Xu, Yu = np.meshgrid(xf, xc, indexing="ij")
    Xv, Yv = np.meshgrid(xc, xf, indexing="ij")
    f = s.initialize(-np.cos(Xu) * np.sin(Yu), np.sin(Xv) * np.cos(Yv))
    e0 = s.field_stats(f).kinetic_energy
    res = TimeStepper(s).run(f, t_end=t_end)
    ratio = s.field_stats(res.fields).kinetic_energy / e0
    assert ratio == pytest.approx(np.exp(-4.0 * nu * res.time), rel=2e-3)


def test_steps_are_bitwise_deterministic():
    spec = cases.STEP_CASES["inout_sym_obstacle_mgcg"]
    out = []
    for _ in range(2):
        cfg = cases.step_config(spec, SimulationConfig, BCSpec, BCKind)
        from oracle.projection import circle_mask_oracle
        solid = circle_mask_oracle(cfg.nx, cfg.ny, cfg.lx, cfg.ly, *spec["circle"])
        s = _solver(cfg, solid)
        f = s.initialize(1.0)
        for _ in range(5):
            f = s.step(f, spec["dt"])
        out.append(f.numpy() + (s.body_force_reaction,))
    for a, b in zip(out[0][:3], out[1][:3]):
        assert np.array_equal(a, b)
    assert out[0][3] == out[1][3]


def test_nonconvergence_raises_runtime_error():
    cfg = _cfg(dict(nx=32, ny=32, re=100.0, pressure_solver="cg", poisson_maxiter=2,
                    poisson_tol=1e-14, boundary_config=cases.bcs(top=("moving_wall", 1.0))))
    s = _solver(cfg)
    with pytest.raises(RuntimeError, match="converge"):
        f = s.initialize()
        for _ in range(3):
            f = s.step(f, 1e-2)


def test_stalled_sor_raises():
    cfg = _cfg(dict(nx=16, ny=16, re=100.0, pressure_solver="sor", poisson_maxiter=10,
                    poisson_tol=1e-14, boundary_config=cases.bcs(top=("moving_wall", 1.0))))
    s = _solver(cfg)
    with pytest.raises(RuntimeError):
        f = s.initialize()
        s.step(f, 1e-2)


def test_nonfinite_state_raises_divergence_error():
    from pycfd_b200.timestepper import TimeStepper, DivergenceError
    cfg = _cfg(dict(nx=16, ny=16, re=100.0, pressure_solver="cg",
                    boundary_config=cases.bcs(top=("moving_wall", 1.0))))
    s = _solver(cfg)
    f = s.initialize()
    f.u[5, 5] = float("nan")
    with pytest.raises(DivergenceError, match="non-finite"):
        TimeStepper(s).run(f, t_end=1.0, max_steps=3)


def test_rejected_configurations():
    from pycfd_b200.solver import GpuOptions, ProjectionSolver
    base = dict(nx=16, ny=16, re=100.0, boundary_config=cases.bcs())
    with pytest.raises(NotImplementedError, match="direct"):
        ProjectionSolver(_cfg(base, pressure_solver="direct"))
    with pytest.raises(NotImplementedError, match="mixed-precision"):
        ProjectionSolver(_cfg(base, pressure_solver="cg"), options=GpuOptions(precision="mixed"))
    with pytest.raises(NotImplementedError, match="simple"):
        ProjectionSolver(_cfg(base, pressure_solver="cg", solver_type="simple"))
    with pytest.raises(ValueError, match="red/black"):
        ProjectionSolver(_cfg(dict(nx=15, ny=16, re=100.0, boundary_config=cases.PER),
                              pressure_solver="sor"))
    with pytest.raises(ValueError, match="shape"):
        ProjectionSolver(_cfg(base, pressure_solver="cg"), obstacle=np.zeros((4, 4), bool))


@pytest.mark.parametrize("solver", ["cg", "mgcg", "sor"])
def test_host_buffer_step_matches_device_step_bitwise(solver):
    """pycfd_step_host (copies in, the recorded step, copies out) against the device step of
    an identically prepared solver, over three steps (the first records, the rest replay)."""
    from pycfd_b200.solver import GpuOptions
    d = dict(nx=40, ny=32, re=100.0, pressure_solver=solver, poisson_tol=1e-12,
             boundary_config=cases.bcs(top=("moving_wall", 1.0)))
    a = _solver(_cfg(d), options=GpuOptions(graphs=False))
    b = _solver(_cfg(d))
    fa = a.initialize()
    fb = b.initialize()
    pin = lambda shape: torch.empty(shape, dtype=torch.float64).pin_memory().numpy()
    out = [(pin(fb.u.shape), pin(fb.v.shape), pin(fb.p.shape)) for _ in range(2)]
    u, v = fb.u.cpu().numpy().copy(), fb.v.cpu().numpy().copy()
    for k in range(3):
        fa = a.step(fa, 2e-3)
        u, v, p = b.step_host(u, v, 2e-3, out=out[k % 2])
        ua, va, pa = fa.numpy()
        assert np.array_equal(ua, u) and np.array_equal(va, v) and np.array_equal(pa, p), k


@pytest.mark.parametrize("solver", ["cg", "mgcg", "multigrid"])
def test_graph_replay_matches_eager_bitwise(solver):
    """A step recorded into a CUDA graph (device-side solve loops) replays the eager launches."""
    from pycfd_b200.obstacles import circle_mask
    from pycfd_b200.mesh import StructuredMesh
    from pycfd_b200.solver import GpuOptions
    d = dict(nx=48, ny=32, lx=3.0, ly=2.0, re=50.0, pressure_solver=solver, poisson_tol=1e-12,
             boundary_config=cases.bcs(left=("inlet", 1.0), right=("outlet",), top=("symmetry",),
                                       bottom=("symmetry",)))
    out = []
    for graphs in (False, True):
        cfg = _cfg(d)
        ob = circle_mask(StructuredMesh.from_config(cfg), (1.0, 1.0), 0.25)
        s = _solver(cfg, ob.mask, options=GpuOptions(graphs=graphs))
        f = s.initialize(1.0)
        its = []
        for _ in range(6):
            f = s.advance(f, 2e-3)
            its.append(s.last_stats.total_iterations)
        out.append((f.numpy(), s.body_force_reaction, its))
    (a, fa, ia), (b, fb, ib) = out
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    assert fa == fb and ia == ib


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_coarse_cluster_matches_per_level_kernels(precision):
    """Coarse levels run in one thread-block cluster agree with the per-kernel V-cycle
    (the two split wide rows over different lane counts, so to rounding: 1e-9)."""
    from pycfd_b200.solver import GpuOptions
    d = dict(nx=96, ny=64, lx=1.5, ly=1.0, re=200.0, pressure_solver="mgcg", poisson_tol=1e-12,
             boundary_config=cases.bcs(top=("moving_wall", 1.0)))
    out = []
    for rows in (0, 20000):   # per-level kernels vs the coarse cluster
        s = _solver(_cfg(d), options=GpuOptions(precision=precision, coarse_cluster_rows=rows, coarse_tail=False))
        f = s.initialize()
        its = []
        for _ in range(4):
            f = s.advance(f, 2e-3)
            its.append(s.last_stats.total_iterations)
        out.append((f.numpy(), its))
    for a, b in zip(out[0][0], out[1][0]):
        assert np.abs(a - b).max() <= 1e-9 * np.abs(b).max()
    assert all(abs(p - q) <= 2 for p, q in zip(out[0][1], out[1][1]))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_programmatic_launch_matches_stream_order(precision):
    """Kernels scheduled early (each waits on its predecessor) give the same bits."""
    from pycfd_b200.solver import GpuOptions
    d = dict(nx=64, ny=48, lx=4.0 / 3.0, ly=1.0, re=150.0, pressure_solver="mgcg",
             poisson_tol=1e-12, boundary_config=cases.bcs(left=("inlet", 1.0), right=("outlet",)))
    out = []
    for pdl in (False, True):
        s = _solver(_cfg(d), options=GpuOptions(precision=precision, programmatic_launch=pdl))
        f = s.initialize(1.0)
        for _ in range(5):
            f = s.advance(f, 2e-3)
        out.append(f.numpy())
    for a, b in zip(*out):
        assert np.array_equal(a, b)
