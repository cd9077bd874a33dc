"""Mixed-precision form: FP32 MG-PCG inner solves inside FP64 iterative refinement.

The outer loop stops on the true FP64 residual ||b - A p|| < tol ||b||, so the
form reaches the same tolerance as the FP64 path; velocity, pressure and
divergence differences against the reference's own step are checked here at
1e-10 relative (the same bar as the FP64 path), and the mixed form's own looser
bars (velocity error <= 1e-6 against the FP64 result, max|div u| <= 1e-8) on a
Taylor-Green vortex.
"""

import numpy as np
import pytest

import cases
from oracle.projection import circle_mask_oracle
from pycfd_b200.config import BCKind, BCSpec, SimulationConfig

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _solver(cfg, solid=None, graphs=True):
    from pycfd_b200.solver import GpuOptions, ProjectionSolver
    return ProjectionSolver(cfg, obstacle=solid,
                            options=GpuOptions(precision="mixed", inner_tol=1e-4, graphs=graphs))


@pytest.mark.parametrize("name", ["periodic_mgcg", "inout_sym_obstacle_mgcg", "periodic_y_sym_mgcg"])
def test_mixed_steps_match_reference(golden, name):
    g = golden("steps.npz")
    spec = cases.STEP_CASES[name]
    cfg = cases.step_config(spec, SimulationConfig, BCSpec, BCKind)
    solid = None
    if "circle" in spec:
        solid = circle_mask_oracle(cfg.nx, cfg.ny, cfg.lx, cfg.ly, *spec["circle"])
    s = _solver(cfg, solid)
    f = s.initialize(*cases.step_init(spec, cfg.nx, cfg.ny, cfg.lx, cfg.ly))
    for _ in range(spec["steps"]):
        f = s.advance(f, spec["dt"])
        assert s.last_stats.ir_iterations >= 1
    u, v, p = f.numpy()
    assert rel(u, g[name + "_u"]) < 1e-10
    assert rel(v, g[name + "_v"]) < 1e-10
    assert rel(p, g[name + "_p"]) < 1e-10
    assert s.max_divergence(f) < 1e-11


def test_mixed_graph_matches_eager_bitwise():
    spec = cases.STEP_CASES["inout_sym_obstacle_mgcg"]
    out = []
    for graphs in (False, True):
        cfg = cases.step_config(spec, SimulationConfig, BCSpec, BCKind)
        solid = circle_mask_oracle(cfg.nx, cfg.ny, cfg.lx, cfg.ly, *spec["circle"])
        s = _solver(cfg, solid, graphs=graphs)
        f = s.initialize(1.0)
        for _ in range(4):
            f = s.advance(f, spec["dt"])
        out.append(f.numpy())
    for a, b in zip(*out):
        assert np.array_equal(a, b)


def test_mixed_taylor_green_against_fp64():
    """128^2 vortex, Re 1000, tol 1e-10: mixed vs FP64 path and the analytic decay."""
    from pycfd_b200.solver import GpuOptions, ProjectionSolver
    n = 128
    cfg = cases.to_config(cases.tgv_cfg(n), SimulationConfig, BCSpec, BCKind)
    u0, v0 = cases.tg_init(n, n, cfg.lx, cfg.ly)
    res = {}
    for prec in ("fp64", "mixed"):
        s = ProjectionSolver(cfg, options=GpuOptions(precision=prec))
        f = s.initialize(u0, v0)
        for _ in range(20):
            f = s.advance(f, cfg.dt)
        res[prec] = (f.numpy(), s.max_divergence(f), f.t)
    (u64, v64, p64), div64, t = res["fp64"]
    (um, vm, pm), divm, _ = res["mixed"]
    assert divm <= 1e-8 and div64 <= 1e-8
    assert np.abs(um - u64).max() <= 1e-6 and np.abs(vm - v64).max() <= 1e-6
    # both decay like exp(-2 nu t) to discretisation accuracy
    decay = np.exp(-2.0 * cfg.nu * t)
    xf, xc = cases.axis(cfg.lx, n)
    exact_u = np.sin(xf)[:, None] * np.cos(xc)[None, :] * decay
    assert np.abs(um[1:n + 2, 1:n + 1] - exact_u).max() < 2e-3
