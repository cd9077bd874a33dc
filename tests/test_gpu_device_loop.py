"""The time loop on the device against the host-driven loop (needs a B200).

With ``GpuOptions(device_loop=K)`` the step, its dt, the health checks, the
end-time clamp and the steady test run in a gated recorded step and the
per-step diagnostics land in a device history read every K steps
(pycfd/core/timestepper.py:145-266).  The dt formula and the step kernels are
the same as the host-driven loop's, so the two give the same bits: fields,
clock, history, steady-state stop, callback cadence and the DivergenceError.
"""

import numpy as np
import pytest

import cases
from pycfd_b200.config import BCKind, BCSpec, SimulationConfig

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _cfg(**kw):
    d = dict(nx=32, ny=24, lx=1.2, ly=1.0, re=150.0, dt=1.0, t_end=1e9, cfl_max=0.5, adaptive_dt=True,
             pressure_solver="mgcg", poisson_tol=1e-11, boundary_config=cases.bcs(top=("moving_wall", 1.0)),
             name="loop")
    d.update(kw)
    return cases.to_config(d, SimulationConfig, BCSpec, BCKind)


def _run(cfg, device_loop, **kw):
    from pycfd_b200.solver import GpuOptions, ProjectionSolver
    from pycfd_b200.timestepper import TimeStepper
    s = ProjectionSolver(cfg, options=GpuOptions(device_loop=device_loop))
    calls = []
    res = TimeStepper(s).run(s.initialize(), callback=lambda f, info: calls.append((f.step, f.t)), **kw)
    return res, calls, s


@pytest.mark.parametrize("window", [1, 8, 64])
def test_device_loop_matches_host_loop_bitwise(window):
    cfg = _cfg()
    a, ca, sa = _run(cfg, 0, max_steps=37, record_every=3, callback_every=5)
    b, cb, sb = _run(cfg, window, max_steps=37, record_every=3, callback_every=5)
    assert (a.steps, a.fields.step) == (b.steps, b.fields.step) == (37, 37) and a.time == b.time
    for x, y in zip(a.fields.numpy(), b.fields.numpy()):
        assert np.array_equal(x, y)
    for k in a.history:
        assert np.array_equal(np.asarray(a.history[k]), np.asarray(b.history[k])), k
    assert ca == cb and [c[0] for c in cb] == [5, 10, 15, 20, 25, 30, 35, 37]
    assert sa.body_force_reaction == sb.body_force_reaction
    assert sa.pressure_solver.last_residual == sb.pressure_solver.last_residual


def test_device_loop_lands_on_t_end_and_stops_when_steady():
    cfg = _cfg()
    a, _, _ = _run(cfg, 0, t_end=0.05)
    b, _, _ = _run(cfg, 16, t_end=0.05)
    assert a.time == b.time and a.steps == b.steps and abs(b.time - 0.05) < 1e-12
    for x, y in zip(a.fields.numpy(), b.fields.numpy()):
        assert np.array_equal(x, y)
    # a steady tolerance reached after some steps: both loops stop at the same step
    cs = _cfg(steady_tol=2.0)
    a, _, _ = _run(cs, 0, max_steps=400)
    b, _, _ = _run(cs, 32, max_steps=400)
    assert a.converged and b.converged and a.steps == b.steps < 400
    for x, y in zip(a.fields.numpy(), b.fields.numpy()):
        assert np.array_equal(x, y)


def test_device_loop_raises_divergence_error_at_the_last_good_step():
    from pycfd_b200.solver import GpuOptions, ProjectionSolver
    from pycfd_b200.timestepper import DivergenceError, TimeStepper
    cfg = _cfg(re=1e6, adaptive_dt=False, dt=5.0, boundary_config=cases.bcs(top=("moving_wall", 1e3)))
    msgs = []
    for loop in (0, 16):
        s = ProjectionSolver(cfg, options=GpuOptions(device_loop=loop))
        with pytest.raises(DivergenceError) as e:
            TimeStepper(s).run(s.initialize(), t_end=1e4, max_steps=100)
        msgs.append(str(e.value))
    assert msgs[0] == msgs[1]
