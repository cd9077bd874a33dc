"""Time loop with adaptive dt, health checks and history (``pycfd/core/timestepper.py``).

Same control flow and formulas as the reference: ``dt = min(cfl/(umax/dx +
vmax/dy), 0.8/(2 nu (1/dx^2+1/dy^2)), cfg.dt)`` from the *exact* device maxima,
health on the un-clamped dt, the clamp that lands on ``t_end``, the steady-state
test on ``max|du|/dt``.  The per-step reductions run as one fused kernel whose
handful of scalars is the only device-to-host traffic of a step.
"""

from __future__ import annotations

import logging
import time
from dataclasses import dataclass, field
from typing import Callable

from .config import (DIVERGENCE_VELOCITY_LIMIT, MIN_TIME_STEP, QUIESCENT_VELOCITY_FLOOR,
                     VISCOUS_SAFETY_FACTOR)
from .fields import FlowField

log = logging.getLogger(__name__)


class DivergenceError(RuntimeError):
    """Raised when the solution blows up or produces non-finite values."""


@dataclass
class SimulationResult:
    fields: FlowField
    steps: int
    time: float
    wall_time: float
    converged: bool = False
    history: dict = field(default_factory=dict)

    def summary(self) -> str:
        rate = self.steps / self.wall_time if self.wall_time > 0 else float("nan")
        status = "steady state reached" if self.converged else "end time reached"
        return (f"{status}: {self.steps} steps, t = {self.time:.4f}, "
                f"{self.wall_time:.2f} s wall ({rate:.0f} steps/s)")


class TimeStepper:
    """Runs a GPU :class:`~pycfd_b200.solver.ProjectionSolver` forward in time."""

    def __init__(self, solver, config=None) -> None:
        self.solver = solver
        self.config = config if config is not None else solver.config
        self.mesh = solver.mesh
        self.viscous_dt_limit = self._viscous_limit()

    def _viscous_limit(self) -> float:
        nu = self.solver.nu
        if nu <= 0:
            return float("inf")
        dx, dy = self.mesh.metrics.min_hx, self.mesh.metrics.min_hy   # the smallest cell
        return VISCOUS_SAFETY_FACTOR / (2.0 * nu * (1.0 / dx ** 2 + 1.0 / dy ** 2))

    def _stats(self, fields: FlowField):
        if fields._stats is None:
            fields._stats = self.solver.field_stats(fields)
        return fields._stats

    def compute_dt(self, fields: FlowField) -> float:
        if not self.config.adaptive_dt:
            return self.config.dt
        st = self._stats(fields)
        m = self.mesh.metrics
        scale = st.max_u / m.min_hx + st.max_v / m.min_hy
        dt_conv = self.config.cfl_max / scale if scale > QUIESCENT_VELOCITY_FLOOR else float("inf")
        return float(min(dt_conv, self.viscous_dt_limit, self.config.dt))

    def cfl_number(self, fields: FlowField, dt: float) -> float:
        st = self._stats(fields)
        m = self.mesh.metrics
        return float(dt * (st.max_u / m.min_hx + st.max_v / m.min_hy))

    def _check_health(self, fields: FlowField, dt: float) -> None:
        st = self._stats(fields)
        if not st.finite:
            raise DivergenceError(
                f"non-finite values at step {fields.step} (t = {fields.t:.6g}). The most common "
                "causes are a time step above the stability limit and a Reynolds number too high "
                "for the grid; try adaptive_dt=True, a smaller cfl_max, or advection_scheme='upwind'.")
        if max(st.max_u, st.max_v) > DIVERGENCE_VELOCITY_LIMIT:
            raise DivergenceError(
                f"solution diverged at step {fields.step} (t = {fields.t:.6g}): max|u| = "
                f"{st.max_u:.3e}, max|v| = {st.max_v:.3e} exceeds the limit "
                f"{DIVERGENCE_VELOCITY_LIMIT:.0e}.")
        if dt < MIN_TIME_STEP:
            raise DivergenceError(
                f"adaptive time step collapsed to {dt:.3e} (< {MIN_TIME_STEP:.0e}) at step "
                f"{fields.step}; the solution is probably diverging.")

    def run(self, fields: FlowField, t_end: float | None = None, max_steps: int | None = None,
            callback: Callable | None = None, callback_every: int = 50, progress: bool = False,
            record_every: int = 1) -> SimulationResult:
        """Integrate until ``t_end`` (``pycfd/core/timestepper.py:145-248``)."""
        t_end = self.config.t_end if t_end is None else t_end
        max_steps = self.config.max_steps if max_steps is None else max_steps
        if self._device_loop() > 0:
            return self._run_device(fields, t_end, max_steps, callback, callback_every, progress,
                                    record_every)
        history = {k: [] for k in ("step", "t", "dt", "cfl", "max_div", "kinetic_energy",
                                   "residual", "fx", "fy")}
        bar = None
        if progress:
            # a bar over simulated time, as the reference shows (timestepper.py:174-181)
            try:
                from tqdm.auto import tqdm
                bar = tqdm(total=float(t_end), initial=float(fields.t), unit="s",
                           desc=self.config.name, dynamic_ncols=True)
            except ImportError:
                log.warning("tqdm not installed; running without a progress bar")
        wall_start = time.perf_counter()
        converged = False
        steps_taken = 0
        try:
            while fields.t < t_end - 1e-12:
                if max_steps is not None and steps_taken >= max_steps:
                    break
                dt = self.compute_dt(fields)
                self._check_health(fields, dt)
                dt = min(dt, t_end - fields.t)
                self.solver.set_upwind_blend(self.solver.upwind_blend_for(fields, dt))
                previous = fields
                fields = self.solver.advance(previous, dt)
                steps_taken += 1
                st = self.solver.field_stats(fields, previous)
                fields._stats = st
                rate_of_change = max(st.max_du, st.max_dv) / dt
                if steps_taken % record_every == 0:
                    info = self._diagnostics(fields, dt, rate_of_change)
                    for k, val in info.items():
                        if k in history:
                            history[k].append(val)
                    fields.diagnostics = info
                if callback is not None and steps_taken % callback_every == 0:
                    callback(fields, fields.diagnostics or self._diagnostics(fields, dt, rate_of_change))
                if bar is not None:
                    bar.update(float(dt))
                if self.config.steady_tol is not None and rate_of_change < self.config.steady_tol:
                    converged = True
                    break
            self._check_health(fields, self.config.dt)
        finally:
            if bar is not None:
                bar.close()
        wall = time.perf_counter() - wall_start
        if callback is not None:
            callback(fields, fields.diagnostics or self._diagnostics(fields, self.config.dt,
                                                                     float("nan")))
        result = SimulationResult(fields, steps_taken, fields.t, wall, converged, history)
        log.info(result.summary())
        return result

    # ------------------------------------------------------------------ #
    def _device_loop(self) -> int:
        from .config import PressureSolver
        opts = getattr(self.solver, "options", None)
        k = int(getattr(opts, "device_loop", 0) or 0)
        kind = PressureSolver(self.config.pressure_solver)
        if k <= 0 or kind in (PressureSolver.SOR, PressureSolver.JACOBI):
            return 0
        return min(k, 4096)

    def _run_device(self, fields, t_end, max_steps, callback, callback_every, progress, record_every):
        """The run loop with the step, its dt, health checks, end-time clamp and steady
        test on the device (one recorded, gated step per step), the per-step
        diagnostics kept in a device history read every ``device_loop`` steps (and
        at each callback step)."""
        from .solver import dt_control_for
        K = self._device_loop()
        keys = ("step", "t", "dt", "cfl", "max_div", "kinetic_energy", "residual", "fx", "fy")
        names = keys + ("rate_of_change",)
        history = {k: [] for k in keys}
        bar = None
        if progress:
            try:
                from tqdm.auto import tqdm
                bar = tqdm(total=float(t_end), initial=float(fields.t), unit="s",
                           desc=self.config.name, dynamic_ncols=True)
            except ImportError:
                log.warning("tqdm not installed; running without a progress bar")
        s = self.solver
        ctl = dt_control_for(self.config, self.mesh, t_end, history=True)
        s.set_clock(fields.t)
        wall_start = time.perf_counter()
        converged = False
        steps_taken = 0
        step0 = fields.step
        cur = fields
        frozen = 0
        try:
            while frozen == 0 and fields.t < t_end - 1e-12:
                n = K
                if max_steps is not None:
                    n = min(n, max_steps - steps_taken)
                if callback is not None:
                    n = min(n, callback_every - steps_taken % callback_every)
                if n <= 0:
                    break
                outs = []
                for _ in range(n):
                    cur = s.advance_adaptive(cur, ctl)
                    outs.append(cur)
                rows, frozen = s.read_history()
                done = len(rows)
                if done == 0 and frozen == 0:
                    raise RuntimeError("the device run loop took no step and reported no stop reason")
                if done:
                    cur = outs[done - 1]
                    fields = FlowField(self.mesh, cur.u, cur.v, cur.p, float(rows[-1][1]),
                                       step0 + int(rows[-1][0]))
                    s._read_stats(raise_on_error=False)
                    if bar is not None:
                        bar.update(float(rows[:, 2].sum()))
                else:
                    cur = fields      # the gate refused the window's first step
                for r in rows:
                    k = int(r[0])
                    if k % record_every == 0:
                        info = dict(zip(names, (float(x) for x in r)))
                        info["step"] = step0 + k
                        for key in keys:
                            history[key].append(info[key])
                        fields.diagnostics = info
                steps_taken += done
                if frozen == 1:
                    fields._stats = None
                    self._check_health(fields, self.compute_dt(fields))
                    raise DivergenceError(f"the device health check stopped the run at step {fields.step}")
                if callback is not None and done and steps_taken % callback_every == 0:
                    callback(fields, fields.diagnostics or self._diagnostics(fields, float(rows[-1][2]),
                                                                              float(rows[-1][9])))
                if frozen == 3:
                    converged = True
            fields = FlowField(self.mesh, fields.u.clone(), fields.v.clone(), fields.p.clone(), fields.t,
                               fields.step, fields.diagnostics)
            self._check_health(fields, self.config.dt)
        finally:
            if bar is not None:
                bar.close()
        wall = time.perf_counter() - wall_start
        if callback is not None:
            callback(fields, fields.diagnostics or self._diagnostics(fields, self.config.dt, float("nan")))
        result = SimulationResult(fields, steps_taken, fields.t, wall, converged, history)
        log.info(result.summary())
        return result

    def _diagnostics(self, fields: FlowField, dt: float, rate_of_change: float) -> dict:
        """``pycfd/core/timestepper.py:251-266`` from the fused reduction."""
        st = self._stats(fields)
        fx, fy = self.solver.body_force_reaction
        return {"step": fields.step, "t": fields.t, "dt": dt, "cfl": self.cfl_number(fields, dt),
                "max_div": st.max_div, "kinetic_energy": st.kinetic_energy,
                "residual": self.solver.pressure_solver.last_residual,
                "rate_of_change": rate_of_change, "fx": fx, "fy": fy}
