"""Projection step, time loop and cylinder mask (oracle; test infrastructure).

Restates ``pycfd/core/solver.py`` (face sets :235-296, face solid flags :62-79,
``initialize`` :301-329, mask/direct forcing :553-599, periodic face wrap
:601-607, ``substep`` :612-640, ``project`` :643-683, ``step`` :686-731,
upwind blend :734-756), ``pycfd/core/timestepper.py`` (dt control :82-113,
health :122-142, ``run`` :145-248, diagnostics :251-266) and
``pycfd/geometry/obstacles.py:87-135`` (8x8 supersampled circle mask), for a
uniform mesh with constant viscosity.
"""

from __future__ import annotations

import time

import numpy as np

from .boundary import Walls, axis_coords
from .poisson import assemble_poisson, make_solver
from .stencil import momentum_rhs, divergence

VISCOUS_SAFETY_FACTOR = 0.8        # config.py:154
DIVERGENCE_VELOCITY_LIMIT = 1.0e6  # config.py:157
MIN_TIME_STEP = 1.0e-8             # config.py:160
QUIESCENT_VELOCITY_FLOOR = 1.0e-12  # config.py:164


class DivergenceError(RuntimeError):
    """timestepper.py:47."""


def _v(x):
    return getattr(x, "value", x)


def face_solid_mask(solid, lo, hi, axis, periodic):
    """Faces in ``[lo, hi)`` touching a solid cell -- solver.py:62-79."""
    m = np.arange(lo, hi)
    if periodic:
        n = solid.shape[axis]
        return np.take(solid, (m - 2) % n, axis=axis) | np.take(solid, (m - 1) % n, axis=axis)
    pad = [(0, 0), (0, 0)]
    pad[axis] = (1, 1)
    padded = np.pad(solid, pad, constant_values=False)
    return np.take(padded, m - 1, axis=axis) | np.take(padded, m, axis=axis)


def circle_mask_oracle(nx, ny, lx, ly, center, radius, subsamples=8):
    """Solid fraction by midpoint supersampling, threshold 0.5 -- obstacles.py:87-135."""
    xf, _ = axis_coords(lx, nx)
    yf, _ = axis_coords(ly, ny)
    dxc = np.full(nx, lx / nx)
    dyc = np.full(ny, ly / ny)
    offs = (np.arange(subsamples) + 0.5) / subsamples
    xs = (xf[:-1, None] + offs[None, :] * dxc[:, None]).ravel()
    ys = (yf[:-1, None] + offs[None, :] * dyc[:, None]).ravel()
    X, Y = np.meshgrid(xs, ys, indexing="ij")
    cx, cy = center
    hits = ((X - cx) ** 2 + (Y - cy) ** 2 <= radius ** 2).astype(float)
    frac = hits.reshape(nx, subsamples, ny, subsamples).mean(axis=(1, 3))
    return frac > 0.5


class OracleSolver:
    """CPU restatement of ``ProjectionSolver`` (uniform mesh, laminar)."""

    def __init__(self, config, solid=None, bodies=None, solver_kind=None):
        self.config = config
        nx, ny = config.nx, config.ny
        self.nx, self.ny = nx, ny
        self.dx, self.dy = config.lx / nx, config.ly / ny
        self.nu = config.u_ref * config.l_ref / config.re
        self.walls = Walls(config.boundary_config, nx, ny, config.lx, config.ly)
        self.periodic_x, self.periodic_y = self.walls.periodic_x, self.walls.periodic_y
        self.solid = np.zeros((nx, ny), bool) if solid is None else np.asarray(solid, bool)
        self.has_obstacle = bool(self.solid.any())
        self.body_masks = tuple(np.asarray(b, bool) for b in bodies) \
            if bodies is not None and len(bodies) > 1 else ()
        self._build_slices()
        self.dirichlet_pressure = self.walls.dirichlet()
        self.poisson = assemble_poisson(nx, ny, self.dx, self.dy, self.periodic_x,
                                        self.periodic_y,
                                        self.solid if self.has_obstacle else None,
                                        self.dirichlet_pressure or None)
        kind = solver_kind if solver_kind is not None else config.pressure_solver
        self.pressure_solver = make_solver(kind, self.poisson, config.poisson_tol,
                                           config.poisson_maxiter, config.sor_omega,
                                           config.mg_sweeps)
        self._p_guess = None
        self.body_force_reaction = (0.0, 0.0)
        self.body_force_reactions = tuple((0.0, 0.0) for _ in self.body_masks)
        self._blend = 0.0

    def _build_slices(self):
        """solver.py:235-296."""
        nx, ny = self.nx, self.ny
        k = self.walls.kinds
        out = "pressure_outlet"
        u_lo = 1 if (self.periodic_x or k["left"] == out) else 2
        u_hi = nx + 2 if (k["right"] == out and not self.periodic_x) else nx + 1
        v_lo = 1 if (self.periodic_y or k["bottom"] == out) else 2
        v_hi = ny + 2 if (k["top"] == out and not self.periodic_y) else ny + 1
        self.u_range, self.v_range = (u_lo, u_hi), (v_lo, v_hi)
        self.u_upd = (slice(u_lo, u_hi), slice(1, ny + 1))
        self.v_upd = (slice(1, nx + 1), slice(v_lo, v_hi))
        self.u_rhs_sel = slice(u_lo - 1, u_hi - 1)
        self.v_rhs_sel = slice(v_lo - 1, v_hi - 1)
        self.area = self.dx * self.dy
        if self.has_obstacle:
            self.u_face_solid = face_solid_mask(self.solid, u_lo, u_hi, 0, self.periodic_x)
            self.v_face_solid = face_solid_mask(self.solid, v_lo, v_hi, 1, self.periodic_y)
        else:
            self.u_face_solid = self.v_face_solid = None
        self.u_face_body = tuple(face_solid_mask(b, u_lo, u_hi, 0, self.periodic_x)
                                 for b in self.body_masks)
        self.v_face_body = tuple(face_solid_mask(b, v_lo, v_hi, 1, self.periodic_y)
                                 for b in self.body_masks)

    # ------------------------------------------------------------------ #
    def initialize(self, u_init=None, v_init=None):
        """solver.py:301-329; returns ``(u, v, p)``."""
        nx, ny = self.nx, self.ny
        u = np.zeros((nx + 3, ny + 2))
        v = np.zeros((nx + 2, ny + 3))
        if u_init is not None:
            u[1:nx + 2, 1:ny + 1] = u_init
        if v_init is not None:
            v[1:nx + 1, 1:ny + 2] = v_init
        self.walls.apply_velocity(u, v, predictor=True)
        self.walls.enforce_global_mass_balance(u, v)
        self.mask_obstacle(u, v, None)
        self.wrap_faces(u, v)
        p = self.project(u, v, 1.0)
        self.mask_obstacle(u, v, None)
        self.wrap_faces(u, v)
        self.walls.apply_velocity(u, v, predictor=False)
        return u, v, p

    def momentum_rhs(self, u, v, blend=0.0):
        fx, fy = self.config.body_force
        return momentum_rhs(u, v, self.dx, self.dy, self.nu, blend, fx, fy)

    def divergence(self, u, v):
        return divergence(u, v, self.dx, self.dy)

    def max_divergence(self, u, v):
        """solver.py:545-550."""
        d = self.divergence(u, v)
        if self.has_obstacle:
            d = d[~self.solid]
        return float(np.abs(d).max()) if d.size else 0.0

    def mask_obstacle(self, u, v, dt, reset=False):
        """Direct forcing with reaction force -- solver.py:553-599."""
        if not self.has_obstacle:
            return
        uf = u[self.u_upd]
        vf = v[self.v_upd]
        if dt is not None:
            fx = float(uf[self.u_face_solid].sum()) * self.area / dt
            fy = float(vf[self.v_face_solid].sum()) * self.area / dt
            if reset:
                self.body_force_reaction = (fx, fy)
            else:
                prev = self.body_force_reaction
                self.body_force_reaction = (prev[0] + fx, prev[1] + fy)
            if self.body_masks:
                per = tuple((float(uf[um].sum()) * self.area / dt,
                             float(vf[vm].sum()) * self.area / dt)
                            for um, vm in zip(self.u_face_body, self.v_face_body))
                if reset:
                    self.body_force_reactions = per
                else:
                    self.body_force_reactions = tuple(
                        (a[0] + b[0], a[1] + b[1])
                        for a, b in zip(self.body_force_reactions, per))
        uf[self.u_face_solid] = 0.0
        vf[self.v_face_solid] = 0.0

    def wrap_faces(self, u, v):
        """solver.py:601-607."""
        if self.periodic_x:
            u[self.nx + 1, :] = u[1, :]
        if self.periodic_y:
            v[:, self.ny + 1] = v[:, 1]

    def project(self, u, v, dt):
        """solver.py:643-683 (uniform mesh)."""
        nx, ny = self.nx, self.ny
        p_int = self.pressure_solver.solve(self.divergence(u, v) / dt, self._p_guess)
        if self.pressure_solver.warm_startable:
            self._p_guess = p_int
        p = np.zeros((nx + 2, ny + 2))
        p[1:nx + 1, 1:ny + 1] = p_int
        self.walls.apply_pressure(p)
        lo_u, hi_u = self.u_range
        lo_v, hi_v = self.v_range
        u[self.u_upd] -= dt * (p[lo_u:hi_u, 1:ny + 1] - p[lo_u - 1:hi_u - 1, 1:ny + 1]) / self.dx
        v[self.v_upd] -= dt * (p[1:nx + 1, lo_v:hi_v] - p[1:nx + 1, lo_v - 1:hi_v - 1]) / self.dy
        return p

    def substep(self, u, v, dt, blend=0.0):
        """solver.py:612-640."""
        rhs_u, rhs_v = self.momentum_rhs(u, v, blend)
        us, vs = u.copy(), v.copy()
        us[self.u_upd] += dt * rhs_u[self.u_rhs_sel, :]
        vs[self.v_upd] += dt * rhs_v[:, self.v_rhs_sel]
        self.walls.apply_velocity(us, vs, predictor=True)
        self.walls.enforce_global_mass_balance(us, vs)
        self.mask_obstacle(us, vs, dt, reset=True)
        self.wrap_faces(us, vs)
        p = self.project(us, vs, dt)
        self.mask_obstacle(us, vs, dt, reset=False)
        self.wrap_faces(us, vs)
        self.walls.apply_velocity(us, vs, predictor=False)
        return us, vs, p

    def step(self, u0, v0, dt):
        """solver.py:686-731; returns ``(u, v, p)``."""
        blend = self._blend
        scheme = _v(self.config.time_scheme)
        if scheme == "euler":
            u, v, p = self.substep(u0, v0, dt, blend)
        elif scheme == "rk2":
            u1, v1, _ = self.substep(u0, v0, dt, blend)
            u2, v2, p = self.substep(u1, v1, dt, blend)
            u = 0.5 * u0 + 0.5 * u2
            v = 0.5 * v0 + 0.5 * v2
        else:
            u1, v1, _ = self.substep(u0, v0, dt, blend)
            ue, ve, _ = self.substep(u1, v1, dt, blend)
            u2 = 0.75 * u0 + 0.25 * ue
            v2 = 0.75 * v0 + 0.25 * ve
            ue2, ve2, p = self.substep(u2, v2, dt, blend)
            u = (1.0 / 3.0) * u0 + (2.0 / 3.0) * ue2
            v = (1.0 / 3.0) * v0 + (2.0 / 3.0) * ve2
        if scheme != "euler":
            self.walls.apply_velocity(u, v, predictor=False)
            self.wrap_faces(u, v)
        return u, v, p

    def set_upwind_blend(self, blend):
        self._blend = float(np.clip(blend, 0.0, 1.0))

    def upwind_blend_for(self, u, v, dt):
        """solver.py:734-756."""
        if _v(self.config.advection_scheme) == "central":
            return 0.0
        if self.config.upwind_blend is not None:
            return self.config.upwind_blend
        umax, vmax = max_velocity(u, v, self.nx, self.ny)
        courant = max(umax * dt / self.dx, vmax * dt / self.dy)
        return float(min(1.0, 1.2 * courant))


def max_velocity(u, v, nx, ny):
    """fields.py:86-88."""
    return (float(np.abs(u[1:nx + 2, 1:ny + 1]).max()),
            float(np.abs(v[1:nx + 1, 1:ny + 2]).max()))


def kinetic_energy(u, v, nx, ny, area, mask=None):
    """postprocess.py:73-79 with fields.py:70-79."""
    uc = 0.5 * (u[1:nx + 1, 1:ny + 1] + u[2:nx + 2, 1:ny + 1])
    vc = 0.5 * (v[1:nx + 1, 1:ny + 1] + v[1:nx + 1, 2:ny + 2])
    e = 0.5 * (uc ** 2 + vc ** 2)
    if mask is not None:
        e = np.where(mask, 0.0, e)
    return float(np.sum(e)) * area


class OracleStepper:
    """CPU restatement of ``TimeStepper`` -- timestepper.py:72-266."""

    def __init__(self, solver):
        self.solver = solver
        self.config = solver.config
        nu = solver.nu
        dx, dy = solver.dx, solver.dy
        self.viscous_dt_limit = (float("inf") if nu <= 0 else
                                 VISCOUS_SAFETY_FACTOR / (2.0 * nu * (1.0 / dx ** 2 + 1.0 / dy ** 2)))

    def compute_dt(self, u, v):
        """timestepper.py:94-113."""
        if not self.config.adaptive_dt:
            return self.config.dt
        s = self.solver
        umax, vmax = max_velocity(u, v, s.nx, s.ny)
        scale = umax / s.dx + vmax / s.dy
        dt_conv = self.config.cfl_max / scale if scale > QUIESCENT_VELOCITY_FLOOR else float("inf")
        return float(min(dt_conv, self.viscous_dt_limit, self.config.dt))

    def check_health(self, u, v, p, dt, step):
        """timestepper.py:122-142."""
        s = self.solver
        if not (np.all(np.isfinite(u)) and np.all(np.isfinite(v)) and np.all(np.isfinite(p))):
            raise DivergenceError(f"non-finite values at step {step}")
        umax, vmax = max_velocity(u, v, s.nx, s.ny)
        if max(umax, vmax) > DIVERGENCE_VELOCITY_LIMIT:
            raise DivergenceError(f"solution diverged at step {step}")
        if dt < MIN_TIME_STEP:
            raise DivergenceError(f"adaptive time step collapsed to {dt:.3e}")

    def run(self, state, t_end=None, max_steps=None):
        """timestepper.py:145-248 without callbacks/progress; ``state = (u, v, p, t, step)``."""
        u, v, p, t, step = state
        s = self.solver
        t_end = self.config.t_end if t_end is None else t_end
        max_steps = self.config.max_steps if max_steps is None else max_steps
        hist = {k: [] for k in ("step", "t", "dt", "max_div", "kinetic_energy", "fx", "fy")}
        taken = 0
        converged = False
        wall0 = time.perf_counter()
        while t < t_end - 1e-12:
            if max_steps is not None and taken >= max_steps:
                break
            dt = self.compute_dt(u, v)
            self.check_health(u, v, p, dt, step)
            dt = min(dt, t_end - t)
            s.set_upwind_blend(s.upwind_blend_for(u, v, dt))
            un, vn, p = s.step(u, v, dt)
            taken += 1
            du = max(float(np.abs(un - u).max()), float(np.abs(vn - v).max()))
            u, v = un, vn
            t, step = t + dt, step + 1
            hist["step"].append(step)
            hist["t"].append(t)
            hist["dt"].append(dt)
            hist["max_div"].append(s.max_divergence(u, v))
            hist["kinetic_energy"].append(kinetic_energy(u, v, s.nx, s.ny, s.area))
            hist["fx"].append(s.body_force_reaction[0])
            hist["fy"].append(s.body_force_reaction[1])
            if self.config.steady_tol is not None and du / dt < self.config.steady_tol:
                converged = True
                break
        self.check_health(u, v, p, self.config.dt, step)
        return (u, v, p, t, step), dict(history=hist, steps=taken, converged=converged,
                                         wall=time.perf_counter() - wall0)
