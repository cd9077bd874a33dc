"""Boundary passes of the MAC grid (oracle; test infrastructure).

Restates ``pycfd/core/boundary.py``: the per-wall normal/ghost/tangential
assignments of ``BoundaryCondition.apply`` (:141-164) with the overrides of each
condition (:175-333), the periodic wrap (:388-420), the pressure ghosts
(:166-169, :293-303) and the outlet mass balance (:423-487).  Walls are applied
in the fixed order left, right, bottom, top, line by line, exactly as the
reference does -- corner ghost values depend on that order.
"""

from __future__ import annotations

import numpy as np

WALL_ORDER = ("left", "right", "bottom", "top")
_MIN_OUTFLOW_FLUX = 1.0e-12          # boundary.py:44


def _kind(spec):
    k = spec.kind
    return getattr(k, "value", k)


def wall_index(wall, nx, ny):
    """``(axis, n_face, n_in, n_ghost, t_ghost, t_in, p_ghost, p_in, outward)`` -- boundary.py:69-80."""
    if wall == "left":
        return (0, 1, 2, 0, 0, 1, 0, 1, -1)
    if wall == "right":
        return (0, nx + 1, nx, nx + 2, nx + 1, nx, nx + 1, nx, +1)
    if wall == "bottom":
        return (1, 1, 2, 0, 0, 1, 0, 1, -1)
    if wall == "top":
        return (1, ny + 1, ny, ny + 2, ny + 1, ny, ny + 1, ny, +1)
    raise ValueError(wall)


def axis_coords(length, n):
    """Face and centre coordinates of a uniform axis -- mesh.py:355-366.

    Built by cumulative sum with the far face pinned, as the reference does, so
    the coordinates carry the same last-bit rounding.
    """
    faces = np.concatenate(([0.0], np.cumsum(np.full(n, length / n, dtype=float))))
    faces[-1] = length
    return faces, 0.5 * (faces[:-1] + faces[1:])


def _get(a, axis, i):
    return a[i, :] if axis == 0 else a[:, i]


def _put(a, axis, i, val):
    if axis == 0:
        a[i, :] = val
    else:
        a[:, i] = val


class Walls:
    """The four wall conditions of a case plus the periodic flags."""

    def __init__(self, boundary_config, nx, ny, lx, ly):
        self.nx, self.ny, self.lx, self.ly = nx, ny, lx, ly
        self.specs = {w: boundary_config[w] for w in WALL_ORDER}
        self.kinds = {w: _kind(self.specs[w]) for w in WALL_ORDER}
        self.periodic_x = self.kinds["left"] == "periodic"
        self.periodic_y = self.kinds["bottom"] == "periodic"
        self.outlets = [w for w in WALL_ORDER if self.kinds[w] == "outlet"]
        self.dx, self.dy = lx / nx, ly / ny
        self.xf, self.xc = axis_coords(lx, nx)
        self.yf, self.yc = axis_coords(ly, ny)

    # -- boundary.py:141-164 with the per-kind hooks ----------------------- #
    def _normal_value(self, wall, wi, normal):
        kind = self.kinds[wall]
        spec = self.specs[wall]
        axis, n_face, n_in = wi[0], wi[1], wi[2]
        if kind == "inlet":                                  # boundary.py:203-215
            speed = -wi[8] * spec.velocity
            if spec.profile == "uniform":
                return speed
            coord, extent = (self.yc, self.ly) if axis == 0 else (self.xc, self.lx)
            prof = 4.0 * coord * (extent - coord) / extent ** 2
            full = np.zeros(normal.shape[1] if axis == 0 else normal.shape[0])
            full[1:1 + coord.size] = speed * prof
            return full
        if kind in ("outlet", "pressure_outlet"):           # boundary.py:234-236
            return _get(normal, axis, n_in).copy()
        return 0.0

    def _tangential_ghost(self, wall, wi, tang):
        kind = self.kinds[wall]
        t_in = _get(tang, wi[0], wi[5])
        if kind == "moving_wall":                            # boundary.py:189-192
            return 2.0 * self.specs[wall].velocity - t_in
        if kind in ("outlet", "pressure_outlet", "symmetry"):  # :238-241, :311-313
            return t_in.copy()
        return -t_in                                          # no-slip / inlet

    def apply_velocity(self, u, v, predictor=True):
        """``BoundaryManager.apply_velocity`` -- boundary.py:375-379."""
        for wall in WALL_ORDER:
            kind = self.kinds[wall]
            if kind == "periodic":
                continue
            wi = wall_index(wall, self.nx, self.ny)
            axis = wi[0]
            normal, tang = (u, v) if axis == 0 else (v, u)
            prescribes = kind != "pressure_outlet"
            derives = kind == "outlet"
            if prescribes and (predictor or not derives):
                _put(normal, axis, wi[1], self._normal_value(wall, wi, normal))
            if kind == "pressure_outlet":                    # boundary.py:288-290
                ghost = _get(normal, axis, wi[1]).copy()
            else:                                            # boundary.py:136-139
                ghost = 2.0 * _get(normal, axis, wi[1]) - _get(normal, axis, wi[2])
            _put(normal, axis, wi[3], ghost)
            _put(tang, axis, wi[4], self._tangential_ghost(wall, wi, tang))
        self.wrap_velocity(u, v)

    def wrap_velocity(self, u, v):
        """boundary.py:388-410."""
        nx, ny = self.nx, self.ny
        if self.periodic_x:
            u[nx + 1, :] = u[1, :]
            u[0, :] = u[nx, :]
            u[nx + 2, :] = u[2, :]
            v[0, :] = v[nx, :]
            v[nx + 1, :] = v[1, :]
        if self.periodic_y:
            v[:, ny + 1] = v[:, 1]
            v[:, 0] = v[:, ny]
            v[:, ny + 2] = v[:, 2]
            u[:, 0] = u[:, ny]
            u[:, ny + 1] = u[:, 1]

    def apply_pressure(self, p):
        """boundary.py:381-385 with :166-169 and :293-303, then :412-420."""
        for wall in WALL_ORDER:
            kind = self.kinds[wall]
            if kind == "periodic":
                continue
            wi = wall_index(wall, self.nx, self.ny)
            inner = _get(p, wi[0], wi[7])
            if kind == "pressure_outlet":
                _put(p, wi[0], wi[6], 2.0 * self.specs[wall].p_ref - inner)
            else:
                _put(p, wi[0], wi[6], inner)
        nx, ny = self.nx, self.ny
        if self.periodic_x:
            p[0, :] = p[nx, :]
            p[nx + 1, :] = p[1, :]
        if self.periodic_y:
            p[:, 0] = p[:, ny]
            p[:, ny + 1] = p[:, 1]

    def enforce_global_mass_balance(self, u, v):
        """boundary.py:423-487 (uniform mesh)."""
        if not self.outlets:
            return
        nx, ny = self.nx, self.ny
        widths = (self.dy, self.dx)
        influx = 0.0
        outflux = 0.0
        faces = []
        for wall in WALL_ORDER:
            if self.kinds[wall] == "periodic":
                continue
            wi = wall_index(wall, nx, ny)
            normal = u if wi[0] == 0 else v
            line = _get(normal, wi[0], wi[1])
            face = line[1:ny + 1] if wi[0] == 0 else line[1:nx + 1]
            width = widths[wi[0]]
            flux_out = wi[8] * (float(face.sum()) * width)
            if wall in self.outlets:
                outflux += flux_out
                faces.append((face, width, wi[8]))
            else:
                influx -= flux_out
        if not faces:
            return
        if outflux > _MIN_OUTFLOW_FLUX:
            scale = influx / outflux
            for face, _, _ in faces:
                face *= scale
        else:
            total = sum(face.size * width for face, width, _ in faces)
            deficit = influx - outflux
            for face, _, outward in faces:
                face += outward * deficit / total

    def dirichlet(self):
        """Walls holding the pressure fixed -- boundary.py:494-500."""
        return {w: self.specs[w].p_ref for w in WALL_ORDER
                if self.kinds[w] == "pressure_outlet"}
