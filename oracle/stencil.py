"""Momentum right-hand side and divergence on the MAC grid (oracle; test infrastructure).

Restates ``pycfd/core/kernels.py:39-110`` (``_momentum_rhs_body``) as whole-array
NumPy expressions with the same operations in the same order, so the result is
bit-identical to the reference's Numba kernel and to its NumPy twin
(``pycfd/core/solver.py:360-465``, pinned equal by the reference's own
``tests/test_solver.py:410-430``).

Layout (``pycfd/core/mesh.py:13-38``): ``u`` is ``(nx+3, ny+2)``, ``v`` is
``(nx+2, ny+3)``, ``p`` is ``(nx+2, ny+2)``, C order with ``y`` fastest.
"""

from __future__ import annotations

import numpy as np


def momentum_rhs(u, v, dx, dy, nu, blend, fx, fy):
    """``-A(u) + nu*lap(u) + f`` on u-faces ``(nx+1, ny)`` and v-faces ``(nx, ny+1)``.

    Follows ``pycfd/core/kernels.py:50-110`` term by term.
    """
    nx = u.shape[0] - 3
    ny = u.shape[1] - 2
    dx2 = dx * dx
    dy2 = dy * dy

    # u-momentum, faces m = 1..nx+1, rows j = 1..ny   (kernels.py:53-80)
    c = u[1:nx + 2, 1:ny + 1]
    e = u[2:nx + 3, 1:ny + 1]
    w = u[0:nx + 1, 1:ny + 1]
    n = u[1:nx + 2, 2:ny + 2]
    s = u[1:nx + 2, 0:ny]
    u_right = 0.5 * (c + e)
    u_left = 0.5 * (w + c)
    duudx = (u_right * u_right - u_left * u_left) / dx
    u_top = 0.5 * (c + n)
    v_top = 0.5 * (v[0:nx + 1, 2:ny + 2] + v[1:nx + 2, 2:ny + 2])
    u_bot = 0.5 * (s + c)
    v_bot = 0.5 * (v[0:nx + 1, 1:ny + 1] + v[1:nx + 2, 1:ny + 1])
    duvdy = (u_top * v_top - u_bot * v_bot) / dy
    if blend > 0.0:
        duudx = duudx + blend / dx * (np.abs(u_right) * (c - e) * 0.5
                                      - np.abs(u_left) * (w - c) * 0.5)
        duvdy = duvdy + blend / dy * (np.abs(v_top) * (c - n) * 0.5
                                      - np.abs(v_bot) * (s - c) * 0.5)
    lap = ((w - 2.0 * c + e) / dx2 + (s - 2.0 * c + n) / dy2)
    rhs_u = -(duudx + duvdy) + nu * lap + fx

    # v-momentum, faces n = 1..ny+1, columns i = 1..nx   (kernels.py:83-110)
    c = v[1:nx + 1, 1:ny + 2]
    n = v[1:nx + 1, 2:ny + 3]
    s = v[1:nx + 1, 0:ny + 1]
    e = v[2:nx + 2, 1:ny + 2]
    w = v[0:nx, 1:ny + 2]
    v_top = 0.5 * (c + n)
    v_bot = 0.5 * (s + c)
    dvvdy = (v_top * v_top - v_bot * v_bot) / dy
    u_right = 0.5 * (u[2:nx + 2, 0:ny + 1] + u[2:nx + 2, 1:ny + 2])
    v_right = 0.5 * (c + e)
    u_left = 0.5 * (u[1:nx + 1, 0:ny + 1] + u[1:nx + 1, 1:ny + 2])
    v_left = 0.5 * (w + c)
    duvdx = (u_right * v_right - u_left * v_left) / dx
    if blend > 0.0:
        dvvdy = dvvdy + blend / dy * (np.abs(v_top) * (c - n) * 0.5
                                      - np.abs(v_bot) * (s - c) * 0.5)
        duvdx = duvdx + blend / dx * (np.abs(u_right) * (c - e) * 0.5
                                      - np.abs(u_left) * (w - c) * 0.5)
    lap = ((w - 2.0 * c + e) / dx2 + (s - 2.0 * c + n) / dy2)
    rhs_v = -(duvdx + dvvdy) + nu * lap + fy
    return rhs_u, rhs_v


def divergence(u, v, dx, dy):
    """Cell divergence ``(nx, ny)`` -- ``pycfd/core/solver.py:532-543`` (uniform mesh)."""
    nx = u.shape[0] - 3
    ny = u.shape[1] - 2
    return ((u[2:nx + 2, 1:ny + 1] - u[1:nx + 1, 1:ny + 1]) / dx
            + (v[1:nx + 1, 2:ny + 2] - v[1:nx + 1, 1:ny + 1]) / dy)
