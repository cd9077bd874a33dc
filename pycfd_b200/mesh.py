"""Uniform MAC mesh: coordinates and array shapes (``pycfd/core/mesh.py:258-529``).

Index convention (``pycfd/core/mesh.py:13-38``): ``p`` is ``(nx+2, ny+2)``,
``u`` is ``(nx+3, ny+2)``, ``v`` is ``(nx+2, ny+3)``; one ghost layer per side;
y is the contiguous axis.  Face coordinates are built by cumulative sum with
the far face pinned, exactly as the reference builds them, so initial
conditions and masks sampled on them match bit for bit.  The GPU path is
discretised for uniform spacing only; a stretched configuration is refused.
"""

from __future__ import annotations

import numpy as np


class NonUniformMeshError(RuntimeError):
    """Raised when the uniform-spacing GPU path is handed a stretched mesh."""


def _axis(length: float, n: int):
    faces = np.concatenate(([0.0], np.cumsum(np.full(n, length / n, dtype=float))))
    faces[-1] = length
    return faces, 0.5 * (faces[:-1] + faces[1:])


class _Metrics:
    """The scalar spacings of a uniform mesh (``pycfd/core/mesh.py:122-233``)."""

    def __init__(self, mesh: "StructuredMesh") -> None:
        self.hx = self.hxu = self.hx_ext = mesh.dx
        self.hy = self.hyv = self.hy_ext = mesh.dy
        self.min_hx, self.min_hy = mesh.dx, mesh.dy
        self.wx_corner = self.wy_corner = 0.5
        self.uniform_area = mesh.dx * mesh.dy
        self.cell_areas = np.full((mesh.nx, mesh.ny), self.uniform_area)

    def integrate(self, field) -> float:
        return float(np.sum(field)) * self.uniform_area


class StructuredMesh:
    """Uniform structured mesh on ``[0, lx] x [0, ly]`` with ``nx x ny`` cells."""

    def __init__(self, nx: int, ny: int, lx: float = 1.0, ly: float = 1.0,
                 stretch_x: float = 1.0, stretch_y: float = 1.0, **_ignored) -> None:
        if nx < 4 or ny < 4:
            raise ValueError(f"mesh must be at least 4x4 cells, got {nx}x{ny}")
        if lx <= 0 or ly <= 0:
            raise ValueError(f"domain extents must be positive, got {lx}x{ly}")
        if abs(stretch_x - 1.0) > 1e-14 or abs(stretch_y - 1.0) > 1e-14:
            raise NotImplementedError(
                "the GPU projection path is discretised for uniform spacing; stretched "
                f"meshes (stretch_x={stretch_x}, stretch_y={stretch_y}) are not provided")
        self.nx, self.ny = int(nx), int(ny)
        self.lx, self.ly = float(lx), float(ly)
        self.stretch_x = self.stretch_y = 1.0
        self.dx_cells = np.full(self.nx, self.lx / self.nx)
        self.dy_cells = np.full(self.ny, self.ly / self.ny)
        self.xf, self.xc = _axis(self.lx, self.nx)
        self.yf, self.yc = _axis(self.ly, self.ny)
        self._dx = float(self.dx_cells[0])
        self._dy = float(self.dy_cells[0])
        self._metrics = None

    is_uniform = True
    stretched_x = stretched_y = False

    @property
    def dx(self) -> float:
        return self._dx

    @property
    def dy(self) -> float:
        return self._dy

    @property
    def cell_area(self) -> float:
        return self._dx * self._dy

    @property
    def metrics(self) -> _Metrics:
        if self._metrics is None:
            self._metrics = _Metrics(self)
        return self._metrics

    @property
    def shape(self):
        return (self.nx, self.ny)

    @property
    def n_cells(self) -> int:
        return self.nx * self.ny

    @property
    def u_shape(self):
        return (self.nx + 3, self.ny + 2)

    @property
    def v_shape(self):
        return (self.nx + 2, self.ny + 3)

    @property
    def p_shape(self):
        return (self.nx + 2, self.ny + 2)

    def cell_centers(self):
        return self.xc, self.yc

    def face_centers(self):
        return self.xf, self.yf

    def u_coords(self):
        return self.xf, self.yc

    def v_coords(self):
        return self.xc, self.yf

    def cell_center_grid(self):
        return np.meshgrid(self.xc, self.yc, indexing="ij")

    def u_grid(self):
        return np.meshgrid(self.xf, self.yc, indexing="ij")

    def v_grid(self):
        return np.meshgrid(self.xc, self.yf, indexing="ij")

    def zeros_u(self):
        return np.zeros(self.u_shape)

    def zeros_v(self):
        return np.zeros(self.v_shape)

    def zeros_p(self):
        return np.zeros(self.p_shape)

    def __repr__(self) -> str:
        return (f"StructuredMesh({self.nx}x{self.ny} cells, domain [0,{self.lx:g}]x[0,{self.ly:g}], "
                f"uniform, dx={self.dx:.6g}, dy={self.dy:.6g})")

    @classmethod
    def from_config(cls, cfg) -> "StructuredMesh":
        return cls(cfg.nx, cfg.ny, cfg.lx, cfg.ly, cfg.stretch_x, cfg.stretch_y)
