"""Uniform or geometrically stretched MAC mesh (``pycfd/core/mesh.py:236-529``).

Index convention (``pycfd/core/mesh.py:13-38``): ``p`` is ``(nx+2, ny+2)``,
``u`` is ``(nx+3, ny+2)``, ``v`` is ``(nx+2, ny+3)``; one ghost layer per side;
y is the contiguous axis.  Cell widths come from the geometric series of
``pycfd/core/mesh.py:271-311`` (ratio and cluster mode per axis), faces by
cumulative sum with the far face pinned, exactly as the reference builds them,
so initial conditions and masks sampled on them match bit for bit.  The metric
arrays of a stretched mesh (``pycfd/core/mesh.py:122-218``) are formed with the
reference's operations and handed to the device as one packed array.
"""

from __future__ import annotations

import numpy as np

#: Relative tolerance of the uniformity test (``pycfd/core/mesh.py:119``).
UNIFORMITY_RTOL = 1.0e-12
#: Where a stretched axis puts its smallest cells (``pycfd/core/mesh.py:236-252``).
CLUSTER_MODES = ("low", "walls", "centre")


class NonUniformMeshError(RuntimeError):
    """Raised when a uniform-spacing quantity is asked of a stretched mesh."""


def normalise_cluster(mode: str) -> str:
    mode = str(mode).lower()
    if mode == "center":
        return "centre"
    if mode not in CLUSTER_MODES:
        raise ValueError(f"cluster mode must be one of {CLUSTER_MODES}, got {mode!r}")
    return mode


def geometric_widths(length: float, n: int, ratio: float, cluster: str = "low") -> np.ndarray:
    """``n`` widths growing by ``ratio`` per cell, summing to ``length``
    (``pycfd/core/mesh.py:271-311``): smallest at the low end (``low``), at both
    ends (``walls``) or in the middle (``centre``); an odd count gets one
    unpaired middle cell continuing the series."""
    if ratio <= 0:
        raise ValueError(f"stretch ratio must be positive, got {ratio}")
    cluster = normalise_cluster(cluster)
    if abs(ratio - 1.0) < 1.0e-14:
        return np.full(n, length / n, dtype=float)
    if cluster == "low":
        first = length * (ratio - 1.0) / (ratio ** n - 1.0)
        return first * ratio ** np.arange(n, dtype=float)
    half, odd = divmod(n, 2)
    if cluster == "walls":
        grow = ratio ** np.arange(half, dtype=float)
        first = length / (2.0 * grow.sum() + odd * ratio ** half)
        grow = first * grow
        mid = [first * ratio ** half] if odd else []
        return np.concatenate([grow, mid, grow[::-1]])
    if odd:
        side = ratio ** np.arange(1, half + 1, dtype=float)
        first = length / (1.0 + 2.0 * side.sum())
        side = first * side
        return np.concatenate([side[::-1], [first], side])
    grow = ratio ** np.arange(half, dtype=float)
    grow = (length / (2.0 * grow.sum())) * grow
    return np.concatenate([grow[::-1], grow])


def _faces(widths: np.ndarray, length: float):
    faces = np.concatenate(([0.0], np.cumsum(widths)))
    faces[-1] = length
    return faces, 0.5 * (faces[:-1] + faces[1:])


class MeshMetrics:
    """The spacings the staggered operators divide by (``pycfd/core/mesh.py:122-218``):
    scalars on a uniform mesh, arrays (shaped to broadcast against the
    ``(nx, ny)`` blocks) on a stretched one.

    hx, hy: cell widths/heights; hxu, hyv: centre-to-centre distances across each
    face, the ghost cell mirroring its neighbour; hx_ext, hy_ext: widths with
    that ghost at each end; wx_corner, wy_corner: weight of the upper node when a
    cell-centred value is interpolated to a corner."""

    def __init__(self, mesh: "StructuredMesh") -> None:
        dxc, dyc = mesh.dx_cells, mesh.dy_cells
        hx_ext = np.concatenate(([dxc[0]], dxc, [dxc[-1]]))
        hy_ext = np.concatenate(([dyc[0]], dyc, [dyc[-1]]))
        hxu = 0.5 * (hx_ext[:-1] + hx_ext[1:])
        hyv = 0.5 * (hy_ext[:-1] + hy_ext[1:])
        wx = 0.5 * hx_ext[:-1] / hxu
        wy = 0.5 * hy_ext[:-1] / hyv
        self.cell_areas = dxc[:, None] * dyc[None, :]
        self.min_hx = float(dxc.min())
        self.min_hy = float(dyc.min())
        self.uniform_area = float(dxc[0] * dyc[0]) if mesh.is_uniform else None
        if mesh.is_uniform:
            self.hx = self.hxu = self.hx_ext = float(dxc[0])
            self.hy = self.hyv = self.hy_ext = float(dyc[0])
            self.wx_corner = self.wy_corner = 0.5
        else:
            self.hx, self.hy = dxc[:, None], dyc[None, :]
            self.hxu, self.hyv = hxu[:, None], hyv[None, :]
            self.hx_ext, self.hy_ext = hx_ext[:, None], hy_ext[None, :]
            self.wx_corner, self.wy_corner = wx[:, None], wy[None, :]
        # flat copies for the device (packed by `device_block`)
        self._flat = dict(hx=dxc, hy=dyc, hxu=hxu, hyv=hyv, hx_ext=hx_ext, hy_ext=hy_ext,
                          wx=wx, wy=wy)

    def integrate(self, field) -> float:
        """Domain integral of a cell-centred field (``pycfd/core/mesh.py:209-218``)."""
        if self.uniform_area is not None:
            return float(np.sum(field)) * self.uniform_area
        return float(np.sum(field * self.cell_areas))

    def device_block(self) -> np.ndarray:
        """The packed metric array the device reads on a stretched mesh, in the
        order of ``pcfd::Metrics`` (csrc/common.cuh): hx, hy, hxu, hyv, hx_ext,
        hy_ext, wx, wy, then the Poisson face denominators hxu*vbar and
        hyv*vbar (``pycfd/core/pressure.py:197-206``) and the mean cell area
        vbar (one element)."""
        f = self._flat
        vbar = float(self.cell_areas.mean())
        return np.ascontiguousarray(np.concatenate(
            [f["hx"], f["hy"], f["hxu"], f["hyv"], f["hx_ext"], f["hy_ext"], f["wx"], f["wy"],
             f["hxu"] * vbar, f["hyv"] * vbar, [vbar]]), dtype=np.float64)


class StructuredMesh:
    """Uniform or stretched structured mesh on ``[0, lx] x [0, ly]`` with ``nx x ny``
    cells (``pycfd/core/mesh.py:312-529``)."""

    def __init__(self, nx: int, ny: int, lx: float = 1.0, ly: float = 1.0,
                 stretch_x: float = 1.0, stretch_y: float = 1.0, cluster_x: str = "low",
                 cluster_y: str = "low", **_ignored) -> None:
        if nx < 4 or ny < 4:
            raise ValueError(f"mesh must be at least 4x4 cells, got {nx}x{ny}")
        if lx <= 0 or ly <= 0:
            raise ValueError(f"domain extents must be positive, got {lx}x{ly}")
        self.nx, self.ny = int(nx), int(ny)
        self.lx, self.ly = float(lx), float(ly)
        self.stretch_x, self.stretch_y = float(stretch_x), float(stretch_y)
        self.cluster_x, self.cluster_y = normalise_cluster(cluster_x), normalise_cluster(cluster_y)
        self.dx_cells = geometric_widths(self.lx, self.nx, self.stretch_x, self.cluster_x)
        self.dy_cells = geometric_widths(self.ly, self.ny, self.stretch_y, self.cluster_y)
        self.xf, self.xc = _faces(self.dx_cells, self.lx)
        self.yf, self.yc = _faces(self.dy_cells, self.ly)
        self._sx = not bool(np.allclose(self.dx_cells, self.dx_cells[0], rtol=UNIFORMITY_RTOL))
        self._sy = not bool(np.allclose(self.dy_cells, self.dy_cells[0], rtol=UNIFORMITY_RTOL))
        self._dx = float(self.dx_cells[0])
        self._dy = float(self.dy_cells[0])
        self._metrics = None

    @property
    def is_uniform(self) -> bool:
        return not (self._sx or self._sy)

    @property
    def stretched_x(self) -> bool:
        return self._sx

    @property
    def stretched_y(self) -> bool:
        return self._sy

    def require_uniform(self, who: str = "operator") -> None:
        if not self.is_uniform:
            raise NonUniformMeshError(
                f"{who} is discretised for uniform spacing but the mesh is stretched "
                f"(stretch_x={self.stretch_x}, stretch_y={self.stretch_y}). Use stretch_x = stretch_y = 1.0.")

    @property
    def dx(self) -> float:
        if not self.is_uniform:
            self.require_uniform("StructuredMesh.dx")
        return self._dx

    @property
    def dy(self) -> float:
        if not self.is_uniform:
            self.require_uniform("StructuredMesh.dy")
        return self._dy

    @property
    def cell_area(self) -> float:
        return self._dx * self._dy

    @property
    def metrics(self) -> MeshMetrics:
        if self._metrics is None:
            self._metrics = MeshMetrics(self)
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
        if self.is_uniform:
            return (f"StructuredMesh({self.nx}x{self.ny} cells, domain [0,{self.lx:g}]x[0,{self.ly:g}], "
                    f"uniform, dx={self.dx:.6g}, dy={self.dy:.6g})")
        return (f"StructuredMesh({self.nx}x{self.ny} cells, domain [0,{self.lx:g}]x[0,{self.ly:g}], "
                f"stretched, stretch=({self.stretch_x:g}, {self.stretch_y:g}), "
                f"cluster=({self.cluster_x}, {self.cluster_y}))")

    @classmethod
    def from_config(cls, cfg) -> "StructuredMesh":
        return cls(cfg.nx, cfg.ny, cfg.lx, cfg.ly, cfg.stretch_x, cfg.stretch_y,
                   getattr(cfg, "cluster_x", "low"), getattr(cfg, "cluster_y", "low"))
