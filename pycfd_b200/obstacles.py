"""Immersed bodies as boolean cell masks (``pycfd/geometry/obstacles.py``).

The solid volume fraction of every cell is the mean of an 8x8 midpoint
supersample of the body's inside test; a cell with fraction > 0.5 is solid.
Sample coordinates are formed from the mesh's own face coordinates, so the
mask agrees bit for bit with the reference's on the same mesh.  Masks are
host set-up; the device consumes them through the solver's face lists.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

DEFAULT_SUBSAMPLES = 8
SOLID_FRACTION_THRESHOLD = 0.5


@dataclass
class Obstacle:
    mask: np.ndarray
    fraction: np.ndarray
    characteristic_length: float
    name: str = "obstacle"

    @property
    def area(self) -> float:
        return float(self.fraction.sum())


def solid_fraction(mesh, inside, subsamples: int = DEFAULT_SUBSAMPLES) -> np.ndarray:
    """Fraction of each cell where ``inside(X, Y)`` holds (``obstacles.py:87-103``)."""
    if subsamples < 1:
        raise ValueError(f"subsamples must be >= 1, got {subsamples}")
    s = (np.arange(subsamples) + 0.5) / subsamples
    X = (mesh.xf[:-1, None] + s[None, :] * mesh.dx_cells[:, None]).ravel()
    Y = (mesh.yf[:-1, None] + s[None, :] * mesh.dy_cells[:, None]).ravel()
    XX, YY = np.meshgrid(X, Y, indexing="ij")
    hit = inside(XX, YY).astype(float).reshape(mesh.nx, subsamples, mesh.ny, subsamples)
    return hit.mean(axis=(1, 3))


def circle_mask(mesh, center, radius, subsamples: int = DEFAULT_SUBSAMPLES,
                name: str = "cylinder") -> Obstacle:
    """Circle of ``radius`` at ``center`` (``obstacles.py:106-135``)."""
    if radius <= 0:
        raise ValueError(f"radius must be positive, got {radius}")
    cx, cy = center
    if not (0 <= cx <= mesh.lx and 0 <= cy <= mesh.ly):
        raise ValueError(f"circle centre {center} lies outside the domain")
    frac = solid_fraction(mesh, lambda X, Y: (X - cx) ** 2 + (Y - cy) ** 2 <= radius ** 2, subsamples)
    mask = frac > SOLID_FRACTION_THRESHOLD
    if not mask.any():
        raise ValueError(f"circle of radius {radius:g} does not cover a single cell")
    return Obstacle(mask, frac, 2.0 * radius, name)


def rectangle_mask(mesh, lower_left, upper_right, subsamples: int = DEFAULT_SUBSAMPLES,
                   name: str = "rectangle") -> Obstacle:
    """Axis-aligned rectangle (``obstacles.py:138-157``)."""
    x0, y0 = lower_left
    x1, y1 = upper_right
    if x1 <= x0 or y1 <= y0:
        raise ValueError(f"rectangle corners are degenerate: {lower_left} -> {upper_right}")
    frac = solid_fraction(mesh, lambda X, Y: (X >= x0) & (X <= x1) & (Y >= y0) & (Y <= y1),
                          subsamples)
    mask = frac > SOLID_FRACTION_THRESHOLD
    if not mask.any():
        raise ValueError("rectangle does not cover a single cell; refine the mesh")
    return Obstacle(mask, frac, y1 - y0, name)


class ObstacleGroup:
    """Several bodies, each reporting its own force (``obstacles.py:445-614``)."""

    def __init__(self, members, name: str = "") -> None:
        self.members = tuple(members)
        if not self.members:
            raise ValueError("an ObstacleGroup needs at least one body")
        shapes = {m.mask.shape for m in self.members}
        if len(shapes) != 1:
            raise ValueError("every body must be built on the same mesh")
        self.name = name or " + ".join(m.name for m in self.members)
        labels = self.labels()
        for a in range(len(self.members)):
            for b in range(a + 1, len(self.members)):
                if np.any(self.members[a].mask & self.members[b].mask):
                    raise ValueError(f"bodies {self.members[a].name!r} and "
                                     f"{self.members[b].name!r} overlap")
        for axis in (0, 1):
            lo = np.take(labels, np.arange(labels.shape[axis] - 1), axis=axis)
            hi = np.take(labels, np.arange(1, labels.shape[axis]), axis=axis)
            if np.any((lo >= 0) & (hi >= 0) & (lo != hi)):
                raise ValueError("two bodies touch along a face; leave a fluid cell between them")

    def labels(self) -> np.ndarray:
        out = np.full(self.members[0].mask.shape, -1, dtype=int)
        for k, m in enumerate(self.members):
            out[m.mask] = k
        return out

    @property
    def masks(self):
        return tuple(m.mask for m in self.members)

    @property
    def names(self):
        return tuple(m.name for m in self.members)

    @property
    def mask(self) -> np.ndarray:
        out = np.zeros(self.members[0].mask.shape, dtype=bool)
        for m in self.members:
            out |= m.mask
        return out

    @property
    def characteristic_length(self) -> float:
        return max(m.characteristic_length for m in self.members)

    def __len__(self) -> int:
        return len(self.members)


def as_obstacle_group(obstacle):
    """Normalise an obstacle argument (``obstacles.py:617-638``)."""
    if obstacle is None:
        return None
    if isinstance(obstacle, ObstacleGroup):
        return obstacle
    if isinstance(obstacle, Obstacle):
        return ObstacleGroup((obstacle,), name=obstacle.name)
    members = tuple(obstacle)
    return ObstacleGroup(members) if members else None
