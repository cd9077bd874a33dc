"""Immersed bodies as boolean cell masks (``pycfd/geometry/obstacles.py``).

The solid volume fraction of every cell is the mean of an S x S (default 8 x 8)
midpoint supersample of the body's inside test; a cell with fraction > 0.5 is
solid.  Sample coordinates are formed from the mesh's own face coordinates, so
the mask agrees bit for bit with the reference's on the same mesh.

Circles, rectangles, polygons and bitmap silhouettes are rasterised on the GPU
(``pycfd_rasterize``: one thread per cell counting its S*S hits) when a CUDA
device is present (``device="auto"``) or asked for (``device="cuda"``), on the
host with NumPy otherwise (``device="cpu"``); both give the same bits.  A
predicate given as a Python function (:func:`mask_from_function`) runs on the
host.  The solver consumes a mask through its face lists.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from pathlib import Path

import numpy as np

DEFAULT_SUBSAMPLES = 8
SOLID_FRACTION_THRESHOLD = 0.5
SHAPE_CIRCLE, SHAPE_RECTANGLE, SHAPE_POLYGON, SHAPE_IMAGE = 0, 1, 2, 3


@dataclass
class Obstacle:
    mask: np.ndarray
    fraction: np.ndarray
    characteristic_length: float
    name: str = "obstacle"

    @property
    def area(self) -> float:
        return float(self.fraction.sum())

    def __repr__(self) -> str:
        return (f"Obstacle({self.name!r}, {int(self.mask.sum())} solid cells, "
                f"L={self.characteristic_length:g})")


def solid_fraction(mesh, inside, subsamples: int = DEFAULT_SUBSAMPLES) -> np.ndarray:
    """Fraction of each cell where ``inside(X, Y)`` holds, on the host (``obstacles.py:87-103``)."""
    if subsamples < 1:
        raise ValueError(f"subsamples must be >= 1, got {subsamples}")
    s = (np.arange(subsamples) + 0.5) / subsamples
    X = (mesh.xf[:-1, None] + s[None, :] * mesh.dx_cells[:, None]).ravel()
    Y = (mesh.yf[:-1, None] + s[None, :] * mesh.dy_cells[:, None]).ravel()
    XX, YY = np.meshgrid(X, Y, indexing="ij")
    hit = inside(XX, YY).astype(float).reshape(mesh.nx, subsamples, mesh.ny, subsamples)
    return hit.mean(axis=(1, 3))


def _use_gpu(device) -> bool:
    if device == "cpu":
        return False
    if device == "cuda":
        return True
    if device != "auto":
        raise ValueError(f"device must be 'auto', 'cuda' or 'cpu', got {device!r}")
    try:
        import torch
    except ImportError:
        return False
    return torch.cuda.is_available()


def rasterize(mesh, kind: int, params=(0.0, 0.0, 0.0, 0.0), verts=None, image=None,
              threshold: float = 0.5, invert: bool = False, subsamples: int = DEFAULT_SUBSAMPLES):
    """Solid fraction and mask of one shape on the GPU (``pycfd_rasterize``);
    returns host ``(fraction, mask)`` arrays."""
    import torch
    from . import _lib
    L = _lib.load()
    if subsamples < 1:
        raise ValueError(f"subsamples must be >= 1, got {subsamples}")
    dev = torch.device("cuda", torch.cuda.current_device())
    d64 = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=dev)
    xf, dxc = d64(mesh.xf[:-1]), d64(mesh.dx_cells)
    yf, dyc = d64(mesh.yf[:-1]), d64(mesh.dy_cells)
    nx, ny = mesh.nx, mesh.ny
    frac = torch.empty((nx, ny), dtype=torch.float64, device=dev)
    mask = torch.empty((nx, ny), dtype=torch.uint8, device=dev)
    sh = _lib.Shape()
    sh.kind = int(kind)
    for k in range(4):
        sh.p[k] = float(params[k])
    keep = []
    if verts is not None:
        vt = d64(verts)
        keep.append(vt)
        sh.verts, sh.n_verts = vt.data_ptr(), int(vt.shape[0])
    if image is not None:
        it = d64(image)
        keep.append(it)
        sh.image, sh.rows, sh.cols = it.data_ptr(), int(it.shape[0]), int(it.shape[1])
        sh.threshold, sh.invert = float(threshold), int(bool(invert))
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    _lib.check(L.pycfd_rasterize(C.byref(sh), _lib.ptr(xf), _lib.ptr(dxc), _lib.ptr(yf), _lib.ptr(dyc),
                                 nx, ny, float(mesh.lx), float(mesh.ly), int(subsamples),
                                 _lib.ptr(frac), _lib.ptr(mask), stream))
    out = frac.cpu().numpy(), mask.cpu().numpy().astype(bool)
    del keep
    return out


def circle_mask(mesh, center, radius, subsamples: int = DEFAULT_SUBSAMPLES,
                name: str = "cylinder", device: str = "auto") -> Obstacle:
    """Circle of ``radius`` at ``center`` (``obstacles.py:106-135``)."""
    if radius <= 0:
        raise ValueError(f"radius must be positive, got {radius}")
    cx, cy = center
    if not (0 <= cx <= mesh.lx and 0 <= cy <= mesh.ly):
        raise ValueError(f"circle centre {center} lies outside the domain")
    if _use_gpu(device):
        frac, mask = rasterize(mesh, SHAPE_CIRCLE, (cx, cy, radius, 0.0), subsamples=subsamples)
    else:
        frac = solid_fraction(mesh, lambda X, Y: (X - cx) ** 2 + (Y - cy) ** 2 <= radius ** 2, subsamples)
        mask = frac > SOLID_FRACTION_THRESHOLD
    if not mask.any():
        raise ValueError(f"circle of radius {radius:g} does not cover a single cell on a "
                         f"{mesh.nx}x{mesh.ny} grid; refine the mesh or enlarge the obstacle")
    return Obstacle(mask, frac, 2.0 * radius, name)


def rectangle_mask(mesh, lower_left, upper_right, subsamples: int = DEFAULT_SUBSAMPLES,
                   name: str = "rectangle", device: str = "auto") -> Obstacle:
    """Axis-aligned rectangle (``obstacles.py:138-157``)."""
    x0, y0 = lower_left
    x1, y1 = upper_right
    if x1 <= x0 or y1 <= y0:
        raise ValueError(f"rectangle corners are degenerate: {lower_left} -> {upper_right}")
    if _use_gpu(device):
        frac, mask = rasterize(mesh, SHAPE_RECTANGLE, (x0, y0, x1, y1), subsamples=subsamples)
    else:
        frac = solid_fraction(mesh, lambda X, Y: (X >= x0) & (X <= x1) & (Y >= y0) & (Y <= y1),
                              subsamples)
        mask = frac > SOLID_FRACTION_THRESHOLD
    if not mask.any():
        raise ValueError("rectangle does not cover a single cell; refine the mesh")
    return Obstacle(mask, frac, y1 - y0, name)


def point_in_polygon(X, Y, verts) -> np.ndarray:
    """Even-odd ray test towards +x with a bounding-box pre-filter, on the host
    (``obstacles.py:160-192``)."""
    inside = np.zeros(X.shape, dtype=bool)
    xv, yv = verts[:, 0], verts[:, 1]
    box = (X >= xv.min()) & (X <= xv.max()) & (Y >= yv.min()) & (Y <= yv.max())
    if not box.any():
        return inside
    xs, ys = X[box], Y[box]
    hit = np.zeros(xs.shape, dtype=bool)
    for x0, y0, x1, y1 in zip(xv, yv, np.roll(xv, -1), np.roll(yv, -1)):
        straddles = (y0 > ys) != (y1 > ys)
        with np.errstate(divide="ignore", invalid="ignore"):
            xc = x0 + (ys - y0) * (x1 - x0) / (y1 - y0)
        hit ^= straddles & (xs < xc)
    inside[box] = hit
    return inside


def load_polygon(path) -> np.ndarray:
    """Closed outline from a text file of ``x, y`` pairs (``obstacles.py:195-234``):
    comma or blank separated, ``#`` comments, a repeated closing vertex dropped."""
    path = Path(path)
    if not path.exists():
        raise FileNotFoundError(f"geometry file not found: {path}")
    rows = []
    for lineno, raw in enumerate(path.read_text().splitlines(), start=1):
        line = raw.split("#", 1)[0].strip()
        if not line:
            continue
        parts = [p for p in line.replace(",", " ").split() if p]
        if len(parts) < 2:
            raise ValueError(f"{path}:{lineno}: expected two numbers 'x y', got {raw.strip()!r}")
        try:
            rows.append((float(parts[0]), float(parts[1])))
        except ValueError:
            raise ValueError(f"{path}:{lineno}: could not parse coordinates from {raw.strip()!r}") from None
    if len(rows) < 3:
        raise ValueError(f"{path}: a polygon needs at least 3 vertices, found {len(rows)}")
    verts = np.asarray(rows, dtype=float)
    if np.allclose(verts[0], verts[-1]):
        verts = verts[:-1]
    return verts


def transform_polygon(verts, scale: float = 1.0, center=None, rotate_deg: float = 0.0) -> np.ndarray:
    """Scale and rotate an outline about its centroid, then move the centroid to
    ``center`` (``obstacles.py:237-258``)."""
    verts = np.asarray(verts, dtype=float)
    if verts.ndim != 2 or verts.shape[1] != 2:
        raise ValueError(f"vertices must have shape (n, 2), got {verts.shape}")
    if scale <= 0:
        raise ValueError(f"scale must be positive, got {scale}")
    centroid = verts.mean(axis=0)
    local = (verts - centroid) * scale
    if rotate_deg:
        th = np.radians(rotate_deg)
        c, s = np.cos(th), np.sin(th)
        local = local @ np.array([[c, s], [-s, c]])
    return local + (centroid if center is None else np.asarray(center, dtype=float))


def polygon_mask(mesh, vertices, characteristic_length: float | None = None,
                 subsamples: int = DEFAULT_SUBSAMPLES, name: str = "polygon",
                 device: str = "auto") -> Obstacle:
    """Body from a closed outline in either winding order (``obstacles.py:261-305``);
    the characteristic length defaults to the outline's height."""
    verts = np.asarray(vertices, dtype=float)
    if verts.ndim != 2 or verts.shape[1] != 2 or len(verts) < 3:
        raise ValueError(f"vertices must be an (n, 2) array with n >= 3, got {verts.shape}")
    lo, hi = verts.min(axis=0), verts.max(axis=0)
    if hi[0] < 0 or lo[0] > mesh.lx or hi[1] < 0 or lo[1] > mesh.ly:
        raise ValueError(f"geometry bounding box x=[{lo[0]:g}, {hi[0]:g}] y=[{lo[1]:g}, {hi[1]:g}] lies "
                         f"entirely outside the domain [0, {mesh.lx:g}] x [0, {mesh.ly:g}]; reposition "
                         "it with transform_polygon()")
    if _use_gpu(device):
        frac, mask = rasterize(mesh, SHAPE_POLYGON, (lo[0], lo[1], hi[0], hi[1]), verts=verts,
                               subsamples=subsamples)
    else:
        frac = solid_fraction(mesh, lambda X, Y: point_in_polygon(X, Y, verts), subsamples)
        mask = frac > SOLID_FRACTION_THRESHOLD
    if not mask.any():
        raise ValueError(f"the outline does not cover a single cell on a {mesh.nx}x{mesh.ny} grid; "
                         "refine the mesh or scale the geometry up with transform_polygon()")
    length = float(hi[1] - lo[1]) if characteristic_length is None else float(characteristic_length)
    return Obstacle(mask, frac, length, name)


def image_luminance(img) -> np.ndarray:
    """A picture as the rasteriser reads it: RGB(A) reduced to the mean of its colour
    channels (alpha ignored), 8-bit values scaled to [0, 1], rows flipped so that row
    0 lies at y = 0 (``obstacles.py:327-335``)."""
    img = np.asarray(img, dtype=float)
    if img.ndim == 3:
        img = img[..., :3].mean(axis=2)
    if img.max() > 1.0:
        img = img / 255.0
    return img[::-1, :]


def _read_image(path):
    path = Path(path)
    if not path.exists():
        raise FileNotFoundError(f"geometry image not found: {path}")
    try:
        import matplotlib.image as mpimg
        return mpimg.imread(path)
    except ImportError:
        pass
    try:
        from PIL import Image
        return np.asarray(Image.open(path))
    except ImportError:
        raise ImportError("reading an image file needs matplotlib or Pillow; pass the pixel array "
                          "instead") from None


def mask_from_image(mesh, image, threshold: float = 0.5, invert: bool = False,
                    characteristic_length: float | None = None, subsamples: int = DEFAULT_SUBSAMPLES,
                    name: str = "image", device: str = "auto") -> Obstacle:
    """Body from a bitmap silhouette stretched over the whole domain
    (``obstacles.py:308-367``): dark pixels (luminance below ``threshold``) are
    solid, the opposite with ``invert``.  ``image`` is a file path or the pixel
    array (rows x cols, optionally x 3/4 channels, row 0 at the top)."""
    raw = _read_image(image) if isinstance(image, (str, Path)) else image
    img = image_luminance(raw)
    rows, cols = img.shape
    label = Path(image).name if isinstance(image, (str, Path)) else "the image"
    if _use_gpu(device):
        frac, mask = rasterize(mesh, SHAPE_IMAGE, image=img, threshold=threshold, invert=invert,
                               subsamples=subsamples)
    else:
        def inside(X, Y):
            col = np.clip((X / mesh.lx * cols).astype(int), 0, cols - 1)
            row = np.clip((Y / mesh.ly * rows).astype(int), 0, rows - 1)
            solid = img[row, col] < threshold
            return ~solid if invert else solid
        frac = solid_fraction(mesh, inside, subsamples)
        mask = frac > SOLID_FRACTION_THRESHOLD
    if not mask.any():
        raise ValueError(f"no cell of the {mesh.nx}x{mesh.ny} grid is solid after thresholding {label} "
                         f"at {threshold}; try a different threshold or invert=True")
    if mask.all():
        raise ValueError(f"every cell is solid after thresholding {label} at {threshold}; the image is "
                         "probably inverted (try invert=True)")
    if characteristic_length is None:
        used = np.flatnonzero(mask.any(axis=0))
        characteristic_length = float(mesh.dy_cells[used[0]:used[-1] + 1].sum())
    return Obstacle(mask, frac, float(characteristic_length), name)


def mask_from_function(mesh, inside, characteristic_length: float = 1.0,
                       subsamples: int = DEFAULT_SUBSAMPLES, name: str = "custom") -> Obstacle:
    """Body from a vectorised predicate ``inside(x, y)`` on NumPy arrays, on the host
    (``obstacles.py:370-396``)."""
    frac = solid_fraction(mesh, inside, subsamples)
    mask = frac > SOLID_FRACTION_THRESHOLD
    if not mask.any():
        raise ValueError(f"the predicate marks no cell solid on a {mesh.nx}x{mesh.ny} grid; check the "
                         "coordinates it expects are in domain units")
    return Obstacle(mask, frac, float(characteristic_length), name)


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
