"""Host set-up of the Poisson operator and its multigrid hierarchy.

Runs once per solver, before anything is uploaded.  The fine operator is
assembled in CSR (the device applies it matrix-free; the CSR form seeds the
Galerkin products), then the smoothed-aggregation hierarchy of
``pycfd/core/multigrid.py`` is built level by level with the same rules --
seeded power-iteration weight, anisotropy-driven coarsening, 2x2 blocks with
singleton leftovers, one damped-Jacobi pass over the 0/1 prolongator,
``A_c = P^T A P`` with identity on dropped aggregates, stop at <= 96 unknowns
or when a level shrinks by less than 1.3x -- and handed to the library as CSR
blocks plus the dense pseudo-inverse of the coarsest operator.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
import scipy.sparse as sp

COARSEST_UNKNOWNS = 96
MAX_LEVELS = 20
MIN_COARSENING_RATIO = 1.3
JACOBI_WEIGHT_FACTOR = 4.0 / 3.0
POWER_ITERATIONS = 12
ANISOTROPY_THRESHOLD = 2.0


@dataclass
class FineOperator:
    """The assembled fine Poisson operator (``pycfd/core/pressure.py:69-94``)."""

    A: sp.csr_matrix
    shape: tuple
    fluid: np.ndarray        # solvable rows, flat
    singular: bool
    pin: int
    bc_rhs: np.ndarray
    row_scale: np.ndarray | float = 1.0   # cell area / mean cell area (1.0 on a uniform mesh)


def assemble(nx, ny, dx, dy, periodic_x, periodic_y, solid=None, dirichlet=None,
             widths=None) -> FineOperator:
    """5-point operator over the projected face set (``pycfd/core/pressure.py:110-270``).

    Couplings are gathered per face direction with index arithmetic; the
    diagonal accumulates the directions in the order left, right, bottom, top,
    Dirichlet walls adding ``-2 c`` in place, which reproduces the reference's
    matrix exactly.  ``widths = (dx_cells, dy_cells)`` of a stretched mesh: each
    face's coefficient is its area over the centre-to-centre distance and the
    mean cell area, and the rows carry the cell area over the mean as their
    scale (``pycfd/core/pressure.py:193-207``).
    """
    n = nx * ny
    fluid = np.ones((nx, ny), bool) if solid is None else ~np.asarray(solid, bool)
    dirichlet = dict(dirichlet or {})
    ii, jj = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    cid = ii * ny + jj
    diag = np.zeros((nx, ny))
    bc = np.zeros((nx, ny))
    rows, cols, vals = [], [], []
    if widths is None:
        cx, cy = 1.0 / (dx * dx), 1.0 / (dy * dy)
        coef = (cx, cx, cy, cy)
        row_scale = 1.0
    else:
        dxc, dyc = (np.asarray(w, dtype=float) for w in widths)
        areas = dxc[:, None] * dyc[None, :]
        vbar = float(areas.mean())
        hxu = 0.5 * (np.concatenate(([dxc[0]], dxc)) + np.concatenate((dxc, [dxc[-1]])))
        hyv = 0.5 * (np.concatenate(([dyc[0]], dyc)) + np.concatenate((dyc, [dyc[-1]])))
        cxf = dyc[None, :] / (hxu[:, None] * vbar)     # (nx+1, ny), by x-face
        cyf = dxc[:, None] / (hyv[None, :] * vbar)     # (nx, ny+1), by y-face
        coef = (cxf[0:nx, :], cxf[1:nx + 1, :], cyf[:, 0:ny], cyf[:, 1:ny + 1])
        row_scale = (areas / vbar).ravel()
    for (wall, di, dj, per), c in zip((("left", -1, 0, periodic_x), ("right", 1, 0, periodic_x),
                                       ("bottom", 0, -1, periodic_y), ("top", 0, 1, periodic_y)), coef):
        ni, nj = ii + di, jj + dj
        inside = (ni >= 0) & (ni < nx) & (nj >= 0) & (nj < ny)
        if per:
            inside[:] = True
        ni, nj = ni % nx, nj % ny
        coupled = fluid & inside & fluid[ni, nj]
        rows.append(cid[coupled])
        cols.append((ni * ny + nj)[coupled])
        vals.append(np.full(int(coupled.sum()), c) if np.isscalar(c) else c[coupled])
        diag -= c * coupled
        if wall in dirichlet:
            on_wall = fluid & ~inside
            diag -= 2.0 * c * on_wall
            bc -= 2.0 * c * dirichlet[wall] * on_wall
    solvable = fluid & (diag != 0.0)
    diag = np.where(solvable, diag, 1.0)
    bc = np.where(solvable, bc, 0.0)
    rows.append(cid.ravel())
    cols.append(cid.ravel())
    vals.append(diag.ravel())
    A = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                      shape=(n, n))
    A.sum_duplicates()
    flat = solvable.ravel()
    pin = int(np.argmax(flat)) if flat.any() else 0
    return FineOperator(A, (nx, ny), flat.copy(), not dirichlet, pin, bc.ravel(), row_scale)


@dataclass
class MgLevelHost:
    n: int
    shape: tuple
    weight: float
    weighted_dinv: np.ndarray
    active: np.ndarray
    A: sp.csr_matrix
    P: sp.csr_matrix | None = None
    arrays: list = field(default_factory=list)   # keeps ctypes-backed buffers alive
    tails: dict = field(default_factory=dict)    # dense cycle operators from this level, by sweeps


def _rho(A, dinv):
    """Power-iteration estimate of rho(D^-1 A), x1.05 (``pycfd/core/multigrid.py:129-157``)."""
    n = A.shape[0]
    if n == 0:
        return 1.0
    v = np.random.default_rng(0).standard_normal(n)
    nv = float(np.linalg.norm(v))
    if nv == 0.0:
        return 1.0
    v = v / nv
    est = 1.0
    for _ in range(POWER_ITERATIONS):
        w = dinv * (A @ v)
        nw = float(np.linalg.norm(w))
        if nw == 0.0:
            return est
        est = nw
        v = w / nw
    return est * 1.05


def _factors(A, shape):
    """Axis coarsening factors from the mean band strengths (``multigrid.py:167-204``)."""
    nx, ny = shape
    if nx < 2 and ny < 2:
        return 1, 1
    band = lambda k: float(np.abs(A.diagonal(k)).mean()) if k < A.shape[0] and A.diagonal(k).size else 0.0
    sx, sy = band(ny), band(1)
    if nx >= 2 and sx > ANISOTROPY_THRESHOLD * sy:
        return 2, 1
    if ny >= 2 and sy > ANISOTROPY_THRESHOLD * sx:
        return 1, 2
    return (2 if nx >= 2 else 1), (2 if ny >= 2 else 1)


def _level(A, shape, active, P):
    d = A.diagonal()
    dinv = 1.0 / np.where(d == 0.0, 1.0, d)
    rho = _rho(A, dinv)
    w = JACOBI_WEIGHT_FACTOR / rho if rho > 0.0 else 1.0
    return MgLevelHost(A.shape[0], tuple(shape), w, w * dinv, active, A, P), dinv


def build_hierarchy(op: FineOperator):
    """Levels (finest first) and the coarsest pseudo-inverse (row-major)."""
    lv, dinv = _level(op.A, op.shape, op.fluid.copy(), None)
    levels = [lv]
    while len(levels) < MAX_LEVELS and lv.n > COARSEST_UNKNOWNS:
        fx, fy = _factors(lv.A, lv.shape)
        nx, ny = lv.shape
        ncx, ncy = max(-(-nx // fx), 1), max(-(-ny // fy), 1)
        nc = ncx * ncy
        if nc == 0 or lv.n < MIN_COARSENING_RATIO * nc:
            break
        ii, jj = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
        agg = ((ii // fx) * ncy + (jj // fy)).ravel()
        rows = np.flatnonzero(lv.active)
        T = sp.csr_matrix((np.ones(rows.size), (rows, agg[rows])), shape=(lv.n, nc))
        cact = np.zeros(nc, bool)
        cact[agg[rows]] = True
        P = (T - sp.diags(lv.weight * dinv) @ (lv.A @ T)).tocsr()
        Ac = sp.csr_matrix(P.T @ lv.A @ P)
        if not cact.all():
            Ac = (Ac + sp.diags((~cact).astype(float))).tocsr()
        Ac.sum_duplicates()
        lv, dinv = _level(Ac, (ncx, ncy), cact, P)
        levels.append(lv)
    return levels, coarsest_pseudo_inverse(levels[-1], op.singular)


def coarsest_pseudo_inverse(level: MgLevelHost, singular: bool) -> np.ndarray:
    """Dense matrix of the coarsest solve (``pycfd/core/multigrid.py:514-543``).

    The reference pins one unknown, factorises, and removes the mean before and
    after; that map is linear in the right-hand side, so it is materialised
    column by column here and applied on the device as one small mat-vec.
    """
    n = level.n
    act = level.active
    M = level.A.toarray()
    pin = int(np.argmax(act)) if act.any() else 0
    if singular and n:
        M[pin, :] = 0.0
        M[pin, pin] = 1.0
    Minv = np.linalg.inv(M)
    E = np.eye(n)
    if singular:
        E[~act, :] = 0.0
        E[act, :] -= E[act, :].mean(axis=0)
        E[pin, :] = 0.0
    X = Minv @ E
    X[~act, :] = 0.0
    if singular and act.any():
        X[act, :] -= X[act, :].mean(axis=0)
    return np.ascontiguousarray(X)


# Levels of at most this many rows may close the V-cycle as one dense operator.
TAIL_MAX_ROWS = 2048


def tail_level(levels, ratio: float | None = None) -> int:
    """First level above the coarsest (index >= 1) with at most TAIL_MAX_ROWS rows, or 0.

    ``ratio``: also require n_l^2 <= ratio * n_0, so the dense operator's bytes stay
    within a few fine-level vectors (for many small solves sharing the GPU, where
    bytes count more than launches).
    """
    n0 = levels[0].n
    for l in range(1, len(levels) - 1):
        n = levels[l].n
        if n <= TAIL_MAX_ROWS and (ratio is None or n * n <= ratio * n0):
            return l
    return 0


def tail_operator(levels, cinv: np.ndarray, t: int, sweeps: int) -> np.ndarray:
    """Dense matrix of the V-cycle from level ``t`` down, as a map of its right-hand side.

    From a zero start the part of the cycle at and below a level -- damped-
    Jacobi sweeps, restriction, the coarser levels, the coarsest pseudo-inverse,
    prolongation and the sweeps back up (``pycfd/core/multigrid.py:430-474``) --
    is linear in that level's right-hand side b, so it equals one matrix M with
    x = M b.  M is built here by running those steps on the identity (columns
    of b at once); the device then replaces the phases below ``t`` by one mat-
    vec.  Row-major, ``n_t x n_t``.
    """
    def cycle(l, B):
        lv = levels[l]
        W = np.asarray(lv.weighted_dinv)[:, None]
        A = lv.A
        x = W * B
        for _ in range(1, sweeps):
            x = x + W * (B - A @ x)
        res = B - A @ x
        nxt = levels[l + 1]
        bc = nxt.P.T @ res
        xc = cinv @ bc if l + 1 == len(levels) - 1 else cycle(l + 1, bc)
        x = x + nxt.P @ xc
        for _ in range(sweeps):
            x = x + W * (B - A @ x)
        return x
    return np.ascontiguousarray(cycle(t, np.eye(levels[t].n)))


def fused_restriction(levels, l: int) -> sp.csr_matrix:
    """``R_l (I - A_{l-1} W_{l-1})``: from a zero start, the first damped-Jacobi
    sweep on level l-1 (x = W b) and the restriction of its residual b - A x
    (``pycfd/core/multigrid.py:436-447``) are one linear map of b onto level l."""
    f = levels[l - 1]
    A = f.A.tocsr()
    W = sp.diags(np.asarray(f.weighted_dinv))
    M = (levels[l].P.T.tocsr() @ (sp.identity(A.shape[0], format="csr") - A @ W)).tocsr()
    M.sort_indices()
    return M


def tail_for(levels, cinv: np.ndarray, sweeps: int, ratio: float | None = None):
    """``(level, operator)`` closing the V-cycle of this hierarchy, or ``(0, None)``;
    built once per hierarchy, sweep count and level."""
    t = tail_level(levels, ratio)
    if t == 0:
        return 0, None
    ops = levels[t].tails
    if sweeps not in ops:
        ops[sweeps] = tail_operator(levels, cinv, t, sweeps)
    return t, ops[sweeps]


def fused_for(levels, t: int):
    """Fused restrictions onto levels 1..t (one sweep per level), built once."""
    out = []
    for l in range(1, t + 1):
        ops = levels[l].tails
        if "M" not in ops:
            ops["M"] = fused_restriction(levels, l)
        out.append(ops["M"])
    return out


_CACHE: dict = {}
_CACHE_ORDER: list = []
_CACHE_MAX = 8


def hierarchy_for(nx, ny, dx, dy, periodic_x, periodic_y, solid=None, dirichlet=None, widths=None):
    """``(fine operator, (levels, coarsest inverse))`` of one Poisson structure.

    The hierarchy is a deterministic function of the assembled operator, so
    problems that share grid, spacing, periodicity, Dirichlet walls and solid
    mask share one build (kept for the last few structures of the process).
    """
    key = (nx, ny, dx, dy, bool(periodic_x), bool(periodic_y),
           tuple(sorted((dirichlet or {}).items())),
           None if solid is None else np.asarray(solid, bool).tobytes(),
           None if widths is None else tuple(np.asarray(w, float).tobytes() for w in widths))
    hit = _CACHE.get(key)
    if hit is None:
        op = assemble(nx, ny, dx, dy, periodic_x, periodic_y, solid, dirichlet, widths)
        hit = _CACHE[key] = (op, build_hierarchy(op))
        _CACHE_ORDER.append(key)
        while len(_CACHE_ORDER) > _CACHE_MAX:
            _CACHE.pop(_CACHE_ORDER.pop(0), None)
    return hit
