"""Smoothed-aggregation multigrid hierarchy and V-cycle (oracle; test infrastructure).

Restates ``pycfd/core/multigrid.py``: damped-Jacobi weight ``(4/3)/rho`` with
``rho`` from 12 power iterations seeded ``default_rng(0)`` times 1.05
(:129-157), anisotropy-driven coarsening factors (:167-204), 2x2 block
aggregation with singleton leftovers (:212-245), tentative and smoothed
prolongators (:248-273), Galerkin ``P^T A P`` with identity on inactive rows
(:276-287, :364-395), the symmetric V-cycle (:424-474), the coarsest
pseudo-inverse by a pinned LU (:514-543) and the stall-guarded standalone loop
(:481-511).  SciPy sparse products and ``splu`` are used as black boxes.
"""

from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

COARSEST_UNKNOWNS = 96            # multigrid.py:93
MAX_LEVELS = 20                   # :98
MIN_COARSENING_RATIO = 1.3        # :103
JACOBI_WEIGHT_FACTOR = 4.0 / 3.0  # :108
POWER_ITERATIONS = 12             # :113
STALL_FACTOR = 0.995              # :119
STALL_PATIENCE = 3                # :123
ANISOTROPY_THRESHOLD = 2.0        # :164


def spectral_radius(A, dinv, seed=0):
    """multigrid.py:129-157."""
    n = A.shape[0]
    if n == 0:
        return 1.0
    x = np.random.default_rng(seed).standard_normal(n)
    norm = float(np.linalg.norm(x))
    if norm == 0.0:
        return 1.0
    x /= norm
    rho = 1.0
    for _ in range(POWER_ITERATIONS):
        y = dinv * (A @ x)
        norm = float(np.linalg.norm(y))
        if norm == 0.0:
            return rho
        rho = norm
        x = y / norm
    return rho * 1.05


def coarsening_factors(A, shape):
    """multigrid.py:167-204."""
    nx, ny = shape
    if nx < 2 and ny < 2:
        return 1, 1

    def strength(offset):
        if offset >= A.shape[0]:
            return 0.0
        band = np.abs(A.diagonal(offset))
        return float(band.mean()) if band.size else 0.0

    sx, sy = strength(ny), strength(1)
    if nx >= 2 and sx > ANISOTROPY_THRESHOLD * sy:
        return 2, 1
    if ny >= 2 and sy > ANISOTROPY_THRESHOLD * sx:
        return 1, 2
    return (2 if nx >= 2 else 1), (2 if ny >= 2 else 1)


def coarse_shape(shape, factors):
    """multigrid.py:207-209."""
    return tuple(max(-(-n // f), 1) for n, f in zip(shape, factors))


def aggregate_blocks(shape, active, factors):
    """multigrid.py:212-245."""
    nx, ny = shape
    fx, fy = factors
    ncx, ncy = coarse_shape(shape, factors)
    i, j = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    block = ((i // fx) * ncy + (j // fy)).ravel()
    labels = np.where(np.asarray(active).ravel(), block, -1)
    coarse_active = np.zeros(ncx * ncy, dtype=bool)
    coarse_active[labels[labels >= 0]] = True
    return labels, coarse_active


class Level:
    """One rung of the hierarchy -- multigrid.py:293-321."""

    def __init__(self, A, shape, active, singular, P):
        self.A = A
        self.shape = shape
        self.active = active
        self.singular = singular
        self.P = P
        diag = A.diagonal()
        self.dinv = 1.0 / np.where(diag == 0.0, 1.0, diag)
        rho = spectral_radius(A, self.dinv)
        self.weight = JACOBI_WEIGHT_FACTOR / rho if rho > 0.0 else 1.0
        self.weighted_dinv = self.weight * self.dinv
        self.lu = None
        self.pin = 0

    @property
    def n(self):
        return self.A.shape[0]


class Hierarchy:
    """multigrid.py:324-511."""

    def __init__(self, A, shape, active, singular, presmooth=1, postsmooth=1):
        if presmooth < 1 or postsmooth < 1 or presmooth != postsmooth:
            raise ValueError("a symmetric V-cycle needs equal sweeps >= 1")
        self.presmooth, self.postsmooth = presmooth, postsmooth
        self.levels = []
        A = sp.csr_matrix(A)
        active = np.asarray(active, bool).ravel()
        level = Level(A, tuple(shape), active, bool(singular), None)
        self.levels.append(level)
        while len(self.levels) < MAX_LEVELS and level.n > COARSEST_UNKNOWNS:
            fx, fy = coarsening_factors(level.A, level.shape)
            labels, coarse_active = aggregate_blocks(level.shape, level.active, (fx, fy))
            next_shape = coarse_shape(level.shape, (fx, fy))
            n_coarse = coarse_active.size
            if n_coarse == 0 or level.n < MIN_COARSENING_RATIO * n_coarse:
                break
            rows = np.flatnonzero(labels >= 0)
            T = sp.coo_matrix((np.ones(rows.size), (rows, labels[rows])),
                              shape=(labels.size, n_coarse)).tocsr()
            P = (T - sp.diags(level.weight * level.dinv) @ (level.A @ T)).tocsr()
            Ac = sp.csr_matrix(P.T @ level.A @ P)
            if not coarse_active.all():
                Ac = (Ac + sp.diags((~coarse_active).astype(float))).tocsr()
            Ac.sum_duplicates()
            level = Level(Ac, next_shape, coarse_active, bool(singular), P)
            self.levels.append(level)
        last = self.levels[-1]
        last.pin = int(np.flatnonzero(last.active)[0]) if last.active.any() else 0
        M = last.A
        if last.singular and M.shape[0]:
            M = M.tolil(copy=True)
            M.rows[last.pin] = [last.pin]
            M.data[last.pin] = [1.0]
            M = M.tocsr()
        last.lu = spla.splu(sp.csc_matrix(M))

    @property
    def unknowns(self):
        return [lv.n for lv in self.levels]

    def _smooth(self, level, b, x, sweeps):
        for _ in range(sweeps):
            x += level.weighted_dinv * (b - level.A @ x)

    def _cycle(self, depth, b, x):
        level = self.levels[depth]
        if depth == len(self.levels) - 1:
            x[:] = solve_coarsest(level, b)
            return
        self._smooth(level, b, x, self.presmooth)
        residual = b - level.A @ x
        P = self.levels[depth + 1].P
        coarse_x = np.zeros(P.shape[1])
        self._cycle(depth + 1, P.T @ residual, coarse_x)
        x += P @ coarse_x
        self._smooth(level, b, x, self.postsmooth)

    @staticmethod
    def project(level, v):
        v[~level.active] = 0.0
        if level.singular and level.active.any():
            v[level.active] -= v[level.active].mean()

    def apply(self, r):
        """One V-cycle from zero -- the preconditioner (multigrid.py:460-474)."""
        top = self.levels[0]
        b = np.array(r, dtype=float).ravel()
        self.project(top, b)
        x = np.zeros_like(b)
        self._cycle(0, b, x)
        self.project(top, x)
        return x

    def cycle_until(self, b, x0, tol, maxiter, residual_norm):
        """multigrid.py:481-511."""
        top = self.levels[0]
        b = np.array(b, dtype=float).ravel()
        self.project(top, b)
        x = np.zeros_like(b) if x0 is None else np.array(x0, dtype=float).ravel()
        self.project(top, x)
        res = residual_norm(x, b)
        cycles = stalled = 0
        while cycles < maxiter and res >= tol and stalled < STALL_PATIENCE:
            previous = res
            self._cycle(0, b, x)
            self.project(top, x)
            res = residual_norm(x, b)
            cycles += 1
            stalled = stalled + 1 if res > STALL_FACTOR * previous else 0
        return x, cycles, res


def solve_coarsest(level, b):
    """Pinned LU followed by mean removal: the pseudo-inverse -- multigrid.py:524-543."""
    rhs = np.array(b, dtype=float)
    active = level.active
    if level.singular:
        rhs[~active] = 0.0
        rhs[active] -= rhs[active].mean()
        rhs[level.pin] = 0.0
    x = level.lu.solve(rhs)
    x[~active] = 0.0
    if level.singular and active.any():
        x[active] -= x[active].mean()
    return x
