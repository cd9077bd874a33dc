"""Pressure Poisson assembly and solvers (oracle; test infrastructure).

Restates ``pycfd/core/pressure.py`` for the uniform mesh: the 5-point operator
over exactly the projected face set (:110-270), the right-hand-side
conditioning and result normalisation (:300-322), and the iterative solvers the
GPU path provides -- Jacobi-preconditioned CG (:366-398), damped Jacobi
(:410-454), red/black SOR (:457-526), standalone multigrid (:545-574) and
multigrid-preconditioned CG (:577-632).

The CG recurrence is SciPy's ``scipy.sparse.linalg.cg`` (SciPy 1.18.1,
``scipy/sparse/linalg/_isolve/iterative.py:311``, pure Python), restated here:
``atol = rtol*||b||``; ``r = b - A x0``; each pass first tests the recurrence
residual ``||r|| < atol``, then ``z = M r``, ``rho = r.z``,
``p = z + (rho/rho_prev) p``, ``q = A p``, ``alpha = rho/(p.q)``,
``x += alpha p``, ``r -= alpha q``.  SciPy's CSR mat-vec is used as a black box.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import scipy.sparse as sp

from .multigrid import Hierarchy

_ZERO_RHS_NORM = 1.0e-300                # pressure.py:59


@dataclass
class PoissonSystem:
    """pressure.py:69-94."""

    A: sp.csr_matrix
    shape: tuple
    fluid: np.ndarray
    singular: bool
    pin: int
    bc_rhs: np.ndarray

    @property
    def n(self):
        return self.A.shape[0]


def assemble_poisson(nx, ny, dx, dy, periodic_x=False, periodic_y=False,
                     solid=None, dirichlet=None):
    """Uniform-mesh ``assemble_poisson_matrix`` -- pressure.py:110-270.

    A face contributes ``1/h**2`` iff both cells are fluid and inside the domain
    (or joined by a periodic wrap); the diagonal is accumulated face by face in
    the order left, right, bottom, top, with a Dirichlet wall adding
    ``-2/h**2`` to the diagonal and ``-2 p_ref/h**2`` to ``bc_rhs``.  Solid and
    isolated cells get the identity row.
    """
    n = nx * ny
    solid = np.zeros((nx, ny), bool) if solid is None else np.asarray(solid, bool)
    fluid = ~solid
    idx = np.arange(n, dtype=np.int64).reshape(nx, ny)
    diag = np.zeros((nx, ny))
    bc = np.zeros((nx, ny))
    rows, cols, data = [], [], []
    dirichlet = dict(dirichlet or {})
    cx, cy = 1.0 / (dx * dx), 1.0 / (dy * dy)
    for axis, shift, coeff, periodic, wall in (
            (0, -1, cx, periodic_x, "left"), (0, +1, cx, periodic_x, "right"),
            (1, -1, cy, periodic_y, "bottom"), (1, +1, cy, periodic_y, "top")):
        nb = np.roll(idx, -shift, axis=axis)                      # pressure.py:97-107
        if not periodic:
            edge = [slice(None), slice(None)]
            edge[axis] = -1 if shift > 0 else 0
            nb[tuple(edge)] = -1
        inside = nb >= 0
        nb_fluid = np.zeros_like(inside)
        nb_fluid[inside] = fluid.ravel()[nb[inside]]
        active = fluid & inside & nb_fluid
        rows.append(idx[active])
        cols.append(nb[active])
        data.append(np.full(int(active.sum()), coeff))
        diag -= coeff * active
        if wall in dirichlet:
            on_wall = fluid & ~inside
            diag -= 2.0 * coeff * on_wall
            bc -= 2.0 * coeff * dirichlet[wall] * on_wall
    isolated = fluid & (diag == 0.0)
    solvable = fluid & ~isolated
    diag = np.where(solvable, diag, 1.0)
    bc = np.where(solvable, bc, 0.0)
    rows.append(idx.ravel())
    cols.append(idx.ravel())
    data.append(diag.ravel())
    A = sp.coo_matrix((np.concatenate(data), (np.concatenate(rows), np.concatenate(cols))),
                      shape=(n, n)).tocsr()
    A.sum_duplicates()
    singular = not dirichlet
    pin = int(np.flatnonzero(solvable.ravel())[0]) if solvable.any() else 0
    return PoissonSystem(A, (nx, ny), solvable.ravel().copy(), singular, pin,
                         bc.ravel().copy())


class _Base:
    """pressure.py:273-327."""

    name = "base"
    warm_startable = False

    def __init__(self, system, tol, maxiter):
        self.system = system
        self.tol = tol
        self.maxiter = maxiter
        self.last_iterations = 0
        self.last_residual = 0.0

    def prepare_rhs(self, rhs):
        """pressure.py:300-308 (row_scale is 1 on a uniform mesh)."""
        b = np.asarray(rhs, dtype=float).ravel() * 1.0 + self.system.bc_rhs
        fluid = self.system.fluid
        b[~fluid] = 0.0
        if self.system.singular:
            b[fluid] -= b[fluid].mean()
        return b

    def normalize(self, p):
        """pressure.py:310-316."""
        fluid = self.system.fluid
        p[~fluid] = 0.0
        if self.system.singular and fluid.any():
            p[fluid] -= p[fluid].mean()
        return p.reshape(self.system.shape)

    def residual_norm(self, p, b):
        """pressure.py:318-322."""
        r = b - self.system.A @ p
        nb = float(np.linalg.norm(b))
        return float(np.linalg.norm(r)) / (nb if nb > _ZERO_RHS_NORM else 1.0)


def cg_recurrence(A, b, x0, rtol, maxiter, psolve, callback=None):
    """SciPy ``cg`` recurrence (iterative.py:311, SciPy 1.18.1), restated.

    Returns ``(x, info)`` with ``info = 0`` on convergence and ``maxiter`` otherwise.
    """
    x = np.zeros_like(b) if x0 is None else np.array(x0, dtype=float).ravel()
    bnrm2 = np.linalg.norm(b)
    atol = max(0.0, float(rtol) * float(bnrm2))
    if bnrm2 == 0:
        return b, 0
    if maxiter is None:
        maxiter = len(b) * 10
    r = b - A @ x if x.any() else b.copy()
    rho_prev, p = None, None
    for iteration in range(maxiter):
        if np.linalg.norm(r) < atol:
            return x, 0
        z = psolve(r)
        rho_cur = np.dot(r, z)
        if iteration > 0:
            beta = rho_cur / rho_prev
            p *= beta
            p += z
        else:
            p = np.empty_like(r)
            p[:] = z[:]
        q = A @ p
        alpha = rho_cur / np.dot(p, q)
        x += alpha * p
        r -= alpha * q
        rho_prev = rho_cur
        if callback:
            callback(x)
    return x, maxiter


class CG(_Base):
    """Jacobi-preconditioned CG -- pressure.py:366-398."""

    name = "cg"
    warm_startable = True

    def __init__(self, system, tol, maxiter):
        super().__init__(system, tol, maxiter)
        self._d = system.A.diagonal()

    def solve(self, rhs, p0=None):
        b = self.prepare_rhs(rhs)
        x0 = None if p0 is None else np.asarray(p0, float).ravel().copy()
        it = [0]
        p, info = cg_recurrence(self.system.A, b, x0, self.tol, self.maxiter,
                                lambda x: x / self._d,
                                lambda _x: it.__setitem__(0, it[0] + 1))
        self.iterations = it[0]
        self.last_residual = self.residual_norm(p, b)
        if info != 0 and self.last_residual > max(self.tol * 10, 1e-8):
            raise RuntimeError(f"pressure CG failed to converge (info={info})")
        return self.normalize(p)


JACOBI_DAMPING = 2.0 / 3.0               # pressure.py:407


class Jacobi(_Base):
    """Damped Jacobi, residual every 20 sweeps -- pressure.py:410-454."""

    name = "jacobi"
    warm_startable = True

    def __init__(self, system, tol, maxiter, omega=JACOBI_DAMPING):
        super().__init__(system, tol, maxiter)
        self.omega = omega
        self._dinv = 1.0 / system.A.diagonal()

    def solve(self, rhs, p0=None):
        b = self.prepare_rhs(rhs)
        A, fluid = self.system.A, self.system.fluid
        p = np.zeros_like(b) if p0 is None else np.asarray(p0, float).ravel().copy()
        p[~fluid] = 0.0
        res = self.residual_norm(p, b)
        it = 0
        for it in range(1, self.maxiter + 1):
            p += self.omega * self._dinv * (b - A @ p)
            if self.system.singular:
                p[fluid] -= p[fluid].mean()
            if it % 20 == 0 or it == self.maxiter:
                res = self.residual_norm(p, b)
                if res < self.tol:
                    break
        self.last_iterations = it
        self.last_residual = res
        if res > self.tol:
            raise RuntimeError("Jacobi pressure solve stalled")
        return self.normalize(p)


class SOR(_Base):
    """Red/black SOR, residual every 5 sweeps -- pressure.py:457-526."""

    name = "sor"
    warm_startable = True

    def __init__(self, system, tol, maxiter, omega=1.8):
        super().__init__(system, tol, maxiter)
        self.omega = omega
        nx, ny = system.shape
        i, j = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
        colour = ((i + j) % 2).ravel()
        self._red = np.flatnonzero(colour == 0)
        self._black = np.flatnonzero(colour == 1)
        A = system.A.tocsr()
        self._A_rb = A[self._red][:, self._black]
        self._A_br = A[self._black][:, self._red]
        d = A.diagonal()
        self._d_red, self._d_black = d[self._red], d[self._black]
        for label, block in (("red", A[self._red][:, self._red]),
                             ("black", A[self._black][:, self._black])):
            off = block - sp.diags(block.diagonal())
            if off.nnz and np.abs(off).max() > 0:
                raise ValueError(f"red/black ordering is invalid for this grid ({label})")

    def solve(self, rhs, p0=None):
        b = self.prepare_rhs(rhs)
        fluid = self.system.fluid
        p = np.zeros_like(b) if p0 is None else np.asarray(p0, float).ravel().copy()
        p[~fluid] = 0.0
        red, black, w = self._red, self._black, self.omega
        b_red, b_black = b[red], b[black]
        res = self.residual_norm(p, b)
        it = 0
        for it in range(1, self.maxiter + 1):
            p[red] = (1 - w) * p[red] + w * (b_red - self._A_rb @ p[black]) / self._d_red
            p[black] = (1 - w) * p[black] + w * (b_black - self._A_br @ p[red]) / self._d_black
            if self.system.singular:
                p[fluid] -= p[fluid].mean()
            if it % 5 == 0 or it == self.maxiter:
                res = self.residual_norm(p, b)
                if res < self.tol:
                    break
        self.last_iterations = it
        self.last_residual = res
        if res > self.tol:
            raise RuntimeError("SOR pressure solve stalled")
        return self.normalize(p)


class Multigrid(_Base):
    """Standalone V-cycles -- pressure.py:545-574."""

    name = "multigrid"
    warm_startable = True

    def __init__(self, system, tol, maxiter, sweeps=1):
        super().__init__(system, tol, maxiter)
        self.hierarchy = Hierarchy(system.A, system.shape, system.fluid,
                                   system.singular, sweeps, sweeps)

    def solve(self, rhs, p0=None):
        b = self.prepare_rhs(rhs)
        x0 = None if p0 is None else np.asarray(p0, float).ravel()
        p, cycles, res = self.hierarchy.cycle_until(b, x0, self.tol, self.maxiter,
                                                    self.residual_norm)
        self.last_iterations = cycles
        self.last_residual = res
        if res > self.tol:
            raise RuntimeError("multigrid pressure solve stalled")
        return self.normalize(p)


class MultigridCG(Multigrid):
    """CG preconditioned by one V-cycle -- pressure.py:577-632."""

    name = "mgcg"

    def solve(self, rhs, p0=None):
        b = self.prepare_rhs(rhs)
        x0 = None if p0 is None else np.asarray(p0, float).ravel().copy()
        it = [0]
        p, info = cg_recurrence(self.system.A, b, x0, self.tol, self.maxiter,
                                self.hierarchy.apply,
                                lambda _x: it.__setitem__(0, it[0] + 1))
        self.last_iterations = it[0]
        self.last_residual = self.residual_norm(p, b)
        if info != 0 and self.last_residual > max(self.tol * 10, 1e-8):
            raise RuntimeError("multigrid-preconditioned CG failed to converge")
        return self.normalize(p)


def make_solver(kind, system, tol=1e-10, maxiter=20000, sor_omega=1.8, mg_sweeps=1):
    """pressure.py:645-660 (no ``direct``: the GPU path does not provide it)."""
    kind = getattr(kind, "value", kind)
    if kind == "cg":
        return CG(system, tol, maxiter)
    if kind == "jacobi":
        return Jacobi(system, tol, maxiter)
    if kind == "sor":
        return SOR(system, tol, maxiter, sor_omega)
    if kind == "multigrid":
        return Multigrid(system, tol, maxiter, mg_sweeps)
    if kind == "mgcg":
        return MultigridCG(system, tol, maxiter, mg_sweeps)
    if kind == "direct":
        return Direct(system, tol, maxiter)
    raise ValueError(kind)


class Direct(_Base):
    """Pinned sparse LU -- pressure.py:330-363; used by the oracle only as a checker."""

    name = "direct"

    def __init__(self, system, tol, maxiter):
        super().__init__(system, tol, maxiter)
        import scipy.sparse.linalg as spla
        A = system.A
        if system.singular:
            A = A.tolil(copy=True)
            A.rows[system.pin] = [system.pin]
            A.data[system.pin] = [1.0]
            A = A.tocsr()
        self._lu = spla.splu(A.tocsc())

    def solve(self, rhs, p0=None):
        b = self.prepare_rhs(rhs)
        bp = b.copy()
        if self.system.singular:
            bp[self.system.pin] = 0.0
        p = self._lu.solve(bp)
        self.last_iterations = 1
        self.last_residual = self.residual_norm(p, b)
        return self.normalize(p)
