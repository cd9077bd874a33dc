"""Hand-written discrete adjoint of the projection step, behind ``torch.autograd.Function``.

The differentiated model is the lid-driven cavity step of the batched and
single-problem paths, extended with the two controls the reference does not
have: a lid-velocity profile and a smoothed immersed obstacle.

* Lid: the top wall's tangential ghost is ``2 U(x) - u_in`` with
  ``U(x) = 1 + sum_k theta_k sin(k pi x)`` on the u-face abscissae (the
  reference's moving wall, ``pycfd/core/boundary.py:141-164``, with a profile).
* Obstacle: ``chi = (1 - tanh((r - R)/w))/2`` at face centres, ``r`` the distance
  to the centre, ``w`` the tanh width; direct forcing multiplies the solvable
  faces by ``1 - chi`` where the reference zeroes the masked faces
  (``pycfd/core/solver.py:553-599``; a 0/1 ``chi`` gives the reference's rule).

One time step is SSP-RK3 over projected Euler substeps (``pycfd/core/solver.py:612-731``):
predictor ``u* = U + dt rhs(U)`` with the central advection-diffusion stencil
(``pycfd/core/kernels.py:54-110``), wall pass, mask, projection (Poisson solve on
the cell grid, gradient correction of the solvable faces), mask, wall pass.
Arrays are float64 tensors in the reference's ghosted layout: ``u`` is
``(nx+3, ny+2)``, ``v`` is ``(nx+2, ny+3)``.

Every primitive exists twice.  On CUDA tensors it runs as a hand-written kernel
of the library (``pycfd_adjoint_apply``: the forward with the library step's own
arithmetic, each transpose in gather form); on CPU tensors it runs as tensor
slicing, so that autograd can run through the forward when the Poisson solve is
a differentiable dense solve (the small dense reference the kernels and the
hand-written backward are checked against).  The backward is hand-written:
each primitive has its transpose (:func:`rhs_adjoint` is the transposed
Jacobian of the advection-diffusion operator; :func:`walls_adjoint` reverses the
ordered line assignments; :func:`project_adjoint` applies the transposed
projection with the same Poisson solver -- the operator is symmetric, so the
adjoint solve is one more solve with the same multigrid).  Long rollouts keep a
checkpoint every ``checkpoint`` steps and recompute each segment during the
backward pass.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np


def _torch():
    import torch
    return torch


# ---------------------------------------------------------------------------
# the kernels (CUDA tensors)
# ---------------------------------------------------------------------------
OP = dict(predictor=1, walls=2, mask=3, div=4, correct=5, lincomb=6, objective=7, predictor_t=8,
          walls_t=9, mask_t=10, grad_t=11, div_t=12, objective_t=13)


def _on_device(t) -> bool:
    return getattr(t, "is_cuda", False)


def _k(op, **kw):
    """One adjoint-primitive kernel launch on the current stream."""
    import ctypes as C
    from . import _lib
    torch = _torch()
    L = _lib.load()
    a = _lib.AdjArgs()
    for k, val in kw.items():
        if isinstance(val, torch.Tensor):
            if val.dtype != torch.float64 or not val.is_contiguous():
                raise ValueError(f"{k}: contiguous float64 tensors only")
            setattr(a, k, val.data_ptr())
        else:
            setattr(a, k, val)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    _lib.check(L.pycfd_adjoint_apply(OP[op], C.byref(a), stream))


def lincomb(a, ca, b=None, cb=0.0):
    """``ca a + cb b`` (``b`` absent: ``ca a``)."""
    if b is None:
        b, cb = a, 0.0
    if _on_device(a):
        out = _torch().empty_like(a)
        _k("lincomb", out=out, a=a.contiguous(), b=b.contiguous(), ca=float(ca), cb=float(cb),
           count=a.numel())
        return out
    return ca * a + cb * b if cb != 0.0 else ca * a


# ---------------------------------------------------------------------------
# problem description
# ---------------------------------------------------------------------------
@dataclass
class AdjointCavity:
    """Lid-driven unit-square cavity with a lid profile and a smoothed disk."""

    n: int = 256                  #: cells per side
    re: float = 400.0             #: Reynolds number (u_ref = l_ref = 1)
    dt: float = 1.2e-3            #: fixed time step
    steps: int = 200              #: rollout length
    modes: int = 32               #: lid-profile sine modes
    centre: tuple = (0.5, 0.3)    #: disk centre
    radius: float = 0.08          #: disk radius (differentiated)
    width_cells: float = 2.0      #: tanh width in cells
    checkpoint: int = 10          #: steps per checkpoint segment
    tol: float = 1e-13            #: Poisson tolerance (tight, so J is smooth in theta)
    seed: int = 0                 #: seed of the default lid amplitudes
    y_split: float = 0.5          #: J = kinetic energy of the cells with yc below this

    @property
    def dx(self) -> float:
        return 1.0 / self.n

    @property
    def nu(self) -> float:
        return 1.0 / self.re

    def default_theta(self):
        """Seeded lid amplitudes theta_k = 0.05 N(0, 1) / k."""
        rng = np.random.default_rng(self.seed)
        return 0.05 * rng.standard_normal(self.modes) / np.arange(1, self.modes + 1)


class Geometry:
    """Face coordinates, lid sine basis and disk distances of one cavity, on a device."""

    def __init__(self, cav: AdjointCavity, device="cpu"):
        torch = _torch()
        n, h = cav.n, cav.dx
        self.cav, self.n, self.h = cav, n, h
        self.device = device
        f64 = dict(dtype=torch.float64, device=device)
        # u faces: x = (m-1) h, m = 0..n+2; y = (j - 1/2) h, j = 0..n+1
        xm = (torch.arange(n + 3, **f64) - 1.0) * h
        yj = (torch.arange(n + 2, **f64) - 0.5) * h
        # v faces: x = (i - 1/2) h, i = 0..n+1; y = (k - 1) h, k = 0..n+2
        xi = (torch.arange(n + 2, **f64) - 0.5) * h
        yk = (torch.arange(n + 3, **f64) - 1.0) * h
        cx, cy = cav.centre
        self.r_u = torch.sqrt((xm[:, None] - cx) ** 2 + (yj[None, :] - cy) ** 2)
        self.r_v = torch.sqrt((xi[:, None] - cx) ** 2 + (yk[None, :] - cy) ** 2)
        k = torch.arange(1, cav.modes + 1, **f64)
        self.lid_basis = torch.sin(math.pi * k[:, None] * xm[None, :])     # (modes, n+3)
        self.w = cav.width_cells * h
        # J: cells with yc below the split
        yc = (torch.arange(n, **f64) + 0.5) * h
        self.lower = (yc < cav.y_split).to(torch.float64)                  # (n,)

    def lid(self, theta):
        return 1.0 + theta @ self.lid_basis

    def chi(self, radius):
        torch = _torch()
        cu = 0.5 * (1.0 - torch.tanh((self.r_u - radius) / self.w))
        cv = 0.5 * (1.0 - torch.tanh((self.r_v - radius) / self.w))
        return cu, cv

    def dchi_dr(self, radius):
        torch = _torch()
        tu = torch.tanh((self.r_u - radius) / self.w)
        tv = torch.tanh((self.r_v - radius) / self.w)
        return 0.5 * (1.0 - tu * tu) / self.w, 0.5 * (1.0 - tv * tv) / self.w


# ---------------------------------------------------------------------------
# forward primitives (tensor slicing only)
# ---------------------------------------------------------------------------
def rhs(u, v, n, h, nu):
    """Central advection-diffusion right-hand side on all u faces (n+1, n) and v faces (n, n+1)."""
    U0, UE, UW = u[1:n + 2, 1:n + 1], u[2:n + 3, 1:n + 1], u[0:n + 1, 1:n + 1]
    UN, US = u[1:n + 2, 2:n + 2], u[1:n + 2, 0:n]
    VT = 0.5 * (v[0:n + 1, 2:n + 2] + v[1:n + 2, 2:n + 2])
    VB = 0.5 * (v[0:n + 1, 1:n + 1] + v[1:n + 2, 1:n + 1])
    ur, ul = 0.5 * (U0 + UE), 0.5 * (UW + U0)
    ut, ub = 0.5 * (U0 + UN), 0.5 * (US + U0)
    ru = -((ur * ur - ul * ul) / h + (ut * VT - ub * VB) / h) + nu * (
        (UW - 2.0 * U0 + UE) / (h * h) + (US - 2.0 * U0 + UN) / (h * h))
    V0, VN, VS = v[1:n + 1, 1:n + 2], v[1:n + 1, 2:n + 3], v[1:n + 1, 0:n + 1]
    VE, VW = v[2:n + 2, 1:n + 2], v[0:n, 1:n + 2]
    UR = 0.5 * (u[2:n + 2, 0:n + 1] + u[2:n + 2, 1:n + 2])
    UL = 0.5 * (u[1:n + 1, 0:n + 1] + u[1:n + 1, 1:n + 2])
    vt, vb = 0.5 * (V0 + VN), 0.5 * (VS + V0)
    vr, vl = 0.5 * (V0 + VE), 0.5 * (VW + V0)
    rv = -((UR * vr - UL * vl) / h + (vt * vt - vb * vb) / h) + nu * (
        (VW - 2.0 * V0 + VE) / (h * h) + (VS - 2.0 * V0 + VN) / (h * h))
    return ru, rv


def predictor(U, V, n, h, nu, dt):
    """u* = U + dt rhs(U) on the solvable faces (u: m = 2..n, v: k = 2..n), U elsewhere."""
    if _on_device(U):
        us, vs = _torch().empty_like(U), _torch().empty_like(V)
        _k("predictor", n=n, h=h, nu=nu, dt=dt, u=U, v=V, out_u=us, out_v=vs)
        return us, vs
    ru, rv = rhs(U, V, n, h, nu)
    us, vs = U.clone(), V.clone()
    us[2:n + 1, 1:n + 1] = U[2:n + 1, 1:n + 1] + dt * ru[1:n]
    vs[1:n + 1, 2:n + 1] = V[1:n + 1, 2:n + 1] + dt * rv[:, 1:n]
    return us, vs


def walls(u, v, lid, n):
    """Wall pass of the cavity, walls in the reference's order (left, right,
    bottom, top), each line assignment in sequence so corner ghosts agree."""
    u, v = u.clone(), v.clone()
    if _on_device(u):
        _k("walls", n=n, h=1.0, out_u=u, out_v=v, lid=lid.contiguous())
        return u, v
    # left: normal face, normal ghost, tangential ghost
    u[1, :] = 0.0
    u[0, :] = 2.0 * u[1, :] - u[2, :]
    v[0, :] = -v[1, :]
    # right
    u[n + 1, :] = 0.0
    u[n + 2, :] = 2.0 * u[n + 1, :] - u[n, :]
    v[n + 1, :] = -v[n, :]
    # bottom
    v[:, 1] = 0.0
    v[:, 0] = 2.0 * v[:, 1] - v[:, 2]
    u[:, 0] = -u[:, 1]
    # top (moving wall with the lid profile)
    v[:, n + 1] = 0.0
    v[:, n + 2] = 2.0 * v[:, n + 1] - v[:, n]
    u[:, n + 1] = 2.0 * lid - u[:, n]
    return u, v


def mask(u, v, cu, cv, n):
    """Direct forcing: solvable faces times (1 - chi)."""
    if _on_device(u):
        uo, vo = _torch().empty_like(u), _torch().empty_like(v)
        _k("mask", n=n, h=1.0, u=u, v=v, out_u=uo, out_v=vo, cu=cu, cv=cv)
        return uo, vo
    uo, vo = u.clone(), v.clone()
    uo[2:n + 1, 1:n + 1] = (1.0 - cu[2:n + 1, 1:n + 1]) * u[2:n + 1, 1:n + 1]
    vo[1:n + 1, 2:n + 1] = (1.0 - cv[1:n + 1, 2:n + 1]) * v[1:n + 1, 2:n + 1]
    return uo, vo


def divergence(u, v, n, h):
    return (u[2:n + 2, 1:n + 1] - u[1:n + 1, 1:n + 1]) / h + (v[1:n + 1, 2:n + 2] - v[1:n + 1, 1:n + 1]) / h


def project(u, v, n, h, dt, solve):
    """Projection: p from lap p = div(u)/dt (``solve``: mean-free, singular
    Neumann system), then u -= dt grad p on the solvable faces."""
    if _on_device(u):
        torch = _torch()
        b = torch.empty((n, n), dtype=u.dtype, device=u.device)
        _k("div", n=n, h=h, dt=dt, u=u, v=v, out=b)
        p = solve(b).contiguous()
        u, v = u.clone(), v.clone()
        _k("correct", n=n, h=h, dt=dt, out_u=u, out_v=v, a=p)
        return u, v
    p = solve(divergence(u, v, n, h) / dt)
    u, v = u.clone(), v.clone()
    u[2:n + 1, 1:n + 1] = u[2:n + 1, 1:n + 1] - dt * (p[1:n] - p[0:n - 1]) / h
    v[1:n + 1, 2:n + 1] = v[1:n + 1, 2:n + 1] - dt * (p[:, 1:n] - p[:, 0:n - 1]) / h
    return u, v


def substep(U, V, lid, cu, cv, g, dt, solve, tape=None):
    n, h, nu = g.n, g.h, g.cav.nu
    a, b = predictor(U, V, n, h, nu, dt)
    a, b = walls(a, b, lid, n)
    if tape is not None:
        tape.append((a, b))
    a, b = mask(a, b, cu, cv, n)
    a, b = project(a, b, n, h, dt, solve)
    if tape is not None:
        tape.append((a, b))
    a, b = mask(a, b, cu, cv, n)
    return walls(a, b, lid, n)


def step(u, v, lid, cu, cv, g, dt, solve, tape=None):
    """One SSP-RK3 step; ``tape`` (a list) receives each substep's input and the
    states in front of its two masks."""
    def sub(U, V):
        if tape is not None:
            tape.append((U, V))
        return substep(U, V, lid, cu, cv, g, dt, solve, tape)
    u1, v1 = sub(u, v)
    u2, v2 = sub(u1, v1)
    u3, v3 = sub(lincomb(u, 0.75, u2, 0.25), lincomb(v, 0.75, v2, 0.25))
    # the library step's weights (pycfd/core/solver.py:716-721)
    return walls(lincomb(u, 1.0 / 3.0, u3, 2.0 / 3.0), lincomb(v, 1.0 / 3.0, v3, 2.0 / 3.0), lid, g.n)


def initial(lid, cu, cv, g, solve, tape=None):
    """Projected initial state from rest (``ProjectionSolver.initialize``, dt = 1)."""
    torch = _torch()
    n = g.n
    z = dict(dtype=torch.float64, device=g.device)
    a, b = walls(torch.zeros(n + 3, n + 2, **z), torch.zeros(n + 2, n + 3, **z), lid, n)
    if tape is not None:
        tape.append((a, b))
    a, b = mask(a, b, cu, cv, n)
    a, b = project(a, b, n, g.h, 1.0, solve)
    if tape is not None:
        tape.append((a, b))
    a, b = mask(a, b, cu, cv, n)
    return walls(a, b, lid, n)


def objective(u, v, g):
    """Kinetic energy of the cells with yc below the split (``pycfd/analysis/postprocess.py:73-79``)."""
    n, h = g.n, g.h
    if _on_device(u):
        out = _torch().empty((), dtype=u.dtype, device=u.device)
        _k("objective", n=n, h=h, u=u, v=v, lower=g.lower, out=out)
        return out
    uc = 0.5 * (u[1:n + 1, 1:n + 1] + u[2:n + 2, 1:n + 1])
    vc = 0.5 * (v[1:n + 1, 1:n + 1] + v[1:n + 1, 2:n + 2])
    return (0.5 * (uc * uc + vc * vc) * g.lower[None, :]).sum() * h * h


# ---------------------------------------------------------------------------
# hand-written adjoints
# ---------------------------------------------------------------------------
def rhs_adjoint(u, v, gru, grv, n, h, nu):
    """Transposed Jacobian of :func:`rhs` at (u, v) applied to (gru, grv)."""
    torch = _torch()
    gu, gv = torch.zeros_like(u), torch.zeros_like(v)
    # ---- u-momentum
    U0, UE, UW = u[1:n + 2, 1:n + 1], u[2:n + 3, 1:n + 1], u[0:n + 1, 1:n + 1]
    UN, US = u[1:n + 2, 2:n + 2], u[1:n + 2, 0:n]
    VT = 0.5 * (v[0:n + 1, 2:n + 2] + v[1:n + 2, 2:n + 2])
    VB = 0.5 * (v[0:n + 1, 1:n + 1] + v[1:n + 2, 1:n + 1])
    ur, ul = 0.5 * (U0 + UE), 0.5 * (UW + U0)
    ut, ub = 0.5 * (U0 + UN), 0.5 * (US + U0)
    g = gru
    gur = -2.0 * ur * g / h
    gul = 2.0 * ul * g / h
    gut = -VT * g / h
    gVT = -ut * g / h
    gub = VB * g / h
    gVB = ub * g / h
    gl = nu * g / (h * h)
    gu[1:n + 2, 1:n + 1] += 0.5 * gur + 0.5 * gul + 0.5 * gut + 0.5 * gub - 4.0 * gl
    gu[2:n + 3, 1:n + 1] += 0.5 * gur + gl
    gu[0:n + 1, 1:n + 1] += 0.5 * gul + gl
    gu[1:n + 2, 2:n + 2] += 0.5 * gut + gl
    gu[1:n + 2, 0:n] += 0.5 * gub + gl
    gv[0:n + 1, 2:n + 2] += 0.5 * gVT
    gv[1:n + 2, 2:n + 2] += 0.5 * gVT
    gv[0:n + 1, 1:n + 1] += 0.5 * gVB
    gv[1:n + 2, 1:n + 1] += 0.5 * gVB
    # ---- v-momentum
    V0, VN, VS = v[1:n + 1, 1:n + 2], v[1:n + 1, 2:n + 3], v[1:n + 1, 0:n + 1]
    VE, VW = v[2:n + 2, 1:n + 2], v[0:n, 1:n + 2]
    UR = 0.5 * (u[2:n + 2, 0:n + 1] + u[2:n + 2, 1:n + 2])
    UL = 0.5 * (u[1:n + 1, 0:n + 1] + u[1:n + 1, 1:n + 2])
    vt, vb = 0.5 * (V0 + VN), 0.5 * (VS + V0)
    vr, vl = 0.5 * (V0 + VE), 0.5 * (VW + V0)
    g = grv
    gUR = -vr * g / h
    gvr = -UR * g / h
    gUL = vl * g / h
    gvl = UL * g / h
    gvt = -2.0 * vt * g / h
    gvb = 2.0 * vb * g / h
    gl = nu * g / (h * h)
    gv[1:n + 1, 1:n + 2] += 0.5 * gvr + 0.5 * gvl + 0.5 * gvt + 0.5 * gvb - 4.0 * gl
    gv[2:n + 2, 1:n + 2] += 0.5 * gvr + gl
    gv[0:n, 1:n + 2] += 0.5 * gvl + gl
    gv[1:n + 1, 2:n + 3] += 0.5 * gvt + gl
    gv[1:n + 1, 0:n + 1] += 0.5 * gvb + gl
    gu[2:n + 2, 0:n + 1] += 0.5 * gUR
    gu[2:n + 2, 1:n + 2] += 0.5 * gUR
    gu[1:n + 1, 0:n + 1] += 0.5 * gUL
    gu[1:n + 1, 1:n + 2] += 0.5 * gUL
    return gu, gv


def predictor_adjoint(U, V, gus, gvs, n, h, nu, dt):
    """Transpose of :func:`predictor` at (U, V)."""
    torch = _torch()
    if _on_device(U):
        gU, gV = torch.empty_like(U), torch.empty_like(V)
        _k("predictor_t", n=n, h=h, nu=nu, dt=dt, u=U, v=V, gu=gus.contiguous(), gv=gvs.contiguous(),
           out_u=gU, out_v=gV)
        return gU, gV
    gru = torch.zeros(n + 1, n, dtype=U.dtype, device=U.device)
    grv = torch.zeros(n, n + 1, dtype=U.dtype, device=U.device)
    gru[1:n] = dt * gus[2:n + 1, 1:n + 1]
    grv[:, 1:n] = dt * gvs[1:n + 1, 2:n + 1]
    gU, gV = rhs_adjoint(U, V, gru, grv, n, h, nu)
    return gU + gus, gV + gvs


def walls_adjoint(gu, gv, n):
    """Transpose of :func:`walls`: the line assignments in reverse order.  Returns
    the input gradients and the gradient of the lid profile."""
    gu, gv = gu.clone(), gv.clone()
    # top
    glid = 2.0 * gu[:, n + 1]
    gu[:, n] -= gu[:, n + 1]
    gu[:, n + 1] = 0.0
    g = gv[:, n + 2].clone()
    gv[:, n + 2] = 0.0
    gv[:, n + 1] += 2.0 * g
    gv[:, n] -= g
    gv[:, n + 1] = 0.0
    # bottom
    gu[:, 1] -= gu[:, 0]
    gu[:, 0] = 0.0
    g = gv[:, 0].clone()
    gv[:, 0] = 0.0
    gv[:, 1] += 2.0 * g
    gv[:, 2] -= g
    gv[:, 1] = 0.0
    # right
    gv[n, :] -= gv[n + 1, :]
    gv[n + 1, :] = 0.0
    g = gu[n + 2, :].clone()
    gu[n + 2, :] = 0.0
    gu[n + 1, :] += 2.0 * g
    gu[n, :] -= g
    gu[n + 1, :] = 0.0
    # left
    gv[1, :] -= gv[0, :]
    gv[0, :] = 0.0
    g = gu[0, :].clone()
    gu[0, :] = 0.0
    gu[1, :] += 2.0 * g
    gu[2, :] -= g
    gu[1, :] = 0.0
    return gu, gv, glid


def mask_adjoint(u_in, v_in, gu, gv, cu, cv, n):
    """Transpose of :func:`mask` (state gradients) and the gradients of chi."""
    torch = _torch()
    gu, gv = gu.clone(), gv.clone()
    gcu, gcv = torch.zeros_like(cu), torch.zeros_like(cv)
    gcu[2:n + 1, 1:n + 1] = -u_in[2:n + 1, 1:n + 1] * gu[2:n + 1, 1:n + 1]
    gcv[1:n + 1, 2:n + 1] = -v_in[1:n + 1, 2:n + 1] * gv[1:n + 1, 2:n + 1]
    gu[2:n + 1, 1:n + 1] = (1.0 - cu[2:n + 1, 1:n + 1]) * gu[2:n + 1, 1:n + 1]
    gv[1:n + 1, 2:n + 1] = (1.0 - cv[1:n + 1, 2:n + 1]) * gv[1:n + 1, 2:n + 1]
    return gu, gv, gcu, gcv


def project_adjoint(gu, gv, n, h, solve):
    """Transpose of :func:`project`.  With u_out = u - G A^+ D u (dt cancels), the
    transpose is g - D^T A^+ G^T g: one solve with the same (symmetric) operator."""
    torch = _torch()
    if _on_device(gu):
        q = torch.empty((n, n), dtype=gu.dtype, device=gu.device)
        _k("grad_t", n=n, h=h, gu=gu.contiguous(), gv=gv.contiguous(), out=q)
        psi = solve(q).contiguous()
        gu, gv = gu.clone(), gv.clone()
        _k("div_t", n=n, h=h, out_u=gu, out_v=gv, a=psi)
        return gu, gv
    gui, gvi = gu[2:n + 1, 1:n + 1], gv[1:n + 1, 2:n + 1]
    q = torch.zeros(n, n, dtype=gu.dtype, device=gu.device)      # G^T g on the cells
    q[1:n] += gui / h
    q[0:n - 1] -= gui / h
    q[:, 1:n] += gvi / h
    q[:, 0:n - 1] -= gvi / h
    psi = solve(q)
    gu, gv = gu.clone(), gv.clone()
    # minus D^T psi: div(u)[c] has +u(high face)/h - u(low face)/h
    gu[2:n + 2, 1:n + 1] -= psi / h
    gu[1:n + 1, 1:n + 1] += psi / h
    gv[1:n + 1, 2:n + 2] -= psi / h
    gv[1:n + 1, 1:n + 1] += psi / h
    return gu, gv


def walls_adjoint_acc(gu, gv, n, acc):
    """:func:`walls_adjoint` with the lid gradient added into ``acc["lid"]``."""
    if _on_device(gu):
        gu, gv = gu.clone(), gv.clone()
        _k("walls_t", n=n, h=1.0, out_u=gu, out_v=gv, acc_u=acc["lid"])
        return gu, gv
    gu, gv, gl = walls_adjoint(gu, gv, n)
    acc["lid"] += gl
    return gu, gv


def mask_adjoint_acc(u_in, v_in, gu, gv, cu, cv, n, acc):
    """:func:`mask_adjoint` with the chi gradients added into ``acc["cu"]``, ``acc["cv"]``."""
    if _on_device(gu):
        gu, gv = gu.clone(), gv.clone()
        _k("mask_t", n=n, h=1.0, u=u_in, v=v_in, out_u=gu, out_v=gv, cu=cu, cv=cv, acc_u=acc["cu"],
           acc_v=acc["cv"])
        return gu, gv
    gu, gv, gcu, gcv = mask_adjoint(u_in, v_in, gu, gv, cu, cv, n)
    acc["cu"] += gcu
    acc["cv"] += gcv
    return gu, gv


def substep_adjoint(U, V, pre1, pre2, gu, gv, lid, cu, cv, g, dt, solve, acc):
    """Adjoint of :func:`substep`; ``pre1``/``pre2`` are the states in front of its
    masks (from the tape).  Lid and chi gradients accumulate into ``acc``."""
    n, h, nu = g.n, g.h, g.cav.nu
    gu, gv = walls_adjoint_acc(gu, gv, n, acc)
    gu, gv = mask_adjoint_acc(pre2[0], pre2[1], gu, gv, cu, cv, n, acc)
    gu, gv = project_adjoint(gu, gv, n, h, solve)
    gu, gv = mask_adjoint_acc(pre1[0], pre1[1], gu, gv, cu, cv, n, acc)
    gu, gv = walls_adjoint_acc(gu, gv, n, acc)
    return predictor_adjoint(U, V, gu, gv, n, h, nu, dt)


def step_adjoint(tape, gu, gv, lid, cu, cv, g, dt, solve, acc):
    """Adjoint of :func:`step` from its tape (9 entries: per substep its input and
    the two pre-mask states); returns the gradient at the step's input."""
    gu, gv = walls_adjoint_acc(gu, gv, g.n, acc)
    gu0, gv0 = lincomb(gu, 1.0 / 3.0), lincomb(gv, 1.0 / 3.0)
    gu3, gv3 = lincomb(gu, 2.0 / 3.0), lincomb(gv, 2.0 / 3.0)
    (U3, V3), p31, p32 = tape[6], tape[7], tape[8]
    gU3, gV3 = substep_adjoint(U3, V3, p31, p32, gu3, gv3, lid, cu, cv, g, dt, solve, acc)
    gu0 = lincomb(gu0, 1.0, gU3, 0.75)
    gv0 = lincomb(gv0, 1.0, gV3, 0.75)
    (U2, V2), p21, p22 = tape[3], tape[4], tape[5]
    gU2, gV2 = substep_adjoint(U2, V2, p21, p22, lincomb(gU3, 0.25), lincomb(gV3, 0.25), lid, cu, cv, g, dt,
                               solve, acc)
    (U1, V1), p11, p12 = tape[0], tape[1], tape[2]
    gU1, gV1 = substep_adjoint(U1, V1, p11, p12, gU2, gV2, lid, cu, cv, g, dt, solve, acc)
    return lincomb(gu0, 1.0, gU1, 1.0), lincomb(gv0, 1.0, gV1, 1.0)


def initial_adjoint(tape, gu, gv, cu, cv, g, solve, acc):
    """Adjoint of :func:`initial` (its tape: the two pre-mask states)."""
    n = g.n
    gu, gv = walls_adjoint_acc(gu, gv, n, acc)
    gu, gv = mask_adjoint_acc(tape[1][0], tape[1][1], gu, gv, cu, cv, n, acc)
    gu, gv = project_adjoint(gu, gv, n, g.h, solve)
    gu, gv = mask_adjoint_acc(tape[0][0], tape[0][1], gu, gv, cu, cv, n, acc)
    walls_adjoint_acc(gu, gv, n, acc)   # from rest: only the lid carries on


def objective_adjoint(u, v, g):
    torch = _torch()
    n, h = g.n, g.h
    if _on_device(u):
        gu, gv = torch.empty_like(u), torch.empty_like(v)
        _k("objective_t", n=n, h=h, u=u, v=v, lower=g.lower, out_u=gu, out_v=gv)
        return gu, gv
    uc = 0.5 * (u[1:n + 1, 1:n + 1] + u[2:n + 2, 1:n + 1])
    vc = 0.5 * (v[1:n + 1, 1:n + 1] + v[1:n + 1, 2:n + 2])
    w = g.lower[None, :] * h * h
    gu, gv = torch.zeros_like(u), torch.zeros_like(v)
    gu[1:n + 1, 1:n + 1] += 0.5 * uc * w
    gu[2:n + 2, 1:n + 1] += 0.5 * uc * w
    gv[1:n + 1, 1:n + 1] += 0.5 * vc * w
    gv[1:n + 1, 2:n + 2] += 0.5 * vc * w
    return gu, gv


# ---------------------------------------------------------------------------
# Poisson solves
# ---------------------------------------------------------------------------
class DenseSolve:
    """Mean-free solve of the cavity's singular Neumann Poisson system with a dense
    pseudo-inverse (small grids; differentiable, the dense reference)."""

    def __init__(self, n, h, device="cpu"):
        torch = _torch()
        from .hierarchy import assemble
        op = assemble(n, n, h, h, False, False)
        A = torch.as_tensor(op.A.toarray(), dtype=torch.float64, device=device)
        self.Ap = torch.linalg.pinv(A)
        self.n = n

    def __call__(self, b):
        torch = _torch()
        b = b.reshape(-1)
        b = b - b.mean()
        p = self.Ap @ b
        return (p - p.mean()).reshape(self.n, self.n)


class MultigridSolve:
    """Mean-free solve with the library's MG-PCG (GPU), the solver of the forward step."""

    def __init__(self, n, tol=1e-13):
        from .config import BCKind, BCSpec, SimulationConfig
        from .solver import ProjectionSolver
        walls_ = {w: BCSpec(BCKind.NO_SLIP) for w in ("left", "right", "bottom", "top")}
        cfg = SimulationConfig(nx=n, ny=n, re=400.0, pressure_solver="mgcg", poisson_tol=tol,
                               poisson_maxiter=2000, boundary_config=walls_)
        self.solver = ProjectionSolver(cfg)
        self.calls = 0

    def __call__(self, b):
        self.calls += 1
        return self.solver.pressure_solver.solve(b.contiguous())


# ---------------------------------------------------------------------------
# rollout with checkpoints and the autograd.Function
# ---------------------------------------------------------------------------
def rollout(theta, radius, g, solve, steps=None, keep_every=None):
    """J after ``steps`` steps; with ``keep_every`` also the checkpoints."""
    cav = g.cav
    steps = cav.steps if steps is None else steps
    lid = g.lid(theta)
    cu, cv = g.chi(radius)
    u, v = initial(lid, cu, cv, g, solve)
    ckpt = {0: (u, v)} if keep_every else None
    for s in range(steps):
        u, v = step(u, v, lid, cu, cv, g, cav.dt, solve)
        if keep_every and (s + 1) % keep_every == 0 and s + 1 < steps:
            ckpt[s + 1] = (u, v)
    return objective(u, v, g), ckpt


def gradient(theta, radius, g, solve, steps=None):
    """J and dJ/d(theta, radius) by the hand-written adjoint with checkpointed recomputation."""
    torch = _torch()
    cav = g.cav
    steps = cav.steps if steps is None else steps
    ce = cav.checkpoint
    with torch.no_grad():
        J, ckpt = rollout(theta, radius, g, solve, steps, keep_every=ce)
        lid = g.lid(theta)
        cu, cv = g.chi(radius)
        acc = {"lid": torch.zeros_like(lid), "cu": torch.zeros_like(cu), "cv": torch.zeros_like(cv)}
        starts = sorted(ckpt)
        gu = gv = None
        for si in range(len(starts) - 1, -1, -1):
            s0 = starts[si]
            s1 = starts[si + 1] if si + 1 < len(starts) else steps
            # recompute the segment, taping every step
            u, v = ckpt[s0]
            tapes = []
            for _ in range(s0, s1):
                tape = []
                u, v = step(u, v, lid, cu, cv, g, cav.dt, solve, tape)
                tapes.append(tape)
            if gu is None:
                gu, gv = objective_adjoint(u, v, g)
            for tape in reversed(tapes):
                gu, gv = step_adjoint(tape, gu, gv, lid, cu, cv, g, cav.dt, solve, acc)
        tape0 = []
        initial(lid, cu, cv, g, solve, tape0)
        initial_adjoint(tape0, gu, gv, cu, cv, g, solve, acc)
        du, dv = g.dchi_dr(radius)
        g_theta = g.lid_basis @ acc["lid"]
        g_radius = (acc["cu"] * du).sum() + (acc["cv"] * dv).sum()
    return J, g_theta, g_radius


class CavityObjective:
    """``J(theta, radius)`` as a ``torch.autograd.Function``: forward runs the rollout,
    backward the hand-written adjoint (recomputing checkpointed segments)."""

    @staticmethod
    def function():
        torch = _torch()

        class _Fn(torch.autograd.Function):
            @staticmethod
            def forward(ctx, theta, radius, g, solve):
                ctx.save_for_backward(theta.detach().clone(), radius.detach().clone())
                ctx.g, ctx.solve = g, solve
                with torch.no_grad():
                    J, _ = rollout(theta.detach(), radius.detach(), g, solve)
                return J

            @staticmethod
            def backward(ctx, gJ):
                theta, radius = ctx.saved_tensors
                _, gt, gr = gradient(theta, radius, ctx.g, ctx.solve)
                return gJ * gt, gJ * gr, None, None

        return _Fn


def objective_fn(theta, radius, g, solve):
    """Differentiable J(theta, radius): call ``.backward()`` on the result."""
    return CavityObjective.function().apply(theta, radius, g, solve)
