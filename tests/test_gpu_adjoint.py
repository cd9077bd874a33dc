"""Discrete adjoint on the GPU, Poisson solves by the library's MG-PCG (needs a B200).

Gradient of the lower-half kinetic energy with respect to the lid-profile modes
and the smoothed-disk radius, through ``torch.autograd.Function`` (forward: the
checkpointed rollout; backward: the hand-written adjoint with recomputation),
checked against central finite differences with h = 1e-6 at the 1e-5 relative
bar, on a 48x48 cavity over 30 steps with the solve at 1e-13.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def test_adjoint_function_matches_central_differences():
    from pycfd_b200.adjoint import AdjointCavity, Geometry, MultigridSolve, objective_fn, rollout
    cav = AdjointCavity(n=48, steps=30, checkpoint=10, dt=2e-3, re=400.0)
    g = Geometry(cav, device="cuda")
    solve = MultigridSolve(cav.n, tol=cav.tol)
    theta = torch.tensor(cav.default_theta(), dtype=torch.float64, device="cuda", requires_grad=True)
    radius = torch.tensor(cav.radius, dtype=torch.float64, device="cuda", requires_grad=True)
    J = objective_fn(theta, radius, g, solve)
    J.backward()
    gt, gr = theta.grad.detach(), float(radius.grad)
    h = 1e-6
    th0 = theta.detach()
    with torch.no_grad():
        for k in (0, 1, 5):
            e = torch.zeros_like(th0)
            e[k] = h
            fd = (rollout(th0 + e, radius.detach(), g, solve)[0]
                  - rollout(th0 - e, radius.detach(), g, solve)[0]) / (2 * h)
            assert float(fd) == pytest.approx(float(gt[k]), rel=1e-5), k
        r0 = radius.detach()
        fd = (rollout(th0, r0 + h, g, solve)[0] - rollout(th0, r0 - h, g, solve)[0]) / (2 * h)
        assert float(fd) == pytest.approx(gr, rel=1e-5)


def _rand_state(n, seed, device):
    gen = torch.Generator().manual_seed(seed)
    u = torch.randn(n + 3, n + 2, generator=gen, dtype=torch.float64)
    v = torch.randn(n + 2, n + 3, generator=gen, dtype=torch.float64)
    return u.to(device), v.to(device)


def test_kernels_match_the_tensor_reference_primitive_by_primitive():
    """Each hand-written kernel (forward primitive and transpose) against the same
    primitive written as tensor slicing, on random inputs; the transposes are also
    checked as transposes (<J x, y> = <x, J^T y>)."""
    from pycfd_b200 import adjoint as A
    n, h, nu, dt = 20, 1.0 / 20, 1.0 / 300.0, 3e-3
    U, V = _rand_state(n, 1, "cpu")
    gU, gV = _rand_state(n, 2, "cpu")
    cu, cv = (0.5 * (1 + torch.tanh(x)) for x in _rand_state(n, 3, "cpu"))
    lid = 1.0 + 0.1 * torch.randn(n + 3, dtype=torch.float64, generator=torch.Generator().manual_seed(4))
    lower = (torch.arange(n, dtype=torch.float64) < n // 2).to(torch.float64)
    d = lambda *xs: [x.cuda() for x in xs]

    def close(a, b, tag):
        a = a.cpu() if hasattr(a, "cpu") else a
        scale = float(b.abs().max()) or 1.0
        assert float((a - b).abs().max()) <= 1e-14 * scale, tag

    for x, y in zip(A.predictor(*d(U, V), n, h, nu, dt), A.predictor(U, V, n, h, nu, dt)):
        close(x, y, "predictor")
    for x, y in zip(A.walls(*d(U, V, lid), n), A.walls(U, V, lid, n)):
        close(x, y, "walls")
    for x, y in zip(A.mask(*d(U, V, cu, cv), n), A.mask(U, V, cu, cv, n)):
        close(x, y, "mask")
    for x, y in zip(A.predictor_adjoint(*d(U, V, gU, gV), n, h, nu, dt),
                    A.predictor_adjoint(U, V, gU, gV, n, h, nu, dt)):
        close(x, y, "predictor_adjoint")
    acc_d = {"lid": torch.zeros(n + 3, dtype=torch.float64, device="cuda")}
    acc_h = {"lid": torch.zeros(n + 3, dtype=torch.float64)}
    for x, y in zip(A.walls_adjoint_acc(*d(gU, gV), n, acc_d), A.walls_adjoint_acc(gU, gV, n, acc_h)):
        close(x, y, "walls_adjoint")
    close(acc_d["lid"], acc_h["lid"], "lid gradient")
    acc_d = {"cu": torch.zeros_like(cu).cuda(), "cv": torch.zeros_like(cv).cuda()}
    acc_h = {"cu": torch.zeros_like(cu), "cv": torch.zeros_like(cv)}
    for x, y in zip(A.mask_adjoint_acc(*d(U, V, gU, gV, cu, cv), n, acc_d),
                    A.mask_adjoint_acc(U, V, gU, gV, cu, cv, n, acc_h)):
        close(x, y, "mask_adjoint")
    close(acc_d["cu"], acc_h["cu"], "chi_u gradient")
    close(acc_d["cv"], acc_h["cv"], "chi_v gradient")
    ident = lambda q: q                 # the projection's transposed halves without the solve
    for x, y in zip(A.project_adjoint(*d(gU, gV), n, h, ident), A.project_adjoint(gU, gV, n, h, ident)):
        close(x, y, "project_adjoint")

    class G:
        pass
    g = G()
    g.n, g.h, g.lower = n, h, lower
    gd = G()
    gd.n, gd.h, gd.lower = n, h, lower.cuda()
    close(A.objective(*d(U, V), gd), A.objective(U, V, g), "objective")
    for x, y in zip(A.objective_adjoint(*d(U, V), gd), A.objective_adjoint(U, V, g)):
        close(x, y, "objective_adjoint")
    # the predictor's transpose is the transpose of its linearisation: <J dU, W> = <dU, J^T W>
    eps = 1e-7
    dU, dV = _rand_state(n, 5, "cpu")
    up, vp = A.predictor(*d(U + eps * dU, V + eps * dV), n, h, nu, dt)
    um, vm = A.predictor(*d(U - eps * dU, V - eps * dV), n, h, nu, dt)
    lhs = float(((up - um) / (2 * eps) * gU.cuda()).sum() + ((vp - vm) / (2 * eps) * gV.cuda()).sum())
    tU, tV = A.predictor_adjoint(*d(U, V, gU, gV), n, h, nu, dt)
    rhs_ = float(((tU.cpu() - gU) * dU).sum() + ((tV.cpu() - gV) * dV).sum()) + float((gU * dU).sum() +
                                                                                        (gV * dV).sum())
    assert lhs == pytest.approx(rhs_, rel=1e-6)


def test_kernel_forward_is_the_library_step():
    """With a flat lid and chi = 0 the adjoint's forward (kernels + the library's
    Poisson solve) is the library's own cavity step; with a 0/1 chi on the faces of
    a solid body and the body's Poisson operator it is the library's step with that
    obstacle (pycfd/core/solver.py:553-599, :612-731)."""
    from pycfd_b200 import adjoint as A
    from pycfd_b200.config import BCKind, BCSpec, SimulationConfig
    from pycfd_b200.solver import ProjectionSolver, face_solid_mask
    n, dt, re = 32, 2e-3, 200.0
    walls_ = {w: BCSpec(BCKind.NO_SLIP) for w in ("left", "right", "bottom")}
    walls_["top"] = BCSpec(BCKind.MOVING_WALL, velocity=1.0)
    cfg = SimulationConfig(nx=n, ny=n, re=re, pressure_solver="mgcg", poisson_tol=1e-13, poisson_maxiter=2000,
                           boundary_config=walls_)
    cav = A.AdjointCavity(n=n, re=re, dt=dt, steps=4, modes=4)
    g = A.Geometry(cav, device="cuda")
    lid = g.lid(torch.zeros(cav.modes, dtype=torch.float64, device="cuda"))
    solid = np.zeros((n, n), dtype=bool)
    solid[12:18, 10:15] = True
    for body in (None, solid):
        s = ProjectionSolver(cfg, obstacle=body)
        f = s.initialize()
        if body is None:
            cu = torch.zeros_like(g.r_u)
            cv = torch.zeros_like(g.r_v)
        else:
            cu = torch.zeros_like(g.r_u)
            cv = torch.zeros_like(g.r_v)
            cu[2:n + 1, 1:n + 1] = torch.as_tensor(face_solid_mask(solid, 2, n + 1, 0, False), dtype=torch.float64)
            cv[1:n + 1, 2:n + 1] = torch.as_tensor(face_solid_mask(solid, 2, n + 1, 1, False), dtype=torch.float64)
        solve = lambda b, s=s: s.pressure_solver.solve(b.contiguous())
        u, v = A.initial(lid, cu, cv, g, solve)
        fu, fv, _ = f.numpy()
        assert np.abs(u.cpu().numpy() - fu).max() <= 1e-10 * np.abs(fu).max()
        for _ in range(cav.steps):
            f = s.step(f, dt)
            u, v = A.step(u, v, lid, cu, cv, g, dt, solve)
        fu, fv, _ = f.numpy()
        scale = max(np.abs(fu).max(), np.abs(fv).max())
        err = max(np.abs(u.cpu().numpy() - fu).max(), np.abs(v.cpu().numpy() - fv).max()) / scale
        assert err <= 1e-10, (body is not None, err)
