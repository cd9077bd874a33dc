"""Discrete adjoint on the GPU, Poisson solves by the library's MG-PCG (needs a B200).

Gradient of the lower-half kinetic energy with respect to the lid-profile modes
and the smoothed-disk radius, through ``torch.autograd.Function`` (forward: the
checkpointed rollout; backward: the hand-written adjoint with recomputation),
checked against central finite differences with h = 1e-6 at the 1e-5 relative
bar, on a 48x48 cavity over 30 steps with the solve at 1e-13.
"""

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
