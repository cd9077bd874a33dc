"""Hand-written discrete adjoint against autograd through the small dense reference (CPU).

The forward step is written with tensor slicing, so with a dense pseudo-inverse
Poisson solve autograd differentiates it exactly; the hand-written adjoint
(transposed advection Jacobian, reversed wall assignments, transposed mask and
projection, checkpointed recomputation) must give the same gradient to
rounding, and central finite differences (h = 1e-6) must agree too.
"""

import pytest

torch = pytest.importorskip("torch")

from pycfd_b200.adjoint import AdjointCavity, DenseSolve, Geometry, gradient, rollout


def _small():
    cav = AdjointCavity(n=10, steps=7, checkpoint=3, dt=4e-3, modes=5, radius=0.18,
                        centre=(0.5, 0.4), re=100.0)
    g = Geometry(cav)
    solve = DenseSolve(cav.n, cav.dx)
    theta = torch.tensor(cav.default_theta(), dtype=torch.float64)
    radius = torch.tensor(cav.radius, dtype=torch.float64)
    return cav, g, solve, theta, radius


def test_adjoint_matches_autograd_of_dense_reference():
    cav, g, solve, theta, radius = _small()
    J, gt, gr = gradient(theta, radius, g, solve)
    th = theta.clone().requires_grad_(True)
    r = radius.clone().requires_grad_(True)
    J2, _ = rollout(th, r, g, solve)
    J2.backward()
    assert float(J) == pytest.approx(float(J2), rel=1e-14)
    assert (th.grad - gt).abs().max() <= 1e-10 * th.grad.abs().max()
    assert abs(float(r.grad) - float(gr)) <= 1e-10 * abs(float(r.grad))


def test_adjoint_matches_central_differences():
    cav, g, solve, theta, radius = _small()
    _, gt, gr = gradient(theta, radius, g, solve)
    h = 1e-6
    for k in (0, 2):
        e = torch.zeros_like(theta)
        e[k] = h
        fd = (rollout(theta + e, radius, g, solve)[0] - rollout(theta - e, radius, g, solve)[0]) / (2 * h)
        assert float(fd) == pytest.approx(float(gt[k]), rel=1e-6)
    fd = (rollout(theta, radius + h, g, solve)[0] - rollout(theta, radius - h, g, solve)[0]) / (2 * h)
    assert float(fd) == pytest.approx(float(gr), rel=1e-6)


def test_checkpointing_does_not_change_the_gradient():
    cav, g, solve, theta, radius = _small()
    _, g1, r1 = gradient(theta, radius, g, solve)
    cav.checkpoint = 1
    _, g2, r2 = gradient(theta, radius, g, solve)
    cav.checkpoint = 100
    _, g3, r3 = gradient(theta, radius, g, solve)
    assert torch.equal(g1, g2) and torch.equal(g1, g3)
    assert float(r1) == float(r2) == float(r3)
