"""Derived quantities on the device state (``pycfd/analysis/postprocess.py``)."""

from __future__ import annotations


def vorticity_corner(fields):
    """``dv/dx - du/dy`` at the ``(nx+1, ny+1)`` corners (``postprocess.py:21-33``)."""
    nx, ny = fields.mesh.shape
    m = fields.mesh.metrics
    hxu, hyv = m.hxu, m.hyv   # scalars, or the face distances of a stretched mesh
    if not fields.mesh.is_uniform:
        import torch
        hxu = torch.as_tensor(hxu, device=fields.u.device)
        hyv = torch.as_tensor(hyv, device=fields.u.device)
    u, v = fields.u, fields.v
    return ((v[1:nx + 2, 1:ny + 2] - v[0:nx + 1, 1:ny + 2]) / hxu
            - (u[1:nx + 2, 1:ny + 2] - u[1:nx + 2, 0:ny + 1]) / hyv)


def vorticity(fields):
    """Corner vorticity averaged to cell centres (``postprocess.py:36-40``)."""
    w = vorticity_corner(fields)
    return 0.25 * (w[:-1, :-1] + w[1:, :-1] + w[:-1, 1:] + w[1:, 1:])


def kinetic_energy(fields, mask=None) -> float:
    """``0.5 sum(uc^2 + vc^2) dA`` with solid cells zeroed (``postprocess.py:73-79``)."""
    import torch
    uc, vc = fields.cell_velocities()
    e = 0.5 * (uc ** 2 + vc ** 2)
    if mask is not None:
        e = torch.where(torch.as_tensor(mask, device=e.device), torch.zeros_like(e), e)
    m = fields.mesh.metrics
    if m.uniform_area is not None:
        return float(e.sum()) * fields.mesh.dx * fields.mesh.dy
    return float((e * torch.as_tensor(m.cell_areas, device=e.device)).sum())


def force_coefficients(force, u_ref: float, l_ref: float, density: float = 1.0):
    """``C = F / (0.5 rho u_ref^2 l_ref)`` (``postprocess.py:104-113``)."""
    if u_ref <= 0 or l_ref <= 0:
        raise ValueError("u_ref and l_ref must be positive to form a coefficient")
    q = 0.5 * density * u_ref ** 2 * l_ref
    return force[0] / q, force[1] / q
