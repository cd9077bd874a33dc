"""Staggered state on the device (``pycfd/core/fields.py:18-96``).

``u``, ``v`` and ``p`` are float64 CUDA tensors with the reference's ghosted
shapes and y-fastest layout, so ``.cpu().numpy()`` gives arrays laid out exactly
like the reference's.  Reductions go through the solver's native kernel.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class FlowField:
    """``(u, v, p)`` plus the simulation clock; tensors live on the GPU."""

    mesh: object
    u: object
    v: object
    p: object
    t: float = 0.0
    step: int = 0
    diagnostics: dict = field(default_factory=dict)
    #: cached :class:`pycfd_b200._lib.FieldStats` of this state (set by the stepper)
    _stats: object = field(default=None, repr=False, compare=False)

    @classmethod
    def zeros(cls, mesh, device="cuda") -> "FlowField":
        import torch
        z = lambda s: torch.zeros(s, dtype=torch.float64, device=device)
        return cls(mesh, z(mesh.u_shape), z(mesh.v_shape), z(mesh.p_shape))

    def copy(self) -> "FlowField":
        return FlowField(self.mesh, self.u.clone(), self.v.clone(), self.p.clone(), self.t,
                         self.step, dict(self.diagnostics))

    @property
    def u_phys(self):
        nx, ny = self.mesh.shape
        return self.u[1:nx + 2, 1:ny + 1]

    @property
    def v_phys(self):
        nx, ny = self.mesh.shape
        return self.v[1:nx + 1, 1:ny + 2]

    @property
    def p_phys(self):
        nx, ny = self.mesh.shape
        return self.p[1:nx + 1, 1:ny + 1]

    def cell_velocities(self):
        nx, ny = self.mesh.shape
        uc = 0.5 * (self.u[1:nx + 1, 1:ny + 1] + self.u[2:nx + 2, 1:ny + 1])
        vc = 0.5 * (self.v[1:nx + 1, 1:ny + 1] + self.v[1:nx + 1, 2:ny + 2])
        return uc, vc

    def speed(self):
        import torch
        uc, vc = self.cell_velocities()
        return torch.hypot(uc, vc)

    def max_velocity(self):
        """``(max|u|, max|v|)`` over the physical faces."""
        return (float(self.u_phys.abs().max()), float(self.v_phys.abs().max()))

    def is_finite(self) -> bool:
        import torch
        return bool(torch.isfinite(self.u).all() and torch.isfinite(self.v).all()
                    and torch.isfinite(self.p).all())

    def numpy(self):
        """Host copies ``(u, v, p)`` as NumPy arrays in the reference layout."""
        return (self.u.detach().cpu().numpy(), self.v.detach().cpu().numpy(),
                self.p.detach().cpu().numpy())

    @classmethod
    def from_numpy(cls, mesh, u, v, p, t=0.0, step=0, device="cuda") -> "FlowField":
        import torch
        T = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=device)
        return cls(mesh, T(u), T(v), T(p), float(t), int(step))
