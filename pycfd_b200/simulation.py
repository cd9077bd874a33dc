"""High-level driver with the reference's ``Simulation`` surface
(``pycfd/physics/incompressible.py:29-256``): mesh, GPU solver, time stepper
and state wired in the same order, ``run()``/``diagnostics()``/forces/checkpoints.
"""

from __future__ import annotations

import logging

import numpy as np

from . import export as export_mod
from .config import SimulationConfig
from .mesh import StructuredMesh
from .obstacles import Obstacle, ObstacleGroup, as_obstacle_group
from .postprocess import force_coefficients
from .solver import GpuOptions, ProjectionSolver
from .timestepper import SimulationResult, TimeStepper

log = logging.getLogger(__name__)


class Simulation:
    """A configured, ready-to-run incompressible flow problem on the GPU."""

    def __init__(self, config: SimulationConfig, obstacle=None, u_init=None, v_init=None,
                 options: GpuOptions | None = None) -> None:
        self.config = config
        self.mesh = StructuredMesh.from_config(config)
        self.bodies = as_obstacle_group(obstacle)
        self.obstacle = obstacle if isinstance(obstacle, (Obstacle, ObstacleGroup)) else self.bodies
        self.solver = ProjectionSolver(
            config, self.mesh, self.bodies.mask if self.bodies is not None else None,
            bodies=self.bodies.masks if self.bodies is not None else None, options=options)
        self.stepper = TimeStepper(self.solver, config)
        self.fields = self.solver.initialize(u_init, v_init)
        self.result: SimulationResult | None = None

    @classmethod
    def from_checkpoint(cls, path, obstacle=None, options=None) -> "Simulation":
        fields, config = export_mod.load_checkpoint(path)
        sim = cls(config, obstacle, options=options)
        sim.fields = fields
        return sim

    def run(self, t_end=None, max_steps=None, callback=None, callback_every=50,
            progress=False) -> SimulationResult:
        self.result = self.stepper.run(self.fields, t_end=t_end, max_steps=max_steps,
                                       callback=callback, callback_every=callback_every,
                                       progress=progress)
        self.fields = self.result.fields
        return self.result

    @property
    def solid_mask(self):
        return self.bodies.mask if self.bodies is not None else None

    def force_coefficients(self):
        if self.bodies is None:
            return 0.0, 0.0
        return force_coefficients(self.solver.body_force_reaction, self.config.u_ref,
                                  self.config.l_ref)

    def force_coefficients_by_body(self):
        if self.bodies is None:
            return {}
        reactions = self.solver.body_force_reactions or (self.solver.body_force_reaction,)
        return {name: force_coefficients(f, self.config.u_ref, self.config.l_ref)
                for name, f in zip(self.bodies.names, reactions)}

    def diagnostics(self) -> dict:
        """``pycfd/physics/incompressible.py:193-208`` from one fused reduction."""
        st = self.solver.field_stats(self.fields)
        cd, cl = self.force_coefficients()
        out = {"t": self.fields.t, "step": self.fields.step, "kinetic_energy": st.kinetic_energy,
               "max_divergence": st.max_div, "max_vorticity": st.max_vorticity, "cd": cd, "cl": cl}
        if self.solver.dirichlet_pressure:
            out["outlet_pressure_dev"] = self.outlet_pressure_deviation()
        return out

    def outlet_pressure_deviation(self) -> float:
        walls = self.solver.dirichlet_pressure
        if not walls:
            return float("nan")
        p = self.fields.p.detach().cpu().numpy()
        nx, ny = self.mesh.shape
        idx = {"left": (0, 0, 1), "right": (0, nx + 1, nx), "bottom": (1, 0, 1), "top": (1, ny + 1, ny)}
        worst = 0.0
        for wall, p_ref in walls.items():
            axis, g, i = idx[wall]
            ghost = p[g, :] if axis == 0 else p[:, g]
            inner = p[i, :] if axis == 0 else p[:, i]
            worst = max(worst, float(np.abs(0.5 * (ghost + inner) - p_ref).max()))
        return worst

    def save_checkpoint(self, path):
        return export_mod.save_checkpoint(self.fields, self.config, path)

    def __repr__(self) -> str:
        return (f"Simulation({self.config.name!r}, {self.mesh.nx}x{self.mesh.ny}, "
                f"Re={self.config.re:g}, t={self.fields.t:.4g}, GPU)")
