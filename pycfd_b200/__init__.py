"""B200-native projection hot path for 2D incompressible MAC-grid flow.

A drop-in for the per-timestep path of the reference solver (kiliancmd/pycfd):
the same ``SimulationConfig``/``BCSpec``, ``Simulation.run()``/``diagnostics()``
and pressure-solver selection, with the step, the Poisson solvers and the
immersed-boundary mask running as hand-written sm_100a CUDA behind a C-ABI
shared library (``libpycfd_b200.so``).  There is no CPU fallback: constructing a
GPU solver without the library or without a CUDA device raises.
"""

from .config import (AdvectionScheme, BCKind, BCSpec, PressureSolver,
                     SimulationConfig, SolverType, TimeScheme, WALLS)

__all__ = ["AdvectionScheme", "BCKind", "BCSpec", "PressureSolver", "SimulationConfig",
           "SolverType", "TimeScheme", "WALLS"]


def __getattr__(name):
    # Heavy pieces (torch, the CUDA library) load on first use only, so that the
    # configuration surface imports on machines without a GPU.
    if name in ("Simulation",):
        from .simulation import Simulation
        return Simulation
    if name in ("ProjectionSolver", "GpuOptions"):
        from . import solver
        return getattr(solver, name)
    if name in ("TimeStepper", "DivergenceError", "SimulationResult"):
        from . import timestepper
        return getattr(timestepper, name)
    if name in ("circle_mask", "rectangle_mask", "polygon_mask", "mask_from_image", "mask_from_function",
                "load_polygon", "transform_polygon", "Obstacle", "ObstacleGroup"):
        from . import obstacles
        return getattr(obstacles, name)
    raise AttributeError(name)
