"""Run configuration: the same surface as the reference's ``pycfd.config``.

``SimulationConfig``, ``BCSpec`` and the enums keep the reference's field names,
defaults, validation rules and JSON round-trip (``pycfd/config.py:39-405``), so a
case written for the reference configures this package unchanged.  No GPU knob
lives here: precision form and launch options belong to
:class:`pycfd_b200.solver.GpuOptions`.
"""

from __future__ import annotations

import json
from dataclasses import asdict, dataclass, field, replace
from enum import Enum
from typing import Any


class SolverType(str, Enum):
    """Pressure-velocity coupling (``pycfd/config.py:39-43``)."""
    PROJECTION = "projection"
    SIMPLE = "simple"


class TimeScheme(str, Enum):
    """Explicit integrator (``pycfd/config.py:46-59``)."""
    EULER = "euler"
    RK2 = "rk2"
    RK3 = "rk3"


class AdvectionScheme(str, Enum):
    """Convective discretisation (``pycfd/config.py:62-66``)."""
    CENTRAL = "central"
    UPWIND = "upwind"


class PressureSolver(str, Enum):
    """Poisson solver selection (``pycfd/config.py:74-82``)."""
    DIRECT = "direct"
    CG = "cg"
    JACOBI = "jacobi"
    SOR = "sor"
    MULTIGRID = "multigrid"
    MGCG = "mgcg"


class BCKind(str, Enum):
    """Boundary condition kinds (``pycfd/config.py:85-94``)."""
    NO_SLIP = "no_slip"
    MOVING_WALL = "moving_wall"
    INLET = "inlet"
    OUTLET = "outlet"
    PRESSURE_OUTLET = "pressure_outlet"
    PERIODIC = "periodic"
    SYMMETRY = "symmetry"


@dataclass(frozen=True)
class BCSpec:
    """One wall's condition (``pycfd/config.py:100-133``)."""

    kind: BCKind = BCKind.NO_SLIP
    velocity: float = 0.0
    profile: str = "uniform"
    p_ref: float = 0.0

    def __post_init__(self) -> None:
        object.__setattr__(self, "kind", BCKind(self.kind))
        if self.profile not in ("uniform", "parabolic"):
            raise ValueError(
                f"BCSpec.profile must be 'uniform' or 'parabolic', got {self.profile!r}")


WALLS = ("left", "right", "bottom", "top")

VISCOUS_SAFETY_FACTOR = 0.8
DIVERGENCE_VELOCITY_LIMIT = 1.0e6
MIN_TIME_STEP = 1.0e-8
QUIESCENT_VELOCITY_FLOOR = 1.0e-12
DEFAULT_POISSON_TOL = 1.0e-10
DEFAULT_POISSON_MAXITER = 20_000
DEFAULT_SOR_OMEGA = 1.8
DEFAULT_MG_SWEEPS = 1

CLUSTER_MODES = ("low", "walls", "centre")


def _default_boundaries() -> dict:
    return {w: BCSpec(BCKind.NO_SLIP) for w in WALLS}


def _cluster(mode: str) -> str:
    mode = str(mode).lower()
    if mode == "center":
        return "centre"
    if mode not in CLUSTER_MODES:
        raise ValueError(f"cluster mode must be one of {CLUSTER_MODES}, got {mode!r}")
    return mode


@dataclass
class SimulationConfig:
    """Complete description of one run (``pycfd/config.py:179-405``)."""

    nx: int = 128
    ny: int = 128
    lx: float = 1.0
    ly: float = 1.0
    stretch_x: float = 1.0
    stretch_y: float = 1.0
    cluster_x: str = "low"
    cluster_y: str = "low"

    dt: float = 1.0e-3
    t_end: float = 10.0
    max_steps: int | None = None
    adaptive_dt: bool = True
    cfl_max: float = 0.5

    re: float = 100.0
    u_ref: float = 1.0
    l_ref: float = 1.0
    body_force: tuple = (0.0, 0.0)

    solver_type: SolverType = SolverType.PROJECTION
    time_scheme: TimeScheme = TimeScheme.RK3
    advection_scheme: AdvectionScheme = AdvectionScheme.CENTRAL
    upwind_blend: float | None = None
    pressure_solver: PressureSolver = PressureSolver.DIRECT
    poisson_tol: float = DEFAULT_POISSON_TOL
    poisson_maxiter: int = DEFAULT_POISSON_MAXITER
    sor_omega: float = DEFAULT_SOR_OMEGA
    mg_sweeps: int = DEFAULT_MG_SWEEPS

    use_numba: bool = True

    use_les: bool = False
    smagorinsky_cs: float = 0.17

    boundary_config: dict = field(default_factory=_default_boundaries)

    steady_tol: float | None = None

    name: str = "simulation"

    def __post_init__(self) -> None:
        self.solver_type = SolverType(self.solver_type)
        self.time_scheme = TimeScheme(self.time_scheme)
        self.advection_scheme = AdvectionScheme(self.advection_scheme)
        self.pressure_solver = PressureSolver(self.pressure_solver)
        self.body_force = tuple(float(c) for c in self.body_force)
        self.validate()

    @property
    def nu(self) -> float:
        """Kinematic viscosity ``u_ref * l_ref / re``."""
        return self.u_ref * self.l_ref / self.re

    @property
    def dx(self) -> float:
        return self.lx / self.nx

    @property
    def dy(self) -> float:
        return self.ly / self.ny

    def is_periodic(self, axis: str) -> bool:
        pair = ("left", "right") if axis == "x" else ("bottom", "top")
        return all(BCKind(self.boundary_config[w].kind) is BCKind.PERIODIC for w in pair)

    def dirichlet_pressure_walls(self) -> dict:
        return {w: s.p_ref for w, s in self.boundary_config.items()
                if BCKind(s.kind) is BCKind.PRESSURE_OUTLET}

    def validate(self) -> None:
        """Same rules and messages as ``pycfd/config.py:280-354``."""
        if self.nx < 4 or self.ny < 4:
            raise ValueError(f"grid must be at least 4x4, got {self.nx}x{self.ny}")
        if self.lx <= 0 or self.ly <= 0:
            raise ValueError(f"domain size must be positive, got {self.lx}x{self.ly}")
        if self.re <= 0:
            raise ValueError(f"Reynolds number must be positive, got {self.re}")
        if self.u_ref <= 0 or self.l_ref <= 0:
            raise ValueError("u_ref and l_ref must be positive")
        if self.dt <= 0:
            raise ValueError(f"dt must be positive, got {self.dt}")
        if self.t_end <= 0:
            raise ValueError(f"t_end must be positive, got {self.t_end}")
        if not 0 < self.cfl_max <= 1.0:
            raise ValueError(f"cfl_max must lie in (0, 1], got {self.cfl_max}")
        if self.stretch_x <= 0 or self.stretch_y <= 0:
            raise ValueError("stretch ratios must be positive")
        object.__setattr__(self, "cluster_x", _cluster(self.cluster_x))
        object.__setattr__(self, "cluster_y", _cluster(self.cluster_y))
        if self.upwind_blend is not None and not 0.0 <= self.upwind_blend <= 1.0:
            raise ValueError(f"upwind_blend must lie in [0, 1], got {self.upwind_blend}")
        if not 0 < self.sor_omega < 2:
            raise ValueError(f"sor_omega must lie in (0, 2), got {self.sor_omega}")
        if self.mg_sweeps < 1:
            raise ValueError(f"mg_sweeps must be at least 1, got {self.mg_sweeps}")
        if self.smagorinsky_cs < 0:
            raise ValueError("smagorinsky_cs must be non-negative")
        if self.max_steps is not None and self.max_steps < 1:
            raise ValueError("max_steps must be >= 1 when given")
        missing = set(WALLS) - set(self.boundary_config)
        if missing:
            raise ValueError(f"boundary_config is missing walls: {sorted(missing)}")
        unknown = set(self.boundary_config) - set(WALLS)
        if unknown:
            raise ValueError(f"boundary_config has unknown walls: {sorted(unknown)}")
        for wall, spec in self.boundary_config.items():
            speed = abs(spec.velocity)
            if BCKind(spec.kind) is BCKind.INLET and speed > 0 and \
                    abs(speed - self.u_ref) > 1e-12 * max(1.0, self.u_ref):
                raise ValueError(
                    f"the {wall} inlet drives the flow at {spec.velocity:g} but u_ref is "
                    f"{self.u_ref:g}; forces are normalised by u_ref^2, so the two must be "
                    "the same speed")
        for axis, (a, b) in (("x", ("left", "right")), ("y", ("bottom", "top"))):
            pa = BCKind(self.boundary_config[a].kind) is BCKind.PERIODIC
            pb = BCKind(self.boundary_config[b].kind) is BCKind.PERIODIC
            if pa != pb:
                raise ValueError(f"periodicity on the {axis}-axis must be set on both "
                                 f"'{a}' and '{b}'")

    def replace(self, **changes: Any) -> "SimulationConfig":
        return replace(self, **changes)

    def to_dict(self) -> dict:
        d = asdict(self)
        d["boundary_config"] = {
            w: {"kind": BCKind(s.kind).value, "velocity": s.velocity,
                "profile": s.profile, "p_ref": s.p_ref}
            for w, s in self.boundary_config.items()}
        d["solver_type"] = self.solver_type.value
        d["time_scheme"] = self.time_scheme.value
        d["advection_scheme"] = self.advection_scheme.value
        d["pressure_solver"] = self.pressure_solver.value
        d["body_force"] = list(self.body_force)
        return d

    @classmethod
    def from_dict(cls, d: dict) -> "SimulationConfig":
        d = dict(d)
        if "boundary_config" in d:
            d["boundary_config"] = {
                w: BCSpec(BCKind(s["kind"]), s.get("velocity", 0.0),
                          s.get("profile", "uniform"), s.get("p_ref", 0.0))
                for w, s in d["boundary_config"].items()}
        if "body_force" in d:
            d["body_force"] = tuple(d["body_force"])
        return cls(**d)

    def to_json(self, indent: int = 2) -> str:
        return json.dumps(self.to_dict(), indent=indent)

    def summary(self) -> str:
        bcs = ", ".join(f"{w}={BCKind(self.boundary_config[w].kind).value}" for w in WALLS)
        return (f"case={self.name}  grid={self.nx}x{self.ny}  domain={self.lx}x{self.ly}\n"
                f"Re={self.re:g}  nu={self.nu:.4g}  u_ref={self.u_ref:g}  l_ref={self.l_ref:g}\n"
                f"time={self.time_scheme.value}  advection={self.advection_scheme.value}  "
                f"poisson={self.pressure_solver.value}\n"
                f"dt={self.dt:g} (adaptive={self.adaptive_dt}, CFL_max={self.cfl_max:g})  "
                f"t_end={self.t_end:g}\nBCs: {bcs}")
