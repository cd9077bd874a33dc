"""GPU projection solver with the reference's ``ProjectionSolver`` surface.

Construction does the host set-up the reference does (face ranges, face
solid flags, Poisson assembly, multigrid hierarchy) and hands it to the native
library; every per-step operation -- momentum RHS, predictor, boundary passes,
mask, divergence, Poisson solve, correction, stage combination -- runs as
sm_100a kernels on the current CUDA stream.  Public methods and attributes
follow ``pycfd/core/solver.py:82-756``; arrays are float64 CUDA tensors in the
reference's ghosted layout.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from .config import (AdvectionScheme, BCKind, PressureSolver, SimulationConfig, SolverType,
                     TimeScheme, WALLS)
from .fields import FlowField
from .hierarchy import assemble, fused_for, hierarchy_for, tail_for
from .mesh import NonUniformMeshError, StructuredMesh

#: solve status of a persistent (cooperative) solve whose grid barrier ran out of time
PERSISTENT_TIMEOUT = -6


@dataclass
class GpuOptions:
    """Knobs of the GPU path that the reference configuration has no field for.

    precision: ``"fp64"`` (drop-in) or ``"mixed"`` (FP32 multigrid-preconditioned
    CG inside FP64 iterative refinement; MG-PCG only).
    inner_tol: relative tolerance of each FP32 inner solve of the mixed form.
    """

    precision: str = "fp64"
    inner_tol: float = 1e-4
    #: TimeStepper.run on the device: dt, health checks, the end-time clamp and the
    #: steady test run in the recorded step, each step appends a row to a device
    #: history, and the host reads the rows every ``device_loop`` steps (0: the
    #: host-driven loop, one small read per step).  cg / multigrid / mgcg only.
    device_loop: int = 64
    #: record each step once into a CUDA graph (device-side Poisson loops) and
    #: replay it; ``advance()`` and the time stepper use it.
    graphs: bool = True
    #: multigrid levels with at most this many rows run inside one thread-block
    #: cluster per V-cycle (0, the default: one kernel per phase on every level;
    #: the cluster form agrees to rounding but is slower while coarse stencils are wide).
    coarse_cluster_rows: int = 0
    #: let each step kernel be scheduled while its predecessor runs
    #: (programmatic dependent launch); False keeps plain stream order.
    programmatic_launch: bool = True
    #: CG and MG-PCG solves (FP64) as one cooperative launch whose phases are
    #: separated by grid barriers; False launches one kernel per phase.  The
    #: launch fills the GPU, so solvers stepped concurrently on several streams
    #: use the per-phase form.
    persistent_solve: bool = False
    #: MG-PCG: apply the V-cycle at and below the first level of at most 2048
    #: rows as one precomputed dense operator (the same linear map, so the same
    #: preconditioner up to rounding) instead of level by level.
    coarse_tail: bool = True
    #: with ``coarse_tail``: also keep the dense operator within ``tail_ratio``
    #: fine-level vectors (n_t^2 <= tail_ratio * n_0); None takes the first level
    #: of at most 2048 rows (fewest launches: best for one solve on the GPU).
    tail_ratio: float | None = None
    #: MG-PCG with a dense tail and one sweep per level: the first sweep of each
    #: level above the tail and the restriction of its residual as one sparse
    #: product R (I - A W) (the same map), so the down sweep takes one launch per
    #: level.
    fused_restriction: bool = True
    #: resident threads a coarse-level pass may spread its rows over (lanes per
    #: row follow from it); 0 = eight 256-thread blocks per SM, -1 = the lane
    #: count of the stored layout.
    ell_thread_budget: int = 0


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("pycfd_b200 needs a CUDA device; there is no CPU fallback")
    return torch


def _stream():
    torch = _torch()
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def face_solid_mask(solid, lo, hi, axis, periodic):
    """Faces in ``[lo, hi)`` touching a solid cell (``pycfd/core/solver.py:62-79``)."""
    m = np.arange(lo, hi)
    if periodic:
        n = solid.shape[axis]
        return np.take(solid, (m - 2) % n, axis=axis) | np.take(solid, (m - 1) % n, axis=axis)
    pad = [(0, 0), (0, 0)]
    pad[axis] = (1, 1)
    padded = np.pad(solid, pad, constant_values=False)
    return np.take(padded, m - 1, axis=axis) | np.take(padded, m, axis=axis)


class BoundaryInfo:
    """Host view of the wall conditions (``pycfd/core/boundary.py:359-504``)."""

    def __init__(self, boundary_config, mesh):
        self.mesh = mesh
        self.specs = {w: boundary_config[w] for w in WALLS}
        self.kinds = {w: BCKind(self.specs[w].kind) for w in WALLS}
        self.periodic_x = self.kinds["left"] is BCKind.PERIODIC
        self.periodic_y = self.kinds["bottom"] is BCKind.PERIODIC

    def pressure_boundary_kinds(self):
        return {w: ("periodic" if k is BCKind.PERIODIC else
                    "dirichlet" if k is BCKind.PRESSURE_OUTLET else "neumann")
                for w, k in self.kinds.items()}

    def dirichlet_pressure(self):
        return {w: self.specs[w].p_ref for w in WALLS
                if self.kinds[w] is BCKind.PRESSURE_OUTLET}

    def profile(self, wall):
        """Normal-face line of a parabolic inlet (``pycfd/core/boundary.py:203-215``)."""
        spec = self.specs[wall]
        outward = -1.0 if wall in ("left", "bottom") else 1.0
        speed = -outward * spec.velocity
        m = self.mesh
        if wall in ("left", "right"):
            coord, extent, length = m.yc, m.ly, m.ny + 2
        else:
            coord, extent, length = m.xc, m.lx, m.nx + 2
        prof = 4.0 * coord * (extent - coord) / extent ** 2
        full = np.zeros(length)
        full[1:1 + coord.size] = speed * prof
        return full


def les_coefficient(cs: float, mesh):
    """``(Cs Delta)^2`` (``pycfd/physics/turbulence.py:38-58``): one number with the
    filter width Delta = sqrt(dx dy) of a uniform mesh; on a stretched mesh the
    per-cell width sqrt(dx_i dy_j) on the ghosted cell grid, the ghost ring
    repeating its neighbour."""
    if mesh.is_uniform:
        delta = float(np.sqrt(mesh.dx * mesh.dy))
        return (float(cs) * delta) ** 2
    nx, ny = mesh.shape
    delta = np.sqrt(mesh.dx_cells[:, None] * mesh.dy_cells[None, :])
    coeff = np.empty((nx + 2, ny + 2))
    coeff[1:nx + 1, 1:ny + 1] = (float(cs) * delta) ** 2
    coeff[0, :], coeff[nx + 1, :] = coeff[1, :], coeff[nx, :]
    coeff[:, 0], coeff[:, ny + 1] = coeff[:, 1], coeff[:, ny]
    return coeff


class GpuSmagorinsky:
    """The Smagorinsky closure of a GPU solver (``pycfd/physics/turbulence.py:25-118``):
    its constant, filter width and the eddy viscosity evaluated on the device."""

    def __init__(self, solver, cs: float) -> None:
        self.solver = solver
        self.mesh = solver.mesh
        self.cs = float(cs)
        self.delta = (float(np.sqrt(self.mesh.dx * self.mesh.dy)) if self.mesh.is_uniform
                      else np.sqrt(self.mesh.dx_cells[:, None] * self.mesh.dy_cells[None, :]))
        self._coeff = les_coefficient(cs, self.mesh)
        self.last_nu_t_max = 0.0

    def eddy_viscosity(self, u, v, nu_molecular: float):
        """``(nu_c, nu_corner)``: nu + nu_t at the ghosted cell centres and at the corners."""
        nu_c, nu_k, _, _ = self.solver._les_rhs(u, v, 0.0)
        self.last_nu_t_max = float((nu_c - nu_molecular).max())
        return nu_c, nu_k

    def __repr__(self) -> str:
        delta = (f"{self.delta:.4g}" if np.isscalar(self.delta)
                 else f"[{self.delta.min():.4g}, {self.delta.max():.4g}]")
        return f"SmagorinskyModel(cs={self.cs:g}, delta={delta})"


def native_desc(config, mesh, boundaries, solid, has_obstacle, body_masks, kind, options,
                levels=None, cinv=None):
    """The ``pycfd_solver_desc`` of one problem and the host arrays it points into.

    Keep the returned list alive until the native call that reads the descriptor returns.
    """
    cfg = config
    nx, ny = mesh.shape
    d = _lib.SolverDesc()
    m = mesh.metrics
    # dx, dy: the uniform spacing, or the smallest cell of a stretched mesh (the
    # time-step limits answer to it, pycfd/core/timestepper.py:91-119)
    d.nx, d.ny, d.dx, d.dy, d.nu = nx, ny, m.min_hx, m.min_hy, config.nu
    d.body_fx, d.body_fy = cfg.body_force
    keep = []
    d.les_coeff_field = _lib.cast(None, C.c_double)
    if cfg.use_les:
        d.use_les = 1
        coeff = les_coefficient(cfg.smagorinsky_cs, mesh)
        if np.isscalar(coeff):
            d.les_coeff = coeff
        else:
            field_ = np.ascontiguousarray(coeff, dtype=np.float64)
            keep.append(field_)
            d.les_coeff_field = _lib.cast(field_, C.c_double)
    if not mesh.is_uniform:
        block = m.device_block()
        keep.append(block)
        d.metrics = _lib.cast(block, C.c_double)
        # summed outlet face widths, outlet walls in wall order (pycfd/core/boundary.py:480-483)
        total = 0.0
        for wall in WALLS:
            if boundaries.kinds[wall] is BCKind.OUTLET:
                total += float((mesh.dy_cells if wall in ("left", "right") else mesh.dx_cells).sum())
        d.outlet_width = total
    else:
        d.metrics = _lib.cast(None, C.c_double)
    for w, wall in enumerate(WALLS):
        spec = boundaries.specs[wall]
        d.bc_kind[w] = _lib.BC_CODES[boundaries.kinds[wall].value]
        d.bc_velocity[w] = spec.velocity
        d.bc_p_ref[w] = spec.p_ref
        if boundaries.kinds[wall] is BCKind.INLET and spec.profile == "parabolic":
            prof = boundaries.profile(wall)
            keep.append(prof)
            d.bc_profile[w] = _lib.cast(prof, C.c_double)
        else:
            d.bc_profile[w] = _lib.cast(None, C.c_double)
    solid_u8 = np.ascontiguousarray(solid.astype(np.uint8))
    keep.append(solid_u8)
    d.solid = _lib.cast(solid_u8 if has_obstacle else None, C.c_uint8)
    if body_masks:
        bid = np.zeros((nx, ny), np.uint8)
        for kb, b in enumerate(body_masks):
            bid[b] = kb + 1
        keep.append(bid)
        d.body_id = _lib.cast(bid, C.c_uint8)
        d.n_bodies = len(body_masks)
    else:
        d.body_id = _lib.cast(None, C.c_uint8)
        d.n_bodies = 0
    d.solver_kind = _lib.SOLVER_CODES[kind.value]
    d.tol = cfg.poisson_tol
    d.maxiter = cfg.poisson_maxiter
    d.sor_omega = cfg.sor_omega
    d.mg_sweeps = cfg.mg_sweeps
    d.time_scheme = _lib.SCHEME_CODES[TimeScheme(cfg.time_scheme).value]
    d.precision = 1 if options.precision == "mixed" else 0
    d.inner_tol = options.inner_tol
    d.coarse_cluster_rows = int(options.coarse_cluster_rows)
    d.sequential_launch = 0 if options.programmatic_launch else 1
    d.persistent_solve = 1 if options.persistent_solve else 0
    d.ell_thread_budget = int(options.ell_thread_budget)
    if levels is not None:
        arr = (_lib.MgLevel * len(levels))()
        for l, lv in enumerate(levels):
            e = arr[l]
            e.n, e.shape_x, e.shape_y, e.weight = lv.n, lv.shape[0], lv.shape[1], lv.weight
            wd = np.ascontiguousarray(lv.weighted_dinv, dtype=np.float64)
            act = np.ascontiguousarray(lv.active.astype(np.uint8))
            keep += [wd, act]
            e.weighted_dinv = _lib.cast(wd, C.c_double)
            e.active = _lib.cast(act, C.c_uint8)
            A = lv.A.tocsr()
            ap = np.ascontiguousarray(A.indptr, np.int64)
            ai = np.ascontiguousarray(A.indices, np.int32)
            ad = np.ascontiguousarray(A.data, np.float64)
            keep += [ap, ai, ad]
            e.a_indptr, e.a_indices, e.a_data = (_lib.cast(ap, C.c_int64), _lib.cast(ai, C.c_int32),
                                                 _lib.cast(ad, C.c_double))
            if lv.P is not None:
                P = lv.P.tocsr()
                pp = np.ascontiguousarray(P.indptr, np.int64)
                pi = np.ascontiguousarray(P.indices, np.int32)
                pd = np.ascontiguousarray(P.data, np.float64)
                keep += [pp, pi, pd]
                e.p_indptr, e.p_indices, e.p_data = (_lib.cast(pp, C.c_int64),
                                                     _lib.cast(pi, C.c_int32),
                                                     _lib.cast(pd, C.c_double))
            else:
                e.p_indptr = _lib.cast(None, C.c_int64)
                e.p_indices = _lib.cast(None, C.c_int32)
                e.p_data = _lib.cast(None, C.c_double)
        cinv = np.ascontiguousarray(cinv, np.float64)
        keep.append(cinv)
        d.n_levels = len(levels)
        d.levels = arr
        d.coarsest_inverse = _lib.cast(cinv, C.c_double)
        keep.append(arr)
        tl, top = (0, None)
        if options.coarse_tail and kind is PressureSolver.MGCG:
            tl, top = tail_for(levels, cinv, cfg.mg_sweeps, options.tail_ratio)
        d.tail_level = tl
        d.tail_operator = _lib.cast(top, C.c_double)
        if tl and options.fused_restriction and cfg.mg_sweeps == 1:
            for l, M in enumerate(fused_for(levels, tl), start=1):
                mp = np.ascontiguousarray(M.indptr, np.int64)
                mi = np.ascontiguousarray(M.indices, np.int32)
                md = np.ascontiguousarray(M.data, np.float64)
                keep += [mp, mi, md]
                e = arr[l]
                e.m_indptr, e.m_indices, e.m_data = (_lib.cast(mp, C.c_int64), _lib.cast(mi, C.c_int32),
                                                     _lib.cast(md, C.c_double))
    else:
        d.n_levels = 0
        d.levels = C.cast(C.c_void_p(0), C.POINTER(_lib.MgLevel))
        d.coarsest_inverse = _lib.cast(None, C.c_double)
        d.tail_level = 0
        d.tail_operator = _lib.cast(None, C.c_double)
    return d, keep


def dt_control_for(config, mesh, t_end: float = float("inf"), history: bool = False):
    """Device-side time-step control matching :class:`TimeStepper` for ``config``.

    ``pycfd/core/timestepper.py:94-142``: CFL and viscous limits capped by ``config.dt``
    (fixed ``config.dt`` when ``adaptive_dt`` is off), donor-cell blend policy.
    """
    nu = config.nu
    dx, dy = mesh.metrics.min_hx, mesh.metrics.min_hy
    visc = float("inf") if nu <= 0 else 0.8 / (2.0 * nu * (1.0 / dx ** 2 + 1.0 / dy ** 2))
    c = _lib.DtControl()
    c.adaptive = int(bool(config.adaptive_dt))
    c.cfl = config.cfl_max
    c.visc_limit = visc
    c.dt_cap = config.dt
    c.t_end = float(t_end)
    central = AdvectionScheme(config.advection_scheme) is AdvectionScheme.CENTRAL
    c.blend_mode = 0 if (central or config.upwind_blend is not None) else 1
    c.blend = 0.0 if central else float(config.upwind_blend or 0.0)
    c.steady_tol = float(config.steady_tol) if (history and config.steady_tol is not None) else 0.0
    c.history = int(bool(history))
    return c


class GpuPoissonSolver:
    """``PoissonSolverBase`` surface over the native solve (``pycfd/core/pressure.py:273-327``)."""

    warm_startable = True

    def __init__(self, owner: "ProjectionSolver", kind: PressureSolver):
        self._owner = owner
        self.name = kind.value
        self.system = owner.poisson
        self.tol = owner.config.poisson_tol
        self.maxiter = owner.config.poisson_maxiter
        self.last_iterations = 0
        self.last_residual = 0.0
        self.hierarchy_levels = owner._levels

    def solve(self, rhs, p0=None):
        """Solve ``lap(p) = rhs`` and return ``p`` with shape ``(nx, ny)`` (device tensor)."""
        torch = _torch()
        o = self._owner
        nx, ny = o.mesh.shape
        rhs_t = o._dev(rhs).reshape(nx, ny).contiguous()
        p0_t = None if p0 is None else o._dev(p0).reshape(nx, ny).contiguous()
        out = torch.empty((nx, ny), dtype=torch.float64, device=rhs_t.device)
        _lib.check(o._L.pycfd_poisson_solve(o._h, _lib.ptr(rhs_t), _lib.ptr(p0_t),
                                            _lib.ptr(out), _stream()))
        o._read_stats(raise_on_error=True)
        return out


class ProjectionSolver:
    """Fractional-step solver whose hot path runs on one B200 (see module doc)."""

    def __init__(self, config: SimulationConfig, mesh: StructuredMesh | None = None,
                 obstacle=None, bodies=None, options: GpuOptions | None = None) -> None:
        if SolverType(config.solver_type) is SolverType.SIMPLE:
            raise NotImplementedError(
                "solver_type='simple' is reserved for a future SIMPLE implementation; only "
                "'projection' is available. Set solver_type='projection'.")
        kind = PressureSolver(config.pressure_solver)
        if kind is PressureSolver.DIRECT:
            raise NotImplementedError(
                "pressure_solver='direct' (sparse LU) is not provided on the GPU path; use "
                "'mgcg', 'cg', 'multigrid', 'sor' or 'jacobi'")
        self.options = options or GpuOptions()
        if self.options.precision not in ("fp64", "mixed"):
            raise ValueError(f"precision must be 'fp64' or 'mixed', got {self.options.precision!r}")
        if self.options.precision == "mixed" and kind is not PressureSolver.MGCG:
            raise NotImplementedError("the mixed-precision form is provided for pressure_solver='mgcg'")
        self._L = _lib.load()
        _torch()
        self.config = config
        self.mesh = mesh if mesh is not None else StructuredMesh.from_config(config)
        self.metrics = self.mesh.metrics
        self.nu = config.nu
        self.boundaries = BoundaryInfo(config.boundary_config, self.mesh)
        self.periodic_x, self.periodic_y = self.boundaries.periodic_x, self.boundaries.periodic_y
        self._reject_stretched_periodic()
        nx, ny = self.mesh.shape
        if obstacle is None:
            self.solid = np.zeros((nx, ny), dtype=bool)
        else:
            self.solid = np.asarray(getattr(obstacle, "mask", obstacle), dtype=bool)
            if self.solid.shape != (nx, ny):
                raise ValueError(f"obstacle mask must have shape {(nx, ny)}, got {self.solid.shape}")
        self.has_obstacle = bool(self.solid.any())
        self.body_masks = ()
        if bodies is not None and len(bodies) > 1:
            if len(bodies) > _lib.MAX_BODIES:
                raise ValueError(f"at most {_lib.MAX_BODIES} bodies report separate forces")
            self.body_masks = tuple(np.asarray(b, dtype=bool) for b in bodies)
            for k, b in enumerate(self.body_masks):
                if b.shape != (nx, ny):
                    raise ValueError(f"body {k} mask must have shape {(nx, ny)}, got {b.shape}")
        self._build_slices()
        self.dirichlet_pressure = self.boundaries.dirichlet_pressure()
        m = self.mesh.metrics
        widths = None if self.mesh.is_uniform else (self.mesh.dx_cells, self.mesh.dy_cells)
        args = (nx, ny, m.min_hx, m.min_hy, self.periodic_x, self.periodic_y,
                self.solid if self.has_obstacle else None, self.dirichlet_pressure or None, widths)
        self._levels, self._cinv = (None, None)
        if kind in (PressureSolver.MULTIGRID, PressureSolver.MGCG):
            self.poisson, (self._levels, self._cinv) = hierarchy_for(*args)
        else:
            self.poisson = assemble(*args)
        self._create_native(kind)
        self.pressure_solver = GpuPoissonSolver(self, kind)
        self.turbulence = GpuSmagorinsky(self, config.smagorinsky_cs) if config.use_les else None
        self.body_force_reaction = (0.0, 0.0)
        self.body_force_reactions = tuple((0.0, 0.0) for _ in self.body_masks)
        self._blend = 0.0
        self.last_stats = None
        self._ring = None

    def _reject_stretched_periodic(self) -> None:
        """A stretched axis cannot be periodic: its first and last cells differ, so the
        domain does not repeat (``pycfd/core/solver.py:209-230``)."""
        for axis, stretched, periodic, ratio in (
                ("x", self.mesh.stretched_x, self.periodic_x, self.mesh.stretch_x),
                ("y", self.mesh.stretched_y, self.periodic_y, self.mesh.stretch_y)):
            if stretched and periodic:
                raise NonUniformMeshError(
                    f"the {axis} axis is periodic and stretched (stretch_{axis}={ratio}): the first and "
                    "last cells differ in width, so the spacing jumps across the seam and the domain "
                    f"does not repeat. Use stretch_{axis}=1.0 on a periodic axis, or a non-periodic "
                    "boundary condition.")

    # ------------------------------------------------------------------ #
    def _build_slices(self) -> None:
        """Solvable face ranges and face solid flags (``pycfd/core/solver.py:235-296``)."""
        nx, ny = self.mesh.shape
        k = self.boundaries.kinds
        out = BCKind.PRESSURE_OUTLET
        u_lo = 1 if (self.periodic_x or k["left"] is out) else 2
        u_hi = nx + 2 if (k["right"] is out and not self.periodic_x) else nx + 1
        v_lo = 1 if (self.periodic_y or k["bottom"] is out) else 2
        v_hi = ny + 2 if (k["top"] is out and not self.periodic_y) else ny + 1
        self.u_upd = (slice(u_lo, u_hi), slice(1, ny + 1))
        self.v_upd = (slice(1, nx + 1), slice(v_lo, v_hi))
        self.u_rhs_sel = slice(u_lo - 1, u_hi - 1)
        self.v_rhs_sel = slice(v_lo - 1, v_hi - 1)
        if self.has_obstacle:
            self.u_face_solid = face_solid_mask(self.solid, u_lo, u_hi, 0, self.periodic_x)
            self.v_face_solid = face_solid_mask(self.solid, v_lo, v_hi, 1, self.periodic_y)
        else:
            self.u_face_solid = self.v_face_solid = None

    def _create_native(self, kind: PressureSolver) -> None:
        d, keep = native_desc(self.config, self.mesh, self.boundaries, self.solid,
                              self.has_obstacle, self.body_masks, kind, self.options,
                              self._levels, self._cinv)
        h = C.c_void_p()
        _lib.check(self._L.pycfd_solver_create(C.byref(d), C.byref(h)))
        self._h = h
        del keep
        ctas = C.c_int()
        _lib.check(self._L.pycfd_solver_persistent(h, C.byref(ctas)))
        #: CTAs of the cooperative launch of each CG / MG-PCG solve (0: per-phase kernels)
        self._persistent = int(ctas.value)

    def set_wait_limit(self, seconds: float) -> None:
        """Limit of one grid-barrier wait of the persistent solve (default 2 s).  A
        wait that runs out ends the solve with a ``RuntimeError``; the solver stays
        usable.  Only solvers built with ``GpuOptions(persistent_solve=True)``."""
        ns = max(1, int(round(seconds * 1e9)))
        _lib.check(self._L.pycfd_solver_set_wait_limit(self._h, C.c_ulonglong(ns)))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                self._L.pycfd_solver_destroy(h)
            except Exception:
                pass
            self._h = None

    # ------------------------------------------------------------------ #
    def _dev(self, a):
        torch = _torch()
        if isinstance(a, torch.Tensor):
            return a.to(device="cuda", dtype=torch.float64)
        return torch.as_tensor(np.asarray(a, dtype=np.float64), device="cuda")

    def _read_stats(self, raise_on_error: bool = True):
        st = _lib.Stats()
        _lib.check(self._L.pycfd_get_stats(self._h, C.byref(st), _stream()))
        self.last_stats = st
        ps = self.pressure_solver if hasattr(self, "pressure_solver") else None
        if ps is not None:
            ps.last_iterations = st.iterations
            ps.last_residual = st.last_residual
        if self.has_obstacle:
            self.body_force_reaction = (st.fx, st.fy)
            if self.body_masks:
                self.body_force_reactions = tuple((st.body_fx[k], st.body_fy[k])
                                                  for k in range(len(self.body_masks)))
        if raise_on_error and st.status == PERSISTENT_TIMEOUT:
            raise RuntimeError(
                "the persistent pressure solve stopped: a grid barrier waited longer than its limit "
                "(a CTA did not arrive); the result of this solve is not valid")
        if raise_on_error and st.status != 0:
            kind = self.config.pressure_solver
            raise RuntimeError(
                f"{PressureSolver(kind).value} pressure solve failed to converge: relative "
                f"residual {st.last_residual:.3e} after {st.iterations} iterations "
                f"(tol {self.config.poisson_tol:.1e})")
        return st

    def _empty_state(self):
        torch = _torch()
        m = self.mesh
        e = lambda s: torch.empty(s, dtype=torch.float64, device="cuda")
        return e(m.u_shape), e(m.v_shape), e(m.p_shape)

    # ------------------------------------------------------------------ #
    def initialize(self, u_init=None, v_init=None) -> FlowField:
        """Initial field with BCs applied and projected (``pycfd/core/solver.py:301-329``)."""
        fields = FlowField.zeros(self.mesh)
        if u_init is not None:
            fields.u_phys[...] = self._dev(u_init) if not np.isscalar(u_init) else float(u_init)
        if v_init is not None:
            fields.v_phys[...] = self._dev(v_init) if not np.isscalar(v_init) else float(v_init)
        _lib.check(self._L.pycfd_initialize(self._h, _lib.ptr(fields.u), _lib.ptr(fields.v),
                                            _lib.ptr(fields.p), _stream()))
        self._read_stats()
        return fields

    def _les_rhs(self, u, v, blend):
        torch = _torch()
        u, v = self._dev(u).contiguous(), self._dev(v).contiguous()
        nx, ny = self.mesh.shape
        f64 = dict(dtype=torch.float64, device="cuda")
        nu_c, nu_k = torch.empty((nx + 2, ny + 2), **f64), torch.empty((nx + 1, ny + 1), **f64)
        ru, rv = torch.empty((nx + 1, ny), **f64), torch.empty((nx, ny + 1), **f64)
        if not self.mesh.is_uniform:   # the solver's own metrics and per-cell coefficient
            _lib.check(self._L.pycfd_solver_momentum_rhs_les(
                self._h, _lib.ptr(u), _lib.ptr(v), float(blend), _lib.ptr(nu_c), _lib.ptr(nu_k),
                _lib.ptr(ru), _lib.ptr(rv), _stream()))
            return nu_c, nu_k, ru, rv
        fx, fy = self.config.body_force
        _lib.check(self._L.pycfd_momentum_rhs_les(
            _lib.ptr(u), _lib.ptr(v), nx, ny, self.mesh.dx, self.mesh.dy, self.nu, self.turbulence._coeff,
            float(blend), fx, fy, _lib.ptr(nu_c), _lib.ptr(nu_k), _lib.ptr(ru), _lib.ptr(rv), _stream()))
        return nu_c, nu_k, ru, rv

    def momentum_rhs(self, u, v, blend: float = 0.0):
        """``-A(u) + D(u) + f`` as ``(nx+1, ny)`` and ``(nx, ny+1)`` tensors; D is
        ``nu lap(u)``, or the stress divergence of ``nu + nu_t`` with the Smagorinsky
        closure (``pycfd/core/solver.py:501-529``)."""
        torch = _torch()
        if self.turbulence is not None:
            return self._les_rhs(u, v, blend)[2:]
        u, v = self._dev(u).contiguous(), self._dev(v).contiguous()
        nx, ny = self.mesh.shape
        ru = torch.empty((nx + 1, ny), dtype=torch.float64, device="cuda")
        rv = torch.empty((nx, ny + 1), dtype=torch.float64, device="cuda")
        if not self.mesh.is_uniform:   # the stretched array stencils (pycfd/core/solver.py:336-466)
            _lib.check(self._L.pycfd_solver_momentum_rhs(self._h, _lib.ptr(u), _lib.ptr(v), float(blend),
                                                         _lib.ptr(ru), _lib.ptr(rv), _stream()))
            return ru, rv
        fx, fy = self.config.body_force
        _lib.check(self._L.pycfd_momentum_rhs(_lib.ptr(u), _lib.ptr(v), nx, ny, self.mesh.dx,
                                              self.mesh.dy, self.nu, float(blend), fx, fy,
                                              _lib.ptr(ru), _lib.ptr(rv), _stream()))
        return ru, rv

    def divergence(self, u, v):
        """Cell divergence ``(nx, ny)`` (``pycfd/core/solver.py:532-543``)."""
        torch = _torch()
        u, v = self._dev(u).contiguous(), self._dev(v).contiguous()
        nx, ny = self.mesh.shape
        out = torch.empty((nx, ny), dtype=torch.float64, device="cuda")
        if not self.mesh.is_uniform:
            _lib.check(self._L.pycfd_solver_divergence(self._h, _lib.ptr(u), _lib.ptr(v), _lib.ptr(out),
                                                       _stream()))
            return out
        _lib.check(self._L.pycfd_divergence(_lib.ptr(u), _lib.ptr(v), nx, ny, self.mesh.dx,
                                            self.mesh.dy, _lib.ptr(out), _stream()))
        return out

    def field_stats(self, fields: FlowField, previous: FlowField | None = None):
        """One fused reduction over a state (max |u|, |v|, |du|, |div|, KE, finiteness)."""
        st = _lib.FieldStats()
        _lib.check(self._L.pycfd_reduce_fields(
            self._h, _lib.ptr(fields.u), _lib.ptr(fields.v), _lib.ptr(fields.p),
            _lib.ptr(previous.u if previous is not None else None),
            _lib.ptr(previous.v if previous is not None else None), C.byref(st), _stream()))
        return st

    def max_divergence(self, fields: FlowField) -> float:
        """Largest |div u| over fluid cells (``pycfd/core/solver.py:545-550``)."""
        return float(self.field_stats(fields).max_div)

    def project(self, u, v, dt: float):
        """Project ``(u, v)`` in place; return the ghosted pressure (``solver.py:643-683``)."""
        torch = _torch()
        p = torch.empty(self.mesh.p_shape, dtype=torch.float64, device="cuda")
        _lib.check(self._L.pycfd_project(self._h, _lib.ptr(u), _lib.ptr(v), _lib.ptr(p),
                                         float(dt), _stream()))
        self._read_stats()
        return p

    def substep(self, fields: FlowField, dt: float, blend: float = 0.0):
        """One projected Euler substep; returns fresh ``(u, v, p)`` (``solver.py:612-640``)."""
        us, vs, p = self._empty_state()
        _lib.check(self._L.pycfd_substep(self._h, _lib.ptr(fields.u.contiguous()),
                                         _lib.ptr(fields.v.contiguous()), _lib.ptr(us),
                                         _lib.ptr(vs), _lib.ptr(p), float(dt), float(blend),
                                         _stream()))
        self._read_stats()
        return us, vs, p

    def step(self, fields: FlowField, dt: float) -> FlowField:
        """Advance by ``dt`` with the configured scheme (``pycfd/core/solver.py:686-731``)."""
        u, v, p = self._empty_state()
        _lib.check(self._L.pycfd_step(self._h, _lib.ptr(fields.u.contiguous()),
                                      _lib.ptr(fields.v.contiguous()), _lib.ptr(u), _lib.ptr(v),
                                      _lib.ptr(p), float(dt), float(self._blend), _stream()))
        self._read_stats()
        return FlowField(self.mesh, u, v, p, fields.t + dt, fields.step + 1)

    def advance(self, fields: FlowField, dt: float) -> FlowField:
        """``step`` into solver-owned ping-pong buffers, replaying a recorded CUDA graph.

        The returned state lives in one of two buffers the solver reuses: it stays
        valid until the step after next (copy it to keep it longer).
        """
        if not self.options.graphs:
            return self.step(fields, dt)
        if self._ring is None:
            self._ring = [self._empty_state(), self._empty_state()]
        out = self._ring[0] if fields.u.data_ptr() != self._ring[0][0].data_ptr() else self._ring[1]
        u, v, p = out
        _lib.check(self._L.pycfd_step_graph(self._h, _lib.ptr(fields.u.contiguous()),
                                            _lib.ptr(fields.v.contiguous()), _lib.ptr(u),
                                            _lib.ptr(v), _lib.ptr(p), float(dt),
                                            float(self._blend), _stream()))
        self._read_stats()
        return FlowField(self.mesh, u, v, p, fields.t + dt, fields.step + 1)

    def dt_control(self):
        """Device-side time-step control matching :class:`TimeStepper` for this configuration."""
        return dt_control_for(self.config, self.mesh)

    def read_history(self):
        """Rows the device history gained since the last read (step, t, dt, cfl, max_div,
        kinetic energy, residual, fx, fy, max|du|/dt) and the frozen state (0 running,
        1 health stop, 2 end time, 3 steady); clears the history (synchronises)."""
        rows = np.empty((4096, 10), dtype=np.float64)
        n, fr = C.c_int(), C.c_int()
        _lib.check(self._L.pycfd_history_read(self._h, _lib.ptr(rows), 4096, C.byref(n), C.byref(fr),
                                              _stream()))
        return rows[:n.value].copy(), fr.value

    def set_clock(self, t: float = 0.0) -> None:
        """Reset the device clock, step counter and health flags of device-side stepping."""
        _lib.check(self._L.pycfd_set_clock(self._h, float(t), _stream()))

    def clock(self):
        """``(t, last dt, steps, health bits)`` of device-side stepping (synchronises)."""
        t, dt, n, h = C.c_double(), C.c_double(), C.c_int(), C.c_int()
        _lib.check(self._L.pycfd_get_clock(self._h, C.byref(t), C.byref(dt), C.byref(n),
                                           C.byref(h), _stream()))
        return t.value, dt.value, n.value, h.value

    def advance_adaptive(self, fields: FlowField, ctl=None) -> FlowField:
        """One step with dt chosen on the device (no host round trip), into the ring buffers.

        The dt, health checks and clock follow :class:`TimeStepper` exactly but live
        on the device; read them with :meth:`clock`.  The returned field's ``t`` is
        not known on the host (``nan``) until the clock is read.
        """
        if self._ring is None:
            self._ring = [self._empty_state(), self._empty_state()]
        if ctl is None:
            ctl = self._ctl = getattr(self, "_ctl", None) or self.dt_control()
        out = self._ring[0] if fields.u.data_ptr() != self._ring[0][0].data_ptr() else self._ring[1]
        u, v, p = out
        _lib.check(self._L.pycfd_step_adaptive(self._h, _lib.ptr(fields.u), _lib.ptr(fields.v),
                                               _lib.ptr(u), _lib.ptr(v), _lib.ptr(p), C.byref(ctl),
                                               _stream()))
        return FlowField(self.mesh, u, v, p, float("nan"), fields.step + 1)

    def launches_per_step(self, fields: FlowField, dt: float) -> int:
        """Kernels one step of ``fields`` launches, counted on an eager step (inputs untouched).

        A recorded step replays the same kernels; the eager step updates the
        warm start of the next solve like any step does.
        """
        before = self._L.pycfd_launch_count()
        self.step(fields, dt)
        return int(self._L.pycfd_launch_count() - before)

    def step_host(self, u0: np.ndarray, v0: np.ndarray, dt: float, out=None):
        """The same step on host arrays: copies in, steps, copies ``(u, v, p)`` out.

        ``out``: three contiguous float64 arrays of the state shapes to write into
        (pinned ones, e.g. ``torch.empty(...).pin_memory().numpy()``, make the copies
        asynchronous DMA); new arrays otherwise.
        """
        u0 = np.ascontiguousarray(u0, np.float64)
        v0 = np.ascontiguousarray(v0, np.float64)
        if out is None:
            u, v, p = (np.empty(self.mesh.u_shape), np.empty(self.mesh.v_shape),
                       np.empty(self.mesh.p_shape))
        else:
            u, v, p = out
            for a, shape in ((u, self.mesh.u_shape), (v, self.mesh.v_shape), (p, self.mesh.p_shape)):
                if a.shape != tuple(shape) or a.dtype != np.float64 or not a.flags.c_contiguous:
                    raise ValueError(f"out arrays must be contiguous float64 of shape {tuple(shape)}")
        _lib.check(self._L.pycfd_step_host(self._h, _lib.ptr(u0), _lib.ptr(v0), _lib.ptr(u),
                                           _lib.ptr(v), _lib.ptr(p), float(dt), float(self._blend),
                                           _stream()))
        return u, v, p

    # ------------------------------------------------------------------ #
    def set_upwind_blend(self, blend: float) -> None:
        self._blend = float(np.clip(blend, 0.0, 1.0))

    def upwind_blend_for(self, fields: FlowField, dt: float) -> float:
        """Donor-cell blend for the state (``pycfd/core/solver.py:740-756``)."""
        if AdvectionScheme(self.config.advection_scheme) is AdvectionScheme.CENTRAL:
            return 0.0
        if self.config.upwind_blend is not None:
            return self.config.upwind_blend
        st = fields._stats if fields._stats is not None else self.field_stats(fields)
        m = self.mesh.metrics   # the worst cell is the smallest one
        courant = max(st.max_u * dt / m.min_hx, st.max_v * dt / m.min_hy)
        return float(min(1.0, 1.2 * courant))
