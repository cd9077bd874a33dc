"""Batched form: many independent problems advanced together on one GPU.

:class:`BatchedSolver` is the batched engine: every stage of the step -- field
reduction, device-side dt, predictor, boundary programs, divergence, each
phase of the MG-PCG (or FP32-in-FP64 mixed) Poisson solve, correction, stage
combination -- is ONE launch over all problems, whatever their grid sizes,
viscosities, boundary conditions and time steps; the step is recorded once as
a CUDA graph whose solve loops run on the device while any problem still
iterates.  :class:`BatchAutotuner` picks its tile shape, smoothing sweeps and
inner tolerance by timing the batch itself, and caches the choice on disk.

:class:`BatchRunner` is the plain alternative it is measured against: one
single-problem solver per problem, each step a recorded per-problem graph,
replayed on a pool of streams (with its own per-grid-size :class:`Autotuner`).
"""

from __future__ import annotations

import ctypes as C
import json
import os
import time
from dataclasses import dataclass, field, replace

import numpy as np

from . import _lib
from .config import BCKind, BCSpec, PressureSolver, SimulationConfig, SolverType, TimeScheme
from .fields import FlowField
from .hierarchy import hierarchy_for
from .mesh import StructuredMesh
from .solver import (BoundaryInfo, GpuOptions, ProjectionSolver, _stream, _torch, dt_control_for,
                     native_desc)


def cavity_batch_configs(count: int = 256, seed: int = 0, sizes=(64, 96, 128, 192, 256),
                         re_range=(100.0, 2000.0), lid_range=(0.5, 1.5), tol: float = 1e-10):
    """Seeded lid-driven cavities of uneven size, Reynolds number and lid speed.

    N uniform over ``sizes``, Re log-uniform over ``re_range``, lid speed U uniform
    over ``lid_range`` with ``u_ref = U`` (so nu = U / Re), adaptive dt at CFL 0.5,
    MG-PCG to ``tol``.
    """
    rng = np.random.default_rng(seed)
    n = rng.choice(np.asarray(sizes), count)
    re = np.exp(rng.uniform(np.log(re_range[0]), np.log(re_range[1]), count))
    lid = rng.uniform(lid_range[0], lid_range[1], count)
    out = []
    for k in range(count):
        walls = {w: BCSpec(BCKind.NO_SLIP) for w in ("left", "right", "bottom")}
        walls["top"] = BCSpec(BCKind.MOVING_WALL, velocity=float(lid[k]))
        out.append(SimulationConfig(nx=int(n[k]), ny=int(n[k]), re=float(re[k]), u_ref=float(lid[k]),
                                    dt=1.0, t_end=1e9, cfl_max=0.5, adaptive_dt=True,
                                    pressure_solver="mgcg", poisson_tol=tol, boundary_config=walls,
                                    name=f"cavity{k}"))
    return out


def partition_by_cells(configs, parts: int):
    """Split independent problems over ``parts`` ranks by cell count.

    Largest problem first, each to the rank with the fewest cells so far (ties to
    the lower rank): every problem lands on exactly one rank, and the ranks'
    totals differ by at most the largest problem's cells.  Returns one sorted
    list of problem indices per rank.  Deterministic, so every rank computes the
    same split without communicating.
    """
    if parts < 1:
        raise ValueError(f"parts must be >= 1, got {parts}")
    order = sorted(range(len(configs)), key=lambda k: (-configs[k].nx * configs[k].ny, k))
    load = [0] * parts
    out = [[] for _ in range(parts)]
    for k in order:
        r = min(range(parts), key=lambda q: (load[q], q))
        out[r].append(k)
        load[r] += configs[k].nx * configs[k].ny
    return [sorted(o) for o in out]


CANDIDATES = (
    dict(precision="fp64", inner_tol=1e-4, mg_sweeps=1),
    dict(precision="mixed", inner_tol=1e-4, mg_sweeps=1),
    dict(precision="mixed", inner_tol=1e-5, mg_sweeps=1),
    dict(precision="fp64", inner_tol=1e-4, mg_sweeps=2),
)


def _cache_path():
    base = os.environ.get("PYCFD_B200_CACHE", os.path.join(os.path.expanduser("~"), ".cache",
                                                           "pycfd_b200"))
    return os.path.join(base, "autotune.json")


@dataclass
class Autotuner:
    """Per-grid-size choice of solver knobs by measurement, cached on disk."""

    candidates: tuple = CANDIDATES
    steps: int = 8
    warmup: int = 3
    allowed_precisions: tuple = ("fp64", "mixed")
    cache: dict = field(default_factory=dict)

    def __post_init__(self):
        try:
            with open(_cache_path()) as fh:
                self.cache = json.load(fh)
        except Exception:
            self.cache = {}

    def _key(self, cfg) -> str:
        import torch
        name = torch.cuda.get_device_name()
        prec = "+".join(self.allowed_precisions)
        return f"{name}|{cfg.nx}x{cfg.ny}|{cfg.pressure_solver.value}|{cfg.poisson_tol:g}|{prec}"

    def choose(self, cfg) -> dict:
        key = self._key(cfg)
        if key in self.cache:
            return self.cache[key]["choice"]
        import torch
        timings = []
        for cand in self.candidates:
            if cand["precision"] not in self.allowed_precisions:
                continue
            c = cfg.replace(mg_sweeps=cand["mg_sweeps"])
            s = ProjectionSolver(c, options=GpuOptions(precision=cand["precision"],
                                                       inner_tol=cand["inner_tol"]))
            f = s.initialize()
            s.set_clock(0.0)
            for _ in range(self.warmup):
                f = s.advance_adaptive(f)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            for _ in range(self.steps):
                f = s.advance_adaptive(f)
            b.record()
            torch.cuda.synchronize()
            timings.append((a.elapsed_time(b) / self.steps, cand))
            del s
        best = min(timings, key=lambda x: x[0])
        self.cache[key] = {"choice": best[1], "ms_per_step": best[0],
                           "tried": [{"ms_per_step": t, **c} for t, c in timings]}
        try:
            os.makedirs(os.path.dirname(_cache_path()), exist_ok=True)
            with open(_cache_path(), "w") as fh:
                json.dump(self.cache, fh, indent=1)
        except OSError:
            pass
        return best[1]


class BatchRunner:
    """Advance many independent problems together (see the module docstring)."""

    def __init__(self, configs, streams: int = 16, autotuner: Autotuner | None = None,
                 options: GpuOptions | None = None, u_init=None, v_init=None):
        import torch
        self.configs = list(configs)
        self.choices = []
        self.solvers = []
        self.fields = []
        for k, cfg in enumerate(self.configs):
            if autotuner is not None:
                ch = autotuner.choose(cfg)
                cfg = cfg.replace(mg_sweeps=ch["mg_sweeps"])
                opts = GpuOptions(precision=ch["precision"], inner_tol=ch["inner_tol"])
            else:
                ch = None
                opts = options or GpuOptions()
            if streams > 1:   # concurrent solves: one kernel per phase, no grid-filling launch
                opts = replace(opts, persistent_solve=False)
            self.choices.append(ch)
            s = ProjectionSolver(cfg, options=opts)
            self.solvers.append(s)
            self.fields.append(s.initialize(None if u_init is None else u_init[k],
                                            None if v_init is None else v_init[k]))
            s.set_clock(0.0)
        self.streams = [torch.cuda.Stream() for _ in range(max(1, streams))]
        self.cells = sum(c.nx * c.ny for c in self.configs)
        self.steps_done = 0

    def step(self, count: int = 1) -> None:
        """``count`` steps of every problem, queued without host synchronisation."""
        import torch
        main = torch.cuda.current_stream()
        for st in self.streams:
            st.wait_stream(main)
        for _ in range(count):
            for k, s in enumerate(self.solvers):
                with torch.cuda.stream(self.streams[k % len(self.streams)]):
                    self.fields[k] = s.advance_adaptive(self.fields[k])
        for st in self.streams:
            main.wait_stream(st)
        self.steps_done += count

    def report(self):
        """Per-problem clock, step count and health (synchronises)."""
        out = []
        for s in self.solvers:
            t, dt, n, h = s.clock()
            out.append({"t": t, "dt": dt, "steps": n, "health": h,
                        "diverged": bool(h & 3), "dt_collapsed": bool(h & 4)})
        return out


# ---------------------------------------------------------------------------
# Batched engine
# ---------------------------------------------------------------------------
class _Problem:
    """Host set-up of one problem of a batch (the host half of ``ProjectionSolver.__init__``)."""

    def __init__(self, cfg: SimulationConfig, obstacle=None):
        if SolverType(cfg.solver_type) is SolverType.SIMPLE:
            raise NotImplementedError("solver_type='simple' is not provided; use 'projection'")
        if cfg.use_les:
            raise NotImplementedError("the batched path is laminar; use_les=True is not provided")
        if PressureSolver(cfg.pressure_solver) is not PressureSolver.MGCG:
            raise NotImplementedError("the batched path solves the pressure with pressure_solver='mgcg'")
        if TimeScheme(cfg.time_scheme) is not TimeScheme.RK3:
            raise NotImplementedError("the batched path steps with time_scheme='rk3'")
        self.config = cfg
        self.mesh = StructuredMesh.from_config(cfg)
        if not self.mesh.is_uniform:
            raise NotImplementedError("the batched path is discretised for uniform meshes; stretched "
                                      "problems run on ProjectionSolver")
        self.boundaries = BoundaryInfo(cfg.boundary_config, self.mesh)
        nx, ny = self.mesh.shape
        if obstacle is None:
            self.solid = np.zeros((nx, ny), dtype=bool)
        else:
            self.solid = np.asarray(getattr(obstacle, "mask", obstacle), dtype=bool)
            if self.solid.shape != (nx, ny):
                raise ValueError(f"obstacle mask must have shape {(nx, ny)}, got {self.solid.shape}")
        self.has_obstacle = bool(self.solid.any())
        b = self.boundaries
        self.dirichlet = b.dirichlet_pressure()
        self.key = (nx, ny, self.mesh.dx, self.mesh.dy, b.periodic_x, b.periodic_y,
                    tuple(sorted(self.dirichlet.items())),
                    self.solid.tobytes() if self.has_obstacle else None)

    def hierarchy(self):
        """Multigrid hierarchy of this problem's structure (built once per structure)."""
        nx, ny = self.mesh.shape
        b = self.boundaries
        _, h = hierarchy_for(nx, ny, self.mesh.dx, self.mesh.dy, b.periodic_x, b.periodic_y,
                             self.solid if self.has_obstacle else None, self.dirichlet or None)
        return h


@dataclass
class BatchOptions:
    """Knobs of the batched engine (all results stay within the Poisson tolerance)."""

    precision: str = "mixed"     #: "mixed" (FP32 MG-PCG in FP64 refinement) or "fp64"
    inner_tol: float = 1e-4      #: mixed: relative tolerance of each inner FP32 solve
    mg_sweeps: int = 1           #: damped-Jacobi sweeps before/after each coarse correction
    tile_rows: int = 32          #: rows of x per fine-level block (8, 16, 32, 64)
    coarse_level: int = 0        #: multigrid levels from this one down: one block per problem (0: off)
    coarse_tail: bool = True     #: close each structure's V-cycle with its dense tail operator
    tail_ratio: float | None = 16.0   #: bound the tail operator: n_t^2 <= tail_ratio * n_0 (None: none)
    fused_restriction: bool = False   #: down sweep by R (I - A W) products (one sweep, every structure tailed)
    fused_from: int = 1               #: first level so restricted (2: the fine level's restriction stays)
    ell_group: int = 8                #: problems per coarse-level block sharing the matrix loads (1 or 8)
    programmatic_launch: bool = False  #: programmatic dependent launch between the kernels (off: plain order)
    #: with the fused down sweep from the fine level: the level-0 <-> level-1 transfers
    #: as stencils over the fine cells instead of products with the stored matrices
    stencil_transfer: bool = False
    #: mixed form: the FP32 CG and level-0 sweep kernels walk 30-column scalar strips
    #: everywhere (off: 128-column float4 strips on problems whose ny is a multiple of 4)
    scalar_strips: bool = False


class BatchedSolver:
    """Advance many independent problems with one launch per stage (module docstring).

    ``configs``: one :class:`SimulationConfig` per problem (``pressure_solver='mgcg'``,
    ``time_scheme='rk3'``; ``poisson_tol`` and ``poisson_maxiter`` shared).  Each
    problem's state is projected once at construction, like
    ``ProjectionSolver.initialize``; :meth:`step` then advances every problem by
    adaptive steps (``TimeStepper.compute_dt`` per problem, on the device).  A
    problem whose health check fails, whose clock reaches ``t_end`` or that has
    taken ``max_steps`` steps stops; the others go on (:meth:`status`).  ``t_end``
    and ``max_steps`` may be given per problem.
    """

    def __init__(self, configs, options: BatchOptions | None = None, obstacles=None,
                 u_init=None, v_init=None, t_end=float("inf"), max_steps=None):
        torch = _torch()
        self._L = _lib.load()
        self.options = opts = options or BatchOptions()
        if opts.precision not in ("fp64", "mixed"):
            raise ValueError(f"precision must be 'fp64' or 'mixed', got {opts.precision!r}")
        self.configs = list(configs)
        n = len(self.configs)
        if n == 0:
            raise ValueError("a batch needs at least one problem")
        tol, maxiter = self.configs[0].poisson_tol, self.configs[0].poisson_maxiter
        for cfg in self.configs:
            if cfg.poisson_tol != tol or cfg.poisson_maxiter != maxiter:
                raise ValueError("every problem of a batch shares poisson_tol and poisson_maxiter")
        self.problems = [_Problem(cfg, None if obstacles is None else obstacles[k])
                         for k, cfg in enumerate(self.configs)]
        leader: dict = {}
        tailed: dict = {}
        agg2: dict = {}
        structure = (C.c_int * n)()
        descs = (_lib.SolverDesc * n)()
        ctl = (_lib.DtControl * n)()
        keep = []
        gopts = GpuOptions(precision=opts.precision, inner_tol=opts.inner_tol,
                           coarse_tail=opts.coarse_tail and opts.coarse_level == 0, tail_ratio=opts.tail_ratio,
                           fused_restriction=opts.fused_restriction)
        for k, pb in enumerate(self.problems):
            first = pb.key not in leader
            if first:
                leader[pb.key] = k
            levels, cinv = pb.hierarchy() if first else (None, None)
            # the tail operator is built for the batch's sweep count
            d, kp = native_desc(pb.config.replace(mg_sweeps=opts.mg_sweeps), pb.mesh, pb.boundaries, pb.solid,
                                pb.has_obstacle, (), PressureSolver.MGCG, gopts, levels, cinv)
            keep.append((d, kp))
            descs[k] = d
            structure[k] = leader[pb.key]
            if first:
                tailed[pb.key] = d.tail_level > 0
                nx0, ny0 = levels[0].shape
                agg2[pb.key] = len(levels) >= 2 and tuple(levels[1].shape) == (-(-nx0 // 2), -(-ny0 // 2))
            te = t_end[k] if isinstance(t_end, (list, tuple, np.ndarray)) else t_end
            ctl[k] = dt_control_for(pb.config, pb.mesh, float(te))
        self.structures = len(leader)
        #: problems whose structure closes its V-cycle with a dense tail
        self._tailed = sum(1 for pb in self.problems if tailed[pb.key])
        #: the down sweep runs by fused restrictions (the engine's rule: every
        #: structure tailed, one sweep per level, per-level coarse launches)
        self._fused = bool(opts.fused_restriction and opts.mg_sweeps == 1 and opts.coarse_level == 0
                           and self._tailed == n)
        #: the level-0 transfers run as stencils (fused sweep from the fine level, and
        #: every structure's level 1 the 2 x 2 aggregation of its cells)
        self._stencil = bool(opts.stencil_transfer and self._fused and opts.fused_from == 1
                             and all(agg2.values()))
        # state in three flat pools (one host<->device copy per array kind), one view per problem
        shapes = [(pb.mesh.u_shape, pb.mesh.v_shape, pb.mesh.p_shape) for pb in self.problems]
        sizes = [[int(np.prod(sh)) for sh in trio] for trio in shapes]
        self._pools = [torch.zeros(sum(sz[a] for sz in sizes), dtype=torch.float64, device="cuda")
                       for a in range(3)]
        self._offsets = np.zeros((n + 1, 3), dtype=np.int64)
        for k in range(n):
            self._offsets[k + 1] = self._offsets[k] + sizes[k]
        self.fields = []
        for k, pb in enumerate(self.problems):
            views = [self._pools[a][self._offsets[k, a]:self._offsets[k + 1, a]].view(shapes[k][a])
                     for a in range(3)]
            f = FlowField(pb.mesh, *views)
            for init, view in ((u_init, "u_phys"), (v_init, "v_phys")):
                if init is None:
                    continue
                val = init[k] if isinstance(init, (list, tuple)) else init
                if val is None:
                    continue
                tgt = getattr(f, view)
                tgt[...] = float(val) if np.isscalar(val) else torch.as_tensor(
                    np.asarray(val, np.float64) if not isinstance(val, torch.Tensor) else val,
                    dtype=torch.float64, device="cuda")
            self.fields.append(f)
        self._host = None
        U = (C.c_void_p * n)(*[f.u.data_ptr() for f in self.fields])
        V = (C.c_void_p * n)(*[f.v.data_ptr() for f in self.fields])
        P = (C.c_void_p * n)(*[f.p.data_ptr() for f in self.fields])
        bo = _lib.BatchOpts(1 if opts.precision == "mixed" else 0, float(tol), int(maxiter),
                            float(opts.inner_tol), int(opts.mg_sweeps), int(opts.tile_rows),
                            int(opts.coarse_level), int(opts.fused_from), int(opts.ell_group),
                            int(bool(opts.programmatic_launch)), int(self._stencil),
                            int(bool(opts.scalar_strips)))
        if max_steps is None:
            ms = None
        else:
            ms = (C.c_int * n)(*[int(m) for m in (max_steps if isinstance(
                max_steps, (list, tuple, np.ndarray)) else [max_steps] * n)])
        h = C.c_void_p()
        _lib.check(self._L.pycfd_batch_create(descs, structure, ctl, ms, U, V, P, n, C.byref(bo),
                                              C.byref(h)))
        self._h = h
        del keep
        self.cells = int(sum(pb.mesh.shape[0] * pb.mesh.shape[1] for pb in self.problems))
        _lib.check(self._L.pycfd_batch_initialize(self._h, _stream()))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                self._L.pycfd_batch_destroy(h)
            except Exception:
                pass
            self._h = None

    def __len__(self) -> int:
        return len(self.problems)

    def step(self, count: int = 1, record: bool = True) -> None:
        """``count`` adaptive steps of every running problem, queued on the current stream."""
        _lib.check(self._L.pycfd_batch_step(self._h, int(count), int(bool(record)), _stream()))

    def status(self) -> dict:
        """Per-problem ``frozen`` (0 running, 1 health stop, 2 end time), ``steps``,
        ``iterations`` (solver iterations of the last step), ``status``, ``t``, ``dt``."""
        n = len(self)
        fr, st, it, ss = ((C.c_int * n)() for _ in range(4))
        t, dt = (C.c_double * n)(), (C.c_double * n)()
        _lib.check(self._L.pycfd_batch_status(self._h, fr, st, it, ss, t, dt, _stream()))
        return {"frozen": np.array(fr[:]), "steps": np.array(st[:]), "iterations": np.array(it[:]),
                "status": np.array(ss[:]), "t": np.array(t[:]), "dt": np.array(dt[:])}

    def field(self, k: int) -> FlowField:
        """Problem ``k``'s state (the batch's own tensors; copy to keep a snapshot)."""
        st = self.status()
        f = self.fields[k]
        return FlowField(f.mesh, f.u, f.v, f.p, float(st["t"][k]), int(st["steps"][k]))

    def field_stats(self, k: int):
        """max|u|, max|v|, max|div|, kinetic energy, vorticity, finiteness of problem ``k``."""
        out = _lib.FieldStats()
        f = self.fields[k]
        hk = self._L.pycfd_batch_problem(self._h, int(k))
        _lib.check(self._L.pycfd_reduce_fields(C.c_void_p(hk), _lib.ptr(f.u), _lib.ptr(f.v),
                                               _lib.ptr(f.p), _lib.ptr(None), _lib.ptr(None),
                                               C.byref(out), _stream()))
        return out

    def force(self, k: int):
        """Immersed-boundary reaction ``(fx, fy)`` of problem ``k``'s last substep."""
        st = _lib.Stats()
        hk = self._L.pycfd_batch_problem(self._h, int(k))
        _lib.check(self._L.pycfd_get_stats(C.c_void_p(hk), C.byref(st), _stream()))
        return st.fx, st.fy

    def state_bytes(self):
        """Bytes of the (u, v) inputs and (u, v, p) outputs of one host round trip."""
        return (8 * int(self._offsets[-1, 0] + self._offsets[-1, 1]),
                8 * int(self._offsets[-1].sum()))

    def step_host(self, count: int = 1, sync: bool = True) -> None:
        """``count`` times: (u, v) of every problem from pinned host memory, one recorded
        step, (u, v, p) back to pinned host memory -- the host-buffer call of
        ``pycfd_step_host`` for the whole batch.  The host copies start as the state.
        ``sync=False`` leaves the work queued on the current stream."""
        torch = _torch()
        if self._host is None:
            self._host = [torch.empty(p.numel(), dtype=torch.float64, pin_memory=True)
                          for p in self._pools]
            for h, p in zip(self._host, self._pools):
                h.copy_(p)
        for _ in range(count):
            self._pools[0].copy_(self._host[0], non_blocking=True)
            self._pools[1].copy_(self._host[1], non_blocking=True)
            self.step(1)
            for h, p in zip(self._host, self._pools):
                h.copy_(p, non_blocking=True)
        if sync:
            torch.cuda.current_stream().synchronize()

    def profile(self, kernel_id: int, steps: int = 1):
        """Device time (ms) and launch count of one kernel kind over ``steps`` eager steps,
        plus the CG iterations per problem of the last step (ids in the C header)."""
        _lib.check(self._L.pycfd_batch_profile(self._h, int(kernel_id)))
        self.step(steps, record=False)
        ms, cnt = C.c_double(), C.c_int()
        _lib.check(self._L.pycfd_batch_profile_read(self._h, C.byref(ms), C.byref(cnt), _stream()))
        _lib.check(self._L.pycfd_batch_profile(self._h, 0))
        return ms.value, cnt.value, self.status()["iterations"]

    def set_loop_cap(self, cap: int = 0) -> None:
        """Pass cap of the device loops of later steps (0: the built-in caps)."""
        _lib.check(self._L.pycfd_batch_set_loop_cap(self._h, int(cap), _stream()))

    def capped(self) -> int:
        """Which device loops a pass cap ended since the last call (bit 0 CG, bit 1 refinement)."""
        out = C.c_int()
        _lib.check(self._L.pycfd_batch_capped(self._h, C.byref(out), _stream()))
        return int(out.value)

    def launches(self, steps: int) -> int:
        """Kernel launches the device ran for the last ``steps`` recorded steps."""
        n = C.c_longlong()
        _lib.check(self._L.pycfd_batch_launches(self._h, int(steps), C.byref(n), _stream()))
        return int(n.value)


class ConcurrentBatch:
    """One batch run as ``parts`` batched engines stepped concurrently, each on a CUDA
    stream of its own.

    The problems are split by cell count (:func:`partition_by_cells`) and every part
    is a :class:`BatchedSolver` with the same options.  Each batched launch is
    latency-bound -- its blocks wait on dependent loads and on the reductions that
    close each phase -- so while one part's kernel drains, another part's kernel
    fills the idle SM slots: on the 256-cavity batch four parts step in 16.6 ms
    against 19.5 ms for one engine.  Problem ``k`` keeps its index: :attr:`fields`,
    :meth:`status`, :meth:`field_stats` and :meth:`profile` answer in the order of
    ``configs``.
    """

    def __init__(self, configs, options: BatchOptions | None = None, parts: int = 4):
        torch = _torch()
        self.configs = list(configs)
        parts = max(1, min(int(parts), len(self.configs)))
        self.index = [ks for ks in partition_by_cells(self.configs, parts) if ks]
        self.parts = [BatchedSolver([self.configs[k] for k in ks], options) for ks in self.index]
        self.options = self.parts[0].options
        self.streams = [torch.cuda.Stream() for _ in self.parts]
        self._where = [None] * len(self.configs)
        for p, ks in enumerate(self.index):
            for j, k in enumerate(ks):
                self._where[k] = (p, j)

    def __len__(self) -> int:
        return len(self.configs)

    @property
    def fields(self):
        return [self.parts[p].fields[j] for p, j in self._where]

    def _each(self, fn) -> None:
        """fn(part) for every part on its own stream, ordered after the current stream's
        work and before its later work."""
        torch = _torch()
        main = torch.cuda.current_stream()
        for st in self.streams:
            st.wait_stream(main)
        for b, st in zip(self.parts, self.streams):
            with torch.cuda.stream(st):
                fn(b)
        for st in self.streams:
            main.wait_stream(st)

    def step(self, count: int = 1, record: bool = True) -> None:
        """``count`` adaptive steps of every running problem, the parts concurrently."""
        self._each(lambda b: b.step(count, record))

    def step_host(self, count: int = 1) -> None:
        """The host-buffer round trip of every part (:meth:`BatchedSolver.step_host`), the
        parts' copies and steps overlapping; returns when all are done."""
        self._each(lambda b: b.step_host(count, sync=False))
        _torch().cuda.current_stream().synchronize()

    def _merge(self, per_part):
        n = len(self.configs)
        out = {}
        for key in per_part[0]:
            arr = np.empty(n, dtype=per_part[0][key].dtype)
            for p, ks in enumerate(self.index):
                arr[ks] = per_part[p][key]
            out[key] = arr
        return out

    def status(self) -> dict:
        return self._merge([b.status() for b in self.parts])

    def field(self, k: int) -> FlowField:
        p, j = self._where[k]
        return self.parts[p].field(j)

    def field_stats(self, k: int):
        p, j = self._where[k]
        return self.parts[p].field_stats(j)

    def force(self, k: int):
        p, j = self._where[k]
        return self.parts[p].force(j)

    def state_bytes(self):
        sizes = [b.state_bytes() for b in self.parts]
        return sum(a for a, _ in sizes), sum(b for _, b in sizes)

    def profile(self, kernel_id: int, steps: int = 1):
        """Summed device time and launches of one kernel kind over every part, each part
        stepped eagerly on its own (kernels timed without the overlap), and the CG
        iterations per problem in the order of ``configs``."""
        ms = cnt = 0
        its = np.zeros(len(self.configs), dtype=np.int64)
        for ks, b in zip(self.index, self.parts):
            m, c, it = b.profile(kernel_id, steps)
            ms += m
            cnt += c
            its[ks] = it
        return ms, cnt, its

    def set_loop_cap(self, cap: int = 0) -> None:
        for b in self.parts:
            b.set_loop_cap(cap)

    def capped(self) -> int:
        out = 0
        for b in self.parts:
            out |= b.capped()
        return out

    def launches(self, steps: int) -> int:
        return sum(b.launches(steps) for b in self.parts)


BATCH_CANDIDATES = (
    BatchOptions(precision="mixed", inner_tol=1e-4, mg_sweeps=1, tile_rows=32),
    BatchOptions(precision="mixed", inner_tol=1e-3, mg_sweeps=1, tile_rows=32),
    BatchOptions(precision="mixed", inner_tol=3e-3, mg_sweeps=1, tile_rows=32),
    BatchOptions(precision="mixed", inner_tol=1e-4, mg_sweeps=2, tile_rows=32),
    BatchOptions(precision="mixed", inner_tol=1e-4, mg_sweeps=1, tile_rows=32, tail_ratio=None),
    BatchOptions(precision="mixed", inner_tol=1e-4, mg_sweeps=1, tile_rows=32, tail_ratio=4.0),
    BatchOptions(precision="mixed", inner_tol=1e-4, mg_sweeps=1, tile_rows=32, coarse_level=3),
    BatchOptions(precision="mixed", inner_tol=1e-3, mg_sweeps=1, tile_rows=32, fused_restriction=True),
    BatchOptions(precision="mixed", inner_tol=1e-3, mg_sweeps=1, tile_rows=32, fused_restriction=True,
                 stencil_transfer=True),
    BatchOptions(precision="mixed", inner_tol=3e-3, mg_sweeps=1, tile_rows=32, fused_restriction=True,
                 stencil_transfer=True),
    BatchOptions(precision="mixed", inner_tol=3e-3, mg_sweeps=1, tile_rows=32, fused_restriction=True,
                 fused_from=2),
    BatchOptions(precision="mixed", inner_tol=1e-3, mg_sweeps=1, tile_rows=32, fused_restriction=True,
                 tail_ratio=64.0),
    BatchOptions(precision="mixed", inner_tol=1e-3, mg_sweeps=1, tile_rows=32, fused_restriction=True,
                 tail_ratio=None),
    BatchOptions(precision="mixed", inner_tol=3e-3, mg_sweeps=1, tile_rows=32, fused_restriction=True,
                 tail_ratio=64.0),
    BatchOptions(precision="mixed", inner_tol=1e-4, mg_sweeps=1, tile_rows=32, ell_group=1),
    BatchOptions(precision="mixed", inner_tol=1e-3, mg_sweeps=1, tile_rows=32, ell_group=1),
    BatchOptions(precision="mixed", inner_tol=1e-4, mg_sweeps=2, tile_rows=32, ell_group=1),
    BatchOptions(precision="mixed", inner_tol=3e-3, mg_sweeps=1, tile_rows=32, fused_restriction=True,
                 fused_from=2, ell_group=1),
    BatchOptions(precision="fp64", inner_tol=1e-4, mg_sweeps=1, tile_rows=32),
    BatchOptions(precision="fp64", inner_tol=1e-4, mg_sweeps=1, tile_rows=32, fused_restriction=True),
    BatchOptions(precision="fp64", inner_tol=1e-4, mg_sweeps=1, tile_rows=32, fused_restriction=True,
                 stencil_transfer=True),
    BatchOptions(precision="fp64", inner_tol=1e-4, mg_sweeps=1, tile_rows=32, ell_group=1),
    BatchOptions(precision="fp64", inner_tol=1e-4, mg_sweeps=1, tile_rows=32, fused_restriction=True,
                 ell_group=1),
)


@dataclass
class BatchAutotuner:
    """Choose the batched engine's knobs by timing candidate batches, cached on disk.

    Every candidate reaches the same Poisson tolerance, so the choice changes
    speed only.  The key is the device, the multiset of grid sizes, the tolerance
    and the precisions allowed.
    """

    candidates: tuple = BATCH_CANDIDATES
    steps: int = 4
    warmup: int = 3
    allowed_precisions: tuple = ("mixed", "fp64")
    cache: dict = field(default_factory=dict)

    def __post_init__(self):
        try:
            with open(_cache_path()) as fh:
                self.cache = json.load(fh)
        except Exception:
            self.cache = {}

    def key(self, configs) -> str:
        import torch
        sizes = {}
        for c in configs:
            sizes[f"{c.nx}x{c.ny}"] = sizes.get(f"{c.nx}x{c.ny}", 0) + 1
        sig = ",".join(f"{k}:{v}" for k, v in sorted(sizes.items()))
        prec = "+".join(self.allowed_precisions)
        return f"batch|{torch.cuda.get_device_name()}|{sig}|{configs[0].poisson_tol:g}|{prec}"

    def choose(self, configs, **kw) -> BatchOptions:
        key = self.key(configs)
        if key in self.cache:
            return BatchOptions(**self.cache[key]["choice"])
        import torch
        tried = []
        for cand in self.candidates:
            if cand.precision not in self.allowed_precisions:
                continue
            b = BatchedSolver(configs, options=cand, **kw)
            b.step(self.warmup)
            a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            b.step(self.steps)
            e.record()
            torch.cuda.synchronize()
            ms = a.elapsed_time(e) / self.steps
            tried.append((ms, cand))
            del b
        best = min(tried, key=lambda x: x[0])
        self.cache[key] = {"choice": best[1].__dict__, "ms_per_step": best[0],
                           "tried": [{"ms_per_step": t, **c.__dict__} for t, c in tried]}
        try:
            os.makedirs(os.path.dirname(_cache_path()), exist_ok=True)
            with open(_cache_path(), "w") as fh:
                json.dump(self.cache, fh, indent=1)
        except OSError:
            pass
        return best[1]
