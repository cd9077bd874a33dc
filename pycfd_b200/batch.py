"""Batched form: many independent problems advanced together on one GPU.

Each problem keeps its own solver, hierarchy and workspace; its whole time
step -- the field reduction, the device-side dt (the reference's formula), the
three projected substeps with their device-side Poisson loops -- is recorded
once into a CUDA graph and replayed.  A step of the batch replays every
problem's graph on a pool of streams, so the small problems' kernels overlap
and fill the GPU that any one of them would leave mostly idle; nothing returns
to the host until the batch is read.  An autotuner picks, per grid size, the
solver knobs (precision form, inner tolerance, smoothing sweeps) by timing
them on a sample problem, and caches the choice on disk.
"""

from __future__ import annotations

import json
import os
import time
from dataclasses import dataclass, field

import numpy as np

from .config import BCKind, BCSpec, SimulationConfig
from .solver import GpuOptions, ProjectionSolver


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
