"""Batched form and device-side stepping (needs a B200).

Device-side dt uses the reference's formula on exact device maxima, so a
problem advanced inside a batch (its step recorded in a graph with the
reduction and the dt kernel, replayed on a stream shared with other problems)
is bit-identical to the same problem run alone by the host-driven time loop.
"""

import numpy as np
import pytest

import cases
from pycfd_b200.config import BCKind, BCSpec, SimulationConfig

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _cavities():
    from pycfd_b200.batch import cavity_batch_configs
    return cavity_batch_configs(count=6, seed=3, sizes=(16, 24, 32), re_range=(100.0, 800.0))


def test_batch_matches_individual_time_loops_bitwise():
    from pycfd_b200.batch import BatchRunner
    from pycfd_b200.solver import GpuOptions, ProjectionSolver
    from pycfd_b200.timestepper import TimeStepper
    cfgs = _cavities()
    batch = BatchRunner(cfgs, streams=3)   # concurrent streams: one kernel per solve phase
    batch.step(12)
    rep = batch.report()
    for k, cfg in enumerate(cfgs):
        s = ProjectionSolver(cfg, options=GpuOptions(persistent_solve=False))
        res = TimeStepper(s).run(s.initialize(), max_steps=12)
        ua, va, pa = batch.fields[k].numpy()
        ub, vb, pb = res.fields.numpy()
        assert np.array_equal(ua, ub) and np.array_equal(va, vb) and np.array_equal(pa, pb), k
        assert rep[k]["t"] == res.time and rep[k]["steps"] == 12 and rep[k]["health"] == 0


def test_device_clock_reproduces_reference_cavity64(golden):
    """The 64x64 Re 100 cavity (CG 1e-10, adaptive CFL dt), 100 device-timed steps."""
    from pycfd_b200.batch import BatchRunner
    g = golden("cavity64.npz")
    cfg = cases.to_config(cases.CAVITY64, SimulationConfig, BCSpec, BCKind)
    batch = BatchRunner([cfg], streams=1)
    batch.step(100)
    rep = batch.report()[0]
    assert rep["t"] == float(g["s100_t"]) and rep["steps"] == 100
    u, v, p = batch.fields[0].numpy()
    for a, k in ((u, "u"), (v, "v"), (p, "p")):
        ref = g["s100_" + k]
        assert np.abs(a - ref).max() / np.abs(ref).max() < 1e-10


def test_blow_up_is_recorded_not_raised():
    from pycfd_b200.batch import BatchRunner
    walls = {w: BCSpec(BCKind.NO_SLIP) for w in ("left", "right", "bottom")}
    walls["top"] = BCSpec(BCKind.MOVING_WALL, velocity=1e3)
    bad = SimulationConfig(nx=16, ny=16, re=1e6, dt=5.0, adaptive_dt=False, t_end=1e4,
                           pressure_solver="mgcg", boundary_config=walls)
    good = _cavities()[0]
    batch = BatchRunner([bad, good], streams=2)
    batch.step(60)
    rep = batch.report()
    assert rep[0]["diverged"] and not rep[1]["diverged"] and rep[1]["health"] == 0


def test_autotuner_picks_and_caches(tmp_path, monkeypatch):
    from pycfd_b200 import batch as B
    monkeypatch.setenv("PYCFD_B200_CACHE", str(tmp_path))
    tuner = B.Autotuner(steps=2, warmup=1)
    cfg = _cavities()[0]
    choice = tuner.choose(cfg)
    assert choice in [dict(c) for c in B.CANDIDATES]
    again = B.Autotuner(steps=2, warmup=1)
    assert again.choose(cfg) == choice and (tmp_path / "autotune.json").exists()
