"""The 256-cavity batch at its own sizes: a sampled subset against the oracle (needs a B200).

From ``cavity_batch_configs(256, seed=0)`` (N in {64, 96, 128, 192, 256}, Re
log-uniform in [100, 2000], lid speed uniform in [0.5, 1.5], adaptive dt at CFL 0.5,
MG-PCG 1e-10) the first cavity of each size and the highest-Re cavity of the 64^2
group run as ONE batch for 20 steps.  The reference's step for each of them is the
oracle's restatement of ``ProjectionSolver.step`` + ``TimeStepper.compute_dt``
(pycfd/core/solver.py:686-731, pycfd/core/timestepper.py:94-113) with the lid speed as
a ``MovingWall`` velocity (pycfd/core/boundary.py:181-192).

Bars: the batched FP64 path within 1e-10 relative of the oracle on u, v and p with
identical step counts and clocks; the batched mixed path the autotuner picks within
1e-6 (relative to the largest velocity) of the FP64 oracle velocities, with
max|div u| <= 1e-8 in every cavity.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

STEPS = 20


def _subset():
    from pycfd_b200.batch import cavity_batch_configs
    cfgs = cavity_batch_configs(count=256, seed=0)
    pick, seen = [], set()
    for k, c in enumerate(cfgs):
        if c.nx not in seen:
            seen.add(c.nx)
            pick.append(k)
    k64 = max((k for k, c in enumerate(cfgs) if c.nx == 64), key=lambda k: cfgs[k].re)
    if k64 not in pick:
        pick.append(k64)
    return [cfgs[k] for k in pick]


@pytest.fixture(scope="module")
def oracle_runs():
    from oracle import OracleSolver
    from oracle.projection import OracleStepper
    out = []
    for cfg in _subset():
        s = OracleSolver(cfg)
        u, v, p = s.initialize()
        (u, v, p, t, step), info = OracleStepper(s).run((u, v, p, 0.0, 0), max_steps=STEPS)
        assert step == STEPS
        out.append((cfg, u, v, p, t))
    return out


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def test_subset_covers_every_size_and_the_hardest_cavity():
    cfgs = _subset()
    assert sorted({c.nx for c in cfgs}) == [64, 96, 128, 192, 256]
    assert max(c.re for c in cfgs if c.nx == 64) > 1000.0


def test_batched_fp64_matches_oracle_at_config_sizes(oracle_runs):
    from pycfd_b200.batch import BatchedSolver, BatchOptions
    cfgs = [r[0] for r in oracle_runs]
    b = BatchedSolver(cfgs, BatchOptions(precision="fp64"))
    b.step(STEPS)
    st = b.status()
    for k, (cfg, u, v, p, t) in enumerate(oracle_runs):
        assert st["steps"][k] == STEPS and st["frozen"][k] == 0, (cfg.name, st)
        assert st["t"][k] == pytest.approx(t, rel=1e-12), cfg.name
        gu, gv, gp = b.fields[k].numpy()
        errs = (_rel(gu, u), _rel(gv, v), _rel(gp, p))
        assert max(errs) < 1e-10, (cfg.name, cfg.nx, cfg.re, errs)


def test_batched_mixed_autotuned_within_bounds_at_config_sizes(oracle_runs):
    from pycfd_b200.batch import BatchAutotuner, BatchedSolver
    cfgs = [r[0] for r in oracle_runs]
    opts = BatchAutotuner(allowed_precisions=("mixed",)).choose(cfgs)
    assert opts.precision == "mixed"
    b = BatchedSolver(cfgs, opts)
    b.step(STEPS)
    st = b.status()
    for k, (cfg, u, v, p, t) in enumerate(oracle_runs):
        assert st["steps"][k] == STEPS and st["frozen"][k] == 0, cfg.name
        gu, gv, _ = b.fields[k].numpy()
        scale = max(np.abs(u).max(), np.abs(v).max())
        err = max(np.abs(gu - u).max(), np.abs(gv - v).max()) / scale
        assert err <= 1e-6, (cfg.name, cfg.nx, cfg.re, err)
        assert b.field_stats(k).max_div <= 1e-8, cfg.name
