"""Checkpoint interchange with the reference (pycfd/analysis/export.py:214-276).

``golden/ref_checkpoint.npz`` was written by the reference's own
``Simulation.save_checkpoint`` (cavity 32x32, 20 steps) and
``golden/ref_checkpoint_continued.npz`` is the reference's state 10 steps after
resuming from it.  ``golden/interchange.npz`` records that a checkpoint written
by this package's writer was read back by the reference's ``load_checkpoint``
with every array, the clock and the configuration unchanged.
"""

import json
import os

import numpy as np
import pytest

import cases
from pycfd_b200 import export
from pycfd_b200.config import BCKind, BCSpec, SimulationConfig

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_reference_checkpoint_loads_bit_for_bit():
    ref = np.load(os.path.join(GOLDEN, "ref_checkpoint.npz"))
    f, cfg = export.load_checkpoint(os.path.join(GOLDEN, "ref_checkpoint.npz"), device="cpu")
    u, v, p = f.numpy()
    assert np.array_equal(u, ref["u"]) and np.array_equal(v, ref["v"]) and np.array_equal(p, ref["p"])
    assert f.t == float(ref["t"]) and f.step == int(ref["step"]) == 20
    want = cases.to_config(cases.CKPT_CAVITY, SimulationConfig, BCSpec, BCKind)
    assert json.loads(cfg.to_json()) == json.loads(want.to_json())
    assert export.checkpoint_provenance(os.path.join(GOLDEN, "ref_checkpoint.npz"))["config"]["nx"] == 32


def test_written_checkpoint_has_the_reference_schema(tmp_path):
    """Same archive keys and dtypes as the reference's file, a sidecar, the provenance
    fields the reference writes, and an exact round trip."""
    ref = np.load(os.path.join(GOLDEN, "ref_checkpoint.npz"))
    f, cfg = export.load_checkpoint(os.path.join(GOLDEN, "ref_checkpoint.npz"), device="cpu")
    path = export.save_checkpoint(f, cfg, tmp_path / "ours")
    assert path.suffix == ".npz" and (tmp_path / "ours.provenance.json").exists()
    mine = np.load(path)
    assert sorted(mine.files) == sorted(ref.files)
    for k in ref.files:
        assert mine[k].dtype.kind == ref[k].dtype.kind and mine[k].shape == ref[k].shape, k
    rec = json.loads(str(mine["provenance"]))
    theirs = json.loads(str(ref["provenance"]))
    for key in ("pycfd_version", "generated_utc", "command", "python", "platform", "config", "units"):
        assert key in rec and key in theirs
    g, cfg2 = export.load_checkpoint(path, device="cpu")
    for a, b in zip(g.numpy(), f.numpy()):
        assert np.array_equal(a, b)
    assert (g.t, g.step) == (f.t, f.step) and cfg2.to_json() == cfg.to_json()
    assert bool(np.load(os.path.join(GOLDEN, "interchange.npz"))["loaded_by_reference"])


@pytest.mark.gpu
def test_resume_from_reference_checkpoint_continues_like_the_reference():
    pytest.importorskip("torch")
    from pycfd_b200.simulation import Simulation
    sim = Simulation.from_checkpoint(os.path.join(GOLDEN, "ref_checkpoint.npz"))
    assert sim.fields.step == 20
    sim.run(max_steps=10)
    want = np.load(os.path.join(GOLDEN, "ref_checkpoint_continued.npz"))
    assert sim.fields.step == int(want["step"]) == 30
    assert sim.fields.t == pytest.approx(float(want["t"]), rel=1e-13)
    for a, k in zip(sim.fields.numpy(), ("u", "v", "p")):
        assert np.abs(a - want[k]).max() / np.abs(want[k]).max() < 1e-10, k


@pytest.mark.gpu
def test_gpu_state_round_trips_through_a_checkpoint(tmp_path):
    pytest.importorskip("torch")
    from pycfd_b200.simulation import Simulation
    cfg = cases.to_config(cases.CKPT_CAVITY, SimulationConfig, BCSpec, BCKind)
    sim = Simulation(cfg)
    sim.run(max_steps=5)
    path = sim.save_checkpoint(tmp_path / "gpu.npz")
    back = Simulation.from_checkpoint(path)
    again = Simulation.from_checkpoint(path)
    for a, b in zip(back.fields.numpy(), sim.fields.numpy()):
        assert np.array_equal(a, b)
    sim.run(max_steps=3)
    back.run(max_steps=3)
    again.run(max_steps=3)
    # The Poisson warm start is solver state, not checkpoint content (the
    # reference keeps it in the solver object, pycfd/core/solver.py:659-663), so
    # a restored run starts its first solve cold: it agrees with the
    # uninterrupted run to the solve tolerance, and bit for bit with another
    # restore of the same file.
    assert back.fields.step == sim.fields.step and back.fields.t == sim.fields.t
    for a, b, c in zip(back.fields.numpy(), sim.fields.numpy(), again.fields.numpy()):
        assert np.array_equal(a, c)
        assert np.abs(a - b).max() <= 1e-8 * max(np.abs(b).max(), 1.0)
