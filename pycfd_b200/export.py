"""Checkpoints in the reference's ``.npz`` format (``pycfd/analysis/export.py:214-276``).

A checkpoint holds the ghosted ``u, v, p``, ``t``, ``step``, the configuration
as JSON and a provenance record (also written beside the archive as
``<name>.provenance.json``), under the reference's keys, so GPU runs resume in
the reference and the reference's checkpoints resume here.  The provenance
record carries the reference's fields (``generated_utc``, ``command``,
``python``, ``platform``, ``git_commit`` when known, ``config``, ``units``),
with ``pycfd_version`` naming this package as the writer.
"""

from __future__ import annotations

import json
import platform
import shlex
import subprocess
import sys
from datetime import datetime, timezone
from pathlib import Path

import numpy as np

from .config import SimulationConfig
from .fields import FlowField
from .mesh import StructuredMesh

VERSION = "0.2.0"
SOLVER_UNITS = {"system": "solver", "note": "non-dimensional; u_ref = l_ref = 1"}


def _git_commit() -> str | None:
    root = Path(__file__).resolve().parent
    try:
        rev = subprocess.run(["git", "rev-parse", "--short", "HEAD"], cwd=root, capture_output=True,
                             text=True, timeout=2.0)
        if rev.returncode != 0:
            return None
        commit = rev.stdout.strip()
        dirty = subprocess.run(["git", "status", "--porcelain"], cwd=root, capture_output=True, text=True,
                               timeout=2.0)
        if dirty.returncode == 0 and dirty.stdout.strip():
            commit += "+"
        return commit
    except (OSError, subprocess.SubprocessError):
        return None


def provenance_record(config: SimulationConfig | None = None, extra: dict | None = None) -> dict:
    """The record of the run that wrote a file, with the reference's keys
    (``pycfd/analysis/provenance.py:84-118``) and its ``units`` block
    (``pycfd/analysis/export.py:70-92``)."""
    record = {
        "pycfd_version": f"pycfd_b200 {VERSION}",
        "generated_utc": datetime.now(timezone.utc).isoformat(timespec="seconds"),
        "command": shlex.join(sys.argv) if sys.argv else "",
        "python": platform.python_version(),
        "platform": platform.platform(),
    }
    commit = _git_commit()
    if commit is not None:
        record["git_commit"] = commit
    if config is not None:
        record["config"] = config.to_dict()
    if extra:
        record["extra"] = dict(extra)
    record["units"] = dict(SOLVER_UNITS)
    return record


def write_sidecar(path, record: dict) -> Path:
    """``<path>.provenance.json`` beside an output file (suffix replaced)."""
    sidecar = Path(path).with_suffix(".provenance.json")
    sidecar.parent.mkdir(parents=True, exist_ok=True)
    sidecar.write_text(json.dumps(record, indent=2), encoding="utf-8")
    return sidecar


def save_checkpoint(fields: FlowField, config: SimulationConfig, path, provenance=None) -> Path:
    """The ghosted state, clock and configuration for an exact restart."""
    path = Path(path)
    if path.suffix != ".npz":
        path = path.with_suffix(".npz")
    path.parent.mkdir(parents=True, exist_ok=True)
    u, v, p = fields.numpy()
    record = provenance_record(config) if provenance is None else dict(provenance)
    record.setdefault("units", dict(SOLVER_UNITS))
    np.savez_compressed(path, u=u, v=v, p=p, t=np.array(fields.t), step=np.array(fields.step),
                        config=np.array(config.to_json()), provenance=np.array(json.dumps(record)))
    write_sidecar(path, record)
    return path


def checkpoint_provenance(path) -> dict | None:
    """The provenance embedded in a checkpoint, or ``None`` for files without one."""
    path = Path(path)
    if not path.exists():
        raise FileNotFoundError(f"checkpoint not found: {path}")
    with np.load(path, allow_pickle=False) as npz:
        if "provenance" not in npz.files:
            return None
        return json.loads(str(npz["provenance"]))


def load_checkpoint(path, device="cuda"):
    """Return ``(FlowField, SimulationConfig)`` from a checkpoint file."""
    path = Path(path)
    if not path.exists():
        raise FileNotFoundError(f"checkpoint not found: {path}")
    with np.load(path, allow_pickle=False) as npz:
        config = SimulationConfig.from_dict(json.loads(str(npz["config"])))
        mesh = StructuredMesh.from_config(config)
        u, v, p = npz["u"], npz["v"], npz["p"]
        t, step = float(npz["t"]), int(npz["step"])
    for arr, expected, label in ((u, mesh.u_shape, "u"), (v, mesh.v_shape, "v"), (p, mesh.p_shape, "p")):
        if arr.shape != expected:
            raise ValueError(f"checkpoint {label} has shape {arr.shape}, expected {expected}; the file "
                             "does not match its stored configuration")
    return FlowField.from_numpy(mesh, u, v, p, t, step, device=device), config
