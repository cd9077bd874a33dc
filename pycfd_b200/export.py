"""Checkpoints in the reference's ``.npz`` format (``pycfd/analysis/export.py:214-276``).

A checkpoint holds the ghosted ``u, v, p``, ``t``, ``step``, the configuration
as JSON and a provenance record, so GPU runs resume in the reference and the
reference's checkpoints resume here.
"""

from __future__ import annotations

import json
import time
from pathlib import Path

import numpy as np

from .config import SimulationConfig
from .fields import FlowField
from .mesh import StructuredMesh


def save_checkpoint(fields: FlowField, config: SimulationConfig, path, provenance=None) -> Path:
    path = Path(path)
    if path.suffix != ".npz":
        path = path.with_suffix(".npz")
    path.parent.mkdir(parents=True, exist_ok=True)
    u, v, p = fields.numpy()
    record = provenance or {"writer": "pycfd_b200", "time": time.time(), "config": config.to_dict()}
    np.savez_compressed(path, u=u, v=v, p=p, t=np.array(fields.t), step=np.array(fields.step),
                        config=np.array(config.to_json()), provenance=np.array(json.dumps(record)))
    return path


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
            raise ValueError(f"checkpoint {label} has shape {arr.shape}, expected {expected}")
    return FlowField.from_numpy(mesh, u, v, p, t, step, device=device), config
