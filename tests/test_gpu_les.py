"""The Smagorinsky closure on the GPU path against the reference (needs a B200).

``golden/les.npz`` holds the reference's eddy viscosities (cell centres and
corners) and its momentum RHS in stress-divergence form on random fields
(pycfd/physics/turbulence.py:25-118, pycfd/core/solver.py:467-529), blend 0
and 0.6, and 10 steps of a 40x40 cavity at Re 5000 with use_les=True (CG 1e-12).
The viscosities and the RHS must agree bit for bit; the steps within 1e-10.
"""

import ctypes as C

import numpy as np
import pytest

import cases
from pycfd_b200.config import BCKind, BCSpec, SimulationConfig

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _cfg(k):
    nx, ny = ((20, 16), (13, 22))[k]
    return cases.to_config(dict(nx=nx, ny=ny, lx=1.0 + 0.1 * k, ly=1.0, re=2000.0, use_les=True,
                                smagorinsky_cs=0.17, body_force=(0.1, -0.2), dt=1e-3, t_end=1.0,
                                adaptive_dt=False, pressure_solver="cg",
                                boundary_config=cases.bcs(top=("moving_wall", 1.0)), name="les"),
                           SimulationConfig, BCSpec, BCKind)


@pytest.mark.parametrize("k", [0, 1])
def test_les_eddy_viscosity_and_rhs_bit_exact(golden, k):
    from pycfd_b200.solver import ProjectionSolver
    g = golden("les.npz")
    s = ProjectionSolver(_cfg(k))
    nu_c, nu_k = s.turbulence.eddy_viscosity(g[f"c{k}_u"], g[f"c{k}_v"], s.nu)
    assert np.array_equal(nu_c.cpu().numpy(), g[f"c{k}_nu_c"])
    assert np.array_equal(nu_k.cpu().numpy(), g[f"c{k}_nu_k"])
    ru, rv = s.momentum_rhs(g[f"c{k}_u"], g[f"c{k}_v"], float(g[f"c{k}_blend"]))
    assert np.array_equal(ru.cpu().numpy(), g[f"c{k}_rhs_u"])
    assert np.array_equal(rv.cpu().numpy(), g[f"c{k}_rhs_v"])
    assert s.turbulence.last_nu_t_max > 0.0


def test_les_cavity_steps_match_reference(golden):
    from pycfd_b200.solver import ProjectionSolver
    g = golden("les.npz")
    cfg = cases.to_config(cases.LES_CAVITY, SimulationConfig, BCSpec, BCKind)
    s = ProjectionSolver(cfg)
    f = s.initialize()
    for _ in range(10):
        f = s.step(f, cfg.dt)
    for a, key in zip(f.numpy(), ("u", "v", "p")):
        ref = g["cav_" + key]
        assert np.abs(a - ref).max() / np.abs(ref).max() < 1e-10, key
