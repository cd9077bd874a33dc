"""Stretched meshes on the GPU path against the reference's array path (needs a B200).

Bars: bit-exact momentum RHS and divergence (every product formed unfused, in the
reference's order); 1e-10 relative on u, v, p over whole runs at the reference's
solver tolerance (the stretched, row-scaled Poisson operator and its Galerkin
hierarchy with semi-coarsening); force history at 1e-9.  Sources:
pycfd/core/solver.py:336-543 (RHS, divergence), :643-683 (projection),
pycfd/core/pressure.py:193-207 (row scaling), pycfd/core/boundary.py:425-487
(outlet mass balance by face widths), pycfd/core/solver.py:265-274 (control-volume
areas of the reaction force).
"""

import numpy as np
import pytest

import cases
from pycfd_b200.config import BCKind, BCSpec, SimulationConfig
from pycfd_b200.mesh import NonUniformMeshError, StructuredMesh

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _cfg(d, **kw):
    return cases.to_config(d, SimulationConfig, BCSpec, BCKind, **kw)


def _rel(a, ref):
    return float(np.abs(np.asarray(a) - ref).max() / max(np.abs(ref).max(), 1e-300))


@pytest.mark.parametrize("k", range(len(cases.STRETCH_MESHES)))
def test_stretched_rhs_and_divergence_bit_exact(golden, k):
    from pycfd_b200.solver import ProjectionSolver
    g = golden("stretched.npz")
    nx, ny, lx, ly, sx, sy, cx, cy = cases.STRETCH_MESHES[k]
    c = dict(nx=nx, ny=ny, lx=lx, ly=ly, stretch_x=sx, stretch_y=sy, cluster_x=cx, cluster_y=cy,
             re=300.0 + 100 * k, body_force=(0.05 * k, -0.1), dt=1e-3, t_end=1.0, adaptive_dt=False,
             pressure_solver="cg", boundary_config=cases.bcs(top=("moving_wall", 1.0)), name="stretch")
    s = ProjectionSolver(_cfg(c))
    u = torch.as_tensor(g[f"m{k}_u"], device="cuda")
    v = torch.as_tensor(g[f"m{k}_v"], device="cuda")
    for b, blend in enumerate((0.0, 0.6)):
        ru, rv = s.momentum_rhs(u, v, blend)
        assert np.array_equal(ru.cpu().numpy(), g[f"m{k}_b{b}_rhs_u"]), (k, blend)
        assert np.array_equal(rv.cpu().numpy(), g[f"m{k}_b{b}_rhs_v"]), (k, blend)
    assert np.array_equal(s.divergence(u, v).cpu().numpy(), g[f"m{k}_div"])


def test_stretched_cavity_run_matches_reference(golden):
    """Walls-clustered on both axes, adaptive dt on the smallest cell, MG-PCG 1e-12."""
    from pycfd_b200.simulation import Simulation
    g = golden("stretched.npz")
    sim = Simulation(_cfg(cases.STRETCH_CAVITY))
    sim.run(max_steps=12)
    assert sim.fields.step == 12
    assert sim.fields.t == pytest.approx(float(g["cav_t"]), rel=1e-12)
    for a, key in zip(sim.fields.numpy(), ("u", "v", "p")):
        assert _rel(a, g["cav_" + key]) < 1e-10, key


def test_stretched_channel_past_cylinder_matches_reference(golden):
    """Inlet/outlet (mass balance by face widths) past a cylinder: the reaction force
    weighted by the faces' control volumes."""
    from pycfd_b200.obstacles import circle_mask
    from pycfd_b200.solver import ProjectionSolver
    g = golden("stretched.npz")
    cfg = _cfg(cases.STRETCH_CHANNEL)
    mesh = StructuredMesh.from_config(cfg)
    ob = circle_mask(mesh, *cases.STRETCH_CHANNEL_CIRCLE)
    assert np.array_equal(ob.mask, g["ch_solid"])
    s = ProjectionSolver(cfg, obstacle=ob.mask)
    f = s.initialize()
    fx, fy = [], []
    for _ in range(10):
        f = s.step(f, cfg.dt)
        fx.append(s.body_force_reaction[0])
        fy.append(s.body_force_reaction[1])
    for a, key in zip(f.numpy(), ("u", "v", "p")):
        assert _rel(a, g["ch_" + key]) < 1e-10, key
    # the channel is symmetric: lift is round-off (1e-15), so it is held to the drag's scale
    assert _rel(fx, g["ch_fx"]) < 1e-9
    assert np.abs(np.asarray(fy) - g["ch_fy"]).max() <= 1e-9 * np.abs(g["ch_fx"]).max()


def test_stretched_pressure_outlet_channel_matches_reference(golden):
    """Parabolic inlet, a Dirichlet (pressure outlet) wall: row-scaled Dirichlet terms, CG."""
    from pycfd_b200.solver import ProjectionSolver
    g = golden("stretched.npz")
    cfg = _cfg(cases.STRETCH_PRESSURE_OUTLET)
    s = ProjectionSolver(cfg)
    f = s.initialize()
    for _ in range(10):
        f = s.step(f, cfg.dt)
    for a, key in zip(f.numpy(), ("u", "v", "p")):
        assert _rel(a, g["po_" + key]) < 1e-10, key


def test_stretched_mixed_precision_tracks_fp64():
    from pycfd_b200.solver import GpuOptions, ProjectionSolver
    cfg = _cfg(cases.STRETCH_CAVITY, adaptive_dt=False, dt=2e-3)
    out = []
    for prec in ("fp64", "mixed"):
        s = ProjectionSolver(cfg, options=GpuOptions(precision=prec))
        f = s.initialize()
        for _ in range(10):
            f = s.step(f, cfg.dt)
        out.append(f.numpy())
        st = s.field_stats(f)
        assert st.max_div < 1e-8
    assert _rel(out[1][0], out[0][0]) < 1e-6 and _rel(out[1][1], out[0][1]) < 1e-6


def test_stretched_refusals():
    from pycfd_b200.batch import BatchedSolver
    from pycfd_b200.solver import ProjectionSolver
    per = {w: ("periodic",) for w in ("left", "right")}
    per.update(bottom=("no_slip",), top=("moving_wall", 1.0))
    with pytest.raises(NonUniformMeshError, match="periodic and stretched"):
        ProjectionSolver(_cfg(dict(nx=16, ny=16, stretch_x=1.1, re=100.0, pressure_solver="cg",
                                   boundary_config=per)))
    with pytest.raises(NotImplementedError, match="uniform meshes"):
        BatchedSolver([_cfg(dict(nx=16, ny=16, stretch_y=1.1, re=100.0, pressure_solver="mgcg",
                                 time_scheme="rk3", boundary_config=cases.bcs(top=("moving_wall", 1.0))))])


def test_stretched_les_viscosity_and_rhs_bit_exact(golden):
    """Per-cell filter width sqrt(dx_i dy_j), strains over the metric spacings, the
    stress-divergence viscous term after the stretched advection
    (pycfd/physics/turbulence.py:38-118, pycfd/core/solver.py:467-499)."""
    from pycfd_b200.solver import ProjectionSolver
    g = golden("stretched.npz")
    nx, ny, lx, ly, sx, sy, cx, cy = cases.STRETCH_MESHES[1]
    c = dict(nx=nx, ny=ny, lx=lx, ly=ly, stretch_x=sx, stretch_y=sy, cluster_x=cx, cluster_y=cy, re=3000.0,
             use_les=True, smagorinsky_cs=0.17, body_force=(0.1, -0.2), dt=1e-3, t_end=1.0, adaptive_dt=False,
             pressure_solver="cg", boundary_config=cases.bcs(top=("moving_wall", 1.0)), name="stretch_les")
    s = ProjectionSolver(_cfg(c))
    u = torch.as_tensor(g["les_u"], device="cuda")
    v = torch.as_tensor(g["les_v"], device="cuda")
    nu_c, nu_k = s.turbulence.eddy_viscosity(u, v, s.nu)
    assert np.array_equal(nu_c.cpu().numpy(), g["les_nu_c"])
    assert np.array_equal(nu_k.cpu().numpy(), g["les_nu_k"])
    for b, blend in enumerate((0.0, 0.6)):
        ru, rv = s.momentum_rhs(u, v, blend)
        assert np.array_equal(ru.cpu().numpy(), g[f"les_b{b}_rhs_u"]), blend
        assert np.array_equal(rv.cpu().numpy(), g[f"les_b{b}_rhs_v"]), blend


def test_stretched_les_cavity_matches_reference(golden):
    from pycfd_b200.solver import ProjectionSolver
    g = golden("stretched.npz")
    cfg = _cfg(cases.STRETCH_LES_CAVITY)
    s = ProjectionSolver(cfg)
    f = s.initialize()
    for _ in range(10):
        f = s.step(f, cfg.dt)
    for a, key in zip(f.numpy(), ("u", "v", "p")):
        assert _rel(a, g["lescav_" + key]) < 1e-10, key
