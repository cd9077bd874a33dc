"""GPU path against the oracle and the reference's golden vectors (needs a B200).

Every call goes through the C ABI (``libpycfd_b200.so``) via the package's
Python layer.  Bars: bit-exact for the stencil, the divergence, the boundary
passes and the masks; 1e-10 relative (max norm) on u, v, p for whole steps at
the reference's solver tolerance (1e-7 for the slowly converging Jacobi case).
"""

import ctypes as C

import numpy as np
import pytest

import cases
from oracle import OracleSolver, Walls, divergence as oracle_div
from oracle.projection import circle_mask_oracle
from pycfd_b200.config import BCKind, BCSpec, SimulationConfig, PressureSolver

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def rel(a, b):
    a = a.detach().cpu().numpy() if hasattr(a, "detach") else np.asarray(a)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def dev(a):
    return torch.as_tensor(np.ascontiguousarray(a), device="cuda")


def host(t):
    return t.detach().cpu().numpy()


@pytest.fixture(scope="module")
def lib():
    from pycfd_b200 import _lib, build
    build.build()
    return _lib.load()


def _cfg(d, **kw):
    return cases.to_config(d, SimulationConfig, BCSpec, BCKind, **kw)


def _solver(cfg, solid=None, **kw):
    from pycfd_b200.solver import ProjectionSolver
    return ProjectionSolver(cfg, obstacle=solid, **kw)


# --------------------------------------------------------------------------- #
@pytest.mark.parametrize("k", range(4))
def test_momentum_rhs_bit_exact(lib, golden, k):
    from pycfd_b200 import _lib
    g = golden("rhs.npz")
    u, v = dev(g[f"c{k}_u"]), dev(g[f"c{k}_v"])
    nx, ny = u.shape[0] - 3, u.shape[1] - 2
    ru = torch.empty((nx + 1, ny), dtype=torch.float64, device="cuda")
    rv = torch.empty((nx, ny + 1), dtype=torch.float64, device="cuda")
    dx, dy, nu, blend, fx, fy = (float(a) for a in g[f"c{k}_args"])
    _lib.check(lib.pycfd_momentum_rhs(_lib.ptr(u), _lib.ptr(v), nx, ny, dx, dy, nu, blend, fx, fy,
                                      _lib.ptr(ru), _lib.ptr(rv), None))
    torch.cuda.synchronize()
    assert np.array_equal(host(ru), g[f"c{k}_rhs_u"])
    assert np.array_equal(host(rv), g[f"c{k}_rhs_v"])


def test_divergence_bit_exact(lib):
    from pycfd_b200 import _lib
    rng = np.random.default_rng(3)
    nx, ny = 37, 29
    u, v = rng.standard_normal((nx + 3, ny + 2)), rng.standard_normal((nx + 2, ny + 3))
    out = torch.empty((nx, ny), dtype=torch.float64, device="cuda")
    ud, vd = dev(u), dev(v)          # keep the device copies alive across the launch
    _lib.check(lib.pycfd_divergence(_lib.ptr(ud), _lib.ptr(vd), nx, ny, 0.1, 0.07,
                                    _lib.ptr(out), None))
    torch.cuda.synchronize()
    assert np.array_equal(host(out), oracle_div(u, v, 0.1, 0.07))


BC_MIXES = {
    "cavity": cases.bcs(top=("moving_wall", 1.0)),
    "periodic": cases.PER,
    "channel": cases.bcs(left=("periodic",), right=("periodic",)),
    "inlet_outlet": cases.bcs(left=("inlet", 1.0), right=("outlet",), top=("symmetry",),
                              bottom=("symmetry",)),
    "parabolic_pressure_outlet": cases.bcs(left=("inlet", 1.0, "parabolic"),
                                           right=("pressure_outlet", 0.0, "uniform", 0.3)),
    "periodic_y_mixed": cases.bcs(bottom=("periodic",), top=("periodic",),
                                  left=("moving_wall", -0.5), right=("outlet",)),
}


@pytest.mark.parametrize("name", list(BC_MIXES))
@pytest.mark.parametrize("predictor", [True, False])
def test_boundary_pass_bit_exact(lib, name, predictor):
    """Every boundary face and ghost, corners included, with the outlet mass balance."""
    from pycfd_b200 import _lib
    d = dict(nx=14, ny=11, lx=1.4, ly=1.1, re=100.0, pressure_solver="cg",
             boundary_config=BC_MIXES[name])
    cfg = _cfg(d)
    s = _solver(cfg)
    rng = np.random.default_rng(11)
    u, v = rng.standard_normal(s.mesh.u_shape), rng.standard_normal(s.mesh.v_shape)
    ud, vd = dev(u), dev(v)
    _lib.check(lib.pycfd_apply_velocity_bc(s._h, _lib.ptr(ud), _lib.ptr(vd), int(predictor), 1, None))
    torch.cuda.synchronize()
    w = Walls(cfg.boundary_config, cfg.nx, cfg.ny, cfg.lx, cfg.ly)
    w.apply_velocity(u, v, predictor=predictor)
    w.enforce_global_mass_balance(u, v)
    gu, gv = host(ud), host(vd)
    # the mass balance sums in a different order: allow one ulp there, exact elsewhere
    assert np.abs(gu - u).max() <= 4e-16 * max(1.0, np.abs(u).max())
    assert np.abs(gv - v).max() <= 4e-16 * max(1.0, np.abs(v).max())
    if not w.outlets:
        assert np.array_equal(gu, u) and np.array_equal(gv, v)


@pytest.mark.parametrize("case", ["walls", "periodic"])
@pytest.mark.parametrize("kind,tol", [("cg", 1e-12), ("jacobi", 1e-7), ("sor", 1e-11),
                                      ("multigrid", 1e-12), ("mgcg", 1e-12)])
def test_poisson_solvers_match_reference(lib, golden, case, kind, tol):
    g = golden("solvers.npz")
    if case == "walls":
        d = dict(nx=24, ny=24, re=100.0, boundary_config=cases.bcs())
    else:
        d = dict(nx=16, ny=20, lx=1.0, ly=1.25, re=100.0, boundary_config=cases.PER)
    s = _solver(_cfg(d, pressure_solver=kind, poisson_tol=tol, poisson_maxiter=200_000))
    p = s.pressure_solver.solve(g[case + "_rhs"], g[case + "_p0"])
    ref = g[f"{case}_direct_p"]
    assert rel(p, ref) < 50 * tol
    assert rel(p, g[f"{case}_{kind}_p"]) < 50 * tol
    assert s.pressure_solver.last_residual < (tol if kind != "cg" else 10 * tol)
    if kind in ("mgcg", "multigrid"):
        assert abs(s.pressure_solver.last_iterations - int(g[f"{case}_{kind}_it"])) <= 1


@pytest.mark.parametrize("name", ["walls", "periodic", "obstacle", "odd_dirichlet"])
def test_vcycle_matches_reference(lib, golden, name):
    """One V-cycle (the preconditioner) against the reference hierarchy's apply()."""
    from pycfd_b200 import _lib
    g = golden("multigrid.npz")
    geo = {"walls": dict(nx=32, ny=32, boundary_config=cases.bcs()),
           "periodic": dict(nx=24, ny=20, lx=1.2, ly=1.0, boundary_config=cases.PER),
           "obstacle": dict(nx=40, ny=24, lx=5.0 / 3.0, ly=1.0, boundary_config=cases.bcs()),
           "odd_dirichlet": dict(nx=33, ny=17, lx=33 / 17, ly=1.0,
                                 boundary_config=cases.bcs(right=("pressure_outlet",)))}[name]
    cfg = _cfg({**geo, "re": 100.0, "pressure_solver": "mgcg"})
    solid = None
    if name == "obstacle":
        solid = circle_mask_oracle(40, 24, 5.0 / 3.0, 1.0, (0.6, 0.5), 0.2)
    s = _solver(cfg, solid)
    r = dev(g[name + "_r"])
    z = torch.empty_like(r)
    _lib.check(lib.pycfd_mg_apply(s._h, _lib.ptr(r), _lib.ptr(z), None))
    torch.cuda.synchronize()
    assert rel(z, g[name + "_z"]) < 1e-12


def test_vcycle_is_symmetric(lib):
    """The preconditioner materialised column by column is symmetric (test_multigrid.py:339-359)."""
    from pycfd_b200 import _lib
    cfg = _cfg(dict(nx=16, ny=16, re=100.0, pressure_solver="mgcg",
                    boundary_config=cases.bcs(top=("moving_wall", 1.0))))
    s = _solver(cfg)
    n = 256
    M = np.zeros((n, n))
    for k in range(n):
        e = torch.zeros(n, dtype=torch.float64, device="cuda")
        e[k] = 1.0
        z = torch.empty_like(e)
        _lib.check(lib.pycfd_mg_apply(s._h, _lib.ptr(e), _lib.ptr(z), None))
        M[:, k] = host(z)
    assert np.abs(M - M.T).max() < 1e-12 * np.abs(M).max()


def _run_case(name, spec):
    cfg = cases.step_config(spec, SimulationConfig, BCSpec, BCKind)
    solid = None
    if "circle" in spec:
        solid = circle_mask_oracle(cfg.nx, cfg.ny, cfg.lx, cfg.ly, *spec["circle"])
    s = _solver(cfg, solid)
    fields = s.initialize(*cases.step_init(spec, cfg.nx, cfg.ny, cfg.lx, cfg.ly))
    init = fields.numpy()
    if cfg.advection_scheme.value == "upwind":
        s.set_upwind_blend(s.upwind_blend_for(fields, spec["dt"]))
    fx = []
    for _ in range(spec["steps"]):
        fields = s.step(fields, spec["dt"])
        fx.append(s.body_force_reaction[0])
    return s, init, fields, np.array(fx), solid


@pytest.mark.parametrize("name", list(cases.STEP_CASES))
def test_steps_match_reference(lib, golden, name):
    g = golden("steps.npz")
    spec = cases.STEP_CASES[name]
    s, init, f, fx, solid = _run_case(name, spec)
    tol = 1e-7 if "jacobi" in name else 1e-10
    assert rel(init[0], g[name + "_u0"]) < tol and rel(init[1], g[name + "_v0"]) < tol
    u, v, p = f.numpy()
    assert rel(u, g[name + "_u"]) < tol
    assert rel(v, g[name + "_v"]) < tol
    assert rel(p, g[name + "_p"]) < tol
    if solid is not None:
        assert rel(fx, g[name + "_fx"]) < 1e-8
        uu = u[s.u_upd][s.u_face_solid]
        vv = v[s.v_upd][s.v_face_solid]
        assert np.all(uu == 0.0) and np.all(vv == 0.0)


def test_cavity64_against_reference_run(lib, golden):
    """64x64 lid cavity, Re 100, CG 1e-10, adaptive CFL dt: 2000 steps against the reference."""
    from pycfd_b200.simulation import Simulation
    g = golden("cavity64.npz")
    sim = Simulation(_cfg(cases.CAVITY64))
    done = 0
    for target in (100, 500, 2000):
        sim.run(max_steps=target - done)
        done = target
        u, v, p = sim.fields.numpy()
        assert sim.fields.t == pytest.approx(float(g[f"s{target}_t"]), rel=1e-14)
        assert sim.fields.step == target
        for a, k in ((u, "u"), (v, "v"), (p, "p")):
            assert rel(a, g[f"s{target}_{k}"]) < 1e-10, (target, k)
    # at CG tol 1e-10 the divergence is set by the solve; match the reference's own level
    ref_div = np.abs(oracle_div(g["s2000_u"], g["s2000_v"], 1 / 64, 1 / 64)).max()
    assert sim.solver.max_divergence(sim.fields) < 10 * ref_div + 1e-12


def test_cylinder_force_history(lib, golden):
    """256x128 cylinder channel, MG-PCG: 30 steps of Cd/Cl and the final field."""
    from pycfd_b200.obstacles import circle_mask
    from pycfd_b200.simulation import Simulation
    from pycfd_b200.mesh import StructuredMesh
    g = golden("cylinder.npz")
    cfg = _cfg(cases.cylinder_cfg(256, 128))
    ob = circle_mask(StructuredMesh.from_config(cfg), (0.5, 0.5), 0.05)
    assert np.array_equal(ob.mask, g["mask"])
    u0, v0 = cases.cylinder_init(256, 128)
    sim = Simulation(cfg, obstacle=ob, u_init=u0, v_init=v0)
    cd, cl = [], []
    for _ in range(30):
        sim.run(max_steps=1)
        c = sim.force_coefficients()
        cd.append(c[0])
        cl.append(c[1])
    assert rel(np.array(cd), g["cd"]) < 1e-8
    assert np.abs(np.array(cl) - g["cl"]).max() < 1e-8 * np.abs(g["cd"]).max()
    u, v, p = sim.fields.numpy()
    assert rel(u, g["u"]) < 1e-10 and rel(v, g["v"]) < 1e-10 and rel(p, g["p"]) < 1e-10


def test_cylinder_long_force_history(lib, golden):
    """512x256 cylinder channel (the 2048x1024 case at reduced grid), MG-PCG 1e-10,
    adaptive dt: Cd/Cl after each of 2000 steps against the reference's own history,
    the clock step for step, and a 1-in-16 sample of the final u, v, p."""
    from pycfd_b200.obstacles import circle_mask
    from pycfd_b200.simulation import Simulation
    from pycfd_b200.mesh import StructuredMesh
    g = golden("cylinder_long.npz")
    cfg = _cfg(cases.cylinder_cfg(512, 256))
    ob = circle_mask(StructuredMesh.from_config(cfg), (0.5, 0.5), 0.05)
    u0, v0 = cases.cylinder_init(512, 256)
    sim = Simulation(cfg, obstacle=ob, u_init=u0, v_init=v0)
    cd, cl, t = [], [], []
    for _ in range(len(g["cd"])):
        sim.run(max_steps=1)
        c = sim.force_coefficients()
        cd.append(c[0])
        cl.append(c[1])
        t.append(sim.fields.t)
    cd, cl, t = np.array(cd), np.array(cl), np.array(t)
    scale = np.abs(g["cd"]).max()
    print(f"cylinder 512x256, 2000 steps: max|dCd| {np.abs(cd - g['cd']).max():.3e}, "
          f"max|dCl| {np.abs(cl - g['cl']).max():.3e}, max|dt| {np.abs(t - g['t']).max():.3e}")
    assert np.abs(t - g["t"]).max() <= 1e-12 * g["t"][-1]
    assert np.abs(cd - g["cd"]).max() <= 1e-8 * scale
    assert np.abs(cl - g["cl"]).max() <= 1e-8 * scale
    u, v, p = sim.fields.numpy()
    assert rel(u[::16, ::16], g["u16"]) < 1e-8
    assert rel(v[::16, ::16], g["v16"]) < 1e-8
    assert rel(p[::16, ::16], g["p16"]) < 1e-8
