"""Pin the CPU oracle against golden vectors produced by the reference itself.

The fixtures in ``tests/golden`` were written by ``tests/golden/make_golden.py``
running the reference solver.  Integer/bool work and the stencil must match
exactly; solver outputs within a few ulps of their tolerance-limited spread.
"""

import numpy as np
import pytest
import scipy.sparse as sp

import cases
from oracle import momentum_rhs, assemble_poisson, make_solver, Hierarchy, OracleSolver
from oracle.projection import circle_mask_oracle, OracleStepper
from pycfd_b200.config import SimulationConfig, BCSpec, BCKind


def csr(g, prefix):
    return sp.csr_matrix((g[prefix + "_data"], g[prefix + "_indices"], g[prefix + "_indptr"]),
                         shape=tuple(g[prefix + "_shape"]))


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("k", range(4))
def test_momentum_rhs_bit_exact(golden, k):
    g = golden("rhs.npz")
    ru, rv = momentum_rhs(g[f"c{k}_u"], g[f"c{k}_v"], *g[f"c{k}_args"])
    assert np.array_equal(ru, g[f"c{k}_rhs_u"])
    assert np.array_equal(rv, g[f"c{k}_rhs_v"])


@pytest.mark.parametrize("name", ["walls", "periodic", "periodic_x", "obstacle", "dirichlet",
                                  "isolated"])
def test_poisson_assembly_exact(golden, name):
    g = golden("poisson.npz")
    nx, ny, lx, ly, px, py = g[name + "_geom"]
    nx, ny = int(nx), int(ny)
    dirichlet = {"right": 0.3} if name == "dirichlet" else None
    s = assemble_poisson(nx, ny, lx / nx, ly / ny, bool(px), bool(py),
                         g[name + "_solid"] if g[name + "_solid"].any() else None, dirichlet)
    A = s.A.tocsr()
    A.sort_indices()
    ref = csr(g, name + "_A")
    assert np.array_equal(A.indptr, ref.indptr)
    assert np.array_equal(A.indices, ref.indices)
    assert np.array_equal(A.data, ref.data)
    assert np.array_equal(s.fluid, g[name + "_fluid"])
    assert s.singular == bool(g[name + "_singular"])
    assert s.pin == int(g[name + "_pin"])
    assert np.array_equal(s.bc_rhs, g[name + "_bc"])


@pytest.mark.parametrize("name", ["walls", "periodic", "obstacle", "odd_dirichlet"])
def test_multigrid_hierarchy_matches(golden, name):
    g = golden("multigrid.npz")
    A0 = csr(g, name + "_A0")
    h = Hierarchy(A0, tuple(g[name + "_shape0"]), g[name + "_active0"],
                  name != "odd_dirichlet")
    assert len(h.levels) == int(g[name + "_nlev"])
    for l, lv in enumerate(h.levels):
        assert tuple(lv.shape) == tuple(g[f"{name}_shape{l}"])
        assert np.array_equal(lv.active, g[f"{name}_active{l}"])
        assert lv.weight == pytest.approx(float(g[f"{name}_w{l}"]), rel=1e-13)
        ref = csr(g, f"{name}_A{l}").toarray()
        assert np.abs(lv.A.toarray() - ref).max() <= 1e-12 * np.abs(ref).max()
        if l:
            refp = csr(g, f"{name}_P{l}").toarray()
            assert np.abs(lv.P.toarray() - refp).max() <= 1e-13
    z = h.apply(g[name + "_r"])
    assert rel(z, g[name + "_z"]) < 1e-12


@pytest.mark.parametrize("case", ["walls", "periodic"])
@pytest.mark.parametrize("kind,tol", [("cg", 1e-12), ("jacobi", 1e-7), ("sor", 1e-11),
                                      ("multigrid", 1e-12), ("mgcg", 1e-12)])
def test_solvers_match(golden, case, kind, tol):
    g = golden("solvers.npz")
    if case == "walls":
        s = assemble_poisson(24, 24, 1 / 24, 1 / 24)
    else:
        s = assemble_poisson(16, 20, 1 / 16, 1.25 / 20, True, True)
    solver = make_solver(kind, s, tol=tol, maxiter=200_000)
    p = solver.solve(g[case + "_rhs"], g[case + "_p0"])
    assert rel(p, g[f"{case}_{kind}_p"]) < 1e-11
    assert rel(p, g[f"{case}_direct_p"]) < 50 * tol
    if kind not in ("cg",):
        assert solver.last_iterations == int(g[f"{case}_{kind}_it"])


def _cfg(d):
    return cases.to_config(d, SimulationConfig, BCSpec, BCKind)


@pytest.mark.parametrize("name", list(cases.STEP_CASES))
def test_steps_match(golden, name):
    g = golden("steps.npz")
    spec = cases.STEP_CASES[name]
    cfg = cases.step_config(spec, SimulationConfig, BCSpec, BCKind)
    solid = None
    if "circle" in spec:
        solid = circle_mask_oracle(cfg.nx, cfg.ny, cfg.lx, cfg.ly, *spec["circle"])
        assert np.array_equal(solid, g[name + "_solid"])
    s = OracleSolver(cfg, solid)
    u, v, p = s.initialize(*cases.step_init(spec, cfg.nx, cfg.ny, cfg.lx, cfg.ly))
    assert rel(u, g[name + "_u0"]) < 1e-12 and rel(v, g[name + "_v0"]) < 1e-12
    if cfg.advection_scheme.value == "upwind":
        s.set_upwind_blend(s.upwind_blend_for(u, v, spec["dt"]))
    fx = []
    for _ in range(spec["steps"]):
        u, v, p = s.step(u, v, spec["dt"])
        fx.append(s.body_force_reaction[0])
    tol = 1e-7 if "jacobi" in name else 1e-10
    assert rel(u, g[name + "_u"]) < tol
    assert rel(v, g[name + "_v"]) < tol
    assert rel(p, g[name + "_p"]) < tol
    if solid is not None:
        assert rel(np.array(fx), g[name + "_fx"]) < 1e-8


def test_cylinder_mask_bit_exact_full_size(golden):
    g = golden("masks.npz")
    m = circle_mask_oracle(2048, 1024, 2.0, 1.0, (0.5, 0.5), 0.05)
    assert int(m.sum()) == int(g["big_count"])
    assert np.array_equal(np.packbits(m.ravel()), g["big_bits"])
    assert np.array_equal(circle_mask_oracle(256, 128, 2.0, 1.0, (0.5, 0.5), 0.05), g["small"])


def test_cavity64_first_100_steps(golden):
    """Adaptive-dt CG cavity (the 64x64 Re 100 workload) against the reference, 100 steps."""
    g = golden("cavity64.npz")
    cfg = _cfg(cases.CAVITY64)
    s = OracleSolver(cfg)
    st = OracleStepper(s)
    u, v, p = s.initialize()
    (u, v, p, t, step), _ = st.run((u, v, p, 0.0, 0), t_end=1e9, max_steps=100)
    assert t == float(g["s100_t"])
    for a, k in ((u, "u"), (v, "v"), (p, "p")):
        assert rel(a, g["s100_" + k]) < 1e-10
