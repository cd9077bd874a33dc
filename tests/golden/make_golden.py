"""Generate the golden fixtures in this folder by running the reference itself.

The reference (kiliancmd/pycfd, pure Python) is imported from a source tree
given as the first command-line argument, and driven through its own
public API.  Nothing here runs on the GPU host: the fixtures it writes are the
committed ``*.npz`` files beside this script, which the tests read.

    python tests/golden/make_golden.py /path/to/reference

Cases (all seeded, all synthetic):
  rhs.npz        momentum RHS (Numba kernel) on random ghosted fields, blend 0 / 0.6
  poisson.npz    assembled Poisson operators for six boundary/obstacle layouts
  multigrid.npz  hierarchies (A_l, P_l, weights) and one V-cycle for four layouts
  solvers.npz    solve() of every iterative solver on seeded right-hand sides
  steps.npz      initialise + N steps for nine boundary/solver/scheme mixes
  cavity64.npz   64x64 lid cavity, Re 100, CG 1e-10, adaptive dt: steps 100/500/2000
  cylinder.npz   256x128 cylinder channel, MG-PCG, 30 steps with Cd/Cl history
  masks.npz      circle_mask at 2048x1024 (packed bits) and at 256x128
  faces.npz      face ranges and face solid flags (total, per body) for four layouts
  cylinder_long.npz  512x256 cylinder, MG-PCG, 2000 steps: Cd/Cl/t history
  shapes.npz     polygon, rectangle and image masks with their fractions (200x120)
  ref_checkpoint.npz (+ _continued)  a reference checkpoint and the state 10 steps on
  interchange.npz  this package's checkpoint writer read back by the reference's loader
  les.npz        Smagorinsky eddy viscosity, LES momentum RHS, and 10 LES cavity steps
  stretched.npz  stretched meshes: widths/metrics, RHS, divergence, Poisson operator, and
                 runs of a stretched cavity, an inlet/outlet channel past a cylinder and
                 a pressure-outlet channel
"""

from __future__ import annotations

import os
import sys
import time

import numpy as np

if len(sys.argv) < 2:
    sys.exit("usage: python tests/golden/make_golden.py <path to the reference source tree>")
REF = sys.argv[1]
sys.path.insert(0, REF)

from pycfd.config import BCKind, BCSpec, SimulationConfig  # noqa: E402
from pycfd.core import kernels  # noqa: E402
from pycfd.core.mesh import StructuredMesh  # noqa: E402
from pycfd.core.multigrid import MultigridHierarchy  # noqa: E402
from pycfd.core.pressure import assemble_poisson_matrix, make_pressure_solver  # noqa: E402
from pycfd.core.solver import ProjectionSolver  # noqa: E402
from pycfd.core.timestepper import TimeStepper  # noqa: E402
from pycfd.geometry.obstacles import circle_mask  # noqa: E402
from pycfd.physics.incompressible import Simulation  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, OUT)
import cases  # noqa: E402


def save(name, **arrays):
    path = os.path.join(OUT, name)
    np.savez_compressed(path, **arrays)
    print(f"wrote {name}: {os.path.getsize(path) / 1024:.0f} KiB", flush=True)


def csr_parts(prefix, A, out):
    A = A.tocsr()
    A.sort_indices()
    out[prefix + "_data"] = A.data
    out[prefix + "_indices"] = A.indices.astype(np.int32)
    out[prefix + "_indptr"] = A.indptr.astype(np.int64)
    out[prefix + "_shape"] = np.array(A.shape)


def gen_rhs():
    out = {}
    for k, (nx, ny, blend) in enumerate(((24, 24, 0.0), (24, 24, 0.6), (20, 13, 0.6), (9, 31, 0.0))):
        u = np.random.default_rng(10 + k).standard_normal((nx + 3, ny + 2))
        v = np.random.default_rng(20 + k).standard_normal((nx + 2, ny + 3))
        ru, rv = np.empty((nx + 1, ny)), np.empty((nx, ny + 1))
        args = (0.01 * (1 + k), 0.02, 0.001 * (k + 1), blend, 0.1, -0.2)
        kernels._kernel_serial(u, v, *args, ru, rv)
        out.update({f"c{k}_u": u, f"c{k}_v": v, f"c{k}_args": np.array(args),
                    f"c{k}_rhs_u": ru, f"c{k}_rhs_v": rv})
    save("rhs.npz", **out)


def poisson_cases():
    m1 = StructuredMesh(12, 10, 1.2, 1.0)
    m2 = StructuredMesh(8, 12, 1.0, 1.5)
    m3 = StructuredMesh(10, 8)
    m4 = StructuredMesh(16, 16)
    m5 = StructuredMesh(12, 8, 1.5, 1.0)
    m6 = StructuredMesh(8, 8)
    ring = np.zeros((8, 8), bool)
    ring[2:5, 2:5] = True
    ring[3, 3] = False                       # a fluid cell enclosed by solid
    return [
        ("walls", m1, dict()),
        ("periodic", m2, dict(periodic_x=True, periodic_y=True)),
        ("periodic_x", m3, dict(periodic_x=True)),
        ("obstacle", m4, dict(solid_mask=circle_mask(m4, (0.5, 0.5), 0.2).mask)),
        ("dirichlet", m5, dict(dirichlet={"right": 0.3})),
        ("isolated", m6, dict(solid_mask=ring)),
    ]


def gen_poisson():
    out = {}
    for name, mesh, kw in poisson_cases():
        s = assemble_poisson_matrix(mesh, **kw)
        csr_parts(name + "_A", s.A, out)
        out[name + "_fluid"] = s.fluid
        out[name + "_singular"] = np.array(s.singular)
        out[name + "_pin"] = np.array(s.pin)
        out[name + "_bc"] = s.bc_rhs
        out[name + "_solid"] = kw.get("solid_mask", np.zeros(mesh.shape, bool))
        out[name + "_geom"] = np.array([mesh.nx, mesh.ny, mesh.lx, mesh.ly,
                                        kw.get("periodic_x", False), kw.get("periodic_y", False)],
                                       dtype=float)
    save("poisson.npz", **out)


def gen_multigrid():
    out = {}
    m1 = StructuredMesh(32, 32)
    m2 = StructuredMesh(24, 20, 1.2, 1.0)
    m3 = StructuredMesh(40, 24, 5.0 / 3.0, 1.0)
    m4 = StructuredMesh(33, 17, 33 / 17, 1.0)
    mg_cases = [
        ("walls", m1, dict()),
        ("periodic", m2, dict(periodic_x=True, periodic_y=True)),
        ("obstacle", m3, dict(solid_mask=circle_mask(m3, (0.6, 0.5), 0.2).mask)),
        ("odd_dirichlet", m4, dict(dirichlet={"right": 0.0})),
    ]
    for name, mesh, kw in mg_cases:
        s = assemble_poisson_matrix(mesh, **kw)
        h = MultigridHierarchy(s.A, mesh.shape, s.fluid, s.singular)
        out[name + "_nlev"] = np.array(h.n_levels)
        for l, lv in enumerate(h.levels):
            csr_parts(f"{name}_A{l}", lv.A, out)
            if lv.P is not None:
                csr_parts(f"{name}_P{l}", lv.P, out)
            out[f"{name}_w{l}"] = np.array(lv.weight)
            out[f"{name}_shape{l}"] = np.array(lv.shape)
            out[f"{name}_active{l}"] = lv.active
        r = np.random.default_rng(5).standard_normal(s.n)
        out[name + "_r"] = r
        out[name + "_z"] = h.apply(r)
    save("multigrid.npz", **out)


def gen_solvers():
    out = {}
    for case, mesh, kw in (("walls", StructuredMesh(24, 24), {}),
                           ("periodic", StructuredMesh(16, 20, 1.0, 1.25),
                            dict(periodic_x=True, periodic_y=True))):
        s = assemble_poisson_matrix(mesh, **kw)
        rhs = np.random.default_rng(7).standard_normal(mesh.shape)
        p0 = 0.1 * np.random.default_rng(8).standard_normal(mesh.shape)
        out[case + "_rhs"] = rhs
        out[case + "_p0"] = p0
        for kind, tol in (("cg", 1e-12), ("jacobi", 1e-7), ("sor", 1e-11),
                          ("multigrid", 1e-12), ("mgcg", 1e-12), ("direct", 1e-12)):
            solver = make_pressure_solver(kind, s, tol=tol, maxiter=200_000)
            p = solver.solve(rhs, p0 if kind != "direct" else None)
            out[f"{case}_{kind}_p"] = p
            out[f"{case}_{kind}_it"] = np.array(solver.last_iterations)
            out[f"{case}_{kind}_res"] = np.array(solver.last_residual)
    save("solvers.npz", **out)


def ref_config(d):
    return cases.to_config(d, SimulationConfig, BCSpec, BCKind)


def run_step_case(spec):
    cfg = cases.step_config(spec, SimulationConfig, BCSpec, BCKind)
    mesh = StructuredMesh.from_config(cfg)
    solid = None
    if "circle" in spec:
        solid = circle_mask(mesh, *spec["circle"]).mask
    solver = ProjectionSolver(cfg, mesh, solid)
    u_init, v_init = cases.step_init(spec, cfg.nx, cfg.ny, cfg.lx, cfg.ly)
    if spec.get("tg"):                       # the reference's own mesh coordinates
        Xu, Yu = mesh.u_grid()
        Xv, Yv = mesh.v_grid()
        u_init, v_init = np.sin(Xu) * np.cos(Yu), -np.cos(Xv) * np.sin(Yv)
    fields = solver.initialize(u_init, v_init)
    init = (fields.u.copy(), fields.v.copy(), fields.p.copy())
    fx, fy = [], []
    if cfg.advection_scheme.value == "upwind":
        solver.set_upwind_blend(solver.upwind_blend_for(fields, spec["dt"]))
    for _ in range(spec["steps"]):
        fields = solver.step(fields, spec["dt"])
        fx.append(solver.body_force_reaction[0])
        fy.append(solver.body_force_reaction[1])
    return init, fields, np.array(fx), np.array(fy), solid


def gen_steps():
    out = {}
    for name, spec in cases.STEP_CASES.items():
        t0 = time.perf_counter()
        init, f, fx, fy, solid = run_step_case(spec)
        out.update({f"{name}_u0": init[0], f"{name}_v0": init[1], f"{name}_p0": init[2],
                    f"{name}_u": f.u, f"{name}_v": f.v, f"{name}_p": f.p,
                    f"{name}_fx": fx, f"{name}_fy": fy,
                    f"{name}_solid": solid if solid is not None else np.zeros((1, 1), bool)})
        print(f"  {name}: {time.perf_counter() - t0:.1f}s", flush=True)
    save("steps.npz", **out)


def cavity64_config():
    return ref_config(cases.CAVITY64)


def gen_cavity64():
    sim = Simulation(cavity64_config())
    out = {}
    done = 0
    for target in (100, 500, 2000):
        sim.run(max_steps=target - done)
        done = target
        f = sim.fields
        out.update({f"s{target}_u": f.u, f"s{target}_v": f.v, f"s{target}_p": f.p,
                    f"s{target}_t": np.array(f.t), f"s{target}_step": np.array(f.step)})
        print(f"  cavity64 step {target}: t={f.t:.6f}", flush=True)
    save("cavity64.npz", **out)


def gen_cylinder():
    nx, ny = 256, 128
    cfg = ref_config(cases.cylinder_cfg(nx, ny))
    ob = circle_mask(StructuredMesh.from_config(cfg), (0.5, 0.5), 0.05)
    u0, v0 = cases.cylinder_init(nx, ny)
    sim = Simulation(cfg, obstacle=ob, u_init=u0, v_init=v0)
    cd, cl = [], []
    for _ in range(30):
        sim.run(max_steps=1)
        c = sim.force_coefficients()
        cd.append(c[0])
        cl.append(c[1])
    f = sim.fields
    save("cylinder.npz", u=f.u, v=f.v, p=f.p, t=np.array(f.t), cd=np.array(cd),
         cl=np.array(cl), mask=ob.mask)


def gen_faces():
    """Solvable face ranges and face solid flags, total and per body
    (pycfd/core/solver.py:62-79, :235-296), for bodies on periodic seams, at a
    pressure outlet and against walls."""
    out = {}
    for name, case in cases.FACE_CASES.items():
        cfg = ref_config({**dict(dt=1e-3, t_end=1.0, adaptive_dt=False, name=name), **case["cfg"]})
        bodies = cases.face_bodies(case, cfg.nx, cfg.ny)
        solid = np.logical_or.reduce(bodies)
        s = ProjectionSolver(cfg, None, solid, bodies=bodies)
        out[f"{name}_upd"] = np.array([s.u_upd[0].start, s.u_upd[0].stop, s.v_upd[1].start,
                                       s.v_upd[1].stop])
        out[f"{name}_u_face_solid"] = s.u_face_solid
        out[f"{name}_v_face_solid"] = s.v_face_solid
        if s.u_face_body:                      # kept only for two or more bodies
            out[f"{name}_u_face_body"] = np.stack(s.u_face_body)
            out[f"{name}_v_face_body"] = np.stack(s.v_face_body)
    save("faces.npz", **out)


def gen_cylinder_long():
    """512x256 cylinder channel (the 2048x1024 case at reduced grid), MG-PCG 1e-10,
    adaptive dt: Cd, Cl and t after each of 2000 steps, and every 16th value of the
    final u, v, p."""
    nx, ny, steps = 512, 256, 2000
    cfg = ref_config(cases.cylinder_cfg(nx, ny))
    ob = circle_mask(StructuredMesh.from_config(cfg), (0.5, 0.5), 0.05)
    u0, v0 = cases.cylinder_init(nx, ny)
    sim = Simulation(cfg, obstacle=ob, u_init=u0, v_init=v0)
    cd, cl, t = [], [], []
    for k in range(steps):
        sim.run(max_steps=1)
        c = sim.force_coefficients()
        cd.append(c[0])
        cl.append(c[1])
        t.append(sim.fields.t)
        if (k + 1) % 200 == 0:
            print(f"  cylinder_long step {k + 1}: t={t[-1]:.5f} cd={cd[-1]:.8f} cl={cl[-1]:.3e}",
                  flush=True)
    f = sim.fields
    save("cylinder_long.npz", cd=np.array(cd), cl=np.array(cl), t=np.array(t),
         u16=f.u[::16, ::16], v16=f.v[::16, ::16], p16=f.p[::16, ::16])


def gen_shapes():
    """polygon_mask (a 12-point star), rectangle_mask and mask_from_image (the
    picture of cases.shape_image, handed to the reference through a stand-in for
    matplotlib.image.imread, which is not installed here) on a 200x120 mesh:
    fraction and mask of each (pycfd/geometry/obstacles.py:87-367)."""
    import types
    from pycfd.geometry import obstacles as ob
    img = cases.shape_image()
    mpl = types.ModuleType("matplotlib")
    mpl_image = types.ModuleType("matplotlib.image")
    mpl_image.imread = lambda path: img
    mpl.image = mpl_image
    sys.modules.setdefault("matplotlib", mpl)
    sys.modules["matplotlib.image"] = mpl_image
    m = cases.SHAPE_MESH
    mesh = StructuredMesh(m["nx"], m["ny"], m["lx"], m["ly"])
    star = np.array(cases.STAR)
    pg = ob.polygon_mask(mesh, star)
    rc = ob.rectangle_mask(mesh, (0.31, 0.22), (0.93, 0.61))
    path = os.path.join(os.path.dirname(__file__), "_unused.png")
    open(path, "wb").close()                 # the reference checks that the path exists
    try:
        im = ob.mask_from_image(mesh, path, threshold=0.5)
        im2 = ob.mask_from_image(mesh, path, threshold=0.5, invert=True, subsamples=3)
    finally:
        os.remove(path)
    save("shapes.npz", star=star, poly_frac=pg.fraction, poly_mask=pg.mask,
         poly_len=np.array(pg.characteristic_length), rect_frac=rc.fraction, rect_mask=rc.mask,
         image=img, img_frac=im.fraction, img_mask=im.mask, img_len=np.array(im.characteristic_length),
         img_inv_frac=im2.fraction, img_inv_mask=im2.mask)


def gen_checkpoint():
    """A checkpoint written by the reference's own save_checkpoint (cavity 32x32,
    Re 100, MG-PCG 1e-12, 20 adaptive steps) and the reference's state 10 steps
    after resuming from it (pycfd/analysis/export.py:214-276)."""
    cfg = ref_config(cases.CKPT_CAVITY)
    sim = Simulation(cfg)
    sim.run(max_steps=20)
    path = os.path.join(os.path.dirname(__file__), "ref_checkpoint.npz")
    sim.save_checkpoint(path)
    side = os.path.join(os.path.dirname(__file__), "ref_checkpoint.provenance.json")
    if os.path.exists(side):
        os.remove(side)                      # the archive embeds the same record
    sim2 = Simulation.from_checkpoint(path)
    sim2.run(max_steps=10)
    f = sim2.fields
    save("ref_checkpoint_continued.npz", u=f.u, v=f.v, p=f.p, t=np.array(f.t), step=np.array(f.step))


def gen_interchange():
    """A checkpoint written by THIS package's writer (from host arrays, the same code
    path a GPU run takes after its device-to-host copy), loaded with the
    reference's own load_checkpoint (pycfd/analysis/export.py:253-276); records
    that it loaded and matched.  Needs pycfd_b200 importable beside the reference."""
    root = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    sys.path.insert(0, root)
    import json
    from pycfd.analysis.export import load_checkpoint
    from pycfd_b200 import export as ours
    from pycfd_b200.config import BCKind as OK, BCSpec as OS, SimulationConfig as OC
    from pycfd_b200.fields import FlowField as OF
    from pycfd_b200.mesh import StructuredMesh as OM
    g = np.load(os.path.join(os.path.dirname(__file__), "ref_checkpoint_continued.npz"))
    cfg = cases.to_config(cases.CKPT_CAVITY, OC, OS, OK)
    f = OF.from_numpy(OM.from_config(cfg), g["u"], g["v"], g["p"], float(g["t"]), int(g["step"]),
                      device="cpu")
    tmp = os.path.join(os.path.dirname(__file__), "_ours_tmp.npz")
    try:
        ours.save_checkpoint(f, cfg, tmp)
        rf, rcfg = load_checkpoint(tmp)
        same = (np.array_equal(rf.u, g["u"]) and np.array_equal(rf.v, g["v"])
                and np.array_equal(rf.p, g["p"]) and rf.t == float(g["t"]) and rf.step == int(g["step"]))
        cfg_same = rcfg.to_dict() == json.loads(cfg.to_json())
    finally:
        for x in (tmp, tmp.replace(".npz", ".provenance.json")):
            if os.path.exists(x):
                os.remove(x)
    assert same and cfg_same
    save("interchange.npz", loaded_by_reference=np.array(bool(same and cfg_same)))


def gen_les():
    """The Smagorinsky closure (pycfd/physics/turbulence.py:25-118 and the
    stress-divergence viscous term, pycfd/core/solver.py:467-529): eddy
    viscosities and the momentum RHS on random fields (blend 0 and 0.6), and a
    cavity run with use_les=True for 10 steps."""
    out = {}
    for k, (nx, ny, blend) in enumerate(((20, 16, 0.0), (13, 22, 0.6))):
        c = dict(nx=nx, ny=ny, lx=1.0 + 0.1 * k, ly=1.0, re=2000.0, use_les=True, smagorinsky_cs=0.17,
                 body_force=(0.1, -0.2), dt=1e-3, t_end=1.0, adaptive_dt=False, pressure_solver="cg",
                 boundary_config=cases.bcs(top=("moving_wall", 1.0)), name="les")
        cfg = ref_config(c)
        s = ProjectionSolver(cfg)
        rng = np.random.default_rng(30 + k)
        u = rng.standard_normal((nx + 3, ny + 2))
        v = rng.standard_normal((nx + 2, ny + 3))
        nu_c, nu_k = s.turbulence.eddy_viscosity(u, v, s.nu)
        ru, rv = s.momentum_rhs(u, v, blend)
        out.update({f"c{k}_u": u, f"c{k}_v": v, f"c{k}_blend": np.array(blend), f"c{k}_nu_c": nu_c,
                    f"c{k}_nu_k": nu_k, f"c{k}_rhs_u": np.array(ru), f"c{k}_rhs_v": np.array(rv)})
    cfg = ref_config(cases.LES_CAVITY)
    s = ProjectionSolver(cfg)
    f = s.initialize()
    for _ in range(10):
        f = s.step(f, cfg.dt)
    out.update({"cav_u": f.u, "cav_v": f.v, "cav_p": f.p})
    save("les.npz", **out)


def gen_stretched():
    """Stretched meshes on the reference's array path (pycfd/core/mesh.py:236-311,
    pycfd/core/solver.py:336-543, pycfd/core/pressure.py:193-207): widths, faces and
    metrics; momentum RHS and divergence on random fields (blend 0 and 0.6); the
    assembled Poisson operator with an obstacle and a Dirichlet wall; a stretched
    lid cavity (adaptive dt, MG-PCG) for 12 steps, an inlet/outlet channel past a
    cylinder for 10 steps with its force history, and a pressure-outlet channel
    (CG) for 10 steps."""
    out = {}
    for k, (nx, ny, lx, ly, sx, sy, cx_, cy_) in enumerate(cases.STRETCH_MESHES):
        mesh = StructuredMesh(nx, ny, lx, ly, sx, sy, cx_, cy_)
        m = mesh.metrics
        out.update({f"m{k}_dx": mesh.dx_cells, f"m{k}_dy": mesh.dy_cells, f"m{k}_xf": mesh.xf,
                    f"m{k}_yf": mesh.yf, f"m{k}_hxu": np.ravel(m.hxu), f"m{k}_hyv": np.ravel(m.hyv),
                    f"m{k}_wx": np.ravel(m.wx_corner), f"m{k}_wy": np.ravel(m.wy_corner)})
        c = dict(nx=nx, ny=ny, lx=lx, ly=ly, stretch_x=sx, stretch_y=sy, cluster_x=cx_, cluster_y=cy_,
                 re=300.0 + 100 * k, body_force=(0.05 * k, -0.1), dt=1e-3, t_end=1.0, adaptive_dt=False,
                 pressure_solver="cg", boundary_config=cases.bcs(top=("moving_wall", 1.0)), name="stretch")
        s = ProjectionSolver(ref_config(c), mesh)
        rng = np.random.default_rng(40 + k)
        u = rng.standard_normal((nx + 3, ny + 2))
        v = rng.standard_normal((nx + 2, ny + 3))
        for b, blend in enumerate((0.0, 0.6)):
            ru, rv = s.momentum_rhs(u, v, blend)
            out.update({f"m{k}_b{b}_rhs_u": np.array(ru), f"m{k}_b{b}_rhs_v": np.array(rv)})
        out.update({f"m{k}_u": u, f"m{k}_v": v, f"m{k}_div": s.divergence(u, v)})
    # Poisson operator: obstacle, a Dirichlet (pressure outlet) wall on the right
    mesh = StructuredMesh(*cases.STRETCH_MESHES[0])
    solid = circle_mask(mesh, (0.7, 0.5), 0.2).mask
    sysm = assemble_poisson_matrix(mesh, solid_mask=solid, dirichlet={"right": 0.3})
    po = {}
    csr_parts("A", sysm.A, po)
    out.update({f"poisson_{k}": v for k, v in po.items()})
    out.update({"poisson_solid": solid, "poisson_bc": sysm.bc_rhs, "poisson_row_scale": np.asarray(sysm.row_scale)})
    # runs
    cfg = ref_config(cases.STRETCH_CAVITY)
    sim = Simulation(cfg)
    sim.run(max_steps=12)
    f = sim.fields
    out.update({"cav_u": f.u, "cav_v": f.v, "cav_p": f.p, "cav_t": np.array(f.t)})
    cfg = ref_config(cases.STRETCH_CHANNEL)
    mesh = StructuredMesh.from_config(cfg)
    solid = circle_mask(mesh, *cases.STRETCH_CHANNEL_CIRCLE).mask
    s = ProjectionSolver(cfg, mesh, solid)
    f = s.initialize()
    fx, fy = [], []
    for _ in range(10):
        f = s.step(f, cfg.dt)
        fx.append(s.body_force_reaction[0])
        fy.append(s.body_force_reaction[1])
    out.update({"ch_u": f.u, "ch_v": f.v, "ch_p": f.p, "ch_fx": np.array(fx), "ch_fy": np.array(fy),
                "ch_solid": solid})
    cfg = ref_config(cases.STRETCH_PRESSURE_OUTLET)
    s = ProjectionSolver(cfg)
    f = s.initialize()
    for _ in range(10):
        f = s.step(f, cfg.dt)
    out.update({"po_u": f.u, "po_v": f.v, "po_p": f.p})
    # the Smagorinsky closure on a stretched mesh (pycfd/physics/turbulence.py:38-118,
    # pycfd/core/solver.py:467-499 with the metric arrays)
    nx, ny, lx, ly, sx, sy, cx_, cy_ = cases.STRETCH_MESHES[1]
    c = dict(nx=nx, ny=ny, lx=lx, ly=ly, stretch_x=sx, stretch_y=sy, cluster_x=cx_, cluster_y=cy_, re=3000.0,
             use_les=True, smagorinsky_cs=0.17, body_force=(0.1, -0.2), dt=1e-3, t_end=1.0, adaptive_dt=False,
             pressure_solver="cg", boundary_config=cases.bcs(top=("moving_wall", 1.0)), name="stretch_les")
    s = ProjectionSolver(ref_config(c))
    rng = np.random.default_rng(50)
    u = rng.standard_normal((nx + 3, ny + 2))
    v = rng.standard_normal((nx + 2, ny + 3))
    nu_c, nu_k = s.turbulence.eddy_viscosity(u, v, s.nu)
    out.update({"les_u": u, "les_v": v, "les_nu_c": nu_c, "les_nu_k": nu_k})
    for b, blend in enumerate((0.0, 0.6)):
        ru, rv = s.momentum_rhs(u, v, blend)
        out.update({f"les_b{b}_rhs_u": np.array(ru), f"les_b{b}_rhs_v": np.array(rv)})
    cfg = ref_config(cases.STRETCH_LES_CAVITY)
    s = ProjectionSolver(cfg)
    f = s.initialize()
    for _ in range(10):
        f = s.step(f, cfg.dt)
    out.update({"lescav_u": f.u, "lescav_v": f.v, "lescav_p": f.p})
    save("stretched.npz", **out)


def gen_masks():
    big = StructuredMesh(2048, 1024, 2.0, 1.0)
    m = circle_mask(big, (0.5, 0.5), 0.05).mask
    small = StructuredMesh(256, 128, 2.0, 1.0)
    m2 = circle_mask(small, (0.5, 0.5), 0.05).mask
    save("masks.npz", big_bits=np.packbits(m.ravel()), big_count=np.array(int(m.sum())),
         small=m2)


if __name__ == "__main__":
    which = set(sys.argv[2:]) or {"rhs", "poisson", "multigrid", "solvers", "steps",
                                  "cavity64", "cylinder", "masks", "faces", "cylinder_long", "shapes",
                                  "checkpoint", "interchange", "les", "stretched"}
    for name in ("rhs", "poisson", "multigrid", "solvers", "steps", "cavity64",
                 "cylinder", "masks", "faces", "cylinder_long", "shapes", "checkpoint", "interchange",
                 "les", "stretched"):
        if name in which:
            t0 = time.perf_counter()
            globals()["gen_" + name]()
            print(f"{name}: {time.perf_counter() - t0:.1f}s", flush=True)
