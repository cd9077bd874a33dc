"""Case table shared by the golden generator and the tests (plain data, no imports of the reference).

Boundary specs are tuples ``(kind, velocity=0, profile="uniform", p_ref=0)``;
``to_config`` turns a case into a config object of whichever package is given.
"""

from __future__ import annotations

import numpy as np

WALLS = ("left", "right", "bottom", "top")


def bcs(**kw):
    out = {w: ("no_slip",) for w in WALLS}
    out.update(kw)
    return out


PER = {w: ("periodic",) for w in WALLS}

STEP_CASES = {
    "cavity_cg_rk3": dict(cfg=dict(nx=16, ny=16, re=100.0, pressure_solver="cg", poisson_tol=1e-12,
                                   boundary_config=bcs(top=("moving_wall", 1.0))),
                          steps=10, dt=2e-3),
    "periodic_mgcg": dict(cfg=dict(nx=32, ny=32, lx=2 * np.pi, ly=2 * np.pi, re=20.0,
                                   pressure_solver="mgcg", poisson_tol=1e-12, boundary_config=PER),
                          steps=8, dt=0.05, tg=True),
    "channel_sor_force": dict(cfg=dict(nx=8, ny=24, re=10.0, pressure_solver="sor", poisson_tol=1e-12,
                                       body_force=(0.8, 0.0),
                                       boundary_config=bcs(left=("periodic",),
                                                           right=("periodic",))),
                              steps=6, dt=5e-3),
    "inout_sym_obstacle_mgcg": dict(cfg=dict(nx=48, ny=32, lx=3.0, ly=2.0, re=50.0, pressure_solver="mgcg",
                                             poisson_tol=1e-12,
                                             boundary_config=bcs(left=("inlet", 1.0),
                                                                 right=("outlet",),
                                                                 top=("symmetry",),
                                                                 bottom=("symmetry",))),
                                    steps=10, dt=2e-3, circle=((1.0, 1.0), 0.25), u_init=1.0),
    "pressure_outlet_parabolic_mg": dict(cfg=dict(nx=40, ny=20, lx=2.0, ly=1.0, re=40.0, pressure_solver="multigrid",
                                                  poisson_tol=1e-12,
                                                  boundary_config=bcs(left=("inlet", 1.0, "parabolic"),
                                                                      right=("pressure_outlet", 0.0, "uniform", 0.25))),
                                         steps=6, dt=4e-3, circle=((0.6, 0.5), 0.15), u_init=0.5),
    "cavity_upwind_cg": dict(cfg=dict(nx=20, ny=16, re=1000.0, pressure_solver="cg", poisson_tol=1e-12,
                                      advection_scheme="upwind", upwind_blend=0.7,
                                      boundary_config=bcs(top=("moving_wall", 1.0))),
                             steps=8, dt=4e-3),
    "cavity_euler_jacobi": dict(cfg=dict(nx=12, ny=12, re=100.0, pressure_solver="jacobi", poisson_tol=1e-9,
                                         time_scheme="euler",
                                         boundary_config=bcs(top=("moving_wall", 1.0))),
                                steps=4, dt=2e-3),
    "noisy_inout_rk2_cg": dict(cfg=dict(nx=16, ny=16, re=50.0, pressure_solver="cg", poisson_tol=1e-12,
                                        time_scheme="rk2",
                                        boundary_config=bcs(left=("inlet", 1.0),
                                                            right=("outlet",))),
                               steps=6, dt=1e-3, noise=0),
    "periodic_y_sym_mgcg": dict(cfg=dict(nx=20, ny=16, re=80.0, pressure_solver="mgcg", poisson_tol=1e-12,
                                         boundary_config=bcs(bottom=("periodic",),
                                                             top=("periodic",),
                                                             left=("moving_wall", -0.5),
                                                             right=("symmetry",))),
                                steps=6, dt=2e-3, noise=3),
}




CAVITY64 = dict(nx=64, ny=64, re=100.0, dt=1.0, t_end=1e9, cfl_max=0.5, adaptive_dt=True,
                pressure_solver="cg", poisson_tol=1e-10,
                boundary_config=bcs(top=("moving_wall", 1.0)), name="cavity64")


def cylinder_cfg(nx, ny, solver="mgcg", tol=1e-10):
    """Cylinder channel: lx=2, ly=1, D=0.1, inlet 1, convective outlet, slip walls, Re 100."""
    return dict(nx=nx, ny=ny, lx=2.0, ly=1.0, re=100.0, u_ref=1.0, l_ref=0.1, dt=1.0,
                t_end=1e9, cfl_max=0.5, pressure_solver=solver, poisson_tol=tol,
                boundary_config={"left": ("inlet", 1.0), "right": ("outlet",),
                                 "bottom": ("symmetry",), "top": ("symmetry",)},
                name="cylinder")


def cylinder_init(nx, ny, seed=0):
    """u = 1, v = 0 plus 1e-3 seeded Gaussian noise on the physical faces."""
    rng = np.random.default_rng(seed)
    return (1.0 + 1e-3 * rng.standard_normal((nx + 1, ny)),
            1e-3 * rng.standard_normal((nx, ny + 1)))


def tgv_cfg(n, re=1000.0, solver="mgcg", tol=1e-10):
    """Doubly periodic Taylor-Green vortex on [0, 2pi]^2, fixed dt = 0.4*2pi/n."""
    return dict(nx=n, ny=n, lx=2 * np.pi, ly=2 * np.pi, re=re, dt=0.4 * 2 * np.pi / n,
                t_end=1e9, adaptive_dt=False, pressure_solver=solver, poisson_tol=tol,
                boundary_config=PER, name=f"tgv{n}")


def axis(length, n):
    """Face and centre coordinates built like the reference mesh (cumsum, far face pinned)."""
    f = np.concatenate(([0.0], np.cumsum(np.full(n, length / n, dtype=float))))
    f[-1] = length
    return f, 0.5 * (f[:-1] + f[1:])


def tg_init(nx, ny, lx, ly):
    """u = sin x cos y on the u-faces, v = -cos x sin y on the v-faces."""
    xf, xc = axis(lx, nx)
    yf, yc = axis(ly, ny)
    Xu, Yu = np.meshgrid(xf, yc, indexing="ij")
    Xv, Yv = np.meshgrid(xc, yf, indexing="ij")
    return np.sin(Xu) * np.cos(Yu), -np.cos(Xv) * np.sin(Yv)


def to_config(d, SimulationConfig, BCSpec, BCKind, **extra):
    """Build a config of the given package from a case dict."""
    d = dict(d)
    bc = {}
    for w, t in d.pop("boundary_config").items():
        t = tuple(t) + (0.0, "uniform", 0.0)[len(t) - 1:]
        bc[w] = BCSpec(BCKind(t[0]), velocity=t[1], profile=t[2], p_ref=t[3])
    d.update(extra)
    return SimulationConfig(boundary_config=bc, **d)


def step_config(spec, SimulationConfig, BCSpec, BCKind):
    return to_config({**dict(dt=spec["dt"], t_end=10.0, adaptive_dt=False, name="golden"),
                      **spec["cfg"]}, SimulationConfig, BCSpec, BCKind)


def step_init(spec, nx, ny, lx, ly):
    """(u_init, v_init) of a step case."""
    u_init = spec.get("u_init")
    v_init = None
    if spec.get("tg"):
        u_init, v_init = tg_init(nx, ny, lx, ly)
    if "noise" in spec:
        rng = np.random.default_rng(spec["noise"])
        u_init = 0.1 * rng.standard_normal((nx + 1, ny))
        v_init = 0.1 * rng.standard_normal((nx, ny + 1))
    return u_init, v_init


# Face-flag layouts: bodies as index boxes (i0, i1, j0, j1) of solid cells, so both
# packages build the same masks without any rasterisation.  Each body is one
# connected set; a body may span a periodic seam (cells on both sides of it).
FACE_CASES = {
    "seam_x": dict(cfg=dict(nx=24, ny=16, re=50.0, pressure_solver="cg", poisson_tol=1e-10,
                            boundary_config=bcs(left=("periodic",), right=("periodic",))),
                   bodies=[[(0, 3, 5, 9), (21, 24, 5, 9)]]),
    "seam_y": dict(cfg=dict(nx=20, ny=24, re=50.0, pressure_solver="cg", poisson_tol=1e-10,
                            boundary_config=bcs(left=("inlet", 1.0), right=("outlet",),
                                                bottom=("periodic",), top=("periodic",))),
                   bodies=[[(6, 10, 0, 2), (6, 10, 22, 24)]]),
    "outlet_touch": dict(cfg=dict(nx=28, ny=16, re=50.0, pressure_solver="cg", poisson_tol=1e-10,
                                  boundary_config=bcs(left=("inlet", 1.0),
                                                      right=("pressure_outlet", 0.0, "uniform", 0.0),
                                                      bottom=("symmetry",), top=("symmetry",))),
                         bodies=[[(25, 28, 6, 10)], [(8, 12, 3, 7)]]),
    "walls_two_bodies": dict(cfg=dict(nx=18, ny=18, re=50.0, pressure_solver="cg", poisson_tol=1e-10,
                                      boundary_config=bcs(top=("moving_wall", 1.0))),
                             bodies=[[(0, 4, 0, 3)], [(9, 12, 8, 13)], [(14, 18, 15, 18)]]),
}


def face_bodies(case, nx, ny):
    """Per-body boolean masks of a face case."""
    out = []
    for boxes in case["bodies"]:
        m = np.zeros((nx, ny), dtype=bool)
        for i0, i1, j0, j1 in boxes:
            m[i0:i1, j0:j1] = True
        out.append(m)
    return out


# Shapes for the rasteriser fixtures (plain data).
STAR = [(0.55 + (0.28 if k % 2 == 0 else 0.12) * np.cos(np.pi * k / 6),
         0.45 + (0.28 if k % 2 == 0 else 0.12) * np.sin(np.pi * k / 6)) for k in range(12)]
SHAPE_MESH = dict(nx=200, ny=120, lx=1.6, ly=1.0)


def shape_image(rows=37, cols=53, seed=4):
    """An RGBA 8-bit picture: a dark ellipse and a dark bar on a light, noisy background."""
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:rows, 0:cols]
    lum = 0.85 + 0.1 * rng.random((rows, cols))
    lum[((xx - 20) / 9.0) ** 2 + ((yy - 14) / 6.0) ** 2 <= 1.0] = 0.1
    lum[28:32, 30:48] = 0.3
    img = np.empty((rows, cols, 4), dtype=np.uint8)
    img[..., 0] = np.round(255 * lum)
    img[..., 1] = np.round(255 * np.clip(lum * 0.9, 0, 1))
    img[..., 2] = np.round(255 * np.clip(lum * 1.05, 0, 1))
    img[..., 3] = 255
    return img


CKPT_CAVITY = dict(nx=32, ny=32, re=100.0, dt=1.0, t_end=1e9, cfl_max=0.5, adaptive_dt=True,
                   pressure_solver="mgcg", poisson_tol=1e-12,
                   boundary_config=bcs(top=("moving_wall", 1.0)), name="ckpt_cavity")


LES_CAVITY = dict(nx=40, ny=40, re=5000.0, use_les=True, smagorinsky_cs=0.17, dt=2e-3, t_end=10.0,
                  adaptive_dt=False, pressure_solver="cg", poisson_tol=1e-12,
                  boundary_config=bcs(top=("moving_wall", 1.0)), name="les_cavity")


# Stretched meshes (pycfd/core/mesh.py:236-311, the array path of pycfd/core/solver.py)
STRETCH_MESHES = [   # (nx, ny, lx, ly, stretch_x, stretch_y, cluster_x, cluster_y)
    (24, 18, 1.5, 1.0, 1.07, 1.12, "low", "walls"),
    (17, 21, 1.0, 2.0, 1.15, 0.93, "centre", "walls"),
    (31, 16, 2.0, 1.0, 1.04, 1.0, "walls", "low"),
]

STRETCH_CAVITY = dict(nx=40, ny=32, stretch_x=1.06, stretch_y=1.08, cluster_x="walls", cluster_y="walls",
                      re=400.0, dt=1.0, t_end=1e9, cfl_max=0.5, adaptive_dt=True, pressure_solver="mgcg",
                      poisson_tol=1e-12, boundary_config=bcs(top=("moving_wall", 1.0)), name="stretch_cavity")

STRETCH_CHANNEL = dict(nx=48, ny=24, lx=3.0, ly=1.0, stretch_x=1.03, stretch_y=1.1, cluster_x="low",
                       cluster_y="centre", re=100.0, dt=4e-3, t_end=10.0, adaptive_dt=False,
                       pressure_solver="mgcg", poisson_tol=1e-12,
                       boundary_config=bcs(left=("inlet", 1.0), right=("outlet",)), name="stretch_channel")
STRETCH_CHANNEL_CIRCLE = ((1.0, 0.5), 0.15)

STRETCH_PRESSURE_OUTLET = dict(nx=36, ny=20, lx=2.0, ly=1.0, stretch_x=1.05, stretch_y=1.06, cluster_x="low",
                               cluster_y="walls", re=50.0, dt=5e-3, t_end=10.0, adaptive_dt=False,
                               pressure_solver="cg", poisson_tol=1e-12,
                               boundary_config=bcs(left=("inlet", 1.0, "parabolic"),
                                                   right=("pressure_outlet", 0.0, "uniform", 0.0)),
                               name="stretch_po")

STRETCH_LES_CAVITY = dict(nx=32, ny=28, stretch_x=1.05, stretch_y=1.07, cluster_x="walls", cluster_y="walls",
                          re=5000.0, use_les=True, smagorinsky_cs=0.17, dt=2e-3, t_end=10.0, adaptive_dt=False,
                          pressure_solver="cg", poisson_tol=1e-12,
                          boundary_config=bcs(top=("moving_wall", 1.0)), name="stretch_les_cavity")
