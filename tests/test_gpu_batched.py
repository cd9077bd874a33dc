"""Batched engine: every stage one launch over many problems (needs a B200).

Each problem of a batch keeps the single-problem arithmetic; only the
reduction trees differ (per-tile partials), so a batched FP64 problem matches
the reference's own step within the solver tolerance (1e-10 relative on u, v,
p, against the golden fixtures) and the same problem solved alone to rounding.
The mixed form (FP32 MG-PCG inside FP64 refinement to the same outer
tolerance) stays within 1e-6 of the FP64 velocities with max|div u| <= 1e-8.
"""

import numpy as np
import pytest

import cases
from oracle.projection import circle_mask_oracle
from pycfd_b200.config import BCKind, BCSpec, SimulationConfig

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def rel(a, b):
    a = a.detach().cpu().numpy() if hasattr(a, "detach") else np.asarray(a)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _case(name):
    spec = cases.STEP_CASES[name]
    cfg = cases.step_config(spec, SimulationConfig, BCSpec, BCKind)
    solid = circle_mask_oracle(cfg.nx, cfg.ny, cfg.lx, cfg.ly, *spec["circle"]) if "circle" in spec else None
    u0, v0 = cases.step_init(spec, cfg.nx, cfg.ny, cfg.lx, cfg.ly)
    return cfg, solid, u0, v0, spec


# Uneven grids and boundary programs in one batch: periodic vortex, inlet/outlet
# channel with an obstacle (mask forces, outlet mass balance), a periodic-y
# channel with a sliding wall, and the vortex again (a shared structure).
REF_CASES = ("periodic_mgcg", "inout_sym_obstacle_mgcg", "periodic_y_sym_mgcg", "periodic_mgcg")


def _reference_batch(precision):
    from pycfd_b200.batch import BatchedSolver, BatchOptions
    probs = [_case(n) for n in REF_CASES]
    b = BatchedSolver([p[0] for p in probs], BatchOptions(precision=precision),
                      obstacles=[p[1] for p in probs], u_init=[p[2] for p in probs],
                      v_init=[p[3] for p in probs], max_steps=[p[4]["steps"] for p in probs])
    return b, probs


def test_batch_fp64_matches_reference_steps(golden):
    g = golden("steps.npz")
    b, probs = _reference_batch("fp64")
    assert b.structures == 3
    for k, name in enumerate(REF_CASES):
        u, v, p = b.fields[k].numpy()
        assert rel(u, g[name + "_u0"]) < 1e-10 and rel(v, g[name + "_v0"]) < 1e-10, name
    b.step(max(p[4]["steps"] for p in probs) + 1)   # the extra step finds every problem done
    st = b.status()
    for k, name in enumerate(REF_CASES):
        spec = probs[k][4]
        assert st["steps"][k] == spec["steps"] and st["frozen"][k] == 2, (name, st)
        assert st["t"][k] == pytest.approx(spec["steps"] * spec["dt"], rel=1e-13)
        u, v, p = b.fields[k].numpy()
        for a, key in ((u, "u"), (v, "v"), (p, "p")):
            assert rel(a, g[f"{name}_{key}"]) < 1e-10, (name, key)
        if probs[k][1] is not None:
            assert b.force(k)[0] == pytest.approx(float(g[name + "_fx"][-1]), rel=1e-8)


def test_batch_mixed_within_bounds_of_reference(golden):
    g = golden("steps.npz")
    b, probs = _reference_batch("mixed")
    b.step(max(p[4]["steps"] for p in probs))
    for k, name in enumerate(REF_CASES):
        u, v, _ = b.fields[k].numpy()
        scale = max(np.abs(g[name + "_u"]).max(), np.abs(g[name + "_v"]).max())
        err = max(np.abs(u - g[name + "_u"]).max(), np.abs(v - g[name + "_v"]).max()) / scale
        assert err < 1e-6, (name, err)
        assert b.field_stats(k).max_div < 1e-8, name


def _cavities(count=5, seed=7):
    from pycfd_b200.batch import cavity_batch_configs
    return cavity_batch_configs(count=count, seed=seed, sizes=(24, 32, 40, 48), re_range=(100.0, 1000.0),
                                tol=1e-11)


def test_batch_matches_problems_solved_alone():
    """Adaptive-dt cavities of uneven size: batched FP64 vs each problem's own solver."""
    from pycfd_b200.batch import BatchedSolver, BatchOptions
    from pycfd_b200.solver import ProjectionSolver
    cfgs = _cavities()
    b = BatchedSolver(cfgs, BatchOptions(precision="fp64"))
    b.step(8)
    st = b.status()
    for k, cfg in enumerate(cfgs):
        s = ProjectionSolver(cfg)
        f = s.initialize()
        s.set_clock(0.0)
        for _ in range(8):
            f = s.advance_adaptive(f)
        t, dt, n, h = s.clock()
        assert n == st["steps"][k] == 8 and h == 0 and st["frozen"][k] == 0
        assert st["t"][k] == pytest.approx(t, rel=1e-12)
        ua, va, pa = b.fields[k].numpy()
        ub, vb, pb = f.numpy()
        assert rel(ua, ub) < 1e-9 and rel(va, vb) < 1e-9 and rel(pa, pb) < 1e-9, k


def test_recorded_step_equals_eager_step_and_counts_launches():
    from pycfd_b200 import _lib
    from pycfd_b200.batch import BatchedSolver, BatchOptions
    cfgs = _cavities(count=4, seed=11)
    L = _lib.load()
    for prec in ("fp64", "mixed"):
        a = BatchedSolver(cfgs, BatchOptions(precision=prec))
        e = BatchedSolver(cfgs, BatchOptions(precision=prec))
        torch.cuda.synchronize()
        a.launches(0)
        a.step(1, record=True)
        n_rec = a.launches(1)
        before = L.pycfd_launch_count()
        e.step(1, record=False)
        torch.cuda.synchronize()
        n_eager = L.pycfd_launch_count() - before
        assert n_rec == n_eager, (prec, n_rec, n_eager)
        a.step(2, record=True)
        e.step(2, record=False)
        for k in range(len(cfgs)):
            for x, y in zip(a.fields[k].numpy(), e.fields[k].numpy()):
                assert np.array_equal(x, y), (prec, k)


def test_programmatic_launch_gives_the_same_bits():
    """Every batched kernel waits on its predecessor before reading, so launching
    them under programmatic dependent launch changes timing only: the states after
    recorded steps are bit-identical to plain stream order."""
    from pycfd_b200.batch import BatchedSolver, BatchOptions
    cfgs = _cavities(count=4, seed=12)
    for prec in ("fp64", "mixed"):
        a = BatchedSolver(cfgs, BatchOptions(precision=prec))
        b = BatchedSolver(cfgs, BatchOptions(precision=prec, programmatic_launch=True))
        a.step(3, record=True)
        b.step(3, record=True)
        for k in range(len(cfgs)):
            for x, y in zip(a.fields[k].numpy(), b.fields[k].numpy()):
                assert np.array_equal(x, y), (prec, k)


def test_concurrent_parts_equal_one_engine():
    """Split over three engines on their own streams, every problem takes the steps
    it takes in one engine, bit for bit (its arithmetic does not depend on the other
    problems of its engine), and the results come back in the configs' order."""
    from pycfd_b200.batch import BatchedSolver, BatchOptions, ConcurrentBatch
    cfgs = _cavities(count=7, seed=13)
    for prec in ("fp64", "mixed"):
        one = BatchedSolver(cfgs, BatchOptions(precision=prec))
        many = ConcurrentBatch(cfgs, BatchOptions(precision=prec), parts=3)
        assert len(many.parts) == 3 and sorted(k for ks in many.index for k in ks) == list(range(len(cfgs)))
        one.step(3)
        many.step(3)
        st1, st2 = one.status(), many.status()
        assert np.array_equal(st1["steps"], st2["steps"]) and np.array_equal(st1["t"], st2["t"])
        for k in range(len(cfgs)):
            for x, y in zip(one.fields[k].numpy(), many.fields[k].numpy()):
                assert np.array_equal(x, y), (prec, k)
            assert one.field_stats(k).max_div == many.field_stats(k).max_div


def test_mixed_batch_tracks_fp64_batch():
    """Velocity error <= 1e-6 of the FP64 batch and max|div u| <= 1e-8 after 20 steps."""
    from pycfd_b200.batch import BatchedSolver, BatchOptions
    cfgs = _cavities(count=6, seed=5)
    a = BatchedSolver(cfgs, BatchOptions(precision="fp64"))
    m = BatchedSolver(cfgs, BatchOptions(precision="mixed"))
    a.step(20)
    m.step(20)
    sa, sm = a.status(), m.status()
    for k in range(len(cfgs)):
        ua, va, _ = a.fields[k].numpy()
        um, vm, _ = m.fields[k].numpy()
        scale = max(np.abs(ua).max(), np.abs(va).max())
        assert max(np.abs(ua - um).max(), np.abs(va - vm).max()) / scale < 1e-6, k
        assert m.field_stats(k).max_div < 1e-8
        assert sm["t"][k] == pytest.approx(sa["t"][k], rel=1e-6)


def test_stopped_problems_leave_the_others_running():
    """A blow-up freezes its own problem (health flag) and an end time freezes another;
    the rest keep stepping."""
    from pycfd_b200.batch import BatchedSolver, BatchOptions
    cfgs = _cavities(count=3, seed=2)
    walls = {w: BCSpec(BCKind.NO_SLIP) for w in ("left", "right", "bottom")}
    walls["top"] = BCSpec(BCKind.MOVING_WALL, velocity=1e3)
    bad = SimulationConfig(nx=32, ny=32, re=1e6, dt=5.0, adaptive_dt=False, t_end=1e4,
                           pressure_solver="mgcg", poisson_tol=1e-11, boundary_config=walls)
    b = BatchedSolver(cfgs + [bad], BatchOptions(precision="fp64"), t_end=[1e9, 0.01, 1e9, 1e9])
    b.step(30)
    st = b.status()
    assert st["frozen"][3] == 1 and st["steps"][3] < 30
    assert st["frozen"][1] == 2 and st["t"][1] == pytest.approx(0.01, rel=1e-12)
    assert st["frozen"][0] == 0 and st["steps"][0] == 30
    assert st["frozen"][2] == 0 and st["steps"][2] == 30
    for k in (0, 2):
        assert b.field_stats(k).finite


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_dense_tail_matches_level_by_level(precision):
    """Each structure's V-cycle closed by its dense tail operator (one blocked mat-vec
    over the structure's problems) against the level-by-level cycle."""
    from pycfd_b200.batch import BatchedSolver, BatchOptions
    cfgs = _cavities(count=7, seed=3)
    out, its = [], []
    for tail in (True, False):
        b = BatchedSolver(cfgs, BatchOptions(precision=precision, coarse_tail=tail, tail_ratio=None))
        assert not tail or b._tailed == len(cfgs)
        b.step(6)
        out.append([b.fields[k].numpy() for k in range(len(cfgs))])
        st = b.status()
        assert all(f == 0 for f in st["frozen"])
        its.append(st["iterations"])
    bound = 1e-9 if precision == "fp64" else 1e-7
    for fa, fb in zip(*out):
        for x, y in zip(fa[:2], fb[:2]):
            assert rel(x, y) < bound
    # the same preconditioner up to rounding: the same CG passes per step (within one per solve)
    assert np.abs(its[0] - its[1]).max() <= 3, its


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_fused_restriction_matches_two_phase_down_sweep(precision):
    """The down sweep by fused restrictions R (I - A W) -- from the fine level, or from
    level 2 with the fine sweep and restriction kept -- against restriction + first sweep."""
    from pycfd_b200.batch import BatchedSolver, BatchOptions
    cfgs = _cavities(count=7, seed=4)
    out = []
    for fused, start in ((True, 1), (True, 2), (False, 1)):
        # unbounded tail: these small cavities all get one (a tail bound would leave them none)
        b = BatchedSolver(cfgs, BatchOptions(precision=precision, fused_restriction=fused, fused_from=start,
                                             tail_ratio=None))
        assert b._fused == fused
        b.step(6)
        out.append([b.fields[k].numpy() for k in range(len(cfgs))])
        assert all(f == 0 for f in b.status()["frozen"])
    bound = 1e-9 if precision == "fp64" else 1e-7
    for k in (0, 1):
        for fa, fb in zip(out[k], out[2]):
            for x, y in zip(fa[:2], fb[:2]):
                assert rel(x, y) < bound


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_stencil_transfers_match_stored_matrices(precision):
    """Level-0 transfers as stencils over the fine cells (the fused restriction
    T^T (I - A W)^2 and the prolongation (I - W A) T with the last sweep) against the
    products with the stored P_1 and M_1: cavities of odd and even size, and the
    reference cases (periodic axes, an obstacle with an outlet, a periodic-y channel)."""
    from pycfd_b200.batch import BatchedSolver, BatchOptions, cavity_batch_configs
    cav = cavity_batch_configs(count=6, seed=9, sizes=(25, 32, 37, 48), re_range=(100.0, 1000.0), tol=1e-11)
    probs = [_case(n) for n in ("periodic_mgcg", "inout_sym_obstacle_mgcg")]
    # the periodic-y channel on a grid with three levels (its own 20 x 16 has two, so no tail)
    chan = _case("periodic_y_sym_mgcg")[0].replace(nx=40, ny=32)
    probs.append((chan, None, None, None, dict(steps=6)))
    batches = [dict(configs=cav, steps=6),
               dict(configs=[p[0] for p in probs], steps=min(p[4]["steps"] for p in probs) - 1,
                    kw=dict(obstacles=[p[1] for p in probs], u_init=[p[2] for p in probs],
                            v_init=[p[3] for p in probs]))]
    bound = 1e-9 if precision == "fp64" else 1e-7
    for bt in batches:
        out, its = [], []
        for stencil in (True, False):
            b = BatchedSolver(bt["configs"], BatchOptions(precision=precision, fused_restriction=True,
                                                           tail_ratio=None, stencil_transfer=stencil),
                              **bt.get("kw", {}))
            assert b._fused and b._stencil == stencil
            b.step(bt["steps"])
            st = b.status()
            assert all(f == 0 for f in st["frozen"])
            out.append([b.fields[k].numpy() for k in range(len(bt["configs"]))])
            its.append(st["iterations"])
            for k in range(len(bt["configs"])):
                assert b.field_stats(k).max_div < 1e-8
        for fa, fb in zip(*out):
            for x, y in zip(fa[:2], fb[:2]):
                assert rel(x, y) < bound
        assert np.abs(its[0] - its[1]).max() <= 2, its


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_loop_cap_ends_device_loops_and_the_batch_goes_on(precision):
    """The pass cap of the device-side WHILE loops, set low from the host, ends every
    solve of a step early (reported per loop, problems unconverged, no hang); with
    the built-in cap restored the next steps converge again."""
    from pycfd_b200.batch import BatchedSolver, BatchOptions
    cfgs = _cavities(count=3, seed=5)
    b = BatchedSolver(cfgs, BatchOptions(precision=precision))
    b.step(2)
    assert b.capped() == 0
    assert (b.status()["status"] == 0).all()
    b.set_loop_cap(2)
    b.step(1)
    assert b.capped() & 1
    st = b.status()
    assert (st["status"] == -3).any() and (st["frozen"] == 0).all()
    b.set_loop_cap(0)
    b.step(2)
    assert b.capped() == 0
    st = b.status()
    assert (st["status"] == 0).all() and (st["steps"] == 5).all()


def test_vector_strips_match_scalar_strips():
    """The mixed form's FP32 CG and level-0 sweep kernels on 128-column float4 strips
    against the 30-column scalar strips: rows a multiple of 4 long and not (those
    stay scalar in one launch with the vector ones), a second segment one lane wide
    (132 columns), both periodic axes, an obstacle beside an outlet and a periodic-y
    channel (edge columns wrapped across the seam)."""
    from pycfd_b200.batch import BatchedSolver, BatchOptions, cavity_batch_configs
    cav = cavity_batch_configs(count=6, seed=11, sizes=(25, 32, 37, 48, 132), re_range=(100.0, 1000.0),
                               tol=1e-11)
    probs = [_case(n) for n in REF_CASES]
    batches = [dict(configs=cav, steps=5),
               dict(configs=[p[0] for p in probs], steps=min(p[4]["steps"] for p in probs) - 1,
                    kw=dict(obstacles=[p[1] for p in probs], u_init=[p[2] for p in probs],
                            v_init=[p[3] for p in probs]))]
    for bt in batches:
        out, its = [], []
        for scalar in (True, False):
            b = BatchedSolver(bt["configs"], BatchOptions(precision="mixed", scalar_strips=scalar),
                              **bt.get("kw", {}))
            b.step(bt["steps"])
            st = b.status()
            assert all(f == 0 for f in st["frozen"])
            out.append([b.fields[k].numpy() for k in range(len(bt["configs"]))])
            its.append(st["iterations"])
            for k in range(len(bt["configs"])):
                assert b.field_stats(k).max_div < 1e-8
        for fa, fb in zip(*out):
            for x, y in zip(fa[:2], fb[:2]):
                assert rel(x, y) < 1e-7
        assert np.abs(its[0] - its[1]).max() <= 2, its
