"""Throughput of the projection step in cell-updates/s: the 256-cavity batch (default).

Workload (default, ``--workload batch``): 256 seeded lid-driven cavities per GPU,
N in {64, 96, 128, 192, 256}, Re log-uniform in [100, 2000], lid speed uniform
in [0.5, 1.5], adaptive dt at CFL 0.5, MG-PCG to 1e-10, advanced by the batched
engine in the mixed form (FP32 MG-PCG inside FP64 refinement).  One step = one
SSP-RK3 step of every cavity; value = cells of all ranks x steps / device time
(CUDA events on the launching stream, barrier + synchronise on both sides,
max over ranks).  The working set (~0.5 GB) exceeds L2.  Beside it the line
carries the batched engine in FP64 and the plain FP64 path (one single-problem
solver per cavity, recorded steps on 16 streams), their ratios, the per-kernel
roofline of one eager step (each part's launches, and the same kernels at full size
in one engine), the end-to-end figure through host buffers and the CPU baseline.
Under torchrun the 256*N cavities of one seeded draw are split over the ranks by
cell count (no exchange on the data path).

``--workload tgv512``: one SSP-RK3 step of the 512x512 Taylor-Green vortex on the
single-problem path (L2 flushed between steps).  Other workloads: adjoint,
tgv-validation, cylinder.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload batch|tgv512|...] [--precision fp64|mixed]

--impl reference times the reference algorithm's CPU implementation (the NumPy/
SciPy restatement in oracle/, which only this arm and the cpu_baseline leg run)
on the host cores, one single-threaded process per cavity, on the same workload
and metric; under torchrun rank 0 alone runs it.
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N = 512
RE = 1000.0
TOL = 1e-10
METRIC = "cell-updates/s per projection step, mixed vs FP64 at 1e-8 div; HBM % peak"
UNIT = "cell-updates/s"


def tgv_config():
    from pycfd_b200.config import BCKind, BCSpec, SimulationConfig
    per = {w: BCSpec(BCKind.PERIODIC) for w in ("left", "right", "bottom", "top")}
    return SimulationConfig(nx=N, ny=N, lx=2 * np.pi, ly=2 * np.pi, re=RE, dt=0.4 * 2 * np.pi / N,
                            t_end=1e9, adaptive_dt=False, pressure_solver="mgcg", poisson_tol=TOL,
                            boundary_config=per, name="tgv512")


def tgv_init(mesh):
    Xu, Yu = mesh.u_grid()
    Xv, Yv = mesh.v_grid()
    return np.sin(Xu) * np.cos(Yu), -np.cos(Xv) * np.sin(Yv)


def workload_config(extra=None):
    d = {"workload": f"taylor_green_{N}x{N}", "re": RE, "scheme": "ssp-rk3",
         "pressure_solver": "mgcg", "poisson_tol": TOL, "dt": 0.4 * 2 * np.pi / N,
         "cells": N * N, "cell_update": "one cell advanced by one full RK3 step (3 projections)",
         "l2": "flushed between timed steps (256 MB write)"}
    d.update(extra or {})
    return d


def max_over_ranks(value, dist, device):
    """Largest value over all ranks (the slowest rank sets the job's time)."""
    import torch
    t = torch.tensor([float(value)], device=device, dtype=torch.float64)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


class Clocks:
    """nvidia-smi samples of SM clock and throttle reasons while the timed steps run."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.proc = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={index}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        out, _ = self.proc.communicate(timeout=10)
        rows = [r.split(", ") for r in out.strip().splitlines() if r.count(",") >= 6]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[0]) for r in rows]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[3 + k].strip() == "Active"})
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(rows[0][1]),
                "reasons": reasons, "samples": len(rows)}


KERNELS = {1: "k_cg_pq (CG direction p = z + beta p, q = A p, p.q)",
           2: "k_fine_smooth (last fine V-cycle sweep, z and r.z)",
           3: "k_fine_pre (first fine sweep from zero + residual)",
           4: "k_coarse_cycle (coarse V-cycle levels in one thread-block cluster)",
           8: "k_solve_persistent (whole MG-PCG solve, one cooperative launch: V-cycle, p/q and x/r "
              "phases between grid barriers)"}


def solve_bytes(solver, iterations, solves, s_bytes=8):
    """Algorithmic bytes of `solves` whole CG / MG-PCG solves with `iterations` passes
    in total: every array a phase reads or writes, once per phase (ELL entries as value
    + column index), one smoothing sweep per level."""
    nx, ny = solver.mesh.shape
    n0 = nx * ny
    e = s_bytes + 4
    fixed = n0 * (4 * s_bytes + 1) + n0 * (3 * s_bytes + 1)   # b, x0, flags -> b, r; b, x, flags -> x
    per = n0 * (4 * s_bytes + 1) + n0 * (6 * s_bytes + 1)     # p/q; x/r
    lv = getattr(solver, "_levels", None)
    if lv and len(lv) > 1:
        Lv = len(lv)
        n = [l.n for l in lv]
        per += n0 * (3 * s_bytes + 1)                         # first fine sweep + residual
        for l in range(1, Lv):
            per += lv[l].P.nnz * e + s_bytes * (n[l - 1] + n[l])   # restriction
            if l < Lv - 1:
                per += lv[l].A.nnz * e + 4 * s_bytes * n[l]       # first sweep + residual
            else:
                per += n[l] * n[l] * s_bytes + 2 * s_bytes * n[l]  # dense coarsest
        for l in range(Lv - 2, -1, -1):
            per += lv[l + 1].P.nnz * e + s_bytes * (n[l + 1] + 2 * n[l])   # prolongation
            per += lv[l].A.nnz * e + 4 * s_bytes * n[l] if l else n0 * (3 * s_bytes + 1)   # sweep
    return solves * fixed + iterations * per


def algorithmic_bytes(kid, solver, s_bytes=8):
    """Bytes a launch must move at minimum: every array it reads or writes, once."""
    nx, ny = solver.mesh.shape
    n = nx * ny
    if kid == 1:
        return n * (4 * s_bytes + 1)          # read z, p_old, flags; write p, q
    if kid == 2:
        return n * (4 * s_bytes + 1)          # read x, b, r, flags; write x
    if kid == 3:
        return n * (3 * s_bytes + 1)          # read b, flags; write x, res
    if kid == 4:                              # coarse levels: matrices (value + column) and vectors
        lv = solver._levels
        rows = solver.options.coarse_cluster_rows
        lc = next((l for l in range(1, len(lv)) if lv[l].n <= rows), len(lv))
        e = s_bytes + 4
        total = 0
        for l in range(lc, len(lv)):
            n_l, n_up = lv[l].n, lv[l - 1].n
            P = lv[l].P
            total += P.nnz * e + (n_up + n_l) * s_bytes            # restriction R = P^T
            if l == len(lv) - 1:
                total += n_l * n_l * s_bytes + 2 * n_l * s_bytes    # dense coarsest solve
                continue
            A = lv[l].A
            total += 2 * A.nnz * e + 8 * n_l * s_bytes              # first sweep + residual, last sweep
            total += lv[l + 1].P.nnz * e + (2 * n_l + lv[l + 1].n) * s_bytes   # prolongation
        return total
    raise ValueError(kid)


def live_roofline(solver, f, dt, hbm_gbs, peak_src, steps=3):
    """Time the candidate kernels with CUDA events around their eager launches."""
    import ctypes as C
    from pycfd_b200 import _lib
    L = solver._L
    stream = _lib.ptr(None)
    import torch
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    shares = {}
    its = {}
    for kid in KERNELS:
        _lib.check(L.pycfd_profile_kernel(solver._h, kid))
        g = f
        its[kid] = 0
        for _ in range(steps):
            g = solver.step(g, dt)
            its[kid] += solver.last_stats.total_iterations
        tot, cnt = C.c_double(), C.c_int()
        _lib.check(L.pycfd_profile_read(solver._h, C.byref(tot), C.byref(cnt), stream))
        if cnt.value:
            shares[kid] = (tot.value, cnt.value)
    _lib.check(L.pycfd_profile_kernel(solver._h, 0))
    # the persistent solve is the whole step's dominant launch when it runs; in
    # the per-phase form k_cg_pq is the top kernel instance of the launch list
    # (the others are timed for their shares only)
    kid = 8 if 8 in shares else (1 if 1 in shares else max(shares, key=lambda k: shares[k][0]))
    ms, cnt = shares[kid]
    per_launch_s = ms / 1e3 / cnt
    if kid == 8:
        nbytes = solve_bytes(solver, its[8], cnt) / cnt
    else:
        nbytes = algorithmic_bytes(kid, solver, 4 if solver.options.precision == "mixed" and kid == 4 else 8)
    achieved = nbytes / per_launch_s / 1e9
    traffic = None
    try:
        prof = json.load(open(os.path.join(ROOT, "profiles", "roofline_traffic.json")))
        traffic = prof.get(solver.options.precision, {}).get(str(kid))
    except Exception:
        pass
    return {"bound": "hbm", "kernel": KERNELS[kid], "achieved": achieved, "peak": hbm_gbs,
            "unit": "GB/s", "frac": achieved / hbm_gbs, "traffic": traffic,
            "bytes_per_launch": nbytes, "us_per_launch": per_launch_s * 1e6, "launches": cnt,
            "peak_source": peak_src,
            "timing": "CUDA events around each eager launch of the kernel over "
                      f"{steps} replayed steps of the same workload (recorded graphs carry no events)",
            "share_of_candidates": {KERNELS[k]: v[0] for k, v in shares.items()}}


def cpu_baseline(steps=3, warmup=0):
    """The oracle (NumPy/SciPy restatement of the reference) on a bounded sample,
    after `warmup` untimed steps."""
    from oracle import OracleSolver
    from pycfd_b200.mesh import StructuredMesh
    cfg = tgv_config()
    t0 = time.perf_counter()
    s = OracleSolver(cfg)
    u, v, p = s.initialize(*tgv_init(StructuredMesh.from_config(cfg)))
    for _ in range(warmup):
        u, v, p = s.step(u, v, cfg.dt)
    setup = time.perf_counter() - t0
    t0 = time.perf_counter()
    for _ in range(steps):
        u, v, p = s.step(u, v, cfg.dt)
    el = time.perf_counter() - t0
    return {"value": N * N * steps / el, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"{steps} RK3 steps of the 512x512 vortex after initialisation and {warmup} "
                      f"untimed steps ({el:.1f} s; {setup:.1f} s before excluded); NumPy/SciPy, one thread"}


def host_cores():
    """Host threads this process may run on (its CPU affinity)."""
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def _oracle_cavity(cfg, warmup, steps, barrier, out):
    """One worker process: the oracle's adaptive RK3 steps of one cavity.  Set-up and
    `warmup` steps untimed; then wait at the barrier, so all workers time together."""
    from oracle import OracleSolver
    from oracle.projection import OracleStepper
    s = OracleSolver(cfg)
    u, v, p = s.initialize()
    stp = OracleStepper(s)
    for _ in range(warmup):
        u, v, p = s.step(u, v, stp.compute_dt(u, v))
    barrier.wait()
    t0 = time.perf_counter()
    for _ in range(steps):
        u, v, p = s.step(u, v, stp.compute_dt(u, v))
    out.put((cfg.nx * cfg.ny * steps, time.perf_counter() - t0, time.time()))


def batch_cpu_baseline(cfgs, steps=1, warmup=0, workers=None):
    """The oracle (the reference's algorithm restated in NumPy/SciPy) on the host cores:
    one single-threaded process per cavity, `workers` cavities at once (default all
    host threads, capped by the batch), drawn round-robin over the grid sizes so the
    sample keeps the batch's size mix.  Every process sets up and runs `warmup`
    untimed steps, then all time `steps` steps together (barrier); value = the
    sample's cell-updates / the wall time from the barrier to the last finisher."""
    import multiprocessing as mp
    by_size = {}
    for c in cfgs:
        by_size.setdefault(c.nx, []).append(c)
    order = []
    while any(by_size.values()):
        for n in sorted(by_size):
            if by_size[n]:
                order.append(by_size[n].pop(0))
    cores = host_cores()
    workers = min(workers or cores, len(order), cores)
    sample = order[:workers]
    for var in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS", "NUMBA_NUM_THREADS"):
        os.environ[var] = "1"   # one thread per process, inherited by the spawned workers
    ctx = mp.get_context("spawn")
    barrier = ctx.Barrier(workers + 1)
    out = ctx.Queue()
    procs = [ctx.Process(target=_oracle_cavity, args=(c, warmup, steps, barrier, out)) for c in sample]
    for pr in procs:
        pr.start()
    barrier.wait(timeout=900)
    t0 = time.time()
    res = [out.get(timeout=1800) for _ in procs]
    for pr in procs:
        pr.join(timeout=60)
    wall = max(r[2] for r in res) - t0
    cells = sum(r[0] for r in res)
    sizes = {}
    for c in sample:
        sizes[c.nx] = sizes.get(c.nx, 0) + 1
    return {"value": cells / wall, "unit": UNIT, "cores": workers, "kind": "port",
            "host_threads": cores, "wall_s": wall, "steps": steps,
            "sample": f"{workers} cavities of the batch (by grid size: {sizes}), one single-threaded "
                      f"NumPy/SciPy process each, {steps} adaptive RK3 step(s) each after set-up and "
                      f"{warmup} untimed step(s), timed together ({wall:.1f} s wall)"}


def batch_kernel_bytes(kid, cells, its, s_bytes):
    """Algorithmic bytes of one eager step's launches of kernel kind `kid` (ids of
    pycfd_batch_profile), from each problem's CG passes in that step."""
    passes = float((its * cells).sum())
    if kid == 1:     # k_b_cg_pq: read z, p_old, flags; write p, q
        return passes * (4 * s_bytes + 1)
    if kid == 5:     # k_b_cg_xr: read p, x, r, q, flags; write x, r
        return passes * (6 * s_bytes + 1)
    if kid == 2:     # k_b_fine (last sweep): read x0, r, flags; write z
        return passes * (3 * s_bytes + 1)
    if kid == 3:     # k_b_fine (first sweep): read r, flags; write x0, lres0
        return passes * (3 * s_bytes + 1)
    if kid == 6:     # k_b_predictor, 3 per step: read u, v; write u*, v* (FP64 state)
        return 3.0 * float(cells.sum()) * 32
    return None


KERNEL_NAMES = {1: "k_b_cg_pq (batched CG direction p = z + beta p, q = A p, p.q)",
                2: "k_b_fine<FM_LAST> (last level-0 V-cycle sweep, z and r.z)",
                3: "k_b_fine<FM_PRE> (first level-0 sweep and residual)",
                5: "k_b_cg_xr (batched CG update x, r, norms)",
                6: "k_b_predictor (momentum RHS + Runge-Kutta stage, FP64 state)"}


def run_batch(args, world, rank, local):
    """The cavity batch: 256 seeded lid-driven cavities of uneven size, Re and lid
    speed per GPU.  At N GPUs the 256*N cavities of one seeded draw are split over
    the ranks by cell count (no exchange on the data path); every rank advances its
    share with the batched engine (every stage one launch over all its problems).
    Beside it, on the same problems and steps: the plain FP64 path (one
    single-problem solver per cavity, recorded steps replayed on 16 streams) and
    the batched engine in FP64."""
    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    from pycfd_b200 import _lib
    from pycfd_b200.batch import (BatchAutotuner, BatchedSolver, BatchOptions, BatchRunner, ConcurrentBatch,
                                  cavity_batch_configs, partition_by_cells)
    from pycfd_b200.solver import GpuOptions
    all_cfgs = cavity_batch_configs(count=args.batch * world, seed=0)
    cfgs = [all_cfgs[k] for k in partition_by_cells(all_cfgs, world)[rank]]
    my_cells = sum(c.nx * c.ny for c in cfgs)
    total_cells = sum(c.nx * c.ny for c in all_cfgs)
    t0 = time.perf_counter()
    if args.autotune:
        opts = BatchAutotuner(allowed_precisions=(args.precision,)).choose(cfgs)
    else:
        tail = args.batch_tail
        opts = BatchOptions(precision=args.precision, tile_rows=args.tile_rows,
                            mg_sweeps=args.mg_sweeps, inner_tol=args.inner_tol,
                            coarse_level=args.coarse_level, coarse_tail=tail != "off",
                            tail_ratio=None if tail in ("none", "off") else float(tail),
                            fused_restriction=args.fused_from > 0, fused_from=max(1, args.fused_from),
                            ell_group=args.ell_group, programmatic_launch=args.pdl,
                            stencil_transfer=args.stencil)
    if args.scalar_strips:
        import dataclasses
        opts = dataclasses.replace(opts, scalar_strips=True)
    b = ConcurrentBatch(cfgs, opts, parts=args.parts) if args.parts > 1 else BatchedSolver(cfgs, opts)
    setup = time.perf_counter() - t0
    rec = not args.eager

    def timed(step_fn, k):
        """Device ms of k steps (events on the launching stream, barrier + sync both sides)."""
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        ev0.record()
        step_fn(k)
        ev1.record()
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        return max_over_ranks(ev0.elapsed_time(ev1), dist, "cuda")

    b.step(args.spinup, record=rec)
    b.step(args.warmup, record=rec)
    torch.cuda.synchronize()
    b.launches(0)
    n_launch0 = _lib.load().pycfd_launch_count()
    clocks = Clocks(local) if rank == 0 else None
    ms = timed(lambda k: b.step(k, record=rec), args.steps)
    ck = clocks.stop() if clocks else None
    launches = b.launches(args.steps) if rec else int(_lib.load().pycfd_launch_count() - n_launch0)
    value = total_cells * args.steps / (ms / 1e3)
    st = b.status()
    its = st["iterations"]
    divs = np.array([b.field_stats(k).max_div for k in range(len(b))])
    # roofline: the kernel kind with the largest share of one eager step
    s_bytes = 4 if opts.precision == "mixed" else 8
    cells = np.array([c.nx * c.ny for c in cfgs], dtype=np.float64)
    prof = {}
    if not args.no_profile:
        for kid in (1, 2, 3, 5, 6):
            kms, kn, kits = b.profile(kid, 1)
            prof[kid] = (kms, kn, batch_kernel_bytes(kid, cells, kits, s_bytes))
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm = peaks.get("hbm_gbs")
    peak_src = "MEASURED_PEAKS.json hbm_gbs (of measured)"
    if hbm is None:
        hbm, peak_src = 6650.0, "fallback 6.65 TB/s (MEASURED_PEAKS.json absent)"
    roof = None
    if prof:
        top = max(prof, key=lambda k: prof[k][0])
        kms, kn, kbytes = prof[top]
        achieved = kbytes / (kms / 1e3) / 1e9 if kms > 0 else None
        traffic = None
        try:
            tr = json.load(open(os.path.join(ROOT, "profiles", "roofline_traffic.json")))
            traffic = tr.get("batch_" + opts.precision, {}).get(str(top))
        except Exception:
            pass
        roof = {"bound": "hbm", "kernel": KERNEL_NAMES[top], "achieved": achieved, "peak": hbm,
                "unit": "GB/s", "frac": achieved / hbm if achieved else None, "traffic": traffic,
                "bytes_per_launch": kbytes / max(kn, 1), "us_per_launch": 1e3 * kms / max(kn, 1),
                "launches": kn, "peak_source": peak_src,
                "timing": "CUDA events around each eager launch of the kernel over one step; bytes = "
                          "sum over problems of its passes x cells x bytes per cell",
                "kernels": {KERNEL_NAMES[k].split(" ")[0] + ("" if k not in (2, 3) else f"[{k}]"):
                            {"ms": v[0], "launches": v[1],
                             "gb_s": (v[2] / (v[0] / 1e3) / 1e9) if v[0] > 0 and v[2] else None}
                            for k, v in prof.items()},
                "traffic_source": "profiles/roofline_traffic.json (one ncu capture of this kernel)"}
        if args.parts > 1:
            # the same kernel kinds at full size: the whole batch in one engine, so every
            # launch covers every cavity (the timed step's parts launch a quarter each)
            b1 = BatchedSolver(cfgs, opts)
            b1.step(1, record=False)
            one = {}
            for kid in prof:
                kms1, kn1, kits1 = b1.profile(kid, 1)
                kb1 = batch_kernel_bytes(kid, cells, kits1, s_bytes)
                gbs = kb1 / (kms1 / 1e3) / 1e9 if kms1 > 0 and kb1 else None
                one[KERNEL_NAMES[kid].split(" ")[0] + ("" if kid not in (2, 3) else f"[{kid}]")] = {
                    "us_per_launch": 1e3 * kms1 / max(kn1, 1), "launches": kn1, "gb_s": gbs,
                    "frac": gbs / hbm if gbs else None}
            del b1
            roof["one_engine"] = {"note": "each kind timed by CUDA events around its eager launches "
                                          "over one step of the whole batch in one engine",
                                  "kernels": one}
    # end to end: (u, v) of every cavity from pinned host memory, one step, (u, v, p) back
    e2e_steps = 0 if args.no_e2e else max(1, min(args.steps, 10))
    e2e = None
    if e2e_steps:
        b.step_host(1)
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        b.step_host(e2e_steps)
        e2e_s = max_over_ranks(time.perf_counter() - t0, dist, "cuda")
        h2d, d2h = b.state_bytes()
        e2e = {"value": total_cells * e2e_steps / e2e_s, "unit": UNIT,
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
               "note": "per rank; every cavity's (u, v) H2D and (u, v, p) D2H inside each timed step"}
    del b
    fp64b = plain = None
    if not args.no_plain:
        # the batched engine in FP64 on the same problems and steps
        o64 = BatchAutotuner(allowed_precisions=("fp64",)).choose(cfgs) if args.autotune else \
            BatchOptions(precision="fp64")
        b64 = ConcurrentBatch(cfgs, o64, parts=args.parts) if args.parts > 1 else BatchedSolver(cfgs, o64)
        b64.step(args.spinup + args.warmup)
        ms64 = timed(lambda k: b64.step(k), args.steps)
        fp64b = {"value": total_cells * args.steps / (ms64 / 1e3), "ms_per_step": ms64 / args.steps,
                 "max_div": max(b64.field_stats(k).max_div for k in range(len(b64))),
                 "options": o64.__dict__}
        del b64
        # the plain FP64 path on the same problems: per-problem recorded steps on 16 streams
        popts = {"auto": GpuOptions(precision="fp64"),
                 "compact": GpuOptions(precision="fp64", tail_ratio=4.0),
                 "off": GpuOptions(precision="fp64", coarse_tail=False)}[args.plain_tail]
        runner = BatchRunner(cfgs, streams=16, options=popts)
        runner.step(args.spinup + args.warmup)
        pms = timed(runner.step, args.steps)
        plain = {"value": total_cells * args.steps / (pms / 1e3), "ms_per_step": pms / args.steps,
                 "steps": args.steps, "form": "fp64, one single-problem solver per cavity, "
                                             "recorded steps replayed on 16 streams",
                 "dense_tail": args.plain_tail}
        del runner
    if rank == 0:
        sizes = {}
        for c in all_cfgs:
            sizes[str(c.nx)] = sizes.get(str(c.nx), 0) + 1
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64/f32" if opts.precision == "mixed" else "f64", "data": "synthetic",
                "config": {"workload": f"batch of {args.batch} lid-driven cavities per GPU "
                                       f"(seed 0, {args.batch * world} in all, split over ranks by cells)",
                           "cells": total_cells, "cells_rank0": my_cells, "sizes": sizes,
                           "re": "log-uniform 100..2000", "lid": "uniform 0.5..1.5",
                           "pressure_solver": "mgcg", "poisson_tol": cfgs[0].poisson_tol,
                           "dt": "adaptive, CFL 0.5, per cavity",
                           "precision": opts.precision, "options": opts.__dict__,
                           "autotuned": bool(args.autotune), "setup_s": setup,
                           "spinup_steps": args.spinup,
                           "cg_iterations_per_step": float(np.mean(its)),
                           "stopped": int((st["frozen"] != 0).sum()),
                           "max_div": float(divs.max()), "cavities_div_le_1e-8": int((divs <= 1e-8).sum()),
                           "parallelism": f"problem partition x{world}, {args.parts} concurrent parts per GPU",
                           "l2": "working set larger than L2 (no flush needed)",
                           "cell_update": "one cell advanced by one RK3 step, summed over the batch",
                           "batched_fp64": fp64b, "plain_fp64_path": plain,
                           "mixed_batched_vs_plain_fp64": value / plain["value"] if plain else None,
                           "mixed_batched_vs_batched_fp64": value / fp64b["value"] if fp64b else None},
                "e2e": e2e, "clocks": ck, "roofline": roof, "gpu_launches": launches}
        if not args.no_cpu_baseline:
            # a bounded sample: 16 cavities of the batch, enough steps for about 10-30 s of work
            line["cpu_baseline"] = batch_cpu_baseline(cfgs, steps=60, workers=16)
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


def run_tgv_validation(args, local):
    """The 512x512 vortex over 500 steps in the FP64 path and in the mixed form: error of
    each against the analytic decay (u, v ~ exp(-2 nu t), p ~ exp(-4 nu t), mean-free)
    and of the mixed form against FP64."""
    import torch
    torch.cuda.set_device(local)
    from pycfd_b200.solver import GpuOptions, ProjectionSolver
    cfg = tgv_config()
    steps = args.val_steps
    out, fields = {}, {}
    for prec in ("fp64", "mixed"):
        s = ProjectionSolver(cfg, options=GpuOptions(precision=prec))
        f = s.initialize(*tgv_init(s.mesh))
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record()
        for _ in range(steps):
            f = s.advance(f, cfg.dt)
        b.record()
        torch.cuda.synchronize()
        ms = a.elapsed_time(b) / steps
        t = steps * cfg.dt
        nu = cfg.nu
        Xu, Yu = s.mesh.u_grid()
        Xv, Yv = s.mesh.v_grid()
        ue = np.sin(Xu) * np.cos(Yu) * np.exp(-2 * nu * t)
        ve = -np.cos(Xv) * np.sin(Yv) * np.exp(-2 * nu * t)
        xc, yc = s.mesh.xc, s.mesh.yc
        pe = 0.25 * (np.cos(2 * xc)[:, None] + np.cos(2 * yc)[None, :]) * np.exp(-4 * nu * t)
        pe -= pe.mean()
        u = f.u_phys.cpu().numpy()
        v = f.v_phys.cpu().numpy()
        p = f.p[1:-1, 1:-1].cpu().numpy()
        p = p - p.mean()
        st = s.field_stats(f)
        fields[prec] = (u, v, p)
        out[prec] = {"ms_per_step": ms, "cell_updates_per_s": N * N / (ms / 1e3),
                     "err_u": float(np.abs(u - ue).max() / np.abs(ue).max()),
                     "err_v": float(np.abs(v - ve).max() / np.abs(ve).max()),
                     "err_p": float(np.abs(p - pe).max() / np.abs(pe).max()), "max_div": st.max_div}
        del s
    uf, vf, pf = fields["fp64"]
    um, vm, pm = fields["mixed"]
    scale = max(np.abs(uf).max(), np.abs(vf).max())
    out["mixed_vs_fp64"] = {"velocity": float(max(np.abs(um - uf).max(), np.abs(vm - vf).max()) / scale),
                            "pressure": float(np.abs(pm - pf).max() / np.abs(pf).max())}
    line = {"metric": METRIC, "value": out["fp64"]["cell_updates_per_s"], "unit": UNIT, "n_gpus": 1,
            "steps": steps, "warmup": 0, "ms_per_step": out["fp64"]["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config({"validation": out, "t_end": steps * cfg.dt})}
    print(json.dumps(line), flush=True)


def run_cylinder(args, local):
    """Flow past a cylinder on the 2048x1024 channel (Re 100, D 0.1 at (0.5, 0.5), uniform
    inflow 1, convective outlet, slip walls, 1e-3 seeded noise), MG-PCG 1e-10, adaptive dt:
    Cd and Cl histories in the FP64 path and in the mixed form."""
    import torch
    torch.cuda.set_device(local)
    from pycfd_b200.config import BCKind, BCSpec, SimulationConfig
    from pycfd_b200.mesh import StructuredMesh
    from pycfd_b200.obstacles import circle_mask
    from pycfd_b200.solver import GpuOptions, ProjectionSolver
    nx, ny = 2048, 1024
    walls = {"left": BCSpec(BCKind.INLET, velocity=1.0), "right": BCSpec(BCKind.OUTLET),
             "bottom": BCSpec(BCKind.SYMMETRY), "top": BCSpec(BCKind.SYMMETRY)}
    cfg = SimulationConfig(nx=nx, ny=ny, lx=2.0, ly=1.0, re=100.0, u_ref=1.0, l_ref=0.1, dt=1.0,
                           t_end=1e9, cfl_max=0.5, pressure_solver="mgcg", poisson_tol=1e-10,
                           boundary_config=walls, name="cylinder")
    mesh = StructuredMesh.from_config(cfg)
    obstacle = circle_mask(mesh, (0.5, 0.5), 0.05)
    rng = np.random.default_rng(0)
    u0 = 1.0 + 1e-3 * rng.standard_normal((nx + 1, ny))
    v0 = 1e-3 * rng.standard_normal((nx, ny + 1))
    steps, every = args.cyl_steps, 20
    out = {}
    for prec in ("fp64", "mixed"):
        s = ProjectionSolver(cfg, mesh, obstacle, options=GpuOptions(precision=prec))
        f = s.initialize(u0, v0)
        s.set_clock(0.0)
        ts, cd, cl = [], [], []
        dev_ms = 0.0
        for k in range(steps // every):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            for _ in range(every):
                f = s.advance_adaptive(f)
            b.record()
            torch.cuda.synchronize()
            dev_ms += a.elapsed_time(b)
            st = s._read_stats()
            t, dt, n, h = s.clock()
            if h:
                break
            ts.append(t)
            cd.append(st.fx / 0.05)
            cl.append(st.fy / 0.05)
        ts, cd, cl = np.array(ts), np.array(cd), np.array(cl)
        half = ts >= 0.5 * ts[-1]
        clh = cl[half] - cl[half].mean()
        crossings = np.where(np.diff(np.sign(clh)) > 0)[0]
        st_num = None
        if len(crossings) >= 2:
            period = (ts[half][crossings[-1]] - ts[half][crossings[0]]) / (len(crossings) - 1)
            st_num = 0.1 / period
        fs = s.field_stats(f)
        out[prec] = {"steps": int(n), "t_end": float(ts[-1]), "ms_per_step": dev_ms / max(n, 1),
                     "cell_updates_per_s": nx * ny * n / (dev_ms / 1e3),
                     "cd_mean_second_half": float(cd[half].mean()), "cl_amplitude_second_half":
                     float(0.5 * (cl[half].max() - cl[half].min())), "strouhal": st_num,
                     "max_div": fs.max_div, "health": int(h),
                     "cd_every_20": [round(float(x), 6) for x in cd[::10]],
                     "cl_every_20": [round(float(x), 6) for x in cl[::10]]}
        del s
    line = {"metric": METRIC, "value": out["fp64"]["cell_updates_per_s"], "unit": UNIT, "n_gpus": 1,
            "steps": steps, "warmup": 0, "ms_per_step": out["fp64"]["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "cylinder channel 2048x1024, Re 100", "runs": out}}
    print(json.dumps(line), flush=True)


def run_stretched(args, local):
    """A channel past a cylinder on a stretched 1024x512 mesh (cells clustered at both
    walls in y, growing from the inlet in x) against the same channel on the uniform
    mesh: FP64 MG-PCG to 1e-10, parabolic inflow 1, convective outlet, Re 100, fixed dt.
    Times `args.steps` steps of each after `args.warmup`; the stretched mesh's cost is
    its per-face metrics in every stencil and the row-scaled Poisson operator."""
    import torch
    torch.cuda.set_device(local)
    from pycfd_b200.config import BCKind, BCSpec, SimulationConfig
    from pycfd_b200.mesh import StructuredMesh
    from pycfd_b200.obstacles import circle_mask
    from pycfd_b200.solver import ProjectionSolver
    nx, ny = 1024, 512
    walls = {"left": BCSpec(BCKind.INLET, velocity=1.0, profile="parabolic"), "right": BCSpec(BCKind.OUTLET),
             "bottom": BCSpec(BCKind.NO_SLIP), "top": BCSpec(BCKind.NO_SLIP)}
    out = {}
    for name, (sx, sy) in (("stretched", (1.001, 1.006)), ("uniform", (1.0, 1.0))):
        cfg = SimulationConfig(nx=nx, ny=ny, lx=4.0, ly=1.0, stretch_x=sx, stretch_y=sy, cluster_x="low",
                               cluster_y="walls", re=100.0, u_ref=1.0, l_ref=0.2, dt=1e-4, t_end=1e9,
                               adaptive_dt=False, pressure_solver="mgcg", poisson_tol=1e-10,
                               boundary_config=walls, name=f"channel_{name}")
        mesh = StructuredMesh.from_config(cfg)
        s = ProjectionSolver(cfg, mesh, circle_mask(mesh, (1.0, 0.5), 0.1))
        f = s.initialize()
        for _ in range(args.warmup):
            f = s.advance(f, cfg.dt)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record()
        its = 0
        for _ in range(args.steps):
            f = s.advance(f, cfg.dt)
            its += s.last_stats.total_iterations
        b.record()
        torch.cuda.synchronize()
        ms = a.elapsed_time(b) / args.steps
        fs = s.field_stats(f)
        out[name] = {"ms_per_step": ms, "cell_updates_per_s": nx * ny / (ms / 1e3),
                     "mgpcg_iterations_per_step": its / args.steps, "max_div": fs.max_div,
                     "cd": s.body_force_reaction[0] / (0.5 * 1.0 * 0.2), "min_cell": [mesh.metrics.min_hx,
                                                                                      mesh.metrics.min_hy]}
        del s
    line = {"metric": METRIC, "value": out["stretched"]["cell_updates_per_s"], "unit": UNIT, "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": out["stretched"]["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": {"workload": "channel past a cylinder, stretched 1024x512 mesh "
                                                        "against the uniform one", "runs": out}}
    print(json.dumps(line), flush=True)


def run_adjoint(args, world, rank, local):
    """Gradient of the lower-half kinetic energy of the 256x256 Re 400 cavity after 200
    steps w.r.t. 32 lid modes and the smoothed-disk radius: hand-written adjoint with
    10-step checkpoints, checked against central differences (h = 1e-6) on 3 components."""
    import torch
    torch.cuda.set_device(local)
    from pycfd_b200.adjoint import AdjointCavity, Geometry, MultigridSolve, gradient, rollout
    cav = AdjointCavity()
    g = Geometry(cav, device="cuda")
    solve = MultigridSolve(cav.n, tol=cav.tol)
    theta = torch.tensor(cav.default_theta(), dtype=torch.float64, device="cuda")
    radius = torch.tensor(cav.radius, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    solve.calls = 0
    J, gt, gr = gradient(theta, radius, g, solve)
    torch.cuda.synchronize()
    t_grad = time.perf_counter() - t0
    grad_solves = solve.calls
    t0 = time.perf_counter()
    J0, _ = rollout(theta, radius, g, solve)
    torch.cuda.synchronize()
    t_fwd = time.perf_counter() - t0
    h = 1e-6
    checks = []
    with torch.no_grad():
        for k in (0, 7):
            e = torch.zeros_like(theta)
            e[k] = h
            fd = float((rollout(theta + e, radius, g, solve)[0] - rollout(theta - e, radius, g, solve)[0]) / (2 * h))
            checks.append({"param": f"theta_{k + 1}", "adjoint": float(gt[k]), "fd": fd,
                           "rel_err": abs(fd - float(gt[k])) / max(abs(fd), 1e-300)})
        fd = float((rollout(theta, radius + h, g, solve)[0] - rollout(theta, radius - h, g, solve)[0]) / (2 * h))
        checks.append({"param": "radius", "adjoint": float(gr), "fd": fd,
                       "rel_err": abs(fd - float(gr)) / max(abs(fd), 1e-300)})
    cells = cav.n * cav.n
    line = {"metric": "gradient of J (lower-half kinetic energy) w.r.t. 33 parameters, adjoint",
            "value": cells * cav.steps / t_grad, "unit": "cell-updates/s (forward + adjoint sweep)",
            "n_gpus": 1, "steps": cav.steps, "warmup": 0, "ms_per_step": 1e3 * t_grad / cav.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": "lid-driven cavity 256x256, Re 400, 200 steps, dt 1.2e-3, "
                                   "32 sine lid modes (seeded) + tanh disk radius at (0.5, 0.3), "
                                   "r 0.08, width 2 cells",
                       "poisson_tol": cav.tol, "checkpoint_every": cav.checkpoint,
                       "J": float(J), "forward_s": t_fwd, "gradient_s": t_grad,
                       "gradient_over_forward": t_grad / t_fwd, "poisson_solves_in_gradient": grad_solves,
                       "fd_checks": checks, "max_fd_rel_err": max(c["rel_err"] for c in checks)}}
    print(json.dumps(line), flush=True)


def run_reference(args, world, rank):
    if rank != 0:
        return
    import torch  # noqa: F401  (same process layout as the GPU arm)
    if args.workload == "batch":
        from pycfd_b200.batch import cavity_batch_configs
        # the 256 cavities of one GPU's share at N = 1; each timed step of this arm is one
        # RK3 step of as many of them as there are host threads, all processes at once
        w = min(args.warmup, 3)
        k = max(1, min(args.steps, 5))
        cb = batch_cpu_baseline(cavity_batch_configs(count=args.batch, seed=0), steps=k, warmup=w)
        line = {"metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": args.gpus,
                "steps": k, "warmup": w, "ms_per_step": 1e3 * cb["wall_s"] / k,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic", "impl": "reference",
                "config": {"workload": f"batch of {args.batch} lid-driven cavities per GPU (seed 0)",
                           "sample": cb["sample"]},
                "cpu_baseline": cb,
                "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return
    steps = max(1, min(args.steps, 4))
    w = min(args.warmup, 3)   # each oracle step of the 512x512 vortex takes about a second
    cb = cpu_baseline(steps, warmup=w)
    line = {"metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": args.gpus,
            "steps": steps, "warmup": w, "ms_per_step": 1e3 * N * N / cb["value"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "impl": "reference", "config": workload_config(),
            "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args, world, rank, local):
    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    from pycfd_b200.solver import GpuOptions, ProjectionSolver
    from pycfd_b200.mesh import StructuredMesh
    cfg = tgv_config()
    opts = GpuOptions(precision=args.precision, graphs=not args.eager, persistent_solve=args.persistent,
                      coarse_tail=not args.no_tail, ell_thread_budget=args.ell_budget)
    solver = ProjectionSolver(cfg, options=opts)
    f = solver.initialize(*tgv_init(solver.mesh))
    dt = cfg.dt
    for _ in range(args.warmup):
        f = solver.advance(f, dt)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    iters = []
    clocks = Clocks(local) if rank == 0 else None
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    for k in range(args.steps):
        flush.fill_(float(k))
        evs[k][0].record(stream)
        f = solver.advance(f, dt)
        evs[k][1].record(stream)
        iters.append(solver.last_stats.total_iterations)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ck = clocks.stop() if clocks else None
    dev_ms = max_over_ranks(sum(a.elapsed_time(b) for a, b in evs), dist, "cuda")
    value = world * N * N * args.steps / (dev_ms / 1e3)
    st = solver.field_stats(f)
    launches_per_step = solver.launches_per_step(f, dt)

    # end to end through the public host-buffer call: copies inside the timed region
    # (two sets of pinned state buffers, ping-ponged: each step reads one, writes the other)
    pin = lambda shape: torch.empty(shape, dtype=torch.float64).pin_memory().numpy()
    bufs = [(pin(solver.mesh.u_shape), pin(solver.mesh.v_shape), pin(solver.mesh.p_shape)) for _ in range(2)]
    bufs[0][0][...] = f.u.cpu().numpy()
    bufs[0][1][...] = f.v.cpu().numpy()
    un, vn = bufs[0][0], bufs[0][1]
    e2e_steps = 0 if args.no_e2e else args.steps
    if e2e_steps:
        solver.step_host(un, vn, dt, out=bufs[1])   # records the host-buffer step once
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for k in range(e2e_steps):
        un, vn, _ = solver.step_host(un, vn, dt, out=bufs[(k + 1) % 2])
    e2e_s = max_over_ranks(time.perf_counter() - t0, dist, "cuda")
    e2e_value = world * N * N * e2e_steps / e2e_s if e2e_steps else None
    h2d = (un.size + vn.size) * 8
    d2h = (un.size + vn.size + int(np.prod(solver.mesh.p_shape))) * 8

    if rank == 0:
        peaks = {}
        try:
            peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        except Exception:
            pass
        hbm = peaks.get("hbm_gbs")
        peak_src = "MEASURED_PEAKS.json hbm_gbs (of measured)"
        if hbm is None:
            hbm, peak_src = 6650.0, "fallback 6.65 TB/s (MEASURED_PEAKS.json absent)"
        roof = live_roofline(solver, f, dt, hbm, peak_src)
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": dev_ms / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64" if args.precision == "fp64" else "f64/f32",
                "data": "synthetic",
                "config": workload_config({"precision": args.precision,
                                           "solve_form": "one cooperative launch per solve" if solver._persistent
                                           else "one kernel per phase",
                                           "coarse_tail": bool(opts.coarse_tail),
                                           "parallelism": f"replicas x{world}",
                                           "mgpcg_iterations_per_step": float(np.mean(iters)),
                                           "max_div": st.max_div}),
                "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                        "d2h_bytes_per_step": int(d2h)},
                "clocks": ck, "roofline": roof,
                "gpu_launches": launches_per_step * args.steps}
        if not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(2)
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default=None, choices=["fp64", "mixed"],
                    help="default: fp64 for the vortex, mixed for the batch")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer leg (profiling runs)")
    ap.add_argument("--eager", action="store_true", help="launch kernels one by one (no CUDA graph)")
    ap.add_argument("--persistent", action="store_true",
                    help="tgv512: each CG solve as one cooperative launch (phases between grid barriers)")
    ap.add_argument("--ell-budget", type=int, default=0,
                    help="tgv512: resident threads per coarse-level pass (0 default, -1 storage lanes)")
    ap.add_argument("--no-tail", action="store_true",
                    help="tgv512: V-cycle level by level down to the coarsest (no dense tail operator)")
    ap.add_argument("--workload", default="batch",
                    choices=["tgv512", "batch", "adjoint", "tgv-validation", "cylinder", "stretched"],
                    help="batch: the seeded 256-cavity batch (the headline); tgv512: the 512x512 "
                         "vortex on the single-problem path")
    ap.add_argument("--spinup", type=int, default=0,
                    help="batch: untimed steps before the warm-up (later steps of the same flow)")
    ap.add_argument("--batch", type=int, default=256, help="problems in the batch workload")
    ap.add_argument("--val-steps", type=int, default=500, help="tgv-validation: steps")
    ap.add_argument("--cyl-steps", type=int, default=20000, help="cylinder: steps per precision")
    ap.add_argument("--no-autotune", dest="autotune", action="store_false",
                    help="batch: take the options below instead of the autotuner's choice (tiles, sweeps, "
                         "tail bound, coarse level, inner tolerance; timed on the batch, cached)")
    ap.add_argument("--tile-rows", type=int, default=32, choices=[8, 16, 32, 64],
                    help="batch: rows per fine-level tile")
    ap.add_argument("--mg-sweeps", type=int, default=1, help="batch: smoothing sweeps per level")
    ap.add_argument("--coarse-level", type=int, default=0,
                    help="batch: multigrid levels from this one down in one block per problem (0: off)")
    ap.add_argument("--inner-tol", type=float, default=1e-4, help="batch, mixed: inner tolerance")
    ap.add_argument("--batch-tail", default="16",
                    help="batch: dense V-cycle tail per structure -- a bound r (n_t^2 <= r n_0), none, or off")
    ap.add_argument("--plain-tail", default="auto", choices=["auto", "compact", "off"],
                    help="batch: dense V-cycle tail of the plain per-problem leg (compact: n_t^2 <= 4 n_0)")
    ap.add_argument("--fused-from", type=int, default=0, choices=[0, 1, 2],
                    help="batch, --no-autotune: down sweep by fused restrictions from this level (0: off)")
    ap.add_argument("--parts", type=int, default=4,
                    help="batch: batched engines stepped concurrently on their own streams (problems split by cells)")
    ap.add_argument("--pdl", action="store_true",
                    help="batch, --no-autotune: programmatic dependent launch between the kernels")
    ap.add_argument("--stencil", action="store_true",
                    help="batch, --no-autotune, --fused-from 1: level-0 transfers as stencils over the fine cells")
    ap.add_argument("--scalar-strips", action="store_true",
                    help="batch: the FP32 CG and level-0 sweep kernels on 30-column scalar strips "
                         "(default: 128-column float4 strips)")
    ap.add_argument("--ell-group", type=int, default=8, choices=[1, 8],
                    help="batch, --no-autotune: problems per coarse-level block sharing the matrix loads")
    ap.add_argument("--no-profile", action="store_true",
                    help="batch: skip the per-kernel eager timing of the roofline block")
    ap.add_argument("--no-plain", action="store_true",
                    help="batch: skip the plain per-problem FP64 comparison leg")
    args = ap.parse_args()
    if args.precision is None:
        args.precision = "mixed" if args.workload == "batch" else "fp64"
    world, rank, local = dist_setup()
    if args.impl == "reference":
        run_reference(args, world, rank)
    elif args.workload == "batch":
        run_batch(args, world, rank, local)
    elif args.workload == "adjoint":
        if rank == 0:
            run_adjoint(args, world, rank, local)
    elif args.workload == "tgv-validation":
        if rank == 0:
            run_tgv_validation(args, local)
    elif args.workload == "stretched":
        if rank == 0:
            run_stretched(args, local)
    elif args.workload == "cylinder":
        if rank == 0:
            run_cylinder(args, local)
    else:
        run_ours(args, world, rank, local)


if __name__ == "__main__":
    main()
