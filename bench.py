"""Throughput of the projection step: cell-updates/s on the 512x512 Taylor-Green vortex.

One step = one SSP-RK3 time step of the whole 512x512 doubly periodic vortex
(Re 1000, fixed dt = 0.4*2pi/512, MG-PCG to 1e-10, three projections).
value = cells x steps / device time of the timed steps (CUDA events on the
launching stream, barrier + synchronise on both sides, max over ranks).  The
working set (~60 MB) fits in the 126 MB L2, so L2 is flushed between timed
steps by writing a 256 MB buffer outside the timed events.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--precision fp64|mixed]

--impl reference times the reference algorithm's CPU implementation (the NumPy/
SciPy restatement in oracle/, which only this arm and the cpu_baseline leg run)
on the host cores, on the same workload and metric.  Under torchrun every rank
advances its own replica of the vortex (the path does not shard: replicas only)
and rank 0 prints one JSON line.
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


def live_roofline(solver, f, dt, hbm_gbs, steps=3):
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
            "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)",
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
        hbm = peaks.get("hbm_gbs", 6650.0)
        roof = live_roofline(solver, f, dt, hbm)
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
                    choices=["tgv512", "batch", "adjoint", "tgv-validation", "cylinder"],
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
    elif args.workload == "cylinder":
        if rank == 0:
            run_cylinder(args, local)
    else:
        run_ours(args, world, rank, local)


if __name__ == "__main__":
    main()
