"""Multi-process paths on the CPU: two gloo ranks (no GPU).

The bench runs one process per GPU, each advancing its own replica (the path
does not shard a single domain), and reports the slowest rank's device time.
This checks that reduction and the rank environment handling with world size 2.
"""

import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import bench
    w, r, local = bench.dist_setup()
    dist.init_process_group("gloo", rank=r, world_size=w)
    try:
        times = [12.5, 40.25]                       # per-rank device milliseconds
        got = bench.max_over_ranks(times[r], dist, "cpu")
        out[r] = (w, r, local, got)
    finally:
        dist.destroy_process_group()


def test_slowest_rank_sets_the_time():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        procs = [ctx.Process(target=_rank_main, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
            assert p.exitcode == 0
        res = dict(out)
    assert res[0] == (2, 0, 0, 40.25) and res[1] == (2, 1, 1, 40.25)


def test_reference_arm_only_rank0_prints(capsys, monkeypatch):
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    args = type("A", (), dict(gpus=2, steps=1, warmup=0))()
    bench.run_reference(args, 2, 1)        # rank 1 exits without work
    assert capsys.readouterr().out == ""
