"""Multi-process paths on the CPU: two gloo ranks (no GPU).

The bench runs one process per GPU.  A single domain does not shard (replicas
only); the cavity batch is partitioned: each rank takes its share of the
independent problems by cell count, with no exchange on the data path, and the
slowest rank's device time sets the figure.  These tests check that reduction,
the rank environment handling and the batch partition with world size 2.
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


def _partition_rank(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    from pycfd_b200.batch import cavity_batch_configs, partition_by_cells
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        cfgs = cavity_batch_configs(count=256 * world, seed=0)
        mine = partition_by_cells(cfgs, world)[rank]     # each rank computes the split alone
        cells = sum(cfgs[k].nx * cfgs[k].ny for k in mine)
        got = [None] * world
        dist.all_gather_object(got, (mine, cells))
        out[rank] = got
    finally:
        dist.destroy_process_group()


def test_batch_partition_over_two_ranks():
    """The 512-cavity batch of two ranks: every cavity on exactly one rank, the ranks
    agree on the split, and their cell totals differ by at most one cavity's cells."""
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        procs = [ctx.Process(target=_partition_rank, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
            assert p.exitcode == 0
        res = dict(out)
    assert res[0] == res[1]
    parts = [set(m) for m, _ in res[0]]
    assert parts[0].isdisjoint(parts[1]) and parts[0] | parts[1] == set(range(512))
    from pycfd_b200.batch import cavity_batch_configs
    cfgs = cavity_batch_configs(count=512, seed=0)
    biggest = max(c.nx * c.ny for c in cfgs)
    totals = [c for _, c in res[0]]
    assert abs(totals[0] - totals[1]) <= biggest
    assert sum(totals) == sum(c.nx * c.ny for c in cfgs)


def test_partition_is_the_whole_batch_on_one_rank():
    from pycfd_b200.batch import cavity_batch_configs, partition_by_cells
    cfgs = cavity_batch_configs(count=256, seed=0)
    assert partition_by_cells(cfgs, 1) == [list(range(256))]
    with pytest.raises(ValueError):
        partition_by_cells(cfgs, 0)
