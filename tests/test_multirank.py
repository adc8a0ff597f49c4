"""The multi-GPU bench path with two gloo ranks on the CPU: each rank builds
its own seeded shape (weak scaling, no data-path collective) and the only
collective is the MAX all-reduce of the timed totals."""
import os
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    from libfive_b200.shape import slot_tape
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        shape = bench.build_shape(bench.rank_seed(rank))
        n_clauses = len(slot_tape(shape)["clauses"])
        # rank r pretends to take 100 (r + 1) ms for 3 steps
        out = bench.combine_ranks(100.0 * (rank + 1), 50.0 * (rank + 1), world, 3, dist, "cpu")
        q.put((rank, n_clauses, out))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    world = 2
    port = 29500 + os.getpid() % 1000
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0
    got = dict((r, (n, out)) for r, n, out in (q.get(timeout=10) for _ in range(world)))
    # different shapes per rank
    assert got[0][0] != got[1][0]
    for r in range(world):
        total_ms, e2e_ms, value, e2e_value = got[r][1]
        assert total_ms == 200.0 and e2e_ms == 100.0          # slowest rank
        assert value == pytest.approx(world * 3 / 0.2)         # whole-job meshes/s
        assert e2e_value == pytest.approx(world * 3 / 0.1)


def _rank_aux(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # the auxiliary workloads' timing reduction: every rank reports the
        # slowest rank's time
        q.put((rank, bench.rank_max(10.0 * (rank + 1), dist), bench.rank_max(3.5 - rank, dist)))
    finally:
        dist.destroy_process_group()


def test_auxiliary_workloads_take_the_slowest_rank():
    world = 2
    port = 30600 + os.getpid() % 1000
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_aux, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(world))
    assert [g[1:] for g in got] == [(20.0, 3.5), (20.0, 3.5)]
    import bench
    assert bench.rank_max(7.25) == 7.25      # one process: unchanged
