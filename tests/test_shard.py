"""The multi-GPU split of the workloads (libfive_b200/shard.py) with two
gloo ranks on the CPU: the partitioning and the collectives are those of the
GPU runs; the per-rank compute is the CPU oracle standing in for the GPU
entry points.  A split run must give the single-rank result."""
import os
import sys

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HERE = os.path.dirname(os.path.abspath(__file__))

LO, HI = (-1.5, -1.5, -1.5), (1.5, 1.5, 1.5)


def _jobs():
    from libfive_b200 import workloads
    return [(n, seed, mf) for n, seed, mf in
            [(20, 1, 0.1), (60, 2, 0.08), (8, 3, 0.2), (120, 4, 0.1), (30, 5, 0.15)]]


def _oracle_mesher(jobs):
    from libfive_b200 import workloads
    from mesh_compare import oracle_mesh
    from oracle_ffi import OracleTape
    out = []
    for n, seed, mf in jobs:
        o = OracleTape(workloads.random_csg(n, seed=seed, size=(0.1, 0.4)))
        out.append(oracle_mesh(o, LO, HI, mf))
    return out


def _oracle_grad(shape_vals):
    """(f, gx, gy, gz, gvars) of a slice from the oracle's forward
    derivatives and Jacobian (the GPU computes them by reverse mode)."""
    from oracle_ffi import OracleTape
    shape, vals = shape_vals

    def compute(tape, x, y, z, seed):
        o = OracleTape(shape, vals)
        f, dx, dy, dz = o.derivs(x, y, z)
        jac = o.jacobian(x, y, z).astype(np.float64)
        gv = (seed.astype(np.float64) @ jac).astype(np.float32) if len(x) else \
            np.zeros(o.n_vars, np.float32)
        return f, seed * dx, seed * dy, seed * dz, gv
    return compute


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    sys.path.insert(0, HERE)
    from libfive_b200 import shard, workloads
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        jobs = _jobs()
        costs = [shard.tree_cost(n * 10, 5) for n, _, _ in jobs]
        owner, meshes, counts, offsets = shard.mesh_trees(jobs, costs, rank, world,
                                                          compute=_oracle_mesher)
        sv = workloads.blended_spheres_vars(6, seed=2, stable=True)
        x, y, z = workloads.uniform_points(1001, seed=5, lo=-1.2, hi=1.2)
        seed = np.random.default_rng(1).uniform(-1, 1, 1001).astype(np.float32)
        lo, hi, f, gx, gy, gz, gv = shard.grad_points(None, x, y, z, seed, rank, world,
                                                      compute=_oracle_grad(sv))
        q.put((rank, owner, {i: (len(v), len(t)) for i, (v, t) in meshes.items()},
               counts.tolist(), offsets.tolist(), lo, hi, gx.tolist(), gv.tolist()))
    finally:
        dist.destroy_process_group()


def test_assign_trees_is_cost_ordered():
    from libfive_b200.shard import assign_trees
    assert assign_trees([5, 1, 4, 3, 2], 2) == [0, 0, 1, 1, 0]
    assert assign_trees([1.0] * 5, 3) == [0, 1, 2, 0, 1]
    owner = assign_trees(list(range(100, 0, -1)), 4)
    loads = [sum(c for c, o in zip(range(100, 0, -1), owner) if o == r) for r in range(4)]
    assert max(loads) - min(loads) <= 100


def test_point_slices_cover_once():
    from libfive_b200.shard import point_slice
    for n in (0, 1, 7, 1000, 1001):
        for world in (1, 2, 3, 8):
            s = [point_slice(n, r, world) for r in range(world)]
            assert s[0][0] == 0 and s[-1][1] == n
            assert all(s[r][1] == s[r + 1][0] for r in range(world - 1))


def test_two_gloo_ranks_equal_one():
    sys.path.insert(0, HERE)
    from libfive_b200 import shard, workloads
    world = 2
    port = 31700 + os.getpid() % 1000
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=600) for _ in range(world))
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0

    # single rank: everything on one process
    jobs = _jobs()
    costs = [shard.tree_cost(n * 10, 5) for n, _, _ in jobs]
    owner1, meshes1, counts1, offsets1 = shard.mesh_trees(jobs, costs, 0, 1,
                                                          compute=_oracle_mesher)
    sv = workloads.blended_spheres_vars(6, seed=2, stable=True)
    x, y, z = workloads.uniform_points(1001, seed=5, lo=-1.2, hi=1.2)
    seed = np.random.default_rng(1).uniform(-1, 1, 1001).astype(np.float32)
    _, _, f1, gx1, _, _, gv1 = shard.grad_points(None, x, y, z, seed, 0, 1,
                                                 compute=_oracle_grad(sv))

    owners = [g[1] for g in got]
    assert owners[0] == owners[1] and set(owners[0]) == {0, 1}
    # every tree meshed once, by its owner, with the single-rank sizes
    seen = {}
    for rank, _, sizes, counts, offsets, *_ in got:
        assert counts == counts1.tolist() and offsets == offsets1.tolist()
        for i, (nv, nt) in sizes.items():
            assert owners[0][i] == rank and i not in seen
            seen[i] = (nv, nt)
            assert (nv - 1, nt) == tuple(counts1[i])
    assert sorted(seen) == list(range(len(jobs)))
    # point gradients: the ranks' slices concatenate to the single-rank ones;
    # the all-reduced variable gradient equals the single-rank sum
    gx = np.concatenate([np.array(g[7], np.float32) for g in got])
    assert [(g[5], g[6]) for g in got] == [(0, 501), (501, 1001)]
    assert np.array_equal(gx, gx1)
    for g in got:
        assert np.allclose(np.array(g[8]), gv1, rtol=1e-5, atol=1e-6)
