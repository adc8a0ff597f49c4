"""Splitting the evaluate-and-mesh workloads over several GPUs, one process
per GPU (torch.distributed, NCCL between GPUs).

The reference runs on one machine's threads only (WorkerPool, libfive/src/
render/brep/worker_pool.inl:35-255; the dual walk's per-thread buffers merged
by BRep::collect, libfive/include/libfive/render/brep/brep.hpp:51-107).
Across GPUs the work splits without any exchange inside the data path:

* Many trees (`mesh_trees`): each tree is meshed by exactly one rank.  Trees
  are dealt out by estimated cost (tape length x 4^depth, the surface cell
  count of a depth-d octree grows as 4^d), largest first, each to the rank
  with the least cost so far.  One all-gather of every tree's (vertex count,
  triangle count) then gives every rank the sizes and the offsets of all
  meshes in a concatenated output, so that rank 0 (or a file writer) can
  place each rank's meshes without a second round trip.
* Points (`grad_points`): the n points are split into contiguous slices,
  one per rank; each rank computes f and the point gradients of its slice
  and its partial sum of the variable gradient; one all-reduce (sum) of the
  V-float variable gradient gives every rank the whole sum.

`compute` arguments default to this library's GPU entry points; tests pass
stand-ins so that the partitioning and the collectives run on CPU ranks
(gloo).  The process group is torch.distributed's default group unless one
is given.
"""
import numpy as np


def tree_cost(n_clauses, depth):
    """Estimated meshing cost of a tree: tape length x 4^depth."""
    return float(n_clauses + 1) * float(4 ** depth)


def assign_trees(costs, world):
    """Cost-ordered assignment of trees to `world` ranks: trees in
    decreasing cost, each to the rank with the least total so far (ties to
    the lowest rank).  Returns owner[i] for every tree i."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    owner = [0] * len(costs)
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        owner[i] = r
        load[r] += costs[i]
    return owner


def _dist(pg):
    import torch.distributed as dist
    return dist, pg


def mesh_trees(jobs, costs, rank, world, pg=None, compute=None, device="cpu"):
    """Meshes this rank's share of `jobs` and shares every mesh's size.

    jobs: list of job descriptions (for the default compute: tuples
    (tape, lower, upper, min_feature[, max_err]) as shape.render_meshes
    takes); costs: tree_cost of each.  compute(list of jobs) -> list of
    (verts, tris).  Returns (owner, meshes, counts, offsets): owner[i] the
    rank meshing tree i, meshes {i: (verts, tris)} for this rank's trees,
    counts an int64 array [n, 2] of (vertices excluding the placeholder
    vertex 0, triangles) of every tree, and offsets [n + 1, 2] their
    exclusive prefix sums (where tree i's vertices and triangles start in a
    concatenation of all meshes)."""
    import torch
    owner = assign_trees(costs, world)
    mine = [i for i in range(len(jobs)) if owner[i] == rank]
    if compute is None:
        from .shape import render_meshes
        compute = render_meshes
    out = compute([jobs[i] for i in mine]) if mine else []
    meshes = dict(zip(mine, out))
    local = torch.zeros((len(jobs), 2), dtype=torch.int64, device=device)
    for i, (v, t) in meshes.items():
        local[i, 0] = max(len(v) - 1, 0)
        local[i, 1] = len(t)
    if world > 1:
        dist, pg = _dist(pg)
        parts = [torch.zeros_like(local) for _ in range(world)]
        dist.all_gather(parts, local, group=pg)
        counts = torch.stack(parts).sum(dim=0)
    else:
        counts = local
    counts = counts.cpu().numpy()
    offsets = np.zeros((len(jobs) + 1, 2), np.int64)
    offsets[1:] = np.cumsum(counts, axis=0)
    return owner, meshes, counts, offsets


def point_slice(n, rank, world):
    """The contiguous slice [lo, hi) of n points that `rank` evaluates."""
    per = (n + world - 1) // world
    lo = min(n, rank * per)
    return lo, min(n, lo + per)


def grad_points(tape, x, y, z, seed, rank, world, pg=None, compute=None):
    """Reverse-mode gradients of sum_i seed_i f(p_i) over n points split
    across ranks (lfb_eval_grad on each rank's slice).

    x, y, z, seed: every rank passes the full arrays (numpy, or CUDA tensors
    for the default compute); compute(tape, x, y, z, seed) -> (f, gx, gy, gz,
    gvars) on a slice.  Returns (lo, hi, f, gx, gy, gz, gvars): this rank's
    slice with its values and point gradients, and the variable gradient
    summed over all points by one all-reduce."""
    import torch
    n = len(x)
    lo, hi = point_slice(n, rank, world)
    if compute is None:
        compute = _gpu_grad
    f, gx, gy, gz, gv = compute(tape, x[lo:hi], y[lo:hi], z[lo:hi], seed[lo:hi])
    if world > 1:
        dist, pg = _dist(pg)
        t = gv if isinstance(gv, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(gv))
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=pg)
        gv = t if isinstance(gv, torch.Tensor) else t.numpy()
    return lo, hi, f, gx, gy, gz, gv


def _gpu_grad(tape, x, y, z, seed):
    import torch
    n = len(x)
    dev = x.device if isinstance(x, torch.Tensor) else None
    if dev is None or dev.type != "cuda":
        raise ValueError("the GPU gradient takes CUDA tensors")
    f, gx, gy, gz = (torch.empty(n, device=dev) for _ in range(4))
    gv = torch.zeros(tape.n_vars, device=dev)
    if n:
        tape.grad(x.contiguous(), y.contiguous(), z.contiguous(), seed=seed.contiguous(), f=f,
                  gx=gx, gy=gy, gz=gz, gvars=gv,
                  stream=torch.cuda.current_stream().cuda_stream)
    return f, gx, gy, gz, gv
