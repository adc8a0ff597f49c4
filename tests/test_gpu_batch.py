"""Batched meshing (lfb_render_meshes): several tapes in flight at once, each
on its own CUDA stream.  Every mesh of a batch must be the mesh that
lfb_render_mesh gives for the same tape, region and settings (which the
mesh parity tests pin to the oracle): the same vertex count and the same
triangle set, vertex positions bit for bit (vertex numbering follows the
order in which leaf records are appended, which the GPU does not fix),
whatever the number of workers and the order in which the meshes finish.  libfive_tree_save_meshes
(libfive.cpp:419-440) renders through the same path."""
import os
import struct

import pytest

from libfive_b200 import ffi, workloads
from libfive_b200.shape import Tape, render_meshes
from mesh_compare import same_mesh

pytestmark = pytest.mark.gpu

BOX = ((-1.5, -1.5, -1.5), (1.5, 1.5, 1.5))


def jobs_mixed():
    """Shapes of very different cost at different depths."""
    shapes = [
        (workloads.spheres_union(4, seed=1), 0.1),
        (workloads.random_csg(60, seed=5), 3 / 127.5),
        (workloads.spheres_union(16, seed=2), 3 / 63.5),
        (workloads.random_csg(200, seed=6), 3 / 255.5),
        (workloads.sphere((0.1, 0.2, -0.1), 0.7), 0.05),
        (workloads.random_csg(20, seed=7), 0.1),
    ]
    return [(Tape(s), BOX[0], BOX[1], mf) for s, mf in shapes]


def single(job):
    tape, lo, hi, mf = job
    return tape.render_mesh(lo, hi, mf)


@pytest.mark.parametrize("workers", [1, 2, 4])
def test_batch_matches_single_meshes(gpu, workers):
    jobs = jobs_mixed()
    want = [single(j) for j in jobs]
    got = render_meshes(jobs, workers=workers)
    assert len(got) == len(jobs)
    for (wv, wt), (gv, gt) in zip(want, got):
        assert len(wv) == len(gv) and same_mesh(wv, wt, gv, gt)


def test_batch_same_tape_many_times(gpu):
    # One tape shared by every job: the jobs only read it.
    tape = Tape(workloads.random_csg(100, seed=9))
    jobs = [(tape, BOX[0], BOX[1], 3 / 127.5)] * 8
    want = single(jobs[0])
    for v, t in render_meshes(jobs, workers=4):
        assert len(v) == len(want[0]) and same_mesh(v, t, *want)


def test_batch_stats(gpu):
    jobs = jobs_mixed()[:3]
    out = render_meshes(jobs, workers=3, stats=True)
    for (v, t, st), job in zip(out, jobs):
        assert st.triangles == len(t) and st.vertices == len(v) - 1
        assert st.ms_total > 0 and st.levels > 0


def test_batch_empty_and_errors(gpu):
    lib = ffi.load()
    assert lib.lfb_render_meshes(None, 0, None, None, 0, None, None) == 0
    n = 2
    keep = Tape(workloads.spheres_union(4, seed=1))   # alive for the call
    tapes = (ffi.tape_t * n)(keep.ptr, None)
    regions = (ffi.Region3 * n)()
    settings = (ffi.MeshSettings * n)()
    meshes = (ffi.ctypes.POINTER(ffi.Mesh) * n)()
    rc = lib.lfb_render_meshes(tapes, n, regions, settings, 0, meshes, None)
    assert rc != 0 and not meshes[0] and not meshes[1]
    assert "null tape" in ffi.last_error()[1]


def test_save_meshes_writes_every_tree(gpu, tmp_path):
    a, b = workloads.spheres_union(4, seed=1), workloads.random_csg(30, seed=3)
    path = str(tmp_path / "two.stl")
    assert _save_meshes([a, b], path, 10)
    want = sum(len(single((Tape(s), BOX[0], BOX[1], 0.1))[1]) for s in (a, b))
    with open(path, "rb") as f:
        data = f.read()
    assert struct.unpack("<I", data[80:84])[0] == want
    assert len(data) == 84 + 50 * want


def _save_meshes(shapes, path, res):
    lib = ffi.load()
    region = ffi.Region3(*[ffi.Interval(a, b) for a, b in zip(*BOX)])
    trees = (ffi.tree_t * (len(shapes) + 1))(*[s.ptr.value for s in shapes], None)
    return lib.libfive_tree_save_meshes(trees, region, res, 8, path.encode())
