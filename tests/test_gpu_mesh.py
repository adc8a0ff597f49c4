"""GPU dual contouring through the C ABI against the CPU oracle mesher and
the reference's mesh tests (libfive/test/mesh.cpp, api.cpp, xtree.cpp)."""
import ctypes
import os

import numpy as np
import pytest

from libfive_b200 import ffi, workloads
from libfive_b200.shape import Shape, Tape, mesh_arrays
from mesh_compare import edge_pairs_ok, hausdorff, oracle_mesh, same_mesh
from oracle_ffi import OracleTape
from sexpr import parse

pytestmark = pytest.mark.gpu

X, Y, Z = Shape.X, Shape.Y, Shape.Z


def gpu_and_oracle(shape, lo, hi, min_feature, max_err=1e-8):
    v, t = Tape(shape).render_mesh(lo, hi, min_feature, max_err)
    ov, ot = oracle_mesh(OracleTape(shape), lo, hi, min_feature, max_err)
    return v, t, ov, ot


@pytest.mark.parametrize("res", [0.5, 0.2, 0.1, 0.05])
def test_sphere_union_matches_oracle(gpu, res):
    s = workloads.spheres_union(16, seed=1)
    v, t, ov, ot = gpu_and_oracle(s, (-1.5, -1.5, -1.5), (1.5, 1.5, 1.5), res)
    assert len(t) > 0
    assert same_mesh(v, t, ov, ot)
    assert len(v) == len(ov)
    assert edge_pairs_ok(t)


def test_single_leaf_root(gpu):
    # Region already below min_feature: the root is evaluated as a leaf.
    s = workloads.sphere((0.1, 0.05, 0.0), 0.5)
    v, t, ov, ot = gpu_and_oracle(s, (-1, -1, -1), (1, 1, 1), 4.0)
    assert same_mesh(v, t, ov, ot)


def test_no_collapse_matches_oracle(gpu):
    s = workloads.spheres_union(8, seed=4)
    v, t, ov, ot = gpu_and_oracle(s, (-1.5, -1.5, -1.5), (1.5, 1.5, 1.5), 0.1, -1.0)
    assert same_mesh(v, t, ov, ot)


def test_random_csg_exact_ops_matches_oracle(gpu, monkeypatch):
    """Union / intersection / difference only: bit-identical mesh."""
    monkeypatch.setattr(workloads, "CSG_WEIGHTS", (0.7, 0.0, 0.2, 0.1))
    s = workloads.random_csg(60, seed=11, size=(0.1, 0.4))
    v, t, ov, ot = gpu_and_oracle(s, (-1.5, -1.5, -1.5), (1.5, 1.5, 1.5), 0.05)
    assert same_mesh(v, t, ov, ot)
    assert edge_pairs_ok(t)


@pytest.mark.parametrize("n,res", [(60, 0.05), (60, 0.2), (8, 0.1)])
def test_random_csg_with_blends_within_tolerance(gpu, n, res):
    """exp / log blends: CUDA's and the C library's expf / logf differ by a
    few ULPs, so vertices may move by that much; the bar is a bbox-relative
    Hausdorff distance of 1e-4 and the same triangle count."""
    s = workloads.random_csg(n, seed=11, size=(0.1, 0.4))
    v, t, ov, ot = gpu_and_oracle(s, (-1.5, -1.5, -1.5), (1.5, 1.5, 1.5), res)
    assert len(t) == len(ot) and len(v) == len(ov)
    assert hausdorff(v, t, ov, ot) <= 1e-4 * 3.0


def test_api_render_mesh_sphere_radii(gpu, lib):
    # api.cpp:107-146: unit sphere, all vertices of all triangles at r^2 in (0.99, 1.01)
    s = X().square() + Y().square() + Z().square() - 1
    m = s.render_mesh((-2, -2, -2), (2, 2, 2), 10)
    v, t = mesh_arrays(m)
    r2 = (v[t.ravel()] ** 2).sum(axis=1)
    assert r2.min() > 0.99 and r2.max() < 1.01


def test_sphere_normals(gpu):
    # mesh.cpp:25-54
    s = workloads.sphere((0, 0, 0), 0.5)
    v, t = Tape(s).render_mesh((-1, -1, -1), (1, 1, 1), 0.2)
    a, b, c = v[t[:, 0]], v[t[:, 1]], v[t[:, 2]]
    n = np.cross(b - a, c - a)
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    ctr = a + b + c
    ctr /= np.linalg.norm(ctr, axis=1, keepdims=True)
    assert (n * ctr).sum(axis=1).min() > 0.9


def test_edge_pairing_coarse(gpu):
    # mesh.cpp:307-317
    s = workloads.sphere((0, 0, 0), 0.5)
    v, t = Tape(s).render_mesh((-1, -1, -1), (1, 1, 1), 1.1)
    assert edge_pairs_ok(t)


STL_RECORD = np.dtype([("normal", "<f4", 3), ("v", "<f4", (3, 3)), ("attr", "<u2")])


def read_stl(path):
    """Binary STL (mesh.cpp:139-194): 80-byte header, uint32 count, 50-byte
    records.  Returns (header, records)."""
    data = open(path, "rb").read()
    n = int.from_bytes(data[80:84], "little")
    assert len(data) == 84 + 50 * n
    return data[:80], np.frombuffer(data, STL_RECORD, count=n, offset=84)


def stl_matches_mesh(recs, v, t):
    """The records are the mesh's triangles (in any order), with zero
    normals and attributes."""
    assert not recs["normal"].any() and not recs["attr"].any()
    flat = recs["v"].reshape(-1, 3)
    idx = np.arange(len(flat), dtype=np.uint32).reshape(-1, 3)
    return same_mesh(flat, idx, v, t)


@pytest.mark.parametrize("res", [10.0, 300.0])
def test_save_mesh_stl(gpu, lib, tmp_path, res):
    # the records are packed on the device and streamed to the file in
    # chunks of 2^20 triangles: res 300 (depth 10) writes two chunks
    s = workloads.sphere((0, 0, 0), 0.5)
    path = str(tmp_path / "out.stl")
    r = ffi.Region3(ffi.Interval(-1, 1), ffi.Interval(-1, 1), ffi.Interval(-1, 1))
    assert lib.libfive_tree_save_mesh(s.ptr, r, res, path.encode())
    header, recs = read_stl(path)
    assert header.startswith(b"This is a binary STL exported from libfive.")
    assert header.endswith(b" ")
    v, t = mesh_arrays(lib.libfive_tree_render_mesh(s.ptr, r, res))
    assert len(recs) == len(t) > 0
    if res > 100:
        assert len(t) > (1 << 20)
    assert stl_matches_mesh(recs, v, t)


def test_save_mesh_stl_empty_region(gpu, lib, tmp_path):
    # no surface in the region: header and a zero count
    s = workloads.sphere((5, 5, 5), 0.5)
    path = str(tmp_path / "empty.stl")
    r = ffi.Region3(ffi.Interval(-1, 1), ffi.Interval(-1, 1), ffi.Interval(-1, 1))
    assert lib.libfive_tree_save_mesh(s.ptr, r, 10.0, path.encode())
    _, recs = read_stl(path)
    assert len(recs) == 0


def test_save_mesh_unwritable_path(gpu, lib, tmp_path):
    s = workloads.sphere((0, 0, 0), 0.5)
    path = str(tmp_path / "no_such_dir" / "out.stl")
    r = ffi.Region3(ffi.Interval(-1, 1), ffi.Interval(-1, 1), ffi.Interval(-1, 1))
    assert not lib.libfive_tree_save_mesh(s.ptr, r, 10.0, path.encode())


def _cube(h=1.5):
    x, y, z = X(), Y(), Z()
    return (-(x + h)).max(x - h).max((-(y + h)).max(y - h)).max((-(z + h)).max(z - h))


def _box(lo, hi):
    x, y, z = X(), Y(), Z()
    return ((lo[0] - x).max(x - hi[0]).max((lo[1] - y).max(y - hi[1]))).max(
        (lo[2] - z).max(z - hi[2]))


def test_cube_face_count(gpu):
    # mesh.cpp:70-88: corners exactly on the surface and on cube edges
    # (isInside / features path); collapses to 12 triangles, 9 vertices.
    v, t, ov, ot = gpu_and_oracle(_cube(), (-3, -3, -3), (3, 3, 3), 0.15)
    assert same_mesh(v, t, ov, ot)
    assert len(t) == 12 and len(v) == 9


def test_prism_face_count(gpu):
    # mesh.cpp:90-102
    x, y, z = X(), Y(), Z()
    t_ = (-x).max(x - 4).max((-y).max(y - 1)).max((-z).max(z - 0.25))
    v, t, ov, ot = gpu_and_oracle(t_, (-1, -1, -1), (5, 2, 1.25), 0.125)
    assert same_mesh(v, t, ov, ot)
    assert len(v) == 9 and len(t) == 12


def _sphere_box():
    return workloads.sphere((0, 0, 0.1), 0.7).min(_box((-1, -1, -1), (1, 1, 0.1)))


def test_no_line_triangles(gpu):
    # mesh.cpp:136-152
    v, t, ov, ot = gpu_and_oracle(_sphere_box(), (-10, -10, -10), (10, 10, 10), 0.25)
    assert same_mesh(v, t, ov, ot)
    assert np.all(t[:, 0] != t[:, 1]) and np.all(t[:, 1] != t[:, 2]) and np.all(t[:, 0] != t[:, 2])


def test_no_flipped_triangles(gpu):
    # mesh.cpp:154-189
    v, t = Tape(_sphere_box()).render_mesh((-10, -10, -10), (10, 10, 10), 0.25)
    P = v[t]
    top = np.all(np.abs(P[:, :, 2] - 0.1) < 1e-3, axis=1)
    n = np.cross(P[:, 1] - P[:, 0], P[:, 2] - P[:, 0])
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    assert top.any()
    assert np.allclose(n[top], [0, 0, 1], atol=0.01)


def test_cone_renders(gpu):
    # mesh.cpp:118-128
    x, y, z = X(), Y(), Z()
    s = 1 / (-z)
    radius = ((x * s).square() + (y * s).square()).sqrt()
    cone = (radius - 1).max(z.max(-1 - z))
    v, t, ov, ot = gpu_and_oracle(cone, (-10, -10, -10), (10, 10, 10), 0.1)
    assert same_mesh(v, t, ov, ot)


def test_render_mesh_coords_matches_render_mesh(gpu, lib):
    """libfive_tree_render_mesh_coords (libfive.cpp:354-395): the mesh's
    vertices and, per triangle, its three vertex indices then -1."""
    s = workloads.spheres_union(8, seed=2)
    R = ffi.Region3(*[ffi.Interval(-1.5, 1.5)] * 3)
    m = lib.libfive_tree_render_mesh(s.ptr, R, 10.0)
    v, t = mesh_arrays(m)
    mc = lib.libfive_tree_render_mesh_coords(s.ptr, R, 10.0)
    assert mc
    c = mc[0]
    cv = np.ctypeslib.as_array(ctypes.cast(c.verts, ctypes.POINTER(ctypes.c_float)),
                               shape=(c.vert_count * 3,)).reshape(-1, 3).copy()
    ci = np.ctypeslib.as_array(c.coord_indices, shape=(c.coord_index_count,)).copy()
    n_idx = c.coord_index_count
    lib.libfive_mesh_coords_delete(mc)
    assert n_idx == 4 * len(t) > 0
    ci = ci.reshape(-1, 4)
    assert np.all(ci[:, 3] == -1)
    # the same mesh (vertex order may differ between two renders)
    assert same_mesh(cv, ci[:, :3].astype(np.uint32), v, t)
