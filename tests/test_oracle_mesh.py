"""The oracle mesher (oracle/oracle_dc.cpp, the CPU restatement of the
reference's DC pipeline) against the reference's own mesh known answers,
on the CPU: the GPU meshes are compared with this mesher, so it is pinned
here first (libfive/test/mesh.cpp, libfive/test/api.cpp)."""
import numpy as np

from libfive_b200 import workloads
from libfive_b200.shape import X, Y, Z
from mesh_compare import edge_pairs_ok, oracle_mesh
from oracle_ffi import OracleTape


def _mesh(shape, lo, hi, min_feature, max_err=1e-8):
    return oracle_mesh(OracleTape(shape), lo, hi, min_feature, max_err, threads=4)


def _box(lo, hi):
    x, y, z = X(), Y(), Z()
    return ((lo[0] - x).max(x - hi[0]).max((lo[1] - y).max(y - hi[1]))).max(
        (lo[2] - z).max(z - hi[2]))


def test_cube_face_count():
    # mesh.cpp:70-88: 12 triangles, 9 vertices (index 0 unused)
    v, t = _mesh(_box((-1.5,) * 3, (1.5,) * 3), (-3,) * 3, (3,) * 3, 0.15)
    assert len(t) == 12 and len(v) == 9


def test_prism_face_count():
    # mesh.cpp:90-102
    x, y, z = X(), Y(), Z()
    s = (-x).max(x - 4).max((-y).max(y - 1)).max((-z).max(z - 0.25))
    v, t = _mesh(s, (-1, -1, -1), (5, 2, 1.25), 0.125)
    assert len(v) == 9 and len(t) == 12


def test_sphere_normals_point_outwards():
    # mesh.cpp:25-54: every normal within 0.9 (cosine) of the radial direction
    v, t = _mesh(workloads.sphere((0, 0, 0), 0.5), (-1,) * 3, (1,) * 3, 0.2)
    tri = v[t.astype(np.int64)].astype(np.float64)
    n = np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0])
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    c = tri.sum(axis=1)
    c /= np.linalg.norm(c, axis=1, keepdims=True)
    assert len(t) > 0 and np.min(np.sum(n * c, axis=1)) > 0.9


def test_api_sphere_radii():
    # api.cpp:107-146: x^2 + y^2 + z^2 - 1 over [-2, 2]^3 at 10 per unit:
    # every vertex of every triangle has r^2 in (0.99, 1.01)
    x, y, z = X(), Y(), Z()
    v, t = _mesh(x.square() + y.square() + z.square() - 1.0, (-2,) * 3, (2,) * 3, 0.1)
    r2 = np.sum(v[t.ravel().astype(np.int64)].astype(np.float64) ** 2, axis=1)
    assert len(t) > 0 and r2.min() > 0.99 and r2.max() < 1.01


def _sphere_box():
    return workloads.sphere((0, 0, 0.1), 0.7).min(_box((-1, -1, -1), (1, 1, 0.1)))


def test_no_line_triangles_and_no_flipped_top_face():
    # mesh.cpp:137-189: no triangle repeats a vertex; triangles on the top
    # face (z = 0.1) face +z
    v, t = _mesh(_sphere_box(), (-10,) * 3, (10,) * 3, 0.25)
    assert len(t) > 0
    assert np.all((t[:, 0] != t[:, 1]) & (t[:, 0] != t[:, 2]) & (t[:, 1] != t[:, 2]))
    tri = v[t.astype(np.int64)].astype(np.float64)
    top = np.all(np.abs(tri[:, :, 2] - 0.1) < 1e-3, axis=1)
    n = np.cross(tri[top, 1] - tri[top, 0], tri[top, 2] - tri[top, 0])
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    assert top.any()
    assert np.all(np.abs(n[:, 0]) < 0.01) and np.all(np.abs(n[:, 1]) < 0.01)
    assert np.all(np.abs(n[:, 2] - 1.0) < 0.01)


def test_edges_pair_up():
    # util/mesh_checks.cpp:4-35 (CHECK_EDGE_PAIRS) on a sphere union and a
    # small random CSG
    for shape, mf in ((workloads.spheres_union(8, seed=3), 0.1),
                      (workloads.random_csg(30, seed=6), 0.05)):
        _, t = _mesh(shape, (-1.5,) * 3, (1.5,) * 3, mf)
        assert len(t) > 0 and edge_pairs_ok(t)


def test_region_levels():
    # region.cpp:160-167: Region<3>({-1,-1,-1}, {1,1,1}).withResolution(r).level
    import ctypes

    import oracle_ffi
    lib = oracle_ffi.load()
    ora = OracleTape(workloads.sphere((0, 0, 0), 0.5))
    for res, level in ((5, 0), (1, 1), (1.2, 1), (0.9, 2)):
        vp, tp = ctypes.c_void_p(), ctypes.c_void_p()
        nv, nt = ctypes.c_uint32(), ctypes.c_uint32()
        got = lib.ora_render_mesh(ora.h, -1, -1, -1, 1, 1, 1, res, 1e-8, 1, ctypes.byref(vp),
                                  ctypes.byref(nv), ctypes.byref(tp), ctypes.byref(nt))
        lib.ora_free(vp)
        lib.ora_free(tp)
        assert got == level


def test_threaded_mesher_matches_serial():
    """The oracle's task pools (octree build and dual walk on several
    threads) give the serial mesher's triangle set."""
    from libfive_b200 import workloads
    from mesh_compare import oracle_mesh, same_mesh
    from oracle_ffi import OracleTape
    s = workloads.random_csg(300, seed=4)
    o = OracleTape(s)
    v1, t1 = oracle_mesh(o, (-1.5, -1.5, -1.5), (1.5, 1.5, 1.5), 0.02, threads=1)
    v8, t8 = oracle_mesh(o, (-1.5, -1.5, -1.5), (1.5, 1.5, 1.5), 0.02, threads=8)
    assert len(t1) > 1000
    assert len(v1) == len(v8)
    assert same_mesh(v1, t1, v8, t8)
