"""The oracle contourer (oracle/oracle_contours.cpp) against the reference's
own contour tests (libfive/test/contours.cpp:22-83, libfive/test/api.cpp:
75-105), the quadtree tables against libfive/test/marching.cpp:16-27 and
dc_tree2.cpp:17-19, the 2x2 QEF solve against numpy's FP64 eigh, and the
welding rule of Contours::collect (contours.cpp:118-184).  CPU only."""
import ctypes

import numpy as np
import pytest

import oracle_ffi
from mesh_compare import same_contours
from oracle_ffi import OracleTape
from shapes2d import circle, menger, rectangle
from libfive_b200.shape import Shape

X, Y = Shape.X, Shape.Y


def contours(shape, lo, hi, z=0.0, min_feature=0.1, max_err=1e-8):
    return oracle_ffi.render_contours(OracleTape(shape), lo, hi, z, min_feature, max_err)[0]


def closed(c):
    return len(c) > 2 and np.array_equal(c[0], c[-1])


def test_circle_welds_into_one_contour():
    # contours.cpp:22-30 and :32-51 (accuracy)
    cs = contours(circle(0.5), (-1, -1), (1, 1))
    assert len(cs) == 1 and closed(cs[0])
    r = np.linalg.norm(cs[0], axis=1)
    assert r.max() < 0.51 and r.min() > 0.49


def test_contour_with_ambiguities():
    # contours.cpp:53-63: a square whose left side is cut by -x exactly
    t = (-X()).max(X() - 1).max((-Y()).max(Y() - 1)).max(-X())
    cs = contours(t, (-2, -2), (2, 2))
    assert len(cs) == 1 and closed(cs[0])


@pytest.mark.parametrize("sign", [1, -1])
def test_adjacent_rectangles(sign):
    # contours.cpp:65-75
    rects = rectangle(-1, 0, -1, 1).min(rectangle(0, 1, -1, 1))
    cs = contours(rects if sign > 0 else -rects, (-2, -2), (2, 2))
    assert len(cs) == 1


def test_menger_slice_with_perp_offset():
    # contours.cpp:77-83: 74 contours at z = 1.49
    cs = contours(menger(2), (-2.5, -2.5), (2.5, 2.5), z=1.49)
    assert len(cs) == 74


def test_slice_of_unit_circle_through_the_c_api_settings():
    # api.cpp:75-105: x^2 + y^2 - 1 over [-2, 2]^2 at z = 0, 10 per unit
    d = X().square() + Y().square() - 1.0
    cs = contours(d, (-2, -2), (2, 2), min_feature=float(np.float32(1) / np.float32(10)))
    assert len(cs) == 1
    r2 = (cs[0].astype(np.float64) ** 2).sum(axis=1)
    assert r2.min() > 0.99 and r2.max() < 1.01


def test_contours_are_deterministic():
    t = circle(0.3, (0.2, -0.1)).min(rectangle(-0.9, -0.2, -0.5, 0.6))
    a = contours(t, (-1, -1), (1, 1), min_feature=0.02)
    b = contours(t, (-1, -1), (1, 1), min_feature=0.02)
    assert same_contours(a, b)


def test_quadtree_tables():
    v, e, p, manifold, npatch, nedge = oracle_ffi.dc_tables2()
    # marching.cpp:16-27: every mixed mask has a patch, 0 and 15 none
    for m in range(1, 15):
        assert v[m, 0, 0, 0] != -1, m
    assert v[0, 0, 0, 0] == -1 and v[15, 0, 0, 0] == -1
    # dc_tree2.cpp:17-19
    assert manifold.tolist() == [1, 1, 1, 1, 1, 1, 0, 1, 1, 0, 1, 1, 1, 1, 1, 1]
    # every directed edge between two corners that differ in one axis has
    # an id, the eight ids are distinct
    ids = [int(e[a, b]) for a in range(4) for b in range(4)
           if bin(a ^ b).count("1") == 1]
    assert sorted(ids) == list(range(8))
    # each patch edge runs from a filled to an empty corner of its mask
    for m in range(16):
        for q in range(npatch[m]):
            for k in range(nedge[m, q]):
                a, b = v[m, q, k]
                assert (m >> a) & 1 and not (m >> b) & 1
                assert p[m, e[a, b]] == q


def _qef2_lib():
    lib = oracle_ffi.load()
    lib.ora_qef2_vertex.restype = ctypes.c_double
    lib.ora_qef2_vertex.argtypes = [ctypes.c_void_p] * 3
    return lib


@pytest.mark.parametrize("seed", range(5))
def test_qef2_against_fp64_eigh(seed):
    """The 2x2 solve: rank decision and vertex against numpy's eigh (the
    same pseudo-inverse in FP64, eigenvalue cutoff 0.1)."""
    rng = np.random.default_rng(seed)
    lib = _qef2_lib()
    for _ in range(200):
        kind = rng.integers(4)
        if kind == 0:       # one normal: rank 1
            n = rng.normal(size=(1, 2))
        elif kind == 1:     # two close normals: near the cutoff
            a = rng.normal(size=2)
            n = np.stack([a, a + rng.normal(scale=0.2, size=2)])
        elif kind == 2:     # repeated normal
            a = rng.normal(size=2)
            n = np.stack([a, a, a])
        else:
            n = rng.normal(size=(4, 2))
        n /= np.linalg.norm(n, axis=1, keepdims=True)
        pts = rng.uniform(-1, 1, size=(len(n), 2))
        A = n.T @ n
        b = (n * pts).sum(axis=1)
        AtB = n.T @ b
        mass = np.array([pts[:, 0].sum(), pts[:, 1].sum(), len(n)])
        q = np.array([A[0, 0], A[0, 1], A[1, 1], AtB[0], AtB[1], (b * b).sum(), *mass])
        v = np.zeros(2)
        rank = ctypes.c_int()
        err = lib.ora_qef2_vertex(q.ctypes.data, v.ctypes.data, ctypes.addressof(rank))
        w, U = np.linalg.eigh(A)
        D = np.where(np.abs(w) < 0.1, 0.0, 1.0 / np.where(w == 0, 1, w))
        assert rank.value == int((np.abs(w) >= 0.1).sum())
        center = mass[:2] / mass[2]
        want = (U @ np.diag(D) @ U.T) @ (AtB - A @ center) + center
        np.testing.assert_allclose(v, want, rtol=1e-9, atol=1e-9)
        want_err = want @ A @ want - 2 * want @ AtB + (b * b).sum()
        assert abs(err - want_err) <= 1e-9 * max(1.0, abs(want_err))


def test_weld_closes_a_loop_in_any_segment_order():
    loop = [(1, 2), (2, 3), (3, 4), (4, 5), (5, 1)]
    rng = np.random.default_rng(0)
    for _ in range(20):
        order = rng.permutation(len(loop))
        w = oracle_ffi.weld([loop[i] for i in order])
        assert len(w) == 1
        c = w[0]
        assert c[0] == c[-1] and sorted(c[:-1]) == [1, 2, 3, 4, 5]
        # segment direction is kept: each id is followed by its successor
        succ = dict(loop)
        assert all(succ[a] == b for a, b in zip(c, c[1:]))
