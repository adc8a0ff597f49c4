"""2D contours on the GPU (contours.cu: libfive_tree_render_slice /
render_slice3 / save_slice, lfb_render_slice) against the oracle contourer,
itself pinned to the reference's contour tests (test_oracle_contours.py):
the same contours, point for point (as cyclic sequences: the order in
which segments are welded differs between runs, in the reference's
threaded walk as here), and the reference's known answers
(libfive/test/contours.cpp:22-83, libfive/test/api.cpp:75-105)."""
import numpy as np
import pytest

import oracle_ffi
from libfive_b200 import ffi, workloads
from libfive_b200.shape import Shape, Tape, contour_arrays, render_slice
from mesh_compare import same_contours
from oracle_ffi import OracleTape
from shapes2d import circle, menger, rectangle

pytestmark = pytest.mark.gpu

X, Y, Z = Shape.X, Shape.Y, Shape.Z


def gpu_slice(shape, lo, hi, z=0.0, min_feature=0.1, max_err=1e-8):
    return render_slice(Tape(shape), lo, hi, z, min_feature, max_err)


def ora(shape, lo, hi, z=0.0, min_feature=0.1, max_err=1e-8):
    return oracle_ffi.render_contours(OracleTape(shape), lo, hi, z, min_feature, max_err)[0]


def closed(c):
    return len(c) > 2 and np.array_equal(c[0], c[-1])


def test_circle(gpu):
    # contours.cpp:22-51
    cs = gpu_slice(circle(0.5), (-1, -1), (1, 1))
    assert len(cs) == 1 and closed(cs[0])
    r = np.linalg.norm(cs[0], axis=1)
    assert r.max() < 0.51 and r.min() > 0.49


def test_with_ambiguities(gpu):
    # contours.cpp:53-63
    t = (-X()).max(X() - 1).max((-Y()).max(Y() - 1)).max(-X())
    cs = gpu_slice(t, (-2, -2), (2, 2))
    assert len(cs) == 1 and closed(cs[0])


@pytest.mark.parametrize("sign", [1, -1])
def test_adjacent_rectangles(gpu, sign):
    # contours.cpp:65-75
    rects = rectangle(-1, 0, -1, 1).min(rectangle(0, 1, -1, 1))
    assert len(gpu_slice(rects if sign > 0 else -rects, (-2, -2), (2, 2))) == 1


def test_menger_perp_offset(gpu):
    # contours.cpp:77-83
    assert len(gpu_slice(menger(2), (-2.5, -2.5), (2.5, 2.5), z=1.49)) == 74


def test_c_api_slice(gpu, lib):
    # api.cpp:75-105 through libfive_tree_render_slice
    d = X().square() + Y().square() - 1.0
    R = ffi.Region2(ffi.Interval(-2, 2), ffi.Interval(-2, 2))
    cs = contour_arrays(lib.libfive_tree_render_slice(d.ptr, R, 0.0, 10.0))
    assert len(cs) == 1 and len(cs[0]) > 0
    r2 = (cs[0].astype(np.float64) ** 2).sum(axis=1)
    assert r2.min() > 0.99 and r2.max() < 1.01
    # the oracle, with the C API's settings (min_feature = 1 / res in float)
    want = ora(d, (-2, -2), (2, 2), min_feature=float(np.float32(1) / np.float32(10)))
    assert same_contours(cs, want)


def test_slice3_carries_z(gpu, lib):
    s = workloads.sphere((0.1, -0.2, 0.3), 0.8)
    R = ffi.Region2(ffi.Interval(-1, 1), ffi.Interval(-1, 1))
    c2 = contour_arrays(lib.libfive_tree_render_slice(s.ptr, R, 0.25, 20.0))
    c3 = contour_arrays(lib.libfive_tree_render_slice3(s.ptr, R, 0.25, 20.0), dim=3)
    assert len(c2) == len(c3) >= 1
    # two renders: the same contours, each possibly starting elsewhere
    assert same_contours([b[:, :2] for b in c3], c2)
    for b in c3:
        assert np.all(b[:, 2] == np.float32(0.25))


def _shapes():
    out = {
        "circle": (circle(0.6, (0.1, -0.05)), (-1, -1), (1, 1), 0.0, 0.02),
        "rects": (rectangle(-0.8, 0.1, -0.5, 0.7).min(rectangle(-0.2, 0.9, -0.9, 0.2)),
                  (-1, -1), (1, 1), 0.0, 0.03),
        "menger1": (menger(1), (-2, -2), (2, 2), 0.7, 0.05),
        "menger2_z": (menger(2), (-2.5, -2.5), (2.5, 2.5), 1.49, 0.1),
    }
    # slices of 3D shapes
    out["spheres"] = (workloads.spheres_union(24, seed=3), (-1.5, -1.5), (1.5, 1.5), 0.2, 0.02)
    out["csg"] = (workloads.random_csg(80, seed=4), (-1.5, -1.5), (1.5, 1.5), -0.1, 0.01)
    return out


@pytest.mark.parametrize("name", ["circle", "rects", "menger1", "menger2_z", "spheres", "csg"])
def test_matches_oracle(gpu, name):
    shape, lo, hi, z, mf = _shapes()[name]
    got = gpu_slice(shape, lo, hi, z, mf)
    want = ora(shape, lo, hi, z, mf)
    assert len(got) == len(want)
    assert same_contours(got, want)


def test_collapse_matches_oracle(gpu):
    # a coarse max_err so that cells collapse: the collapsed cells' vertices
    # (leaf level > 0) must agree as well
    shape = rectangle(-0.7, 0.6, -0.55, 0.45)
    got = gpu_slice(shape, (-1, -1), (1, 1), 0.0, 0.01, max_err=1e-3)
    want = ora(shape, (-1, -1), (1, 1), 0.0, 0.01, max_err=1e-3)
    assert same_contours(got, want)
    # the square's contour collapses to few points
    assert len(got) == 1 and len(got[0]) < 40


def test_empty_slice(gpu):
    assert gpu_slice(circle(0.2, (5, 5)), (-1, -1), (1, 1)) == []


def test_save_slice_svg(gpu, lib, tmp_path):
    # Contours::saveSVG (contours.cpp:51-116)
    shape = circle(0.5).min(circle(0.2, (0.8, 0.8)))
    R = ffi.Region2(ffi.Interval(-1, 1.5), ffi.Interval(-1, 1.5))
    path = str(tmp_path / "slice.svg")
    lib.libfive_tree_save_slice(shape.ptr, R, 0.0, 20.0, path.encode())
    text = open(path).read()
    assert text.startswith('<?xml version="1.0" encoding="UTF-8" standalone="no"?>\n'
                           '<svg xmlns="http://www.w3.org/2000/svg" version="1.1"\n'
                           ' width="2.5" height="2.5" id="libfive">\n')
    assert text.endswith("\n</svg>")
    cs = contour_arrays(lib.libfive_tree_render_slice(shape.ptr, R, 0.0, 20.0))
    assert text.count("<path d=") == len(cs) == 2
    assert text.count("Z\"") == sum(closed(c) for c in cs)
    # every contour's points, y flipped into the box, in the stream's %g
    # format (the two renders may start a closed contour at different points)
    paths = [p.split('"')[0].split() for p in text.split('<path d="')[1:]]
    got = sorted(sorted((float(p[k + 1]), float(p[k + 2])) for k in range(0, len(p) - 1, 3)
                        if p[k] in "ML") for p in paths)
    want = sorted(sorted((float("%g" % (float(x) + 1.0)), float("%g" % (1.5 - float(y))))
                         for x, y in (c[:-1] if closed(c) else c)) for c in cs)
    assert got == want
