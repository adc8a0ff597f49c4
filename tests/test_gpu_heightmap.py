"""Height maps on the GPU (lfb_render_heightmap, libfive_tree_render_pixels)
against the oracle's restatement of Heightmap::render, which
test_oracle_heightmap.py pins to the reference's own known answers.  Depths
are z sample values, so they must match exactly; normals are packed from
gradients at the same points and must match exactly as well."""
import json
import os

import numpy as np
import pytest

from libfive_b200 import ffi, workloads
from libfive_b200.shape import Shape, Tape, render_heightmap
from oracle_ffi import OracleTape, render_heightmap as oracle_heightmap, voxel_dims
from sexpr import parse

pytestmark = pytest.mark.gpu

KATS = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "heightmap_kats.json")))
X, Y, Z = Shape.X, Shape.Y, Shape.Z


def both(shape, lower, upper, res):
    got = render_heightmap(Tape(shape), lower, upper, res)
    want = oracle_heightmap(OracleTape(shape), lower, upper, res)
    return got, want


def assert_same(got, want):
    (gd, gn), (wd, wn) = got, want
    assert gd.shape == wd.shape
    assert np.array_equal(gd, wd), np.argwhere(gd != wd)[:8]
    bad = np.argwhere(gn != wn)
    assert len(bad) == 0, [(tuple(p), hex(gn[tuple(p)]), hex(wn[tuple(p)])) for p in bad[:8]]


@pytest.mark.parametrize("e", KATS["depth"] + KATS["normals"], ids=lambda e: e["src"])
def test_kat_regions(gpu, e):
    assert_same(*both(parse(e["expr"], {}), e["lower"], e["upper"], e["res"]))


@pytest.mark.parametrize("res", [8, 23, 40])
def test_spheres(gpu, res):
    s = workloads.spheres_union(24, seed=3)
    assert_same(*both(s, (-1.5, -1.5, -1.5), (1.5, 1.5, 1.5), res))


def test_csg_deep_z(gpu):
    # many slabs: the voxel rounds run top-down over 40 z slabs
    s = workloads.random_csg(80, seed=4)
    assert_same(*both(s, (-1.2, -1.0, -1.5), (1.0, 1.3, 1.5), (60, 50, 210)))


def test_thin_and_anisotropic(gpu):
    s = workloads.random_csg(40, seed=8)
    for lo, hi, res in (((-1, -1, 0.2), (1, 1, 0.2), 33),     # one z sample
                        ((-1, -0.1, -1), (1, 0.1, 1), 37),    # a few rows
                        ((0.3, -1, -1), (0.3, 1, 1), (0, 17, 29))):   # one column
        assert_same(*both(s, lo, hi, res))


def test_render_pixels_c_api(gpu):
    # libfive.cpp:442-465: pixels = finite depth of a one-sample-deep region
    lib = ffi.load()
    shape = workloads.spheres_union(24, seed=3)
    R2 = ffi.Region2(ffi.Interval(-1.5, 1.5), ffi.Interval(-1.2, 1.4))
    for z, res in ((0.1, 40.0), (-0.35, 17.5)):
        p = lib.libfive_tree_render_pixels(shape.ptr, R2, z, res)
        assert p
        w, h = p[0].width, p[0].height
        got = np.ctypeslib.as_array(p[0].pixels, shape=(h * w,)).reshape(h, w).copy()
        lib.libfive_pixels_delete(p)
        lo, hi = (-1.5, -1.2, z), (1.5, 1.4, z)
        assert (w, h, 1) == voxel_dims(lo, hi, res)
        depth, _ = oracle_heightmap(OracleTape(shape), lo, hi, res)
        assert np.array_equal(got, np.isfinite(depth))
        assert got.any() and not got.all()


def test_without_normals_and_sizes(gpu):
    tape = Tape(workloads.spheres_union(8, seed=5))
    d1, n1 = render_heightmap(tape, (-1, -1, -1), (1, 1, 1), 12)
    d2, n2 = render_heightmap(tape, (-1, -1, -1), (1, 1, 1), 12, normals=False)
    assert n2 is None and np.array_equal(d1, d2)
    assert d1.shape == (24, 24)
