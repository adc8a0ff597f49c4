"""Pins the oracle's restatement of Heightmap::render (and of the Voxels
sampling grid) to the reference's own known answers
(tests/golden/heightmap_kats.json, restated from libfive/test/heightmap.cpp)."""
import json
import math
import os

import numpy as np
import pytest

from oracle_ffi import OracleTape, render_heightmap, voxel_dims, voxel_pts
from sexpr import parse

KATS = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "heightmap_kats.json")))


def _f(v):
    return -math.inf if v == "-inf" else v


def tape(expr):
    return OracleTape(parse(expr, {}))


@pytest.mark.parametrize("e", KATS["depth"], ids=lambda e: e["src"])
def test_depth_kats(e):
    depth, _ = render_heightmap(tape(e["expr"]), e["lower"], e["upper"], e["res"])
    if "want" in e:
        want = np.array([[_f(v) for v in row] for row in e["want"]], np.float32)
        assert depth.shape == want.shape
        with np.errstate(invalid="ignore"):
            same = (depth == want) | (np.abs(depth - want) <= e["tol"])
        assert same.all(), depth
    else:
        ztop = voxel_pts(e["lower"], e["upper"], e["res"], 2)[-1]
        allowed = [ztop if a == "ztop" else _f(a) for a in e["allowed"]]
        assert np.isin(depth, np.array(allowed, np.float32)).all()
        assert np.isfinite(depth).any() and np.isinf(depth).any()


@pytest.mark.parametrize("e", KATS["shape"], ids=lambda e: e["src"])
def test_image_shape_kats(e):
    cols, rows, _ = voxel_dims(e["lower"], e["upper"], e["res"])
    assert (rows, cols) == (e["rows"], e["cols"])
    depth, _ = render_heightmap(tape(e["expr"]), e["lower"], e["upper"], e["res"])
    assert depth.shape == (e["rows"], e["cols"])


@pytest.mark.parametrize("e", KATS["normals"], ids=lambda e: e["src"])
def test_normal_kats(e):
    _, norm = render_heightmap(tape(e["expr"]), e["lower"], e["upper"], e["res"])
    assert np.isin(norm, np.array(e["allowed"], np.uint32)).all(), [hex(v) for v in np.unique(norm)]


def test_voxel_grid_expands_about_the_centre():
    # voxels.cpp:23-44: 2.5 units at 2 voxels per unit -> 5 voxels, bounds kept;
    # 2.2 units -> 5 voxels, bounds pushed out by 0.15 on each side
    for lo, hi, n in ((-1.25, 1.25, 5), (-1.1, 1.1, 5)):
        pts = voxel_pts((lo, 0, 0), (hi, 1, 1), (2, 2, 2), 0)
        assert len(pts) == n
        assert np.allclose(pts, np.linspace(-1.0, 1.0, n), atol=1e-6)
    # zero resolution: one sample at the middle
    assert voxel_dims((0, 0, -1), (1, 1, 1), (1, 1, 0))[2] == 1
    assert voxel_pts((0, 0, -1), (1, 1, 1), (1, 1, 0), 2)[0] == 0.0


def test_workers_do_not_change_the_image():
    t = tape("(- (sqrt (+ (+ (square (- x 0.1)) (square y)) (square (+ z 0.2)))) 0.8)")
    ref = render_heightmap(t, (-1, -1, -1), (1, 1, 1), 16, workers=1)
    for w in (2, 8):
        d, n = render_heightmap(t, (-1, -1, -1), (1, 1, 1), 16, workers=w)
        assert np.array_equal(d, ref[0]) and np.array_equal(n, ref[1])
