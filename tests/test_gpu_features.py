"""The device feature evaluator (the mesher's path at samples whose value is
exactly zero) through lfb_eval_features, against the reference's isInside
truth tables (libfive/test/eval_feature.cpp:20-95, restated in
tests/golden/eval_kats.json) and the CPU oracle's FeatureEvaluator."""
import json
import os

import numpy as np
import pytest

from libfive_b200 import workloads
from libfive_b200.shape import Shape, Tape
from oracle_ffi import OracleTape
from sexpr import parse

pytestmark = pytest.mark.gpu

KATS = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "eval_kats.json")))


def _build(e):
    vars_ = {}
    t = parse(e["expr"], vars_)
    return t, {vars_[k]: v for k, v in e.get("vars", {}).items()}


@pytest.mark.parametrize("e", KATS["is_inside"], ids=lambda e: e["src"] + str(e["p"]))
def test_is_inside_kats_on_device(gpu, e):
    t, vals = _build(e)
    p = [np.array([v], np.float32) for v in e["p"]]
    inside, _ = Tape(t, vals).features(*p, lists=False)
    assert bool(inside[0]) == e["inside"]


def _zero_points(n, seed):
    """Lattice points of step 1/4 (many exact zeros and ties for shapes
    built from planes and boxes with quarter-integer sizes)."""
    r = np.random.default_rng(seed)
    p = r.integers(-6, 7, (3, n)).astype(np.float32) / 4
    return [np.ascontiguousarray(a) for a in p]


SHAPES = {
    "max_xy": "(max x y)",
    "min_xy": "(min x y)",
    "box": "(max (max (- (abs x) 1) (- (abs y) 1)) (- (abs z) 1))",
    "cross": "(min (max (- (abs x) 0.5) (- (abs y) 1.5)) (max (- (abs x) 1.5) (- (abs y) 0.5)))",
    "diff": "(max (- (abs x) 1) (- 0.5 (abs y)))",
    "planes": "(max (min (- x y) (+ x y)) (- z 0.25))",
}


@pytest.mark.parametrize("name", sorted(SHAPES))
def test_features_match_oracle(gpu, name):
    t = parse(SHAPES[name], {})
    P = _zero_points(600, seed=len(name))
    inside, feats = Tape(t).features(*P)
    o = OracleTape(t)
    for i in range(len(P[0])):
        q = (P[0][i], P[1][i], P[2][i])
        assert bool(inside[i]) == o.is_inside(q), (name, q)
        of = o.features(q)
        assert len(feats[i]) == len(of), (name, q)
        assert np.array_equal(np.sort(feats[i], axis=0), np.sort(of, axis=0)), (name, q)


def test_features_on_csg_zeros(gpu):
    """Exact zeros of a box CSG at cell corners, where the mesher calls the
    feature evaluator."""
    a = workloads.box((0.25, 0.0, 0.0), 0.5)
    b = workloads.box((-0.25, 0.25, 0.0), 0.75)
    c = workloads.sphere((0.0, 0.0, 0.5), 0.5)
    t = workloads.difference(workloads.union(a, b), c)
    P = _zero_points(1500, seed=3)
    inside, feats = Tape(t).features(*P)
    o = OracleTape(t)
    zeros = 0
    for i in range(len(P[0])):
        q = (P[0][i], P[1][i], P[2][i])
        assert bool(inside[i]) == o.is_inside(q), q
        assert len(feats[i]) == len(o.features(q)), q
    v = o.values(*P)
    zeros = int((v == 0).sum())
    assert zeros > 50
