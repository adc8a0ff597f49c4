"""Pins the CPU oracle to the reference's known answers (tests/golden/
eval_kats.json, restated from libfive/test/*.cpp) and to the reference's
procedural unit tests for ambiguity, point specialization and pushing."""
import json
import math
import os

import numpy as np
import pytest

from oracle_ffi import OracleTape
from sexpr import parse

KATS = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "eval_kats.json")))


def _f(v):
    return {"inf": math.inf, "-inf": -math.inf}.get(v, v) if isinstance(v, str) else v


def build(entry):
    vars_ = {}
    t = parse(entry["expr"], vars_)
    vals = {vars_[k]: v for k, v in entry.get("vars", {}).items()}
    return t, vals


def arr(*v):
    return [np.array([float(_f(a))], np.float32) for a in v]


@pytest.mark.parametrize("e", KATS["values"], ids=lambda e: e["src"])
def test_values(e):
    t, vals = build(e)
    o = OracleTape(t, vals)
    got = o.values(*arr(*e["p"]))[0]
    assert abs(got - e["want"]) <= e["tol"], (got, e)


@pytest.mark.parametrize("e", KATS["derivs"], ids=lambda e: e["src"])
def test_derivs(e):
    t, vals = build(e)
    o = OracleTape(t, vals)
    v, dx, dy, dz = o.derivs(*arr(*e["p"]))
    got = [dx[0], dy[0], dz[0], v[0]]
    for g, w in zip(got, e["want"]):
        w = _f(w)
        if math.isinf(w):
            assert math.isinf(g) and (g > 0) == (w > 0)
        else:
            assert abs(g - w) <= e["tol"], (got, e)


@pytest.mark.parametrize("e", KATS["intervals"], ids=lambda e: e["src"])
def test_intervals(e):
    t, vals = build(e)
    o = OracleTape(t, vals)
    lo = np.array([[_f(v)] for v in e["lo"]], np.float32)
    hi = np.array([[_f(v)] for v in e["hi"]], np.float32)
    l, h, _ = o.intervals(lo, hi)
    assert l[0] == _f(e["want"][0]) and h[0] == _f(e["want"][1]), (l, h, e)


@pytest.mark.parametrize("e", KATS["interval_nan"], ids=lambda e: e["src"])
def test_interval_nan_flags(e):
    t, vals = build(e)
    o = OracleTape(t, vals)
    lo = np.array([[_f(v)] for v in e["lo"]], np.float32)
    hi = np.array([[_f(v)] for v in e["hi"]], np.float32)
    _, _, n = o.intervals(lo, hi)
    assert (not n[0]) == e["safe"]


def test_ambiguous():
    # eval_array.cpp:198-216
    o = OracleTape(parse("(min x (- x))"))
    x = np.array([0, 1, 2, 0], np.float32)
    z = np.zeros(4, np.float32)
    assert o.ambiguous(x, z, z).tolist() == [True, False, False, True]


def test_push_shrinks_and_collapses():
    # eval_interval.cpp:64-85: pushing min(x+1, y+1) over a box where the
    # lhs always wins drops the rhs.
    t = parse("(min (+ x 1) (+ y 1))")
    o = OracleTape(t)
    full = len(o.st["clauses"])
    assert o.pushed_size((-5, 8, 0), (-4, 9, 0)) < full
    # eval_interval.cpp:86-98: both sides pick x, tape collapses to nothing
    t = parse("(min (min y x) (min x (+ y 3)))")
    o = OracleTape(t)
    assert o.pushed_size((-5, 0, 0), (-4, 1, 0)) == 0


def test_mod_interval_encloses_values():
    # eval_interval.cpp:128-168: mod enclosure fuzz
    t = parse("(mod x y)")
    o = OracleTape(t)
    ivs = [(a, b) for a in range(-5, 6) for b in range(-5, 6) if a <= b]
    for al, au in ivs[::3]:
        for bl, bu in ivs[::3]:
            lo = np.array([[al], [bl], [0]], np.float32)
            hi = np.array([[au], [bu], [0]], np.float32)
            l, h, n = o.intervals(lo, hi)
            if n[0]:
                continue
            c = np.arange(11, dtype=np.float32) / np.float32(10)
            a_ = np.float32(al) + c * (np.float32(au) - np.float32(al))
            b_ = np.float32(bl) + c * (np.float32(bu) - np.float32(bl))
            A, B = np.meshgrid(a_, b_)
            A = A.ravel().astype(np.float32)
            B = B.ravel().astype(np.float32)
            v = o.values(A, B, np.zeros_like(A))
            assert np.all(v >= l[0]) and np.all(v <= h[0]), (al, au, bl, bu)


def test_is_inside_and_features():
    # eval_feature.cpp:20-95 (isInside truth tables) and feature.cpp tests
    o = OracleTape(parse("(max x y)"))
    assert o.is_inside((-1, -1, 0))
    assert not o.is_inside((1, 0, 0))
    # On the corner of the quadrant: inside (both sides can be approached
    # from the negative side)
    assert o.is_inside((0, 0, 0))
    f = o.features((0, 0, 0))
    assert len(f) == 2
    o = OracleTape(parse("(min x y)"))
    # min(x, y) at the origin: a point of the boundary with an inside cone
    assert o.is_inside((0, 0, 0))


def test_jacobian_known():
    # eval_jacobian.cpp:19-61: gradient of (x * a + y * b) wrt a, b
    vars_ = {}
    t = parse("(+ (* x a) (* y b))", vars_)
    o = OracleTape(t, {vars_["a"]: 1.0, vars_["b"]: 2.0})
    j = o.jacobian(*arr(2, 3, 0))
    got = sorted(j[0].tolist())
    assert got == [2.0, 3.0]


@pytest.mark.parametrize("e", KATS["is_inside"], ids=lambda e: e["src"] + str(e["p"]))
def test_is_inside_kats(e):
    t, vals = build(e)
    assert OracleTape(t, vals).is_inside(tuple(e["p"])) == e["inside"]


@pytest.mark.parametrize("e", KATS["jacobian"], ids=lambda e: e["src"] + str(e["p"]))
def test_jacobian_kats(e):
    vars_ = {}
    t = parse(e["expr"], vars_)
    vals = {vars_[k]: v for k, v in e["vars"].items()}
    o = OracleTape(t, vals)
    j = o.jacobian(*arr(*e["p"]))[0]
    order = {vid: i for i, (_, vid) in enumerate(o.st["vars"])}
    for name, want in e["want"].items():
        assert abs(j[order[vars_[name].id()]] - want) <= e["tol"]
