"""Host-side tree construction, optimizer and tape layout, pinned by the
reference's own known answers (libfive/test/tree.cpp, deck.cpp, api.cpp)."""
import ctypes

import pytest

from libfive_b200.shape import Shape, Tape, slot_tape
from sexpr import parse

X, Y, Z = Shape.X, Shape.Y, Shape.Z


def s(t):
    return str(t)


def test_print_basic():
    # tree.cpp:183-184
    assert s(X() + 5) == "(+ x 5)"


@pytest.mark.parametrize("build,want", [
    # tree.cpp:285-291
    (lambda: (Z() + 2) / (2 * (Z() + 3)), "(/ (+ z 2) (+ (* z 2) 6))"),
    # tree.cpp:293-300
    (lambda: -3 * X().cos() + Z() + 2, "(- (+ z 2) (* (cos x) 3))"),
    # tree.cpp:302-307
    (lambda: (lambda c: X() * 2 + Y() * 5 + c + 5 * c)(Z().cos()),
     "(+ (* x 2) (* y 5) (* (cos z) 6))"),
    # tree.cpp:309-313
    (lambda: (Z() - 10) / -Z(), "(/ (- z 10) (- z))"),
    # tree.cpp:315-321
    (lambda: (2 * X() + Y()) + (2 * X() + Y()), "(+ (* y 2) (* x 4))"),
    # tree.cpp:323-329
    (lambda: (2 * X() + Y()) * (2 * X() + Y()), "(square (+ y (* x 2)))"),
    # tree.cpp:331-337
    (lambda: (lambda a: a + 3 * a.cos())(X() + 2 * Y()),
     "(+ x (* y 2) (* (cos (+ x (* y 2))) 3))"),
    # tree.cpp:339-345
    (lambda: (lambda a: a + 3 * a.sin().cos())(X() + 2 * Y() + 7),
     "(+ x (* y 2) (* (cos (sin (+ x (* y 2) 7))) 3) 7)"),
    # tree.cpp:347-358
    (lambda: ((-Z()) / (Z() - 10)).atan2((-Z()) / (Z() - 100)),
     "(atan2 (/ (- z) (- z 10)) (/ (- z) (- z 100)))"),
    # tree.cpp:377-384
    (lambda: (lambda a: a * a)(-Z()), "(square (- z))"),
])
def test_optimizer_forms(build, want):
    assert s(build().optimized()) == want


def test_print_unoptimized_constants():
    # tree.cpp:386-391
    t = -0.091 - (Z() - 2.7) / 0.6
    assert s(t) == "(- -0.091 (/ (- z 2.7) 0.6))"


def test_min_dedup_size():
    # tree.cpp:360-365: min(X, Y, X, Y) optimizes to 3 unique nodes
    t = X().min(Y()).min(X().min(Y())).optimized()
    st = slot_tape(t)
    assert st["num_clauses"] == 3 + 0 + 1   # x, y, z slots + one min clause


def test_deck_num_clauses():
    # deck.cpp:19-23: X + 1 -> X, Y, Z, 1, +
    assert slot_tape(X() + 1)["num_clauses"] == 5


def test_deck_xyz_slots():
    # deck.cpp:25-31
    st = slot_tape(X() + 2)
    assert (st["X"], st["Y"], st["Z"]) == (3, 4, 5)
    assert st["root"] == 1


def test_deck_constants():
    # deck.cpp:33-41
    st = slot_tape(X() + 5)
    assert st["constants"] == [(2, 5.0)]


def test_walk_order():
    # tree.cpp:219-243 and deck.cpp:24-58: the optimized min list of
    # (x, y, z, 1) becomes three min clauses; the root clause is slot 1 and
    # every argument slot is numbered above the clause that reads it.
    t = X().min(Y()).min(Z().min(1.0))
    st = slot_tape(t)
    assert [c[0] for c in st["clauses"]] == [19, 19, 19]
    assert st["clauses"][0][1] == 1
    for op, cid, a, b in st["clauses"]:
        assert a > cid and b > cid


def test_opcode_enum_and_args(lib):
    # libfive.cpp:75-87
    assert lib.libfive_opcode_enum(b"min") == 19
    assert lib.libfive_opcode_enum(b"MIN") == 19
    assert lib.libfive_opcode_enum(b"nth-root") == 25
    assert lib.libfive_opcode_enum(b"var-free") == 5
    assert lib.libfive_opcode_enum(b"invalid") == -1
    assert lib.libfive_opcode_enum(b"no-such-op") == -1
    assert lib.libfive_opcode_args(19) == 2
    assert lib.libfive_opcode_args(8) == 1
    assert lib.libfive_opcode_args(2) == 0
    assert lib.libfive_opcode_args(0) == -1
    assert lib.libfive_opcode_args(99) == -1


def test_invalid_constructors_return_null(lib):
    # libfive.cpp:116-142: wrong arity or null arguments give NULL
    x = lib.libfive_tree_x()
    assert not lib.libfive_tree_unary(19, x)        # min is binary
    assert not lib.libfive_tree_binary(8, x, x)     # sqrt is unary
    assert not lib.libfive_tree_nullary(19)
    assert not lib.libfive_tree_unary(8, None)
    lib.libfive_tree_delete(x)


def test_get_const_and_is_var(lib):
    c = lib.libfive_tree_const(ctypes.c_float(2.5))
    ok = ctypes.c_bool(False)
    assert lib.libfive_tree_get_const(c, ctypes.byref(ok)) == 2.5 and ok.value
    v = lib.libfive_tree_var()
    assert lib.libfive_tree_is_var(v)
    assert not lib.libfive_tree_is_var(c)
    lib.libfive_tree_get_const(v, ctypes.byref(ok))
    assert not ok.value
    lib.libfive_tree_delete(c)
    lib.libfive_tree_delete(v)


def test_identity_simplifications():
    # tree.cpp:95-230 local simplifications
    assert s(X() + 0) == "x"
    assert s(0 + X()) == "x"
    assert s(X() * 1) == "x"
    assert s(X() * -1) == "(- x)"
    assert s(-(-X())) == "x"
    assert s(X().abs().abs()) == "(abs x)"
    assert s(X().square().abs()) == "(square x)"
    assert s(X() / 1) == "x"
    assert s(X() + (-Y())) == "(- x y)"
    assert s(X() - (-Y())) == "(+ x y)"
    assert s(X().min(X())) == "x"
    assert s(Shape.constant(2) + 3) == "5"


def test_remap():
    # Tree::remap + flatten (tree.cpp:366-528)
    t = (X() + Y()).remap(Y(), X() * 2, Z())
    assert s(t.optimized()) == "(+ y (* x 2))"


def test_register_tape_is_consistent():
    """Every register read is defined earlier; the root is defined last."""
    t = parse("(min (sqrt (+ (square (- x 1)) (square y))) (max (- x 3) (abs z)))")
    st = slot_tape(t)
    assert len(st["clauses"]) > 0
