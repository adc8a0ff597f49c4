"""The dual-contouring mesher's constant tables (libfive_b200/csrc/
dc_tables.hpp) pinned to the reference: its MarchingTable<3> test
(libfive/test/marching.cpp:29-42), its corner-manifold table
(DCTree<3>::cornersAreManifold, libfive/src/render/brep/dc/dc_tree3.cpp:
111-154, restated in tests/golden/dc_corner_manifold.json by
make_dc_manifold_fixture.py), and the properties a dual-marching-cubes patch
table must have.

(libfive/test/manifold_tables.cpp tests ManifoldTables<N>, which only the
hybrid mesher uses, hybrid_tree.inl:450; the DC collapse uses the corner
table checked here.)"""
import ctypes
import json
import os

import numpy as np

import oracle_ffi

HERE = os.path.dirname(os.path.abspath(__file__))

# DcTables field layout (all 8-bit, no padding)
FIELDS = [("v", np.int8, (256, 4, 12, 2)), ("e", np.int8, (8, 8)), ("p", np.int8, (256, 24)),
          ("manifold", np.uint8, (256,)), ("npatch", np.uint8, (256,)),
          ("nedge", np.uint8, (256, 4))]


def tables():
    lib = oracle_ffi.load()
    n = ctypes.c_uint64()
    ptr = lib.ora_dc_tables(ctypes.byref(n))
    raw = np.ctypeslib.as_array(ctypes.cast(ptr, ctypes.POINTER(ctypes.c_uint8)),
                                shape=(n.value,)).copy()
    out, off = {}, 0
    for name, dt, shape in FIELDS:
        size = int(np.prod(shape))
        out[name] = raw[off:off + size].view(dt).reshape(shape)
        off += size
    assert off == n.value
    return out


T = tables()
CUBE_EDGES = [(a, a | (1 << k)) for a in range(8) for k in range(3) if not a & (1 << k)]


def patches(mask):
    out = []
    for p in range(4):
        if T["v"][mask, p, 0, 0] == -1:
            break
        pairs = []
        for e in range(12):
            if T["v"][mask, p, e, 0] == -1:
                break
            pairs.append((int(T["v"][mask, p, e, 0]), int(T["v"][mask, p, e, 1])))
        out.append(pairs)
    return out


def test_every_mask_has_a_patch():
    # marching.cpp:29-42
    for i in range(1, 255):
        assert T["v"][i, 0, 0, 0] != -1, i
    assert T["v"][0, 0, 0, 0] == -1
    assert T["v"][255, 0, 0, 0] == -1


def test_corner_manifold_table_is_the_reference_table():
    want = json.load(open(os.path.join(HERE, "golden", "dc_corner_manifold.json")))["manifold"]
    assert T["manifold"].tolist() == want


def test_patches_cover_each_crossing_edge_once():
    for mask in range(256):
        filled = {c for c in range(8) if mask & (1 << c)}
        crossing = set()
        for a, b in CUBE_EDGES:
            if (a in filled) != (b in filled):
                crossing.add((a, b) if a in filled else (b, a))
        seen = []
        for pairs in patches(mask):
            for a, b in pairs:
                assert a in filled and b not in filled, (mask, a, b)
                seen.append((a, b))
        assert sorted(seen) == sorted(crossing), mask
        assert T["npatch"][mask] == len(patches(mask))


def test_patch_edges_walk_around_faces():
    """Consecutive edges of a patch (cyclically) lie on one cube face: each
    patch is one closed polygon on the cube surface."""
    def face_of(edge_pairs):
        # faces as (axis, side); an edge lies on the two faces its corners share
        fs = set()
        for ax in range(3):
            for side in (0, 1):
                if all(((c >> ax) & 1) == side for c in edge_pairs):
                    fs.add((ax, side))
        return fs
    for mask in range(1, 255):
        for pairs in patches(mask):
            if len(pairs) < 3:
                continue
            for k in range(len(pairs)):
                e0, e1 = pairs[k], pairs[(k + 1) % len(pairs)]
                assert face_of(e0) & face_of(e1), (mask, pairs)


def test_rotations_permute_patches():
    def rot(v, axis):
        c = [1 if v & (1 << k) else -1 for k in range(3)]
        r = {0: (c[0], -c[2], c[1]), 1: (c[2], c[1], -c[0]), 2: (-c[1], c[0], c[2])}[axis]
        return sum((1 << k) for k in range(3) if r[k] > 0)

    def as_sets(ps):
        return sorted(tuple(sorted(p)) for p in ps)

    for mask in range(256):
        for axis in range(3):
            m2 = sum(1 << rot(c, axis) for c in range(8) if mask & (1 << c))
            rotated = [[(rot(a, axis), rot(b, axis)) for a, b in p] for p in patches(mask)]
            assert as_sets(rotated) == as_sets(patches(m2)), (mask, axis)


def test_directed_edge_ids():
    ids = sorted(int(x) for x in T["e"].ravel() if x >= 0)
    assert ids == list(range(24))
    for a, b in CUBE_EDGES:
        assert T["e"][a, b] >= 0 and T["e"][b, a] >= 0
    for mask in range(256):
        for p, pairs in enumerate(patches(mask)):
            for a, b in pairs:
                assert T["p"][mask, T["e"][a, b]] == p
