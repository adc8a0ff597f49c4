"""Mesh comparison helpers for the parity tests."""
import ctypes

import numpy as np

import oracle_ffi


def oracle_mesh(ora, lo, hi, min_feature, max_err=1e-8, threads=1):
    """Mesh of an OracleTape by the CPU oracle mesher: (verts [N,3], tris [M,3])."""
    lib = oracle_ffi.load()
    vp, tp = ctypes.c_void_p(), ctypes.c_void_p()
    nv, nt = ctypes.c_uint32(), ctypes.c_uint32()
    lib.ora_render_mesh(ora.h, *lo, *hi, min_feature, max_err, threads,
                        ctypes.byref(vp), ctypes.byref(nv), ctypes.byref(tp),
                        ctypes.byref(nt))
    v = np.ctypeslib.as_array(ctypes.cast(vp, ctypes.POINTER(ctypes.c_float)),
                              shape=(nv.value * 3,)).reshape(-1, 3).copy()
    t = (np.ctypeslib.as_array(ctypes.cast(tp, ctypes.POINTER(ctypes.c_uint32)),
                               shape=(nt.value * 3,)).reshape(-1, 3).copy()
         if nt.value else np.zeros((0, 3), np.uint32))
    lib.ora_free(vp)
    lib.ora_free(tp)
    return v, t


def canonical_triangles(verts, tris):
    """Triangles as sorted rows of 9 float32 bit patterns, each rotated so
    that the smallest vertex comes first (orientation preserved)."""
    if len(tris) == 0:
        return np.zeros((0, 9), np.uint32)
    P = np.ascontiguousarray(verts, np.float32)[tris].view(np.uint32).reshape(-1, 3, 3)
    # rank of every corner among all corners, in lexicographic order
    _, rank = np.unique(P.reshape(-1, 3), axis=0, return_inverse=True)
    rank = rank.reshape(-1, 3)
    first = np.argmin(rank, axis=1)
    idx = (first[:, None] + np.arange(3)[None, :]) % 3
    out = np.take_along_axis(P, idx[:, :, None], axis=1).reshape(-1, 9)
    order = np.lexsort(out.T[::-1])
    return out[order]


def same_mesh(v1, t1, v2, t2):
    """Identical triangle sets (vertex positions compared bit for bit)."""
    if len(t1) != len(t2):
        return False
    return np.array_equal(canonical_triangles(v1, t1), canonical_triangles(v2, t2))


def edge_pairs_ok(tris):
    """CHECK_EDGE_PAIRS (libfive/test/util/mesh_checks.cpp:4-35): every edge
    is used exactly once in each direction."""
    seen = {}
    for t in tris.tolist():
        for k in range(3):
            a, b = t[k], t[(k + 1) % 3]
            key = (min(a, b), max(a, b))
            bit = 1 if a < b else 2
            cur = seen.get(key, 0)
            if cur & bit:
                return False
            seen[key] = cur | bit
    return all(v == 3 for v in seen.values())


def hausdorff(v1, t1, v2, t2):
    """Symmetric Hausdorff distance between the used vertex sets."""
    from scipy.spatial import cKDTree
    a = v1[np.unique(t1)] if len(t1) else np.zeros((0, 3))
    b = v2[np.unique(t2)] if len(t2) else np.zeros((0, 3))
    if len(a) == 0 or len(b) == 0:
        return 0.0 if len(a) == len(b) else np.inf
    da, _ = cKDTree(b).query(a)
    db, _ = cKDTree(a).query(b)
    return float(max(da.max(), db.max()))


def canonical_contours(contours):
    """Contours as a sorted list of tuples of float32 bit patterns: closed
    contours (first point == last) lose the repeated point and are rotated
    to start at their smallest point, so that the segment order in which
    they were welded does not matter."""
    out = []
    for c in contours:
        c = np.asarray(c, np.float32).reshape(-1, 2)
        bits = [tuple(p) for p in c.view(np.uint32).tolist()]
        if len(bits) > 1 and bits[0] == bits[-1]:
            bits = bits[:-1]
            k = min(range(len(bits)), key=lambda i: bits[i])
            bits = bits[k:] + bits[:k]
            bits.append(bits[0])
        out.append(tuple(bits))
    return sorted(out)


def same_contours(a, b):
    return canonical_contours(a) == canonical_contours(b)
