"""ctypes access to the CPU oracle (oracle/lib/liboracle.so), for tests only."""
import ctypes
import os

import numpy as np

from libfive_b200.shape import slot_tape

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
_lib = None


def load():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "lib", "liboracle.so"))
        vp = ctypes.c_void_p
        _lib.ora_tape_new.restype = vp
        _lib.ora_tape_new.argtypes = [ctypes.c_uint32, ctypes.c_uint32, vp, ctypes.c_uint32,
                                      vp, vp, ctypes.c_uint32, vp, vp, ctypes.c_uint32,
                                      ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32]
        _lib.ora_tape_delete.argtypes = [vp]
        _lib.ora_values.argtypes = [vp, ctypes.c_uint64, vp, vp, vp, vp, ctypes.c_int]
        _lib.ora_derivs.argtypes = [vp, ctypes.c_uint64, vp, vp, vp, vp, vp, vp, vp, ctypes.c_int]
        _lib.ora_ambiguous.argtypes = [vp, ctypes.c_uint64, vp, vp, vp, vp]
        _lib.ora_intervals.argtypes = [vp, ctypes.c_uint64] + [vp] * 9 + [ctypes.c_int]
        _lib.ora_pushed_size.restype = ctypes.c_uint32
        _lib.ora_pushed_size.argtypes = [vp] + [ctypes.c_float] * 6
        _lib.ora_jacobian.argtypes = [vp, ctypes.c_uint64, vp, vp, vp, vp, ctypes.c_int]
        _lib.ora_is_inside.restype = ctypes.c_int
        _lib.ora_is_inside.argtypes = [vp, ctypes.c_float, ctypes.c_float, ctypes.c_float]
        _lib.ora_features.restype = ctypes.c_int
        _lib.ora_features.argtypes = [vp, ctypes.c_float, ctypes.c_float, ctypes.c_float, vp, ctypes.c_int]
        _lib.ora_voxel_dims.argtypes = [vp, vp, vp, vp]
        _lib.ora_voxel_pts.argtypes = [vp, vp, vp, ctypes.c_int, vp]
        _lib.ora_render_heightmap.argtypes = [vp, vp, vp, vp, ctypes.c_int, vp, vp]
        if hasattr(_lib, "ora_render_mesh"):
            _lib.ora_render_mesh.restype = ctypes.c_int
            _lib.ora_render_mesh.argtypes = [vp] + [ctypes.c_float] * 6 + [
                ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.POINTER(vp),
                ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(vp),
                ctypes.POINTER(ctypes.c_uint32)]
            _lib.ora_free.argtypes = [vp]
            _lib.ora_time_mesh.restype = ctypes.c_int
            _lib.ora_time_mesh.argtypes = [vp] + [ctypes.c_float] * 6 + [
                ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int, vp,
                ctypes.POINTER(ctypes.c_uint32)]
        _lib.ora_render_contours.restype = ctypes.c_int
        _lib.ora_render_contours.argtypes = [vp] + [ctypes.c_double] * 7 + [
            ctypes.POINTER(vp), ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(vp),
            ctypes.POINTER(ctypes.c_uint32)]
        _lib.ora_dc_tables2.argtypes = [vp]
        _lib.ora_weld.restype = ctypes.c_uint32
        _lib.ora_weld.argtypes = [vp, ctypes.c_uint32, vp, vp]
        _lib.ora_libm_mode.argtypes = [ctypes.c_int]
        _lib.ora_libm_table.argtypes = [vp, vp, ctypes.c_uint64]
        _lib.ora_libm_take.restype = ctypes.c_uint64
        _lib.ora_libm_take.argtypes = [vp, ctypes.c_uint64]
        _lib.ora_libm_misses.restype = ctypes.c_uint64
        _lib.ora_sym3_eigen.argtypes = [vp, vp, vp]
        _lib.ora_dc_tables.restype = vp
        _lib.ora_dc_tables.argtypes = [ctypes.POINTER(ctypes.c_uint64)]
        _lib.ora_qef_rank.restype = ctypes.c_int
        _lib.ora_qef_rank.argtypes = [vp]
        _lib.ora_qef_vertex.restype = ctypes.c_double
        _lib.ora_qef_vertex.argtypes = [vp, vp, ctypes.c_double, vp, vp, vp]
    return _lib


def _p(a):
    return a.ctypes.data


class OracleTape:
    """The reference-layout tape of a shape, evaluated on the CPU."""

    def __init__(self, shape, var_values=None):
        lib = load()
        st = slot_tape(shape)
        self.st = st
        cl = np.array(st["clauses"], np.int32).reshape(-1, 4) if st["clauses"] else np.zeros((0, 4), np.int32)
        cl = np.ascontiguousarray(cl)
        cs = np.array([c[0] for c in st["constants"]], np.uint32)
        cv = np.array([c[1] for c in st["constants"]], np.float32)
        vs = np.array([v[0] for v in st["vars"]], np.uint32)
        vals = {}
        if var_values:
            for k, v in var_values.items():
                vals[k.id() if hasattr(k, "id") else k] = v
        vv = np.array([vals.get(v[1], 0.0) for v in st["vars"]], np.float32)
        self._keep = (cl, cs, cv, vs, vv)
        self.n_vars = len(st["vars"])
        self.h = lib.ora_tape_new(st["num_clauses"], len(cl), _p(cl), len(cs), _p(cs), _p(cv),
                                  len(vs), _p(vs), _p(vv), st["X"], st["Y"], st["Z"], st["root"])

    def __del__(self):
        try:
            load().ora_tape_delete(self.h)
        except Exception:
            pass

    def values(self, x, y, z, threads=1):
        out = np.empty(len(x), np.float32)
        load().ora_values(self.h, len(x), _p(x), _p(y), _p(z), _p(out), threads)
        return out

    def derivs(self, x, y, z, threads=1):
        outs = [np.empty(len(x), np.float32) for _ in range(4)]
        load().ora_derivs(self.h, len(x), _p(x), _p(y), _p(z), *[_p(o) for o in outs], threads)
        return outs

    def ambiguous(self, x, y, z):
        out = np.empty(len(x), np.uint8)
        load().ora_ambiguous(self.h, len(x), _p(x), _p(y), _p(z), _p(out))
        return out.astype(bool)

    def intervals(self, lo, hi, threads=1):
        lo = np.ascontiguousarray(lo, np.float32)
        hi = np.ascontiguousarray(hi, np.float32)
        n = lo.shape[1]
        olo, ohi = np.empty(n, np.float32), np.empty(n, np.float32)
        onan = np.empty(n, np.uint8)
        load().ora_intervals(self.h, n, _p(lo[0]), _p(hi[0]), _p(lo[1]), _p(hi[1]),
                             _p(lo[2]), _p(hi[2]), _p(olo), _p(ohi), _p(onan), threads)
        return olo, ohi, onan.astype(bool)

    def pushed_size(self, lo, hi):
        return load().ora_pushed_size(self.h, *lo, *hi)

    def jacobian(self, x, y, z, threads=1):
        out = np.zeros((len(x), self.n_vars), np.float32)
        load().ora_jacobian(self.h, len(x), _p(x), _p(y), _p(z), _p(out), threads)
        return out

    def is_inside(self, p):
        return bool(load().ora_is_inside(self.h, *p))

    def features(self, p, max_n=16):
        out = np.zeros((max_n, 3), np.float32)
        n = load().ora_features(self.h, *p, _p(out), max_n)
        return out[:min(n, max_n)]


def _f3(v):
    return np.ascontiguousarray(np.asarray(v, np.float32).reshape(3))


def _region(lower, upper, res):
    res = res if np.ndim(res) else (res, res, res)
    return _f3(lower), _f3(upper), _f3(res)


def voxel_dims(lower, upper, res):
    """(cols, rows, depth samples) of a Voxels region (voxels.cpp:23-44)."""
    lo, hi, r = _region(lower, upper, res)
    dims = np.zeros(3, np.uint32)
    load().ora_voxel_dims(_p(lo), _p(hi), _p(r), _p(dims))
    return tuple(int(d) for d in dims)


def voxel_pts(lower, upper, res, axis):
    lo, hi, r = _region(lower, upper, res)
    out = np.zeros(voxel_dims(lower, upper, res)[axis], np.float32)
    load().ora_voxel_pts(_p(lo), _p(hi), _p(r), axis, _p(out))
    return out


def render_heightmap(tape, lower, upper, res, workers=8):
    """Heightmap::render restated: (depth, norm), rows x cols."""
    lo, hi, r = _region(lower, upper, res)
    w, h, _ = voxel_dims(lower, upper, res)
    depth = np.zeros((h, w), np.float32)
    norm = np.zeros((h, w), np.uint32)
    load().ora_render_heightmap(tape.h, _p(lo), _p(hi), _p(r), workers, _p(depth), _p(norm))
    return depth, norm


def render_contours(tape, lo, hi, z, min_feature, max_err=1e-8):
    """Contours::render restated: (list of [n, 2] float32 point arrays, depth)."""
    lib = load()
    pp, cp = ctypes.c_void_p(), ctypes.c_void_p()
    npt, nc = ctypes.c_uint32(), ctypes.c_uint32()
    depth = lib.ora_render_contours(tape.h, lo[0], lo[1], hi[0], hi[1], z, min_feature, max_err,
                                    ctypes.byref(pp), ctypes.byref(npt), ctypes.byref(cp),
                                    ctypes.byref(nc))
    pts = np.ctypeslib.as_array(ctypes.cast(pp, ctypes.POINTER(ctypes.c_float)),
                                shape=(max(npt.value, 1) * 2,)).reshape(-1, 2)[:npt.value].copy()
    counts = np.ctypeslib.as_array(ctypes.cast(cp, ctypes.POINTER(ctypes.c_uint32)),
                                   shape=(max(nc.value, 1),))[:nc.value].copy()
    lib.ora_free(pp)
    lib.ora_free(cp)
    out, k = [], 0
    for c in counts:
        out.append(pts[k:k + c])
        k += c
    return out, depth


def dc_tables2():
    """DcTables2 as numpy arrays (v, e, p, manifold, npatch, nedge)."""
    raw = np.zeros(16 * 2 * 4 * 2 + 16 + 16 * 8 + 16 + 16 + 32, np.int8)
    load().ora_dc_tables2(raw.ctypes.data)
    o = 0
    v = raw[o:o + 256].reshape(16, 2, 4, 2); o += 256
    e = raw[o:o + 16].reshape(4, 4); o += 16
    p = raw[o:o + 128].reshape(16, 8); o += 128
    manifold = raw[o:o + 16].view(np.uint8); o += 16
    npatch = raw[o:o + 16].view(np.uint8); o += 16
    nedge = raw[o:o + 32].view(np.uint8).reshape(16, 2)
    return v, e, p, manifold, npatch, nedge


def weld(segs):
    """Contours::collect's welding of directed segments [(a, b), ...]:
    lists of vertex ids."""
    segs = np.ascontiguousarray(segs, np.uint32).reshape(-1, 2)
    out = np.zeros(2 * len(segs) + 1, np.uint32)
    counts = np.zeros(len(segs) + 1, np.uint32)
    n = load().ora_weld(segs.ctypes.data, len(segs), out.ctypes.data, counts.ctypes.data)
    res, k = [], 0
    for c in counts[:n]:
        res.append(out[k:k + c].tolist())
        k += c
    return res
