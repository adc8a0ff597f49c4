"""Python mirror of the reference's `libfive.shape.Shape`
(libfive/bind/python/libfive/shape.py:27-277), backed by libfive_b200.

Trees are built through the same C calls (libfive_tree_unary / _binary /
_const ...); `get_mesh` / `save_stl` / `__call__` keep the reference's names,
arguments and return shapes.  `Tape` adds the batched GPU entry points of
include/libfive_b200.h over numpy arrays (host) or torch CUDA tensors
(device, no copies).
"""
import ctypes
import numbers

import numpy as np

from . import ffi


def _lib():
    return ffi.load()


def _opcode(name):
    o = _lib().libfive_opcode_enum(name.encode())
    if o < 0:
        raise ValueError(f"unknown opcode {name}")
    return o


class Shape:
    """Reference-counted handle to a libfive tree."""

    def __init__(self, ptr):
        if not ptr:
            raise ValueError("null tree")
        self.ptr = ctypes.c_void_p(ptr)

    def __del__(self):
        try:
            if self.ptr:
                _lib().libfive_tree_delete(self.ptr)
                self.ptr = None
        except Exception:
            pass

    @classmethod
    def new(cls, op, *args):
        lib = _lib()
        o = _opcode(op)
        if len(args) == 0:
            return cls(lib.libfive_tree_nullary(o))
        if len(args) == 1:
            return cls(lib.libfive_tree_unary(o, args[0].ptr))
        return cls(lib.libfive_tree_binary(o, args[0].ptr, args[1].ptr))

    @classmethod
    def wrap(cls, t):
        if isinstance(t, Shape):
            return t
        if isinstance(t, numbers.Number):
            return cls(_lib().libfive_tree_const(float(t)))
        raise TypeError(f"cannot convert {type(t)} to Shape")

    @classmethod
    def X(cls):
        return cls(_lib().libfive_tree_x())

    @classmethod
    def Y(cls):
        return cls(_lib().libfive_tree_y())

    @classmethod
    def Z(cls):
        return cls(_lib().libfive_tree_z())

    @classmethod
    def var(cls):
        return cls(_lib().libfive_tree_var())

    @classmethod
    def constant(cls, v):
        return cls(_lib().libfive_tree_const(float(v)))

    def id(self):
        return _lib().libfive_tree_id(self.ptr)

    def __str__(self):
        lib = _lib()
        p = lib.libfive_tree_print(self.ptr)
        s = ctypes.cast(p, ctypes.c_char_p).value.decode()
        lib.libfive_free_str(p)
        return s

    __repr__ = __str__

    def _bin(self, op, other, swap=False):
        o = Shape.wrap(other)
        return Shape.new(op, o, self) if swap else Shape.new(op, self, o)

    def __add__(self, o): return self._bin('add', o)
    def __radd__(self, o): return self._bin('add', o, True)
    def __sub__(self, o): return self._bin('sub', o)
    def __rsub__(self, o): return self._bin('sub', o, True)
    def __mul__(self, o): return self._bin('mul', o)
    def __rmul__(self, o): return self._bin('mul', o, True)
    def __truediv__(self, o): return self._bin('div', o)
    def __rtruediv__(self, o): return self._bin('div', o, True)
    def __mod__(self, o): return self._bin('mod', o)
    def __rmod__(self, o): return self._bin('mod', o, True)
    def __pow__(self, o): return self._bin('pow', o)
    def __neg__(self): return Shape.new('neg', self)

    def min(self, o): return self._bin('min', o)
    def max(self, o): return self._bin('max', o)
    def atan2(self, o): return self._bin('atan2', o)
    def nth_root(self, o): return self._bin('nth-root', o)
    def nanfill(self, o): return self._bin('nanfill', o)
    def compare(self, o): return self._bin('compare', o)
    def sqrt(self): return Shape.new('sqrt', self)
    def square(self): return Shape.new('square', self)
    def abs(self): return Shape.new('abs', self)
    def sin(self): return Shape.new('sin', self)
    def cos(self): return Shape.new('cos', self)
    def tan(self): return Shape.new('tan', self)
    def asin(self): return Shape.new('asin', self)
    def acos(self): return Shape.new('acos', self)
    def atan(self): return Shape.new('atan', self)
    def exp(self): return Shape.new('exp', self)
    def log(self): return Shape.new('log', self)
    def with_constant_vars(self): return Shape.new('const-var', self)

    def remap(self, x, y, z):
        x, y, z = (Shape.wrap(t) for t in (x, y, z))
        return Shape(_lib().libfive_tree_remap(self.ptr, x.ptr, y.ptr, z.ptr))

    def optimized(self):
        return Shape(_lib().libfive_tree_optimized(self.ptr))

    def __call__(self, x, y, z):
        """libfive_tree_eval_f at one point (free variables read as zero)."""
        return _lib().libfive_tree_eval_f(self.ptr, ffi.Vec3(x, y, z))

    def eval_interval(self, lower, upper):
        r = ffi.Region3(*[ffi.Interval(a, b) for a, b in zip(lower, upper)])
        i = _lib().libfive_tree_eval_r(self.ptr, r)
        return i.lower, i.upper

    def eval_deriv(self, x, y, z):
        d = _lib().libfive_tree_eval_d(self.ptr, ffi.Vec3(x, y, z))
        return d.x, d.y, d.z

    def get_mesh(self, xyz_min=(-10, -10, -10), xyz_max=(10, 10, 10),
                 resolution=10):
        """Returns (verts, tris) like the reference's Shape.get_mesh."""
        verts, tris = mesh_arrays(self.render_mesh(xyz_min, xyz_max, resolution))
        return [tuple(v) for v in verts.tolist()], [tuple(t) for t in tris.tolist()]

    def render_mesh(self, xyz_min, xyz_max, resolution):
        region = ffi.Region3(*[ffi.Interval(a, b) for a, b in zip(xyz_min, xyz_max)])
        m = _lib().libfive_tree_render_mesh(self.ptr, region, resolution)
        if not m:
            raise RuntimeError("libfive_tree_render_mesh failed: %s" % ffi.last_error()[1])
        return m

    def save_stl(self, filename, xyz_min=(-10, -10, -10), xyz_max=(10, 10, 10),
                 resolution=10, quality=8):
        region = ffi.Region3(*[ffi.Interval(a, b) for a, b in zip(xyz_min, xyz_max)])
        trees = (ffi.tree_t * 2)(self.ptr.value, None)
        return _lib().libfive_tree_save_meshes(trees, region, resolution, quality,
                                               filename.encode())


def contour_arrays(cs_p, dim=2, delete=True):
    """Copies a libfive_contours* (dim 2) or libfive_contours3* (dim 3) into
    a list of float32 [n, dim] arrays."""
    out = []
    cs = cs_p[0]
    for i in range(cs.count):
        c = cs.cs[i]
        a = np.ctypeslib.as_array(ctypes.cast(c.pts, ctypes.POINTER(ctypes.c_float)),
                                  shape=(c.count * dim,)).reshape(c.count, dim).copy()
        out.append(a)
    if delete:
        (_lib().libfive_contours_delete if dim == 2 else _lib().libfive_contours3_delete)(cs_p)
    return out


def mesh_arrays(mesh_p, delete=True):
    """Copies a libfive_mesh* into numpy (verts float32 [N,3], tris uint32 [M,3])."""
    m = mesh_p[0]
    nv, nt = m.vert_count, m.tri_count
    verts = np.ctypeslib.as_array(ctypes.cast(m.verts, ctypes.POINTER(ctypes.c_float)),
                                  shape=(nv * 3,)).reshape(nv, 3).copy() if nv else np.zeros((0, 3), np.float32)
    tris = np.ctypeslib.as_array(ctypes.cast(m.tris, ctypes.POINTER(ctypes.c_uint32)),
                                 shape=(nt * 3,)).reshape(nt, 3).copy() if nt else np.zeros((0, 3), np.uint32)
    if delete:
        _lib().libfive_mesh_delete(mesh_p)
    return verts, tris


def _ptr(a):
    """Host numpy array or torch tensor -> (pointer, is_device)."""
    if a is None:
        return None, None
    if isinstance(a, np.ndarray):
        assert a.flags.c_contiguous
        return a.ctypes.data, False
    # torch tensor
    assert a.is_contiguous()
    return a.data_ptr(), a.is_cuda


class Tape:
    """A tree flattened once and kept on the GPU (lfb_tape)."""

    def __init__(self, shape, var_values=None):
        lib = _lib()
        self.shape = shape
        vars_ = _vars_struct(var_values)
        self.ptr = lib.lfb_tape_new(shape.ptr, vars_)
        if not self.ptr:
            raise RuntimeError("lfb_tape_new failed: %s" % ffi.last_error()[1])
        counts = (ctypes.c_uint32 * 6)()
        ffi.check(lib.lfb_tape_info(self.ptr, counts))
        (self.n_clauses, self.n_regs, self.n_const, self.n_vars,
         self.n_choices, self.n_slots) = list(counts)

    def __del__(self):
        try:
            if self.ptr:
                _lib().lfb_tape_delete(self.ptr)
                self.ptr = None
        except Exception:
            pass

    def set_vars(self, var_values):
        return ffi.check(_lib().lfb_tape_set_vars(self.ptr, _vars_struct(var_values)))

    def var_ids(self):
        arr = (ctypes.c_void_p * max(1, self.n_vars))()
        ffi.check(_lib().lfb_tape_var_ids(self.ptr, arr, self.n_vars))
        return [arr[i] for i in range(self.n_vars)]

    def get_vars(self):
        """Current variable values in var_ids() order (after fit steps on
        the device, the values they wrote)."""
        out = np.zeros(max(1, self.n_vars), np.float32)
        ffi.check(_lib().lfb_tape_get_vars(
            self.ptr, out.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), self.n_vars),
            "get_vars")
        return out[:self.n_vars]

    def _flags(self, arrays):
        devs = {_ptr(a)[1] for a in arrays if a is not None}
        if len(devs) != 1:
            raise ValueError("mix of host and device arrays")
        return ffi.LFB_DEVICE_PTRS if devs.pop() else 0

    def values(self, x, y, z, out=None, stream=None):
        out = np.empty_like(x) if out is None else out
        fl = self._flags([x, y, z, out])
        ffi.check(_lib().lfb_eval_values(self.ptr, len(x), _ptr(x)[0], _ptr(y)[0],
                                         _ptr(z)[0], _ptr(out)[0], stream, fl), "values")
        return out

    def derivs(self, x, y, z, v=None, dx=None, dy=None, dz=None, stream=None):
        if v is None:
            v, dx, dy, dz = (np.empty_like(x) for _ in range(4))
        fl = self._flags([x, y, z, v])
        ffi.check(_lib().lfb_eval_derivs(self.ptr, len(x), _ptr(x)[0], _ptr(y)[0],
                                         _ptr(z)[0], _ptr(v)[0], _ptr(dx)[0],
                                         _ptr(dy)[0], _ptr(dz)[0], stream, fl), "derivs")
        return v, dx, dy, dz

    def intervals(self, lo, hi, stream=None):
        """lo, hi: [3, n] float32 arrays of box bounds."""
        n = lo.shape[1]
        olo, ohi = np.empty(n, np.float32), np.empty(n, np.float32)
        onan = np.empty(n, np.uint8)
        lo = np.ascontiguousarray(lo, np.float32)
        hi = np.ascontiguousarray(hi, np.float32)
        ffi.check(_lib().lfb_eval_intervals(
            self.ptr, n, lo[0].ctypes.data, hi[0].ctypes.data, lo[1].ctypes.data,
            hi[1].ctypes.data, lo[2].ctypes.data, hi[2].ctypes.data,
            olo.ctypes.data, ohi.ctypes.data, onan.ctypes.data, stream, 0), "intervals")
        return olo, ohi, onan.astype(bool)

    def features(self, x, y, z, max_feats=16, lists=True):
        """FeatureEvaluator at host points: (inside [n] bool, list of
        [k, 3] arrays of the distinct feature gradients at each point, or
        None when lists is False)."""
        x, y, z = (np.ascontiguousarray(a, np.float32) for a in (x, y, z))
        n = len(x)
        inside = np.zeros(n, np.uint8)
        feats = np.zeros((n, max_feats, 3), np.float32) if lists else None
        counts = np.zeros(n, np.uint32) if lists else None
        ffi.check(_lib().lfb_eval_features(
            self.ptr, n, x.ctypes.data, y.ctypes.data, z.ctypes.data, inside.ctypes.data,
            feats.ctypes.data if lists else None, max_feats,
            counts.ctypes.data if lists else None), "features")
        if not lists:
            return inside.astype(bool), None
        return inside.astype(bool), [feats[i, :min(int(c), max_feats)] for i, c in enumerate(counts)]

    def jacobian(self, x, y, z, out=None, stream=None):
        out = np.zeros((len(x), self.n_vars), np.float32) if out is None else out
        fl = self._flags([x, y, z, out])
        ffi.check(_lib().lfb_eval_jacobian(self.ptr, len(x), _ptr(x)[0], _ptr(y)[0],
                                           _ptr(z)[0], _ptr(out)[0], stream, fl), "jacobian")
        return out

    def grad(self, x, y, z, seed=None, f=None, gx=None, gy=None, gz=None,
             gvars=None, stream=None):
        fl = self._flags([x, y, z])
        ffi.check(_lib().lfb_eval_grad(
            self.ptr, len(x), _ptr(x)[0], _ptr(y)[0], _ptr(z)[0], _ptr(seed)[0],
            _ptr(f)[0], _ptr(gx)[0], _ptr(gy)[0], _ptr(gz)[0], _ptr(gvars)[0],
            stream, fl), "grad")
        return f, gx, gy, gz, gvars

    def loss_grad(self, x, y, z, f, gx=None, gy=None, gz=None, gvars=None, loss=None,
                  stream=None):
        """loss = mean f^2 and its gradients in one call (CUDA tensors;
        lfb_eval_loss_grad).  gvars accumulates; zero it first."""
        ffi.check(_lib().lfb_eval_loss_grad(
            self.ptr, len(x), _ptr(x)[0], _ptr(y)[0], _ptr(z)[0], _ptr(f)[0], _ptr(gx)[0],
            _ptr(gy)[0], _ptr(gz)[0], _ptr(gvars)[0], _ptr(loss)[0], stream,
            ffi.LFB_DEVICE_PTRS), "loss_grad")
        return f, gx, gy, gz, gvars, loss

    def render_mesh(self, lower, upper, min_feature, max_err=1e-8, stats=False):
        region = ffi.Region3(*[ffi.Interval(a, b) for a, b in zip(lower, upper)])
        st = ffi.MeshStats()
        m = _lib().lfb_render_mesh(self.ptr, region,
                                   ffi.MeshSettings(min_feature, max_err),
                                   ctypes.byref(st))
        if not m:
            raise RuntimeError("lfb_render_mesh failed: %s" % ffi.last_error()[1])
        v, t = mesh_arrays(m)
        return (v, t, st) if stats else (v, t)


def render_slice(tape, lower, upper, z, min_feature, max_err=1e-8):
    """Contours of the slice z of a Tape over [lower, upper] (2D): a list of
    float32 [n, 2] point arrays, closed contours repeating their first
    point."""
    region = ffi.Region2(*[ffi.Interval(a, b) for a, b in zip(lower, upper)])
    cs = _lib().lfb_render_slice(tape.ptr, region, z, min_feature, max_err)
    if not cs:
        raise RuntimeError("lfb_render_slice failed: %s" % ffi.last_error()[1])
    return contour_arrays(cs)


def render_heightmap(tape, lower, upper, res, normals=True):
    """Heightmap::render of a Tape over the Voxels region lower / upper at
    `res` voxels per unit (a number or one per axis): (depth, norm) as
    rows x cols arrays (norm is None when normals is false)."""
    res = res if np.ndim(res) else (res, res, res)
    lo, hi, r = (np.ascontiguousarray(np.asarray(v, np.float32).reshape(3))
                 for v in (lower, upper, res))
    fp = ctypes.POINTER(ctypes.c_float)
    dims = np.zeros(3, np.uint32)
    lib = _lib()
    args = (lo.ctypes.data_as(fp), hi.ctypes.data_as(fp), r.ctypes.data_as(fp),
            dims.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)))
    ffi.check(lib.lfb_render_heightmap(tape.ptr, *args, None, None))
    cols, rows = int(dims[0]), int(dims[1])
    depth = np.empty((rows, cols), np.float32)
    norm = np.empty((rows, cols), np.uint32) if normals else None
    ffi.check(lib.lfb_render_heightmap(
        tape.ptr, *args, depth.ctypes.data_as(fp),
        norm.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)) if normals else None))
    return depth, norm


def render_meshes(jobs, workers=0, stats=False):
    """Meshes of several tapes in one lfb_render_meshes call.

    jobs: sequence of (tape, lower, upper, min_feature[, max_err]); the meshes
    render concurrently, each on its own CUDA stream.  Returns a list of
    (verts, tris) pairs (with an MeshStats third item when stats is true), in
    the order of jobs; raises RuntimeError if any mesh failed.
    """
    n = len(jobs)
    tapes = (ffi.tape_t * n)()
    regions = (ffi.Region3 * n)()
    settings = (ffi.MeshSettings * n)()
    for i, job in enumerate(jobs):
        tape, lower, upper, min_feature = job[:4]
        max_err = job[4] if len(job) > 4 else 1e-8
        tapes[i] = tape.ptr
        regions[i] = ffi.Region3(*[ffi.Interval(a, b) for a, b in zip(lower, upper)])
        settings[i] = ffi.MeshSettings(min_feature, max_err)
    meshes = (ctypes.POINTER(ffi.Mesh) * n)()
    st = (ffi.MeshStats * n)()
    rc = _lib().lfb_render_meshes(tapes, n, regions, settings, workers, meshes,
                                  st if stats else None)
    out = []
    for i in range(n):
        if meshes[i]:
            v, t = mesh_arrays(meshes[i])
            out.append((v, t, st[i]) if stats else (v, t))
    if rc != 0:
        raise RuntimeError("lfb_render_meshes failed: %s" % ffi.last_error()[1])
    return out


def _vars_struct(var_values):
    if not var_values:
        return ffi.Vars(None, None, 0)
    ids = list(var_values.keys())
    vals = [float(var_values[k]) for k in ids]
    n = len(ids)
    idp = (ctypes.c_void_p * n)(*[k.id() if isinstance(k, Shape) else k for k in ids])
    vp = (ctypes.c_float * n)(*vals)
    s = ffi.Vars(ctypes.cast(idp, ctypes.POINTER(ctypes.c_void_p)),
                 ctypes.cast(vp, ctypes.POINTER(ctypes.c_float)), n)
    s._keep = (idp, vp)
    return s


def slot_tape(shape):
    """The reference-layout tape (lfb_tree_slot_tape) as python lists."""
    lib = _lib()
    counts = (ctypes.c_uint32 * 8)()
    ffi.check(lib.lfb_tree_slot_tape(shape.ptr, counts, None, None, None, None, None))
    num_clauses, n, nc, nv, X, Y, Z, root = list(counts)
    clauses = (ctypes.c_int32 * max(1, 4 * n))()
    cslots = (ctypes.c_uint32 * max(1, nc))()
    cvals = (ctypes.c_float * max(1, nc))()
    vslots = (ctypes.c_uint32 * max(1, nv))()
    vids = (ctypes.c_void_p * max(1, nv))()
    ffi.check(lib.lfb_tree_slot_tape(shape.ptr, counts, clauses, cslots, cvals, vslots, vids))
    return dict(num_clauses=num_clauses, X=X, Y=Y, Z=Z, root=root,
                clauses=[tuple(clauses[4 * i:4 * i + 4]) for i in range(n)],
                constants=[(cslots[i], cvals[i]) for i in range(nc)],
                vars=[(vslots[i], vids[i]) for i in range(nv)])


X = Shape.X
Y = Shape.Y
Z = Shape.Z


def _fn(name):
    def f(a, *rest):
        a = Shape.wrap(a)
        return getattr(a, name)(*rest)
    f.__name__ = name
    return f


sqrt, square, abs_, sin, cos, tan, asin, acos, atan, exp, log = (
    _fn(n) for n in ("sqrt", "square", "abs", "sin", "cos", "tan", "asin",
                     "acos", "atan", "exp", "log"))


def min_(a, b):
    return Shape.wrap(a).min(b)


def max_(a, b):
    return Shape.wrap(a).max(b)
