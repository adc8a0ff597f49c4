"""Tapes compiled to straight-line kernels (jit.cpp) against the interpreter.

The compiled value, derivative, reverse-mode and interval kernels must give
the interpreters' bits at every point and box,
transcendental opcodes included (both call the same CUDA functions with
contraction off).  The interpreter's values are computed in a child process
with LFB_JIT=0; lfb_tape_compiled says which path a tape took."""
import os
import subprocess
import sys

import numpy as np
import pytest

from libfive_b200 import ffi, workloads
from libfive_b200.shape import Shape, Tape

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
X, Y, Z = Shape.X, Shape.Y, Shape.Z


def shapes():
    """name -> (shape, var values); every compiled opcode appears."""
    out = {
        "spheres": (workloads.spheres_union(64, seed=1), None),
        "csg": (workloads.random_csg(60, seed=5), None),
    }
    blend, vals = workloads.blended_spheres_vars(16, seed=4)
    out["blend_vars"] = (blend, vals)
    x, y, z = X(), Y(), Z()
    v = Shape.var()
    recip = Shape.new("recip", (z * v).abs())
    misc = ((x / (y.square() + 0.5)) - recip).max(-(x.with_constant_vars() * 0.25))
    out["misc"] = (misc, {v: 1.75})
    # opcodes compiled through the interpreters' own rules (dev_point.cuh)
    trig = ((x.sin() * y.cos() + (z * 0.3).tan() - y.atan2(x) + (x * 0.5).asin()
             + (y * 0.5).acos() + z.atan() + x ** 3 + y.nth_root(3) + z % 0.7
             + x.sqrt().nanfill(y) + x.compare(y)) - 0.5)
    out["trig"] = (trig, None)
    # longer than the straight-line limit (4096 clauses): values and the
    # reverse mode compile in segments; the free variables exercise the
    # checkpointed backward pass's variable sums
    long_, lvals = workloads.blended_spheres_vars(300, seed=6, stable=True)
    out["long"] = (long_, lvals)
    return out


CHILD = r"""
import sys, numpy as np
sys.path.insert(0, sys.argv[1]); sys.path.insert(0, sys.argv[1] + "/tests")
from test_gpu_jit import shapes, points, grad, grad_vars, boxes
from libfive_b200.shape import Tape
from libfive_b200 import ffi
name = sys.argv[2]
s, vals = shapes()[name]
t = Tape(s, vals)
out = t.values(*points())
assert ffi.load().lfb_tape_compiled(t.ptr) == 0
d = t.derivs(*points())
np.save(sys.argv[3], np.stack([out] + list(d)))
np.save(sys.argv[3] + ".grad.npy", np.stack(grad(t)))
np.save(sys.argv[3] + ".gvars.npy", grad_vars(t))
lo, hi, nan = t.intervals(*boxes())
np.save(sys.argv[3] + ".iv.npy", np.stack([lo, hi, nan.astype(np.float32)]))
"""


def boxes():
    """Boxes of several sizes around random centres, a few degenerate."""
    r = np.random.default_rng(4)
    c = r.uniform(-1.5, 1.5, (3, 20000)).astype(np.float32)
    h = (10.0 ** r.uniform(-4, 0, (1, 20000))).astype(np.float32)
    h[:, :100] = 0
    return c - h, c + h


def grad(t):
    """f and the reverse-mode point gradients with a varying seed."""
    x, y, z = points()
    n = len(x)
    seed = np.linspace(-1.0, 1.0, n).astype(np.float32)
    f = np.empty(n, np.float32)
    gx, gy, gz = (np.empty(n, np.float32) for _ in range(3))
    t.grad(x, y, z, seed=seed, f=f, gx=gx, gy=gy, gz=gz)
    return f, gx, gy, gz


def grad_vars(t):
    x, y, z = points()
    gv = np.zeros(max(t.n_vars, 1), np.float32)
    if t.n_vars:
        t.grad(x, y, z, gvars=gv)
    return gv


def points():
    x, y, z = workloads.uniform_points(50000, seed=9, lo=-1.6, hi=1.6)
    # exact zeros and ties: lattice points too
    lx, ly, lz = workloads.lattice(16, lo=-1.0, hi=1.0)
    return (np.concatenate([x, lx]), np.concatenate([y, ly]), np.concatenate([z, lz]))


@pytest.mark.parametrize("name", ["spheres", "csg", "blend_vars", "misc", "trig", "long"])
def test_compiled_matches_interpreter(gpu, name, tmp_path):
    s, vals = shapes()[name]
    t = Tape(s, vals)
    got = t.values(*points())
    assert ffi.load().lfb_tape_compiled(t.ptr) == 1
    path = str(tmp_path / "interp.npy")
    r = subprocess.run([sys.executable, "-c", CHILD, ROOT, name, path],
                       env=dict(os.environ, LFB_JIT="0"), capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    want = np.load(path)
    assert np.array_equal(got.view(np.uint32), want[0].view(np.uint32))
    # values and d/dx, d/dy, d/dz of the compiled derivative kernel
    d = np.stack(list(t.derivs(*points())))
    assert np.array_equal(d.view(np.uint32), want[1:].view(np.uint32))
    # reverse mode: f and point gradients bit for bit (same operations in the
    # same order), variable gradients up to the order of the atomic sums
    g = np.stack(grad(t))
    assert np.array_equal(g.view(np.uint32), np.load(path + ".grad.npy").view(np.uint32))
    gv, gw = grad_vars(t), np.load(path + ".gvars.npy")
    finite = np.isfinite(gw)
    scale = max(1.0, float(np.abs(gw[finite]).max())) if finite.any() else 1.0
    assert np.array_equal(np.isfinite(gv), finite)
    assert np.allclose(gv, gw, rtol=1e-5, atol=1e-5 * scale, equal_nan=True)
    # intervals: the same bounds and NaN flags
    lo, hi, nan = t.intervals(*boxes())
    iv = np.load(path + ".iv.npy")
    assert np.array_equal(lo.view(np.uint32), iv[0].view(np.uint32))
    assert np.array_equal(hi.view(np.uint32), iv[1].view(np.uint32))
    assert np.array_equal(nan, iv[2].astype(bool))


def test_variables_change_without_recompiling(gpu):
    s, vals = shapes()["blend_vars"]
    t = Tape(s, vals)
    p = points()
    a = t.values(*p)
    t.set_vars({k: v + 0.1 for k, v in vals.items()})
    b = t.values(*p)
    assert ffi.load().lfb_tape_compiled(t.ptr) == 1
    assert not np.array_equal(a, b)
    t2 = Tape(s, {k: v + 0.1 for k, v in vals.items()})
    assert np.array_equal(b.view(np.uint32), t2.values(*p).view(np.uint32))


def test_long_tape_compiles_in_segments(gpu):
    t = Tape(workloads.spheres_union(500, seed=2))
    assert t.n_clauses > 4096
    t.values(*points())
    assert ffi.load().lfb_tape_compiled(t.ptr) == 1
