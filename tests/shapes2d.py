"""Shapes of the reference's contour tests (libfive/test/util/shapes.cpp:
circle, rectangle with a 4x4 transform, menger), restated over this
library's Shape class.  Arithmetic on the shapes' parameters is float32,
as in the C++ helpers."""
import numpy as np

from libfive_b200.shape import Shape

f32 = np.float32
IDENTITY = np.eye(4, dtype=np.float32)


def circle(r, center=(0.0, 0.0)):
    """shapes.cpp:98-101"""
    x, y = Shape.X(), Shape.Y()
    return ((x - float(f32(center[0]))).square() + (y - float(f32(center[1]))).square()).sqrt() - float(f32(r))


def _row(M, i):
    x, y, z = Shape.X(), Shape.Y(), Shape.Z()
    return float(M[i, 0]) * x + float(M[i, 1]) * y + float(M[i, 2]) * z + float(M[i, 3])


def rectangle(xmin, xmax, ymin, ymax, M=IDENTITY):
    """shapes.cpp:16-23: max(max(xmin - x, x - xmax), max(ymin - y, y - ymax))
    over the first two rows of the transform M."""
    x, y = _row(M, 0), _row(M, 1)
    return (float(f32(xmin)) - x).max(x - float(f32(xmax))).max(
        (float(f32(ymin)) - y).max(y - float(f32(ymax))))


def _recurse(x, y, scale, M, i):
    """shapes.cpp:44-69"""
    x, y, scale = f32(x), f32(y), f32(scale)
    h = scale / f32(2)
    base = rectangle(x - h, x + h, y - h, y + h, M)
    if i == 0:
        return base
    t = scale / f32(3)
    j = i - 1
    offs = [(scale, 0), (-scale, 0), (0, scale), (0, -scale), (scale, scale), (scale, -scale),
            (-scale, scale), (-scale, -scale)]
    subs = [_recurse(x + f32(dx), y + f32(dy), t, M, j) for dx, dy in offs]
    # min(base, min(s0, min(s1, ... min(s6, s7))))
    acc = subs[-1]
    for s in reversed(subs[:-1]):
        acc = s.min(acc)
    return base.min(acc)


def menger(i):
    """shapes.cpp:71-96, with the two quarter turns (about X, then about Y)
    written with exact 0 / +-1 entries."""
    M = np.zeros((4, 4), np.float32)
    M[:3, :3] = np.eye(3)
    a = _recurse(0, 0, 1, M, i)
    M = np.zeros((4, 4), np.float32)
    M[:3, :3] = [[1, 0, 0], [0, 0, -1], [0, 1, 0]]
    b = _recurse(0, 0, 1, M, i)
    M = np.zeros((4, 4), np.float32)
    M[:3, :3] = [[0, 0, 1], [0, 1, 0], [-1, 0, 0]]
    c = _recurse(0, 0, 1, M, i)
    x, y, z = Shape.X(), Shape.Y(), Shape.Z()
    cube = ((-(x + 1.5)).max(x - 1.5).max((-(y + 1.5)).max(y - 1.5))).max(
        (-(z + 1.5)).max(z - 1.5))
    cutout = -(a.min(b).min(c))
    return cube.max(cutout)
