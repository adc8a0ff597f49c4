"""The gradient the reverse mode is held to, pinned to FP64 central finite
differences (h = 1e-3).

The GPU's variable gradients are compared with the oracle's
JacobianEvaluator (tests/test_gpu_grad.py, rtol 1e-4); here that
Jacobian, restating libfive/src/eval/eval_jacobian.cpp:49-115 in float32, is
compared with central differences of the same shape written out in float64
numpy: the gradient of loss = mean f^2 over fixed points with respect to
every free variable: within 1e-3 relative (vector norm) at h = 1e-3, and
within 1e-6 at h = 1e-5, where the differences' truncation error at the
shape's min / max kinks has shrunk below float32 rounding."""
import numpy as np

from libfive_b200 import workloads
from libfive_b200.shape import Shape, X, Y, Z
from oracle_ffi import OracleTape

H = 1e-3


def _model(n_spheres=5, n_boxes=3, seed=17):
    """Shape and float64 model: union of spheres (cx, cy, cz, r free), minus
    boxes (cx, cy, cz, s free), smooth-unioned (m = 0.3) with one more
    sphere."""
    rng = workloads.SplitMix64(seed)
    x, y, z = X(), Y(), Z()
    vars_, vals = [], []

    def var(v):
        s = Shape.var()
        vars_.append(s)
        vals.append(v)
        return s

    sph = []
    for _ in range(n_spheres + 1):
        c = [var(rng.uniform(-0.6, 0.6)) for _ in range(3)]
        r = var(rng.uniform(0.2, 0.45))
        sph.append((c, r))
    box = []
    for _ in range(n_boxes):
        c = [var(rng.uniform(-0.6, 0.6)) for _ in range(3)]
        s = var(rng.uniform(0.1, 0.3))
        box.append((c, s))

    def sphere_s(c, r):
        return ((x - c[0]).square() + (y - c[1]).square() + (z - c[2]).square()).sqrt() - r

    def box_s(c, s):
        return ((x - c[0]).abs() - s).max(((y - c[1]).abs() - s).max((z - c[2]).abs() - s))

    u = sphere_s(*sph[0])
    for c, r in sph[1:n_spheres]:
        u = u.min(sphere_s(c, r))
    for c, s in box:
        u = workloads.difference(u, box_s(c, s))
    shape = workloads.blend_stable(u, sphere_s(*sph[n_spheres]), 0.3)

    def f64(v, px, py, pz):
        it = iter(v)
        nxt = lambda: next(it)  # noqa: E731
        sp = [([nxt(), nxt(), nxt()], nxt()) for _ in range(n_spheres + 1)]
        bx = [([nxt(), nxt(), nxt()], nxt()) for _ in range(n_boxes)]
        d = [np.sqrt((px - c[0]) ** 2 + (py - c[1]) ** 2 + (pz - c[2]) ** 2) - r for c, r in sp]
        a = np.min(np.stack(d[:n_spheres]), axis=0)
        for c, s in bx:
            b = np.maximum(np.maximum(np.abs(px - c[0]) - s, np.abs(py - c[1]) - s),
                           np.abs(pz - c[2]) - s)
            a = np.maximum(a, -b)
        k = 2.75 / 0.3 ** 2
        return np.minimum(a, d[n_spheres]) - np.log1p(np.exp(-k * np.abs(a - d[n_spheres]))) / k

    return shape, vars_, np.array(vals, np.float32), f64


def test_oracle_gradient_matches_fp64_central_differences():
    shape, vars_, vals, f64 = _model()
    x, y, z = workloads.uniform_points(20000, seed=23, lo=-1.0, hi=1.0)
    ora = OracleTape(shape, dict(zip(vars_, vals.tolist())))
    # float32 oracle: d mean f^2 / dv = (2 / N) sum f_i df_i/dv
    f = ora.values(x, y, z).astype(np.float64)
    jac = ora.jacobian(x, y, z).astype(np.float64)
    col = {s.id(): i for i, s in enumerate(vars_)}
    order = [col[vid] for _, vid in ora.st["vars"]]
    g_ora = np.zeros(len(vars_))
    g_ora[order] = 2.0 / len(f) * (f @ jac)
    # the float64 model agrees with the float32 oracle pointwise
    px, py, pz = (a.astype(np.float64) for a in (x, y, z))
    v64 = vals.astype(np.float64)
    np.testing.assert_allclose(f64(v64, px, py, pz), f, atol=2e-6)
    def central(h):
        g = np.zeros(len(vars_))
        for i in range(len(vars_)):
            up, dn = v64.copy(), v64.copy()
            up[i] += h
            dn[i] -= h
            g[i] = (np.mean(f64(up, px, py, pz) ** 2) - np.mean(f64(dn, px, py, pz) ** 2)) / (2 * h)
        return g

    g_fd = central(H)
    assert np.linalg.norm(g_ora - g_fd) <= 1e-3 * np.linalg.norm(g_fd)
    # the remaining difference is the differences' own truncation error (min /
    # max kinks crossed within +-h): it shrinks with h, to float32 rounding
    g_fine = central(1e-5)
    assert np.linalg.norm(g_ora - g_fine) <= 1e-6 * np.linalg.norm(g_fine)
    big = np.abs(g_fine) > 1e-2 * np.abs(g_fine).max()
    np.testing.assert_allclose(g_ora[big], g_fine[big], rtol=1e-5)
