"""Seeded synthetic shapes for the benchmark and parity workloads.

All randomness comes from SplitMix64 (Steele et al., 2014), so a seed names
a shape exactly.  Primitives follow libfive's stdlib formulas
(libfive/stdlib/stdlib_impl.cpp): sphere 227-230, union/intersection/
difference 51-65 (min / max / max(a, -b)), blend_expt_unit 79-85 (the Python
`blend`), with a box as the max of three slab distances and a z-cylinder as
max(radial distance, |z - cz| - h).
"""
import math

import numpy as np

from .shape import Shape, X, Y, Z

MASK = (1 << 64) - 1


class SplitMix64:
    def __init__(self, seed):
        self.s = seed & MASK

    def next(self):
        self.s = (self.s + 0x9E3779B97F4A7C15) & MASK
        z = self.s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK
        return z ^ (z >> 31)

    def uniform(self, lo=0.0, hi=1.0):
        return lo + (hi - lo) * ((self.next() >> 11) * (1.0 / (1 << 53)))

    def below(self, n):
        return self.next() % n


def sphere(c, r):
    x, y, z = X(), Y(), Z()
    return ((x - c[0]).square() + (y - c[1]).square() + (z - c[2]).square()).sqrt() - r


def box(c, s):
    x, y, z = X(), Y(), Z()
    return ((x - c[0]).abs() - s).max(((y - c[1]).abs() - s).max((z - c[2]).abs() - s))


def zcylinder(c, r, h):
    x, y, z = X(), Y(), Z()
    radial = ((x - c[0]).square() + (y - c[1]).square()).sqrt() - r
    return radial.max((z - c[2]).abs() - h)


def union(a, b):
    return a.min(b)


def intersection(a, b):
    return a.max(b)


def difference(a, b):
    return a.max(-b)


def blend(a, b, m=0.05):
    """blend_expt_unit(a, b, m) = -log(exp(-k a) + exp(-k b)) / k,
    k = 2.75 / m^2, built with the same tree operations as the stdlib."""
    mt = Shape.constant(m)
    k = Shape.constant(2.75) / (mt ** Shape.constant(2))
    ea = ((-k) * a).exp()
    eb = ((-k) * b).exp()
    return -((ea + eb).log()) / k


def blend_stable(a, b, m=0.05):
    """The same smooth union as `blend`, -log(exp(-k a) + exp(-k b)) / k
    with k = 2.75 / m^2, written as min(a, b) - log(1 + exp(-k |a - b|)) / k:
    equal in exact arithmetic, but its exp never overflows, while `blend`'s
    exp(-k a) overflows float32 once a < -88 / k (-0.08 for m = 0.05) and
    its value becomes -inf (or +inf when both terms underflow)."""
    mt = Shape.constant(m)
    k = Shape.constant(2.75) / (mt ** Shape.constant(2))
    e = ((-k) * (a - b).abs()).exp()
    return a.min(b) - (e + 1.0).log() / k


def spheres_union(n=64, seed=1):
    """Union (min) of n spheres, centres U[-1,1]^3, radii U[0.1,0.35]."""
    rng = SplitMix64(seed)
    out = None
    for _ in range(n):
        c = [rng.uniform(-1, 1) for _ in range(3)]
        r = rng.uniform(0.1, 0.35)
        s = sphere(c, r)
        out = s if out is None else out.min(s)
    return out


# Operator weights for the random CSG tree: (union, blend, difference,
# intersection).  Unions dominate so that the combined surface stays large.
CSG_WEIGHTS = (0.63, 0.07, 0.20, 0.10)


def random_csg(n_prims=2000, seed=2, size=(0.02, 0.2)):
    """Random binary CSG tree over n primitives (spheres, boxes, z-cylinders
    in rotation), centres U[-1,1]^3, sizes U[size]."""
    rng = SplitMix64(seed)
    prims = []
    for i in range(n_prims):
        c = [rng.uniform(-1, 1) for _ in range(3)]
        s = rng.uniform(*size)
        kind = i % 3
        if kind == 0:
            prims.append(sphere(c, s))
        elif kind == 1:
            prims.append(box(c, s))
        else:
            prims.append(zcylinder(c, s, rng.uniform(*size)))
    level = prims
    while len(level) > 1:
        nxt = []
        for i in range(0, len(level) - 1, 2):
            u = rng.uniform()
            a, b = level[i], level[i + 1]
            w = CSG_WEIGHTS
            if u < w[0]:
                nxt.append(union(a, b))
            elif u < w[0] + w[1]:
                nxt.append(blend(a, b))
            elif u < w[0] + w[1] + w[2]:
                nxt.append(difference(a, b))
            else:
                nxt.append(intersection(a, b))
        if len(level) % 2:
            nxt.append(level[-1])
        level = nxt
    return level[0]


def batch_specs(n_trees=512, seed=11, prims=(8, 4000), resolutions=(64, 128, 256, 512)):
    """Per-tree (primitive count, tree seed, resolution per unit) of the
    many-tree meshing workload: primitive counts log-uniform over `prims`,
    resolutions drawn uniformly from `resolutions` (over a 3-unit region:
    octree depths 8, 9, 10 and 11)."""
    rng = SplitMix64(seed)
    lo, hi = math.log(prims[0]), math.log(prims[1])
    out = []
    for i in range(n_trees):
        n = int(round(math.exp(rng.uniform(lo, hi))))
        res = resolutions[min(int(rng.uniform() * len(resolutions)), len(resolutions) - 1)]
        out.append((n, seed * 100003 + i, res))
    return out


def blended_spheres_vars(n=256, seed=4, m=0.05, stable=False):
    """n spheres whose centres and radii are free variables, combined by a
    balanced binary tree of blends (`blend`, or with stable=True the
    overflow-free `blend_stable`, whose values and gradients stay finite
    everywhere).  Returns (shape, {var: value})."""
    rng = SplitMix64(seed)
    values = {}
    leaves = []
    x, y, z = X(), Y(), Z()
    for _ in range(n):
        cx, cy, cz, r = Shape.var(), Shape.var(), Shape.var(), Shape.var()
        values[cx] = rng.uniform(-1, 1)
        values[cy] = rng.uniform(-1, 1)
        values[cz] = rng.uniform(-1, 1)
        values[r] = rng.uniform(0.1, 0.35)
        leaves.append(((x - cx).square() + (y - cy).square() + (z - cz).square()).sqrt() - r)
    level = leaves
    while len(level) > 1:
        mix = blend_stable if stable else blend
        nxt = [mix(level[i], level[i + 1], m) for i in range(0, len(level) - 1, 2)]
        if len(level) % 2:
            nxt.append(level[-1])
        level = nxt
    return level[0], values


def fit_csg_vars(n_prims=128, seed=21, m=0.05, size=(0.1, 0.35)):
    """CSG of n primitives with 7 free variables each (the fitting
    workload): spheres sqrt((ax (x-cx))^2 + (ay (y-cy))^2 + (az (z-cz))^2) - r,
    boxes max(|x-cx| - sx, |y-cy| - sy, |z-cz| - sz) - d and z-cylinders
    max(sqrt((ax (x-cx))^2 + (ay (y-cy))^2) - r, |z-cz| - h), in rotation,
    centres U[-1,1]^3, sizes U[size], axis scales 1, box offsets 0; combined
    by a random binary tree with the CSG_WEIGHTS operators (smooth unions of
    radius m, in the overflow-free form of blend_stable, so that f and its
    gradient stay finite everywhere).  Returns (shape, {var: value}, [vars
    in creation order])."""
    rng = SplitMix64(seed)
    x, y, z = X(), Y(), Z()
    values, order, prims = {}, [], []

    def var(v):
        s = Shape.var()
        values[s] = v
        order.append(s)
        return s

    for i in range(n_prims):
        cx, cy, cz = (var(rng.uniform(-1, 1)) for _ in range(3))
        kind = i % 3
        if kind == 0:
            r = var(rng.uniform(*size))
            ax, ay, az = var(1.0), var(1.0), var(1.0)
            prims.append(((ax * (x - cx)).square() + (ay * (y - cy)).square()
                          + (az * (z - cz)).square()).sqrt() - r)
        elif kind == 1:
            sx, sy, sz = (var(rng.uniform(*size)) for _ in range(3))
            d = var(0.0)
            prims.append(((x - cx).abs() - sx).max(((y - cy).abs() - sy).max(
                (z - cz).abs() - sz)) - d)
        else:
            r, h = var(rng.uniform(*size)), var(rng.uniform(*size))
            ax, ay = var(1.0), var(1.0)
            radial = ((ax * (x - cx)).square() + (ay * (y - cy)).square()).sqrt() - r
            prims.append(radial.max((z - cz).abs() - h))
    level = prims
    while len(level) > 1:
        nxt = []
        for i in range(0, len(level) - 1, 2):
            u = rng.uniform()
            a, b = level[i], level[i + 1]
            w = CSG_WEIGHTS
            if u < w[0]:
                nxt.append(union(a, b))
            elif u < w[0] + w[1]:
                nxt.append(blend_stable(a, b, m))
            elif u < w[0] + w[1] + w[2]:
                nxt.append(difference(a, b))
            else:
                nxt.append(intersection(a, b))
        if len(level) % 2:
            nxt.append(level[-1])
        level = nxt
    return level[0], values, order


def perturbed(values, sigma=0.05, seed=0):
    """The variable values plus N(0, sigma) noise (Box-Muller over SplitMix64
    uniforms), in the dict's order."""
    rng = SplitMix64(seed)
    out = {}
    for k, v in values.items():
        u1 = max(rng.uniform(), 1e-300)
        u2 = rng.uniform()
        out[k] = v + sigma * math.sqrt(-2.0 * math.log(u1)) * math.cos(2.0 * math.pi * u2)
    return out


def surface_points(verts, tris, n, seed=7):
    """n points sampled area-uniformly from a triangle mesh, as float32
    x, y, z arrays."""
    tri = verts[tris.astype(np.int64)].astype(np.float64)
    area = 0.5 * np.linalg.norm(np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0]), axis=1)
    rng = np.random.Generator(np.random.PCG64(seed))
    k = rng.choice(len(tri), size=n, p=area / area.sum())
    u, w = rng.random(n), rng.random(n)
    flip = u + w > 1
    u[flip], w[flip] = 1 - u[flip], 1 - w[flip]
    p = tri[k, 0] + u[:, None] * (tri[k, 1] - tri[k, 0]) + w[:, None] * (tri[k, 2] - tri[k, 0])
    return tuple(np.ascontiguousarray(p[:, a], np.float32) for a in range(3))


def lattice(n=128, lo=-1.5, hi=1.5):
    """n^3 inclusive lattice as flat float32 x, y, z arrays."""
    t = (lo + (hi - lo) * np.arange(n, dtype=np.float64) / (n - 1)).astype(np.float32)
    zz, yy, xx = np.meshgrid(t, t, t, indexing="ij")
    return (np.ascontiguousarray(xx.ravel()), np.ascontiguousarray(yy.ravel()),
            np.ascontiguousarray(zz.ravel()))


def uniform_points(n, seed=3, lo=-1.5, hi=1.5):
    r = np.random.Generator(np.random.PCG64(seed))
    p = r.uniform(lo, hi, size=(3, n)).astype(np.float32)
    return p[0].copy(), p[1].copy(), p[2].copy()
