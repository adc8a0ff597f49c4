"""Writes tests/golden/tape_hashes.json: SHA-256 of the slot tape
(lfb_tree_slot_tape: clause order, operands, constants, variable slots) of
seeded trees, as built by the current library.  The optimizer, walk and
slot numbering restate the reference's step for step, so any change to
these tapes is a parity change; test_tape_regression.py fails on one.

    python tests/golden/make_tape_hashes.py     (after a deliberate change)
"""
import hashlib
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from libfive_b200 import workloads  # noqa: E402
from libfive_b200.shape import Shape, X, Y, Z, slot_tape  # noqa: E402

UNARY = ("square", "sqrt", "neg", "abs", "sin", "cos", "tan", "asin", "acos", "atan",
         "exp", "log", "const-var")
BINARY = ("add", "mul", "min", "max", "sub", "div", "atan2", "pow", "nth-root", "mod",
          "nanfill", "compare")


def random_dag(seed, n_nodes):
    """A seeded random expression DAG over every unary and binary opcode:
    operands drawn from all earlier nodes (so subtrees are shared), from a
    small set of repeated constants (0, 1, -1, 2: the optimizer's folding
    and affine cases) or from three free variables; every node is then
    folded into one root by min / max / add / sub / mul, and some trees are
    remapped.  Returns (shape, variables in creation order)."""
    rng = workloads.SplitMix64(seed)
    vs = [Shape.var() for _ in range(3)]
    pool = [X(), Y(), Z()]

    def operand():
        k = rng.below(10)
        if k == 0:
            return Shape.constant((0.0, 1.0, -1.0, 2.0)[rng.below(4)])
        if k == 1:
            return Shape.constant(rng.uniform(-2, 2))
        if k == 2:
            return vs[rng.below(3)]
        return pool[rng.below(len(pool))]

    for _ in range(n_nodes):
        k = rng.below(10)
        if k == 0:
            node = Shape.constant(rng.uniform(-2, 2))
        elif k <= 3:
            node = Shape.new(UNARY[rng.below(len(UNARY))], pool[rng.below(len(pool))])
        else:
            node = Shape.new(BINARY[rng.below(len(BINARY))], operand(), operand())
        pool.append(node)
    level = pool[3:]
    while len(level) > 1:
        nxt = [Shape.new(("min", "max", "add", "sub", "mul")[rng.below(5)], level[i], level[i + 1])
               for i in range(0, len(level) - 1, 2)]
        if len(level) % 2:
            nxt.append(level[-1])
        level = nxt
    root = level[0]
    if rng.below(4) == 0:
        x, y, z = X(), Y(), Z()
        root = root.remap(x + y * 0.5, y.square() - 1, z * 2 + x)
    return root, vs


def trees():
    """name -> (shape, variables in creation order)."""
    out = {}
    for s in range(8):
        out["csg%d" % s] = (workloads.random_csg(50 + 250 * s, seed=100 + s), [])
    for s in range(3):
        sh, _, order = workloads.fit_csg_vars(64, seed=300 + s)
        out["fit%d" % s] = (sh, order)
        sh, vals = workloads.blended_spheres_vars(32, seed=400 + s)
        out["blend%d" % s] = (sh, list(vals))
        out["spheres%d" % s] = (workloads.spheres_union(64, seed=500 + s), [])
    x, y, z = X(), Y(), Z()
    out["affine"] = ((((x * 2 + y * 3 - z / 4) * (x - 1) * (y + 2)).max(-(x + x + x))
                      .min(z * 0.5 - x * 0.5)) / (y.square() + 1), [])
    for s in range(40):
        out["dag%d" % s] = random_dag(600 + s, 20 + 10 * s)
    return out


def tape_hash(shape, var_order):
    st = slot_tape(shape)
    # variable ids are node addresses: name them by creation order
    rank = {v.id(): k for k, v in enumerate(var_order)}
    st["vars"] = [(slot, rank[vid]) for slot, vid in st["vars"]]
    return hashlib.sha256(json.dumps(st, sort_keys=True).encode()).hexdigest()


def main():
    out = {name: tape_hash(s, order) for name, (s, order) in trees().items()}
    with open(os.path.join(HERE, "tape_hashes.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
        f.write("\n")


if __name__ == "__main__":
    main()
