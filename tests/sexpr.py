"""Builds Shapes from libfive-style prefix expressions, e.g. "(+ (* x 2) 1)".

Symbols x, y, z are the axes; any other bare symbol names a free variable
(looked up in / added to `vars`); numbers are float constants.
"""
from libfive_b200.shape import Shape

_ALIAS = {"+": "add", "*": "mul", "/": "div"}


def _tokens(s):
    return s.replace("(", " ( ").replace(")", " ) ").split()


def parse(s, vars=None):
    vars = {} if vars is None else vars
    toks = _tokens(s)
    pos = [0]

    def atom(t):
        if t in ("x", "y", "z"):
            return {"x": Shape.X, "y": Shape.Y, "z": Shape.Z}[t]()
        try:
            return Shape.constant(float(t))
        except ValueError:
            if t not in vars:
                vars[t] = Shape.var()
            return vars[t]

    def expr():
        t = toks[pos[0]]
        pos[0] += 1
        if t != "(":
            return atom(t)
        op = toks[pos[0]]
        pos[0] += 1
        args = []
        while toks[pos[0]] != ")":
            args.append(expr())
        pos[0] += 1
        if op == "-":
            op = "neg" if len(args) == 1 else "sub"
        op = _ALIAS.get(op, op)
        if len(args) > 2:   # commutative n-ary form, left fold
            out = args[0]
            for a in args[1:]:
                out = Shape.new(op, out, a)
            return out
        return Shape.new(op, *args)

    return expr()
