"""Oracle runs with the GPU's library-call results (tests only).

The oracle's point evaluators call the host C library for sin, cos, tan,
asin, acos, atan, exp and log; the GPU calls CUDA's functions, which differ
by a few ULPs (each opcode's bound is checked on its own in
test_gpu_eval.py).  Every other opcode is exactly rounded on both sides, so
when the oracle is given the GPU's result for each library call it meets,
a whole tape -- or a whole mesh -- must come out bit for bit the same.

`with_gpu_libm(run)` calls `run()` once recording the oracle's library-call
inputs, evaluates them on the GPU (one-clause tapes through the C ABI), and
calls `run()` again replaying those results; inputs the replayed run meets
for the first time (its control flow can change) are added and the run
repeated, until none is missing.
"""
import numpy as np

import oracle_ffi
from libfive_b200.shape import Shape, Tape

# opcode value -> stdlib name (libfive/include/libfive/tree/opcode.hpp)
LIBM_OPS = {10: "sin", 11: "cos", 12: "tan", 13: "asin", 14: "acos", 15: "atan",
            16: "exp", 30: "log"}


def _gpu_results(keys):
    ops = (keys >> np.uint64(32)).astype(np.int64)
    xs = (keys & np.uint64(0xffffffff)).astype(np.uint32).view(np.float32)
    out = np.empty(len(keys), np.uint32)
    for op in np.unique(ops):
        sel = ops == op
        x = np.ascontiguousarray(xs[sel])
        z = np.zeros_like(x)
        v = Tape(Shape.new(LIBM_OPS[int(op)], Shape.X())).values(x, z, z)
        out[sel] = v.view(np.uint32)
    return out


def _take(lib):
    n = lib.ora_libm_take(None, 0)
    keys = np.zeros(n, np.uint64)
    if n:
        lib.ora_libm_take(keys.ctypes.data, n)
    return keys


def with_gpu_libm(run, max_rounds=8):
    """run() with the oracle's library calls answered by the GPU; returns
    run()'s result from a replay that missed no input."""
    lib = oracle_ffi.load()
    table_k = np.zeros(0, np.uint64)
    table_v = np.zeros(0, np.uint32)
    try:
        lib.ora_libm_mode(1)
        run()
        new = _take(lib)
        for _ in range(max_rounds):
            if len(new):
                table_k = np.concatenate([table_k, new])
                table_v = np.concatenate([table_v, _gpu_results(new)])
                table_k = np.ascontiguousarray(table_k)
                table_v = np.ascontiguousarray(table_v)
                lib.ora_libm_table(table_k.ctypes.data, table_v.ctypes.data, len(table_k))
            lib.ora_libm_mode(2)
            out = run()
            if lib.ora_libm_misses() == 0:
                return out
            new = np.setdiff1d(_take(lib), table_k)
        raise AssertionError("library-call replay did not settle")
    finally:
        lib.ora_libm_mode(0)
