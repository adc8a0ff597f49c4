"""The oracle's library-call record / replay hook (used to check whole tapes
and meshes bit for bit against the GPU with the GPU's exp / log results),
exercised on the CPU with a stand-in table."""
import numpy as np

import oracle_ffi
from libfive_b200 import workloads
from libfive_b200.shape import Shape
from oracle_ffi import OracleTape


def _take(lib):
    n = lib.ora_libm_take(None, 0)
    keys = np.zeros(n, np.uint64)
    if n:
        lib.ora_libm_take(keys.ctypes.data, n)
    return keys


def test_record_then_replay_uses_the_table():
    lib = oracle_ffi.load()
    x = np.linspace(-3, 3, 1001).astype(np.float32)
    z = np.zeros_like(x)
    t = OracleTape(Shape.X().exp() + Shape.X().log())
    plain = t.values(x, z, z)
    try:
        lib.ora_libm_mode(1)
        assert np.array_equal(t.values(x, z, z), plain, equal_nan=True)
        keys = _take(lib)
        ops = (keys >> np.uint64(32)).astype(np.int64)
        assert set(ops.tolist()) == {16, 30}          # EXP, LOG
        assert len(keys) == 2 * len(np.unique(x))
        # stand-in results: one ULP above the C library's
        xs = (keys & np.uint64(0xffffffff)).astype(np.uint32).view(np.float32)
        host = np.where(ops == 16, np.exp(xs.astype(np.float64)),
                        np.log(np.where(xs > 0, xs, np.nan).astype(np.float64)))
        host = host.astype(np.float32)
        vals = np.nextafter(host, np.float32(np.inf)).view(np.uint32)
        keys = np.ascontiguousarray(keys)
        vals = np.ascontiguousarray(vals)
        lib.ora_libm_table(keys.ctypes.data, vals.ctypes.data, len(keys))
        lib.ora_libm_mode(2)
        got = t.values(x, z, z)
        assert lib.ora_libm_misses() == 0
        e = np.nextafter(np.exp(x.astype(np.float64)).astype(np.float32), np.float32(np.inf))
        lg = np.log(np.where(x > 0, x, np.nan).astype(np.float64)).astype(np.float32)
        want = e + np.nextafter(lg, np.float32(np.inf))
        assert np.array_equal(got, want, equal_nan=True)
        # an input outside the table falls back to the C library and is counted
        y = np.array([7.25], np.float32)
        t.values(y, y * 0, y * 0)
        assert lib.ora_libm_misses() == 2
    finally:
        lib.ora_libm_mode(0)
    assert np.array_equal(t.values(x, z, z), plain, equal_nan=True)


def test_replay_covers_derivatives_and_threads():
    lib = oracle_ffi.load()
    s = workloads.random_csg(40, seed=3)
    P = workloads.uniform_points(20000, seed=4)
    t = OracleTape(s)
    plain = t.derivs(*P, threads=4)
    try:
        lib.ora_libm_mode(1)
        t.derivs(*P, threads=4)
        keys = _take(lib)
        assert len(keys) > 0
        xs = (keys & np.uint64(0xffffffff)).astype(np.uint32).view(np.float32)
        ops = (keys >> np.uint64(32)).astype(np.int64)
        # the C library's own results: replay must reproduce the plain run
        one = np.zeros(1, np.float32)
        vals = np.empty(len(keys), np.float32)
        for i, (op, v) in enumerate(zip(ops, xs)):
            sh = Shape.X().exp() if op == 16 else Shape.X().log()
            vals[i] = OracleTape(sh).values(np.array([v], np.float32), one, one)[0]
        keys = np.ascontiguousarray(keys)
        vb = np.ascontiguousarray(vals.view(np.uint32))
        lib.ora_libm_table(keys.ctypes.data, vb.ctypes.data, len(keys))
        lib.ora_libm_mode(2)
        again = t.derivs(*P, threads=4)
        assert lib.ora_libm_misses() == 0
    finally:
        lib.ora_libm_mode(0)
    for a, b in zip(plain, again):
        assert np.array_equal(a, b, equal_nan=True)
