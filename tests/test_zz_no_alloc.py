"""lfb_eval_derivs_static: the evaluation entry point that allocates no
device memory.

It exists for callers that cannot call cudaMalloc while they run (a frame
loop that must not synchronise the device, or an application whose own
allocator owns all device memory).  It stages points through a fixed array
in the library instead of allocating, so it must give exactly what the
allocating entry point (lfb_eval_derivs) gives, call after call, and must
refuse batches larger than that array.

This file is named to be collected last, so that a run stopping at the first
failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

from libfive_b200 import ffi, workloads
from libfive_b200.shape import Tape

pytestmark = pytest.mark.gpu

MAX_POINTS = 262144


def _static(lib, tape, P):
    n = len(P[0])
    outs = [np.full(n, np.nan, np.float32) for _ in range(4)]
    rc = lib.lfb_eval_derivs_static(tape.ptr, n, *(p.ctypes.data for p in P),
                                    *(o.ctypes.data for o in outs))
    return rc, outs


def test_matches_allocating_entry_on_consecutive_calls(gpu):
    """Two calls in a row on a fresh tape: the first runs the interpreter
    (nothing compiled for the tape yet, and the static path never compiles),
    the second the compiled kernel that lfb_eval_derivs loaded in between.
    The compiled kernel and the interpreter give the same bits, so both
    calls must equal lfb_eval_derivs exactly (tolerance 0)."""
    lib = ffi.load()
    tape = Tape(workloads.spheres_union(32, seed=1))
    for call, n in enumerate([MAX_POINTS, 1000]):
        P = workloads.uniform_points(n, seed=10 + call)
        rc, got = _static(lib, tape, P)
        assert rc == 0, ffi.last_error()
        want = tape.derivs(*P)
        for a, b in zip(got, want):
            assert np.array_equal(a, b)


def test_rejects_batches_beyond_the_fixed_buffer(gpu):
    lib = ffi.load()
    tape = Tape(workloads.sphere((0, 0, 0), 0.5))
    P = workloads.uniform_points(MAX_POINTS + 1, seed=3)
    rc, _ = _static(lib, tape, P)
    assert rc == -1
    assert "262144" in ffi.last_error()[1]
