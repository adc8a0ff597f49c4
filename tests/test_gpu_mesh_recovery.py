"""Cancellation (BRepSettings::cancel, libfive/include/libfive/render/brep/
settings.hpp:73, tested by libfive/test/xtree.cpp:240-272) and the mesher's
recovery paths, driven from the host: a cancel flag set before or during a
mesh, capacities forced to their minimum (every tape-arena, list and
dual-walk growth retry runs) and device allocations made to fail
(lfb_debug_set).  No GPU fault is involved: the failures are made on the
host and every call must end with a clean status or the unforced mesh."""
import ctypes
import threading
import time

import numpy as np
import pytest

from libfive_b200 import ffi, workloads
from libfive_b200.shape import Tape, mesh_arrays
from mesh_compare import same_mesh

pytestmark = pytest.mark.gpu

LO, HI = (-1.5, -1.5, -1.5), (1.5, 1.5, 1.5)
REGION = ffi.Region3(*[ffi.Interval(a, b) for a, b in zip(LO, HI)])


def render(tape, mf, cancel=None):
    lib = ffi.load()
    flag = ctypes.pointer(cancel) if cancel is not None else None
    st = ffi.MeshStats()
    m = lib.lfb_render_mesh(tape.ptr, REGION, ffi.MeshSettings(mf, 1e-8, flag), ctypes.byref(st))
    if not m:
        return None, ffi.last_error()
    v, t = mesh_arrays(m)
    return (v, t), None


@pytest.fixture
def hooks():
    lib = ffi.load()
    yield lib
    lib.lfb_debug_set(b"fail_alloc_after", 0)
    lib.lfb_debug_set(b"small_capacity", 0)


def test_cancel_before_start(gpu):
    tape = Tape(workloads.spheres_union(16, seed=1))
    flag = ctypes.c_int32(1)
    mesh, err = render(tape, 0.05, flag)
    assert mesh is None and err[0] == -5     # LFB_E_CANCELLED
    flag.value = 0
    mesh, err = render(tape, 0.05, flag)
    assert mesh is not None, err
    want, _ = render(tape, 0.05)
    assert same_mesh(*mesh, *want)


def test_cancel_during_a_mesh(gpu):
    """The 2000-primitive benchmark tree at depth 10 (tens of ms on the GPU):
    a flag raised from another thread stops it within 150 ms (the
    reference's bound in xtree.cpp:240-272), or the mesh was already done."""
    tape = Tape(workloads.random_csg(2000, seed=2))
    render(tape, 3.0 / 1000)     # warm: buffers and kernels ready
    flag = ctypes.c_int32(0)
    raised = {}

    def raise_flag():
        time.sleep(0.005)
        raised["t"] = time.perf_counter()
        flag.value = 1

    th = threading.Thread(target=raise_flag)
    th.start()
    mesh, err = render(tape, 3.0 / 1000, flag)
    done = time.perf_counter()
    th.join()
    if mesh is None:
        assert err[0] == -5, err
        assert done - raised["t"] < 0.150
    # the library is usable afterwards
    flag.value = 0
    again, err = render(tape, 3.0 / 1000, flag)
    assert again is not None, err


@pytest.mark.parametrize("seed,mf", [(1, 0.05), (5, 0.02)])
def test_minimal_capacities_give_the_same_mesh(gpu, hooks, seed, mf):
    tape = Tape(workloads.random_csg(200, seed=seed))
    want, err = render(tape, mf)
    assert want is not None, err
    hooks.lfb_debug_set(b"small_capacity", 1)
    got, err = render(tape, mf)
    assert got is not None, err
    assert same_mesh(*got, *want)
    assert len(got[0]) == len(want[0])


def test_allocation_failures_end_cleanly(gpu, hooks):
    tape = Tape(workloads.spheres_union(16, seed=3))
    want, err = render(tape, 0.05)
    assert want is not None, err
    hooks.lfb_debug_set(b"small_capacity", 1)
    failures = 0
    for k in range(1, 200):
        hooks.lfb_debug_set(b"fail_alloc_after", k)
        got, err = render(tape, 0.05)
        hooks.lfb_debug_set(b"fail_alloc_after", 0)
        if got is None:
            failures += 1
            assert err[0] == -3 and "injected" in err[1], err
            # the next call, without injection, is whole
            again, err2 = render(tape, 0.05)
            assert again is not None, err2
            assert same_mesh(*again, *want)
        else:
            # k is past the allocations of one mesh: nothing failed
            assert same_mesh(*got, *want)
            break
    assert failures >= 5


def test_batch_retries_a_mesh_that_ran_out_of_memory(gpu, hooks):
    lib = hooks
    shapes = [workloads.spheres_union(8 + 4 * i, seed=i) for i in range(4)]
    tapes = [Tape(s) for s in shapes]
    wants = [render(t, 0.05)[0] for t in tapes]
    n = len(tapes)
    b_tapes = (ffi.tape_t * n)(*[t.ptr for t in tapes])
    b_regions = (ffi.Region3 * n)(*[REGION] * n)
    b_settings = (ffi.MeshSettings * n)(*[ffi.MeshSettings(0.05, 1e-8, None)] * n)
    lib.lfb_debug_set(b"small_capacity", 1)
    lib.lfb_debug_set(b"fail_alloc_after", 6)
    meshes = (ctypes.POINTER(ffi.Mesh) * n)()
    rc = lib.lfb_render_meshes(b_tapes, n, b_regions, b_settings, 2, meshes, None)
    lib.lfb_debug_set(b"fail_alloc_after", 0)
    assert rc == 0, ffi.last_error()
    for m, want in zip(meshes, wants):
        assert m
        assert same_mesh(*mesh_arrays(m), *want)   # mesh_arrays frees the mesh
