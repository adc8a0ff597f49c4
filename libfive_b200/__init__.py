"""libfive_b200: libfive's evaluate-and-mesh path on NVIDIA B200.

The C ABI (include/libfive.h, include/libfive_b200.h) lives in
lib/libfive.so, built by `python -m libfive_b200.build`.  This package adds a
Python mirror of the reference's Shape class and the batched GPU tapes;
`libfive_b200.autograd` (a differentiable torch operation) and
`libfive_b200.fit` (batched Adam fitting of free variables) need torch and
are imported on their own.
"""
from . import ffi  # noqa: F401
from .shape import Shape, Tape, mesh_arrays, slot_tape  # noqa: F401
