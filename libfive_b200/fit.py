"""Batched least-squares fitting of many shapes' free variables on the GPU.

`BatchedFit(tapes, points)` fits each Tape's free variables so that its
shape passes through its own points (CUDA float32 tensors x, y, z per
shape): loss_j = mean f_j(p)^2, one Adam step of every shape per `step()`
call through lfb_fit_adam_step (reverse-mode gradients, loss and update on
the device; the variables stay in the tapes' device constant pools, where
evaluation and meshing read them).  The reference has no optimiser; its
closest piece is JacobianEvaluator (libfive/src/eval/eval_jacobian.cpp
:49-115), which gives df/dvar one point at a time.
"""
import ctypes

import numpy as np
import torch

from . import ffi


class BatchedFit:
    def __init__(self, tapes, points, lr=1e-3, betas=(0.9, 0.999), eps=1e-8):
        if len(tapes) != len(points) or not tapes:
            raise ValueError("one (x, y, z) per tape, at least one tape")
        self.tapes = list(tapes)
        dev = points[0][0].device
        self.x, self.y, self.z = (torch.cat([p[a].reshape(-1).float() for p in points])
                                  .contiguous() for a in range(3))
        counts = [int(p[0].numel()) for p in points]
        self.point_offsets = np.concatenate([[0], np.cumsum(counts)]).astype(np.uint64)
        nv = [t.n_vars for t in self.tapes]
        self.var_offsets = np.concatenate([[0], np.cumsum(nv)]).astype(np.uint64)
        n_vars = int(self.var_offsets[-1])
        self.m = torch.zeros(max(1, n_vars), dtype=torch.float32, device=dev)
        self.v = torch.zeros(max(1, n_vars), dtype=torch.float32, device=dev)
        self.losses = torch.empty(len(tapes), dtype=torch.float32, device=dev)
        self.settings = ffi.AdamSettings(lr, betas[0], betas[1], eps)
        self.t = 0
        self._ptrs = (ctypes.c_void_p * len(tapes))(*[t.ptr for t in self.tapes])

    @property
    def n_points(self):
        return int(self.point_offsets[-1])

    @property
    def n_vars(self):
        return int(self.var_offsets[-1])

    def step(self, stream=None):
        """One Adam step of every shape; returns the device tensor of losses
        at the values before the step (valid once the stream reaches it)."""
        self.t += 1
        s = torch.cuda.current_stream().cuda_stream if stream is None else stream
        u64 = ctypes.POINTER(ctypes.c_uint64)
        ffi.check(ffi.load().lfb_fit_adam_step(
            self._ptrs, len(self.tapes), self.point_offsets.ctypes.data_as(u64),
            self.x.data_ptr(), self.y.data_ptr(), self.z.data_ptr(),
            self.var_offsets.ctypes.data_as(u64), self.m.data_ptr(), self.v.data_ptr(),
            self.settings, self.t, self.losses.data_ptr(), s), "fit step")
        return self.losses

    def values(self):
        """Each tape's current variable values (host arrays)."""
        return [t.get_vars() for t in self.tapes]
