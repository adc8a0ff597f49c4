"""torch.autograd binding of the batched GPU tapes.

`shape_value(tape, x, y, z, vars=None)` returns f at the points (CUDA float32
tensors of one shape) and is differentiable with respect to the point
coordinates and, when given, to the free variables (`vars`: a 1-D CUDA
float32 tensor of the tape's variables in `tape.var_ids()` order).  The
forward pass is lfb_eval_values, the backward pass the reverse-mode
lfb_eval_grad: one launch pair per call, no CPU work on the data (the
variables are copied device to device into the tape on the current stream).
"""
import torch

from . import ffi
from .shape import Tape


def _stream():
    return torch.cuda.current_stream().cuda_stream


class _ShapeValue(torch.autograd.Function):
    @staticmethod
    def forward(ctx, tape, x, y, z, vars_):
        if vars_ is not None:
            v = vars_.detach().to(torch.float32).contiguous()
            if v.numel() != tape.n_vars or not v.is_cuda:
                raise ValueError("vars must be a CUDA tensor of the tape's %d variables"
                                 % tape.n_vars)
            ffi.check(ffi.load().lfb_tape_set_vars_device(tape.ptr, v.data_ptr(), v.numel(),
                                                          _stream()), "set_vars_device")
        x, y, z = (t.detach().contiguous() for t in (x, y, z))
        f = torch.empty_like(x)
        tape.values(x, y, z, out=f, stream=_stream())
        ctx.tape = tape
        ctx.has_vars = vars_ is not None
        ctx.save_for_backward(x, y, z)
        return f

    @staticmethod
    def backward(ctx, grad_f):
        x, y, z = ctx.saved_tensors
        tape = ctx.tape
        seed = grad_f.detach().contiguous()
        need = ctx.needs_input_grad
        gx = torch.empty_like(x) if need[1] else None
        gy = torch.empty_like(x) if need[2] else None
        gz = torch.empty_like(x) if need[3] else None
        gv = None
        if ctx.has_vars and need[4]:
            gv = torch.zeros(tape.n_vars, dtype=torch.float32, device=x.device)
        if gx is not None or gy is not None or gz is not None or gv is not None:
            tape.grad(x, y, z, seed=seed, gx=gx, gy=gy, gz=gz, gvars=gv, stream=_stream())
        return None, gx, gy, gz, gv


def shape_value(tape: Tape, x, y, z, vars=None):
    """f(x, y, z) of a Tape as a differentiable torch operation."""
    return _ShapeValue.apply(tape, x, y, z, vars)
