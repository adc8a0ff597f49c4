"""Adam restated in float32 numpy, operation by operation as
lfb_fit_adam_step's update kernel does it (test infrastructure: the checker
of the fit step, pinned against torch.optim.Adam by test_fit_host.py)."""
import math

import numpy as np

f32 = np.float32


def adam_step(params, grad, m, v, t, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8):
    """One step; returns new (params, m, v), all float32 arrays."""
    params, grad, m, v = (np.asarray(a, f32) for a in (params, grad, m, v))
    one_minus_b1 = f32(1.0) - f32(beta1)
    one_minus_b2 = f32(1.0) - f32(beta2)
    step_size = f32(float(f32(lr)) / (1.0 - float(f32(beta1)) ** t))
    bc2_sqrt = f32(math.sqrt(1.0 - float(f32(beta2)) ** t))
    m = m + one_minus_b1 * (grad - m)
    v = v * f32(beta2) + (one_minus_b2 * grad) * grad
    denom = np.sqrt(v) / bc2_sqrt + f32(eps)
    params = params + (-step_size) * (m / denom)
    return params.astype(f32), m.astype(f32), v.astype(f32)
