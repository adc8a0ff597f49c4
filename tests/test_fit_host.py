"""Host side of the batched fit: the Adam restatement that checks
lfb_fit_adam_step against torch.optim.Adam, and the fitting workload's
generators (no GPU)."""
import numpy as np
import torch

from adam_ref import adam_step
from libfive_b200 import workloads


def test_adam_restatement_matches_torch_adam():
    rng = np.random.default_rng(5)
    p0 = rng.normal(size=300).astype(np.float32)
    grads = [rng.normal(scale=10.0 ** rng.uniform(-6, 1), size=300).astype(np.float32)
             for _ in range(6)]
    for lr, betas, eps in [(1e-3, (0.9, 0.999), 1e-8), (0.05, (0.5, 0.9), 1e-6)]:
        p = torch.tensor(p0, requires_grad=True)
        opt = torch.optim.Adam([p], lr=lr, betas=betas, eps=eps, foreach=False)
        q, m, v = p0.copy(), np.zeros(300, np.float32), np.zeros(300, np.float32)
        for t, g in enumerate(grads, start=1):
            p.grad = torch.tensor(g)
            opt.step()
            q, m, v = adam_step(q, g, m, v, t, lr, betas[0], betas[1], eps)
            np.testing.assert_allclose(q, p.detach().numpy(), rtol=2e-6, atol=1e-7)


def test_fit_workload_has_seven_variables_per_primitive():
    shape, values, order = workloads.fit_csg_vars(128, seed=21)
    assert len(values) == len(order) == 896
    again = workloads.fit_csg_vars(128, seed=21)[1]
    assert list(values.values()) == list(again.values())


def test_perturbation_is_seeded_gaussian():
    values = {i: 0.0 for i in range(20000)}
    a = np.array(list(workloads.perturbed(values, 0.05, seed=3).values()))
    b = np.array(list(workloads.perturbed(values, 0.05, seed=3).values()))
    assert np.array_equal(a, b)
    assert abs(a.mean()) < 3 * 0.05 / np.sqrt(len(a))
    assert abs(a.std() - 0.05) < 0.002


def test_surface_points_lie_on_the_mesh():
    # unit square in z = 0.25 as two triangles
    verts = np.array([[0, 0, 0.25], [1, 0, 0.25], [1, 1, 0.25], [0, 1, 0.25]], np.float32)
    tris = np.array([[0, 1, 2], [0, 2, 3]], np.uint32)
    x, y, z = workloads.surface_points(verts, tris, 4000, seed=1)
    assert np.all(z == np.float32(0.25))
    assert np.all((x >= 0) & (x <= 1) & (y >= 0) & (y <= 1))
    # area-uniform: both triangles get about half the points
    assert abs(np.mean(y < x) - 0.5) < 0.05


def test_reverse_mode_ops_follow_the_tape():
    # sqrt(x^2 + y^2) - 0.5: per clause twice its value weight (forward and
    # local partials) and a multiply-add per operand: square 2 + 2 (x2),
    # add 2 + 4, sqrt 2 + 2, sub 2 + 4
    import bench
    from libfive_b200.shape import X, Y
    shape = (X().square() + Y().square()).sqrt() - 0.5
    assert bench.reverse_mode_ops_per_point(shape) == 2 * 4 + 6 + 4 + 6
    # library calls count 20 each
    assert bench.reverse_mode_ops_per_point(X().sin()) == 2 * 20 + 2
