"""lfb_fit_adam_step against its parts: the loss against mean f^2 of
lfb_eval_values, and each Adam step against the Adam restatement
(adam_ref.py, pinned to torch.optim.Adam) applied to the reverse-mode
gradient of lfb_eval_grad.  The gradient sums variable adjoints with
atomics, so the comparison has a tolerance; variables whose gradient is
tiny next to the shape's largest may take Adam's first step with either
sign and are only held to the step size."""
import ctypes

import numpy as np
import pytest
import torch

from adam_ref import adam_step
from libfive_b200 import ffi, workloads
from libfive_b200.fit import BatchedFit
from libfive_b200.shape import Tape
from mesh_compare import same_mesh

pytestmark = pytest.mark.gpu

LR = 1e-2
REGION = ((-1.5,) * 3, (1.5,) * 3)


def _problem(seed, n_prims, n_points):
    """(shape, initial values, host points on the perturbed copy's surface)."""
    shape, vals, _ = workloads.fit_csg_vars(n_prims, seed=seed)
    target = Tape(shape, workloads.perturbed(vals, 0.05, seed=seed + 1))
    verts, tris = target.render_mesh(*REGION, 1.0 / 32)
    assert len(tris) > 0
    return shape, vals, workloads.surface_points(verts, tris, n_points, seed=seed + 2)


def _ref_grad(shape, ids, values, pts):
    """f at the points and the gradient of mean f^2 (float32), through a
    separate tape."""
    t = Tape(shape, dict(zip(ids, values.tolist())))
    f = t.values(*pts)
    gv = np.zeros(t.n_vars, np.float32)
    t.grad(*pts, seed=f, gvars=gv)
    return f, gv * np.float32(2.0 / len(f))


def _check_params(got, want, g, lr):
    big = np.abs(g) > 1e-3 * np.abs(g).max()
    np.testing.assert_allclose(got[big], want[big], rtol=1e-5, atol=1e-6)
    assert np.all(np.abs(got - want) <= 2 * lr + 1e-6)


@pytest.fixture(scope="module")
def problems():
    return [_problem(31, 8, 3000), _problem(41, 12, 5000), _problem(51, 16, 1234)]


def _fit(problems, lr=LR):
    tapes = [Tape(s, v) for s, v, _ in problems]
    pts = [tuple(torch.from_numpy(a).cuda() for a in p) for _, _, p in problems]
    return tapes, BatchedFit(tapes, pts, lr=lr)


def test_two_steps_match_gradient_and_adam(gpu, problems):
    tapes, fit = _fit(problems)
    ids = [t.var_ids() for t in tapes]
    p0 = [t.get_vars() for t in tapes]
    losses = fit.step().cpu().numpy()
    torch.cuda.synchronize()
    m_ref, v_ref = [], []
    for j, (shape, _, pts) in enumerate(problems):
        f, g = _ref_grad(shape, ids[j], p0[j], pts)
        np.testing.assert_allclose(losses[j], np.mean(f.astype(np.float64) ** 2), rtol=1e-5)
        z = np.zeros_like(g)
        want, m1, v1 = adam_step(p0[j], g, z, z, 1, lr=LR)
        _check_params(tapes[j].get_vars(), want, g, LR)
        m_ref.append(m1)
        v_ref.append(v1)
    # second step from the values and moments the first one left
    p1 = [t.get_vars() for t in tapes]
    m_dev, v_dev = fit.m.cpu().numpy(), fit.v.cpu().numpy()
    losses = fit.step().cpu().numpy()
    for j, (shape, _, pts) in enumerate(problems):
        a, b = int(fit.var_offsets[j]), int(fit.var_offsets[j + 1])
        f, g = _ref_grad(shape, ids[j], p1[j], pts)
        np.testing.assert_allclose(losses[j], np.mean(f.astype(np.float64) ** 2), rtol=1e-5)
        want, m2, v2 = adam_step(p1[j], g, m_dev[a:b], v_dev[a:b], 2, lr=LR)
        _check_params(tapes[j].get_vars(), want, g, LR)
        big = np.abs(g) > 1e-3 * np.abs(g).max()
        np.testing.assert_allclose(fit.m.cpu().numpy()[a:b][big], m2[big], rtol=1e-4, atol=1e-9)
        np.testing.assert_allclose(fit.v.cpu().numpy()[a:b][big], v2[big], rtol=1e-4, atol=1e-12)


def test_fitted_values_reach_evaluation_and_meshing(gpu, problems):
    tapes, fit = _fit(problems[:2])
    for _ in range(3):
        fit.step()
    torch.cuda.synchronize()
    for t, (shape, _, pts) in zip(tapes, problems):
        fresh = Tape(shape, dict(zip(t.var_ids(), t.get_vars().tolist())))
        assert np.array_equal(t.values(*pts), fresh.values(*pts))
        # vertex numbering varies from run to run: compare triangle sets
        va, ta = t.render_mesh(*REGION, 1.0 / 16)
        vb, tb = fresh.render_mesh(*REGION, 1.0 / 16)
        assert len(ta) > 0 and len(va) == len(vb) and same_mesh(va, ta, vb, tb)


def test_set_vars_after_fit_keeps_fitted_values(gpu, problems):
    tapes, fit = _fit(problems[:1])
    fit.step()
    t = tapes[0]
    before = t.get_vars()
    ids = t.var_ids()
    t.set_vars({ids[0]: 0.125})
    after = t.get_vars()
    assert after[0] == np.float32(0.125)
    assert np.array_equal(after[1:], before[1:])


def test_loss_falls_over_a_short_fit(gpu, problems):
    tapes, fit = _fit(problems[:1], lr=5e-3)
    hist = [float(fit.step().cpu()[0]) for _ in range(40)]
    assert min(hist[-5:]) < hist[0]


def test_rejects_inconsistent_arguments(gpu, problems):
    lib = ffi.load()
    tapes, fit = _fit(problems[:2])
    u64 = ctypes.POINTER(ctypes.c_uint64)

    def call(ptrs, voff, step=1):
        return lib.lfb_fit_adam_step(
            ptrs, len(ptrs), fit.point_offsets.ctypes.data_as(u64), fit.x.data_ptr(),
            fit.y.data_ptr(), fit.z.data_ptr(), voff.ctypes.data_as(u64), fit.m.data_ptr(),
            fit.v.data_ptr(), fit.settings, step, fit.losses.data_ptr(), None)

    ptrs = (ctypes.c_void_p * 2)(tapes[0].ptr, tapes[1].ptr)
    bad = fit.var_offsets.copy()
    bad[1] += 1
    assert call(ptrs, bad) == -1
    assert "variables" in ffi.last_error()[1]
    twice = (ctypes.c_void_p * 2)(tapes[0].ptr, tapes[0].ptr)
    same = np.array([0, tapes[0].n_vars, 2 * tapes[0].n_vars], np.uint64)
    assert call(twice, same) == -1
    assert "twice" in ffi.last_error()[1]
    assert call(ptrs, fit.var_offsets, step=0) == -1
