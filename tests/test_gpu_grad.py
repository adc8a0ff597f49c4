"""Gradients with respect to free variables (JacobianEvaluator::gradient,
libfive/test/eval_jacobian.cpp) and the reverse-mode gradient, through the
C ABI against the CPU oracle."""
import json
import os

import numpy as np
import pytest

from libfive_b200 import workloads
from libfive_b200.shape import Shape, Tape
from libm_replay import with_gpu_libm
from oracle_ffi import OracleTape
from sexpr import parse

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
KATS = json.load(open(os.path.join(HERE, "golden", "eval_kats.json")))
X, Y, Z = Shape.X, Shape.Y, Shape.Z


def pts(*p):
    return [np.array([float(a)], np.float32) for a in p]


def var_index(tape):
    return {vid: i for i, vid in enumerate(tape.var_ids())}


@pytest.mark.parametrize("e", KATS["jacobian"], ids=lambda e: e["src"] + str(e["p"]))
def test_jacobian_kats(gpu, e):
    vars_ = {}
    t = parse(e["expr"], vars_)
    tape = Tape(t, {vars_[k]: v for k, v in e["vars"].items()})
    j = tape.jacobian(*pts(*e["p"]))[0]
    idx = var_index(tape)
    for name, want in e["want"].items():
        assert abs(j[idx[vars_[name].id()]] - want) <= e["tol"]


def test_jacobian_dependency_on_xyz(gpu):
    # eval_jacobian.cpp:95-113
    a, b, c = Shape.var(), Shape.var(), Shape.var()
    tape = Tape(a * X() + b * Y() + c * Z(), {a: 3, b: 7, c: 5})
    j = tape.jacobian(*pts(1, 2, 4))[0]
    idx = var_index(tape)
    assert [j[idx[v.id()]] for v in (a, b, c)] == [1.0, 2.0, 4.0]
    v, dx, dy, dz = tape.derivs(*pts(0, 0, 0))
    assert (dx[0], dy[0], dz[0]) == (3.0, 7.0, 5.0)


def test_jacobian_const_var(gpu):
    # eval_jacobian.cpp:115-124: CONST_VAR blocks the gradient
    vars_ = {}
    tape = Tape(parse("(const-var (+ v 1))", vars_), {vars_["v"]: 3.14})
    j = tape.jacobian(*pts(1, 2, 3))
    assert j.shape == (1, 1) and j[0, 0] == 0.0


def test_jacobian_1024_vars(gpu):
    # eval_jacobian.cpp:63-93: pairwise sum of v_i * i; v_0 * 0 folds away
    vs = [Shape.var() for _ in range(1024)]
    ts = [v * float(i) for i, v in enumerate(vs)]
    while len(ts) > 1:
        ts = [ts[k + 1] + ts[k] for k in range(0, len(ts), 2)]
    tape = Tape(ts[0], {v: float(i) for i, v in enumerate(vs)})
    assert tape.n_vars == 1023
    j = tape.jacobian(*pts(0, 0, 0))[0]
    idx = var_index(tape)
    for i, v in enumerate(vs[1:], start=1):
        assert j[idx[v.id()]] == float(i)


def sphere_vars(n, seed):
    """Union of n spheres with free centres and radii (exact ops only)."""
    rng = workloads.SplitMix64(seed)
    vals, out = {}, None
    for _ in range(n):
        cx, cy, cz, r = Shape.var(), Shape.var(), Shape.var(), Shape.var()
        for v, lo, hi in ((cx, -1, 1), (cy, -1, 1), (cz, -1, 1), (r, 0.1, 0.35)):
            vals[v] = rng.uniform(lo, hi)
        s = ((X() - cx).square() + (Y() - cy).square() + (Z() - cz).square()).sqrt() - r
        out = s if out is None else out.min(s)
    return out, vals


def test_jacobian_matches_oracle_exact_ops(gpu):
    s, vals = sphere_vars(12, seed=7)
    x, y, z = workloads.uniform_points(3000, seed=5)
    j = Tape(s, vals).jacobian(x, y, z)
    o = OracleTape(s, vals).jacobian(x, y, z)
    assert np.array_equal(j, o)


def test_jacobian_matches_oracle_blends(gpu):
    s, vals = workloads.blended_spheres_vars(16, seed=4)
    x, y, z = workloads.uniform_points(2000, seed=6, lo=-1.2, hi=1.2)
    j = Tape(s, vals).jacobian(x, y, z)
    o = OracleTape(s, vals).jacobian(x, y, z)
    ok = np.isfinite(o)
    assert np.array_equal(ok, np.isfinite(j))
    # CUDA's expf/logf differ from the C library's by a few ULPs
    assert np.allclose(j[ok], o[ok], rtol=1e-4, atol=1e-5)
    # with the GPU's exp / log results, the oracle's forward Jacobian is the
    # GPU's bit for bit
    ora = OracleTape(s, vals)
    o2 = with_gpu_libm(lambda: ora.jacobian(x, y, z))
    assert np.array_equal(j, o2, equal_nan=True)


@pytest.mark.parametrize("maker", ["spheres", "blends"])
def test_reverse_gradient_matches_forward(gpu, maker):
    n = 4096
    if maker == "spheres":
        s, vals = sphere_vars(12, seed=9)
        x, y, z = workloads.uniform_points(n, seed=11, lo=-1.2, hi=1.2)
    else:
        s, vals = workloads.blended_spheres_vars(16, seed=8, stable=True)
        x, y, z = workloads.uniform_points(n, seed=11, lo=-1.2, hi=1.2)
    seed = np.random.default_rng(3).uniform(-1, 1, n).astype(np.float32)
    tape = Tape(s, vals)
    f = np.empty(n, np.float32)
    gx, gy, gz = (np.empty(n, np.float32) for _ in range(3))
    gvars = np.zeros(tape.n_vars, np.float32)
    tape.grad(x, y, z, seed=seed, f=f, gx=gx, gy=gy, gz=gz, gvars=gvars)
    ora = OracleTape(s, vals)
    ov, odx, ody, odz = ora.derivs(x, y, z)
    assert np.array_equal(f, tape.values(x, y, z))
    keep = np.isfinite(odx) & np.isfinite(ody) & np.isfinite(odz)
    for g, od in ((gx, odx), (gy, ody), (gz, odz)):
        assert np.allclose(g[keep], seed[keep] * od[keep], rtol=1e-4, atol=1e-5)
    # Variable gradients: points whose Jacobian row is finite (blends
    # overflow deep inside a shape, and a non-finite local partial makes the
    # whole sum non-finite), run again on their own.
    jac = ora.jacobian(x, y, z).astype(np.float64)
    rows = np.isfinite(jac).all(axis=1) & np.isfinite(ov)
    assert rows.sum() >= n // 4
    xs, ys, zs, ss = (np.ascontiguousarray(a[rows]) for a in (x, y, z, seed))
    gvars = np.zeros(tape.n_vars, np.float32)
    tape.grad(xs, ys, zs, seed=ss, gvars=gvars)
    want = ss.astype(np.float64) @ jac[rows]
    scale = np.abs(ss[:, None] * jac[rows]).sum(axis=0) + 1e-6
    assert np.all(np.abs(gvars - want) <= 1e-4 * scale)


def test_reverse_gradient_blended_spheres_256_chunked(gpu):
    """The adjoint configuration's shape (256 spheres blended pairwise, 1024
    free variables; the blend in its overflow-free form, so that gradients
    are finite everywhere) over more points than one 4 GiB partials chunk
    holds at this tape's stored partials per point: 2048 points, each
    repeated, so the summed variable gradient is 512 times that of the 2048
    and the per-point gradients repeat the oracle's derivatives."""
    s, vals = workloads.blended_spheres_vars(256, seed=4, stable=True)
    tape = Tape(s, vals)
    assert tape.n_vars == 1024
    ora = OracleTape(s, vals)
    cx, cy, cz = workloads.uniform_points(8192, seed=21, lo=-1.2, hi=1.2)
    ov, odx, ody, odz = ora.derivs(cx, cy, cz, threads=8)
    fin = np.isfinite(ov) & np.isfinite(odx) & np.isfinite(ody) & np.isfinite(odz)
    idx = np.flatnonzero(fin)[:2048]
    assert len(idx) == 2048
    bx, by, bz = (np.ascontiguousarray(a[idx]) for a in (cx, cy, cz))
    jac = ora.jacobian(bx, by, bz, threads=8).astype(np.float64)
    assert np.isfinite(jac).all()
    bseed = np.random.default_rng(5).uniform(-1, 1, 2048).astype(np.float32)
    reps = 512
    x, y, z, seed = (np.ascontiguousarray(np.tile(a, reps)) for a in (bx, by, bz, bseed))
    n = len(x)
    f = np.empty(n, np.float32)
    gx, gy, gz = (np.empty(n, np.float32) for _ in range(3))
    gvars = np.zeros(1024, np.float32)
    tape.grad(x, y, z, seed=seed, f=f, gx=gx, gy=gy, gz=gz, gvars=gvars)
    assert np.array_equal(f, np.tile(tape.values(bx, by, bz), reps))
    for g, od in ((gx, odx), (gy, ody), (gz, odz)):
        w = np.tile(bseed * od[idx], reps)
        assert np.allclose(g, w, rtol=1e-4, atol=1e-5)
    want = reps * (bseed.astype(np.float64) @ jac)
    scale = reps * np.abs(bseed[:, None] * jac).sum(axis=0) + 1e-6
    assert np.all(np.abs(gvars - want) <= 1e-4 * scale)


def test_reverse_gradient_const_var(gpu):
    # CONST_VAR blocks variable gradients but passes point gradients
    vars_ = {}
    s = parse("(+ (const-var (* v x)) (* v y))", vars_)
    v = vars_["v"]
    tape = Tape(s, {v: 2.0})
    x, y, z = (np.array([0.5, -1.0], np.float32) for _ in range(3))
    gx, gy, gz = (np.empty(2, np.float32) for _ in range(3))
    gvars = np.zeros(1, np.float32)
    tape.grad(x, y, z, gx=gx, gy=gy, gz=gz, gvars=gvars)
    assert np.array_equal(gx, [2.0, 2.0]) and np.array_equal(gy, [2.0, 2.0])
    assert np.array_equal(gz, [0.0, 0.0])
    assert gvars[0] == pytest.approx(float(y.sum()))


def test_jacobian_device_pointers(gpu):
    torch = pytest.importorskip("torch")
    s, vals = sphere_vars(6, seed=2)
    x, y, z = workloads.uniform_points(1000, seed=1)
    tape = Tape(s, vals)
    host = tape.jacobian(x, y, z)
    dx, dy, dz = (torch.from_numpy(a).cuda() for a in (x, y, z))
    out = torch.empty((1000, tape.n_vars), dtype=torch.float32, device="cuda")
    tape.jacobian(dx, dy, dz, out=out)
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), host)


def test_torch_autograd(gpu):
    torch = pytest.importorskip("torch")
    from libfive_b200.autograd import shape_value
    s, vals = sphere_vars(6, seed=3)
    tape = Tape(s, vals)
    by_id = {k.id(): v for k, v in vals.items()}
    pts_np = workloads.uniform_points(512, seed=2)
    x, y, z = (torch.from_numpy(a).cuda().requires_grad_() for a in pts_np)
    v = torch.tensor([by_id[i] for i in tape.var_ids()], device="cuda", requires_grad=True)
    f = shape_value(tape, x, y, z, v)
    loss = (f * f).sum()
    loss.backward()
    ora = OracleTape(s, vals)
    ov, odx, ody, odz = ora.derivs(*pts_np)
    assert np.array_equal(f.detach().cpu().numpy(), ov)
    for g, od in ((x.grad, odx), (y.grad, ody), (z.grad, odz)):
        assert np.allclose(g.cpu().numpy(), 2 * ov * od, rtol=1e-4, atol=1e-5)
    jac = ora.jacobian(*pts_np).astype(np.float64)
    want = (2 * ov.astype(np.float64)) @ jac
    scale = np.abs(2 * ov[:, None] * jac).sum(axis=0) + 1e-6
    assert np.all(np.abs(v.grad.cpu().numpy() - want) <= 1e-4 * scale)


def test_loss_grad_equals_values_then_grad(gpu):
    """lfb_eval_loss_grad (one forward pass for f and the gradient of
    mean f^2) against lfb_eval_values then lfb_eval_grad with seed 2 f / n."""
    torch = pytest.importorskip("torch")
    s, vals = workloads.blended_spheres_vars(64, seed=3, stable=True)
    tape = Tape(s, vals)
    n = 100003
    x, y, z = (torch.from_numpy(a).cuda() for a in workloads.uniform_points(n, seed=2, lo=-1.2, hi=1.2))
    st = torch.cuda.current_stream().cuda_stream
    f1 = torch.empty(n, device="cuda")
    tape.values(x, y, z, out=f1, stream=st)
    seed = f1 * (2.0 / n)
    g1 = [torch.empty(n, device="cuda") for _ in range(3)]
    gv1 = torch.zeros(tape.n_vars, device="cuda")
    tape.grad(x, y, z, seed=seed, gx=g1[0], gy=g1[1], gz=g1[2], gvars=gv1, stream=st)
    f2 = torch.empty(n, device="cuda")
    g2 = [torch.empty(n, device="cuda") for _ in range(3)]
    gv2 = torch.zeros(tape.n_vars, device="cuda")
    loss = torch.zeros(1, device="cuda")
    tape.loss_grad(x, y, z, f2, *g2, gvars=gv2, loss=loss, stream=st)
    torch.cuda.synchronize()
    assert torch.equal(f1, f2)
    for a, b in zip(g1, g2):
        assert torch.equal(a, b)
    assert torch.allclose(gv1, gv2, rtol=1e-5, atol=1e-7)
    want = (f1.double() ** 2).mean().item()
    assert abs(loss.item() - want) <= 1e-6 * want
