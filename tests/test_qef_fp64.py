"""The mesher's FP64 QEF solve (libfive_b200/csrc/qef.h, compiled into the
device kernels and, unchanged, into the CPU oracle) pinned against an
independent eigensolver: numpy.linalg.eigh (LAPACK dsyevd) in FP64.

qef.h replaces Eigen's SelfAdjointEigenSolver used by the reference's
DCTree::findVertex (libfive/src/render/brep/dc/dc_tree.inl:740-813) and
Intersection::get_rank (libfive/include/libfive/render/brep/dc/
intersection.hpp:67-88) with a cyclic Jacobi solver.  These checks cover the
matrices the mesher builds (sums of unit-normal outer products: full rank,
rank 2 on edges, rank 1 on faces), repeated eigenvalues and eigenvalues next
to the 0.1 truncation cutoff (dc_flags.hpp:12), which decides feature
preservation."""
import ctypes

import numpy as np
import pytest

import oracle_ffi

CUTOFF = 0.1


def _p(a):
    return a.ctypes.data


def sym6(A):
    return np.ascontiguousarray([A[0, 0], A[0, 1], A[0, 2], A[1, 1], A[1, 2], A[2, 2]],
                                np.float64)


def jacobi(A):
    lib = oracle_ffi.load()
    ev = np.zeros(3)
    U = np.zeros(9)
    lib.ora_sym3_eigen(_p(sym6(A)), _p(ev), _p(U))
    return ev, U.reshape(3, 3)


def normals_ata(normals):
    n = np.asarray(normals, np.float64)
    n = n / np.linalg.norm(n, axis=1, keepdims=True)
    return n.T @ n


def random_unit(rng, k):
    return rng.normal(size=(k, 3))


def cases():
    rng = np.random.default_rng(1234)
    out = []
    for k in range(2, 14):                      # generic: full rank
        for _ in range(20):
            out.append(("full", normals_ata(random_unit(rng, k))))
    for _ in range(60):                          # one plane of normals: rank 2
        a, b = random_unit(rng, 2)
        w = rng.normal(size=(rng.integers(2, 9), 2))
        out.append(("rank2", normals_ata(w @ np.stack([a, b]))))
    for _ in range(60):                          # one normal repeated: rank 1
        a = random_unit(rng, 1)[0]
        s = rng.choice([-1, 1], size=rng.integers(1, 9))
        out.append(("rank1", normals_ata(s[:, None] * a)))
    for _ in range(40):                          # repeated eigenvalues
        Q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
        lam = rng.choice([[2.0, 2.0, 0.5], [1.0, 1.0, 1.0], [3.0, 0.0, 0.0],
                          [1.5, 1.5, 0.0]])
        out.append(("repeated", Q @ np.diag(lam) @ Q.T))
    for _ in range(80):                          # next to the cutoff
        Q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
        d = rng.choice([-1, 1]) * rng.uniform(1e-6, 1e-3)
        lam = np.array([rng.uniform(0.5, 4), CUTOFF + d, rng.uniform(0, 0.05)])
        out.append(("cutoff", Q @ np.diag(rng.permutation(lam)) @ Q.T))
    for (a, b, c) in ([1, 0, 0], [0, 1, 0], [0, 0, 1]), ([1, 1, 0], [1, -1, 0], [0, 0, 1]):
        out.append(("axes", normals_ata([a, b, c])))
    return out


CASES = cases()


KINDS = ["full", "rank2", "rank1", "repeated", "cutoff", "axes"]


@pytest.mark.parametrize("kind", KINDS)
def test_eigenpairs_match_lapack(kind):
    for k, A in CASES:
        if k != kind:
            continue
        ev, U = jacobi(A)
        w = np.linalg.eigvalsh(A)
        scale = max(1.0, np.abs(w).max())
        assert np.allclose(np.sort(ev), w, rtol=0, atol=1e-13 * scale)
        # orthonormal eigenvectors with small residuals
        assert np.allclose(U.T @ U, np.eye(3), atol=1e-13)
        assert np.abs(A @ U - U * ev).max() <= 1e-13 * scale


def reference_vertex(ata, atb, btb, mass):
    """findVertex (dc_tree.inl:740-813) with LAPACK's eigenpairs."""
    w, U = np.linalg.eigh(ata)
    D = np.where(np.abs(w) < CUTOFF, 0.0, 1.0 / np.where(w == 0, 1, w))
    P = U @ np.diag(D) @ U.T
    c = mass[:3] / mass[3]
    v = P @ (atb - ata @ c) + c
    err = v @ ata @ v - 2 * v @ atb + btb
    return v, err, int((D != 0).sum())


@pytest.mark.parametrize("kind", KINDS)
def test_vertex_and_rank_match_lapack(kind):
    rng = np.random.default_rng(len(kind))
    lib = oracle_ffi.load()
    worst = 0.0
    n = 0
    for k, A in CASES:
        if k != kind:
            continue
        w = np.linalg.eigvalsh(A)
        # rank decision: identical unless an eigenvalue is within rounding of
        # the cutoff (none of these cases is closer than 1e-6)
        assert not np.any(np.abs(np.abs(w) - CUTOFF) < 1e-9)
        rank = lib.ora_qef_rank(_p(sym6(A)))
        assert rank == int((np.abs(w) < CUTOFF).sum())
        # a QEF with this A^T A: positions near the unit cube
        c = rng.uniform(-1, 1, 3)
        mass = np.ascontiguousarray(np.append(c * 4, 4.0))
        atb = np.ascontiguousarray(A @ (c + rng.normal(scale=0.05, size=3)))
        btb = float(rng.uniform(0, 1))
        v = np.zeros(3)
        r = ctypes.c_int()
        err = lib.ora_qef_vertex(_p(sym6(A)), _p(atb), btb, _p(mass), _p(v), ctypes.byref(r))
        rv, rerr, rrank = reference_vertex(A, atb, btb, mass)
        assert r.value == rrank
        worst = max(worst, np.abs(v - rv).max())
        assert abs(err - rerr) <= 1e-12 * max(1.0, abs(btb))
        n += 1
    assert n > 0
    # vertex error of the Jacobi solve against the LAPACK solve, FP64
    assert worst <= 1e-12, worst
