"""The solvers' host pieces on the CPU.

The N-GMRES combination step's least-squares solve (linalg.hpp lsq_sym)
against numpy's minimum-norm least squares: symmetric positive definite and
rank-deficient Gram matrices of up to 16 unknowns, the sizes N-GMRES(m <= 16)
forms.  Tolerance: 1e-10 relative on well-conditioned systems; on
rank-deficient ones both drop the null space (singular values below 2.2e-16
of the largest), so the solutions agree to 1e-8.

The stretch solver's N-GMRES(3) with the critical-point line search
(ngmres.hpp) on synthetic three-unknown residuals: a linear one, which the
subspace spans after three iterates, and a mildly nonlinear one; both must
reach the tolerance at the known root with three evaluations per
iteration."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from conftest import HOSTMODEL_DIR, ROOT

SRC = os.path.join(HOSTMODEL_DIR, "linalg_shim.cpp")
SO = os.path.join(HOSTMODEL_DIR, "_build", "liblinalg_shim.so")


lsq_lib = [None]


@pytest.fixture(scope="module")
def lsq():
    hdrs = [os.path.join(ROOT, "bt-am_b200", "csrc", h) for h in ("linalg.hpp", "ngmres.hpp")]
    if (not os.path.exists(SO) or
            os.path.getmtime(SO) < max(os.path.getmtime(f) for f in [SRC] + hdrs)):
        os.makedirs(os.path.dirname(SO), exist_ok=True)
        subprocess.run(["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-o", SO, SRC],
                       check=True)
    L = ctypes.CDLL(SO)
    D = ctypes.POINTER(ctypes.c_double)
    L.lsq_sym_c.argtypes = [ctypes.c_int, D, D]
    lsq_lib[0] = L

    def solve(H, b):
        H = np.ascontiguousarray(H, np.float64)
        x = np.ascontiguousarray(b, np.float64).copy()
        L.lsq_sym_c(len(x), H.ctypes.data_as(D), x.ctypes.data_as(D))
        return x
    return solve


@pytest.mark.parametrize("n", [1, 2, 3, 5, 8, 16])
def test_spd_systems(lsq, n):
    g = np.random.default_rng(n)
    A = g.normal(size=(n + 4, n))
    H = A.T @ A
    b = g.normal(size=n)
    want = np.linalg.solve(H, b)
    got = lsq(H, b)
    assert np.abs(got - want).max() <= 1e-10 * max(1.0, np.abs(want).max())


@pytest.mark.parametrize("n,rank", [(3, 2), (5, 3), (8, 1), (16, 9)])
def test_rank_deficient_min_norm(lsq, n, rank):
    g = np.random.default_rng(10 * n + rank)
    A = g.normal(size=(rank, n))
    H = A.T @ A  # rank `rank`, as the Gram matrix of dependent residual differences
    b = H @ g.normal(size=n)  # consistent right-hand side
    want = np.linalg.lstsq(H, b, rcond=2.220446049250313e-16)[0]
    got = lsq(H, b)
    assert np.abs(got - want).max() <= 1e-8 * max(1.0, np.abs(want).max())
    assert np.abs(H @ got - b).max() <= 1e-8 * max(1.0, np.abs(b).max())


def test_zero_matrix_gives_zero(lsq):
    assert np.array_equal(lsq(np.zeros((4, 4)), np.ones(4)), np.zeros(4))


RESFN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                         ctypes.POINTER(ctypes.c_double))


def run_ngmres(L, F, x0, m=3, atol=1e-12, rtol=1e-10, max_iter=200):
    D = ctypes.POINTER(ctypes.c_double)
    calls = [0]

    @RESFN
    def res(x, f):
        calls[0] += 1
        y = F(np.array([x[0], x[1], x[2]]))
        for a in range(3):
            f[a] = y[a]
        return 0

    L.ngmres3_c.argtypes = [RESFN, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                            D, D, ctypes.c_double, ctypes.POINTER(ctypes.c_int),
                            ctypes.POINTER(ctypes.c_int)]
    X = np.array(x0, np.float64)
    Y = F(X).astype(np.float64)
    n0 = float(np.linalg.norm(Y))
    it, status = ctypes.c_int(0), ctypes.c_int(0)
    rc = L.ngmres3_c(res, m, atol, rtol, max_iter, X.ctypes.data_as(D), Y.ctypes.data_as(D), n0,
                     ctypes.byref(it), ctypes.byref(status))
    return rc, X, Y, it.value, status.value, calls[0]


def test_ngmres_linear_residual(lsq):
    L = lsq_lib[0]
    A = np.array([[3.0, 0.5, 0.2], [0.5, 2.0, 0.1], [0.2, 0.1, 1.5]])
    root = np.array([1.01, 0.99, 1.02])
    rc, X, Y, it, status, calls = run_ngmres(L, lambda x: A @ (x - root), [1.0, 1.0, 1.0])
    assert rc == 0 and status == 1, (rc, status, it)
    assert np.abs(X - root).max() <= 1e-11 and np.linalg.norm(Y) <= 1e-12
    assert it <= 12 and calls <= 3 * it


def test_ngmres_nonlinear_residual(lsq):
    L = lsq_lib[0]
    root = np.array([1.0115, 1.0116, 1.0205])

    def F(x):
        d = x - root
        return np.array([2.0 * d[0] + 0.3 * d[1] + 5.0 * d[0] ** 3,
                         0.3 * d[0] + 1.5 * d[1] + 0.2 * d[2] + 4.0 * d[1] ** 3,
                         0.2 * d[1] + 1.2 * d[2] + 3.0 * d[2] ** 2])

    rc, X, Y, it, status, calls = run_ngmres(L, F, [1.0, 1.0, 1.0])
    assert rc == 0 and status == 1, (rc, status, it)
    assert np.abs(X - root).max() <= 1e-10 and np.linalg.norm(Y) <= 1e-12
    assert calls <= 3 * it
