"""The N-GMRES combination step's least-squares solve (linalg.hpp lsq_sym)
on the CPU against numpy's minimum-norm least squares: symmetric positive
definite and rank-deficient Gram matrices of up to 16 unknowns, the sizes
N-GMRES(m <= 16) forms.  Tolerance: 1e-10 relative on well-conditioned
systems; on rank-deficient ones both drop the null space (singular values
below 2.2e-16 of the largest), so the solutions agree to 1e-8."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from conftest import HOSTMODEL_DIR, ROOT

SRC = os.path.join(HOSTMODEL_DIR, "linalg_shim.cpp")
SO = os.path.join(HOSTMODEL_DIR, "_build", "liblinalg_shim.so")


@pytest.fixture(scope="module")
def lsq():
    hdr = os.path.join(ROOT, "bt-am_b200", "csrc", "linalg.hpp")
    if (not os.path.exists(SO) or os.path.getmtime(SO) < max(os.path.getmtime(SRC),
                                                             os.path.getmtime(hdr))):
        os.makedirs(os.path.dirname(SO), exist_ok=True)
        subprocess.run(["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-o", SO, SRC],
                       check=True)
    L = ctypes.CDLL(SO)
    D = ctypes.POINTER(ctypes.c_double)
    L.lsq_sym_c.argtypes = [ctypes.c_int, D, D]

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
