"""Host-only entry points of the C ABI (no GPU): the GLL grid of CreatePDEPlan
(helm_gll_grid) against the oracle, and the FP64 LU pair behind the shim's
LUDecomposition / LUSolve (helm_lu_factor / helm_lu_solve) against numpy."""
import ctypes

import numpy as np
import pytest

from mpi_b200 import _lib as L
from oracle import oracle as O


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


@pytest.mark.parametrize("N,Ns,Lg", [(5, 1, 2.0), (10, 52, 1.0), (33, 1, 2.0), (65, 3, 0.7), (129, 2, 5.0)])
def test_gll_grid_matches_oracle(N, Ns, Lg):
    lib = L.lib()
    y = np.zeros(Ns * (N - 1) + 1)
    D = np.zeros((N, N))
    D2 = np.zeros((N, N))
    assert lib.helm_gll_grid(N, Ns, Lg, _p(y), _p(D), _p(D2)) == 0
    yo, Do, D2o = O.gll_grid(N, Ns, Lg)
    assert np.abs(y - yo).max() < 1e-14 * Lg
    assert np.abs(D - Do).max() < 1e-11 * np.abs(Do).max()
    assert np.abs(D2 - D2o).max() < 1e-10 * np.abs(D2o).max()
    assert lib.helm_gll_grid(1, 1, 1.0, None, None, None) == L.HELM_ERR_INVALID


@pytest.mark.parametrize("n", [1, 7, 31, 127])
def test_lu_factor_solve_determinant(n):
    lib = L.lib()
    rng = np.random.default_rng(n)
    A = rng.standard_normal((n, n)) + n * np.eye(n) * 0.1
    b = rng.standard_normal(n)
    LU = A.copy()
    perm = np.zeros(n, dtype=np.int32)
    det = ctypes.c_double()
    assert lib.helm_lu_factor(n, _p(LU), _p(perm), ctypes.byref(det)) == 0
    assert sorted(perm.tolist()) == list(range(n))
    x = b.copy()
    assert lib.helm_lu_solve(n, _p(LU), _p(perm), _p(x)) == 0
    assert np.abs(A @ x - b).max() < 1e-10 * np.abs(b).max() * n
    assert abs(det.value - np.linalg.det(A)) < 1e-9 * abs(np.linalg.det(A))


def test_lu_factor_singular():
    lib = L.lib()
    A = np.zeros((4, 4))
    perm = np.zeros(4, dtype=np.int32)
    assert lib.helm_lu_factor(4, _p(A), _p(perm), None) == L.HELM_ERR_SINGULAR
