"""The product's FP64 host setup (GLL grid, LU with scaled partial pivoting,
eigen-decomposition of the interior GLL operator) checked on the CPU against
the oracle and numpy."""
import ctypes
import os
import subprocess
import tempfile

import numpy as np
import pytest

from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
P = ctypes.POINTER(ctypes.c_double)


@pytest.fixture(scope="module")
def shim():
    d = tempfile.mkdtemp()
    so = os.path.join(d, "libhostsetup.so")
    subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-o", so, os.path.join(HERE, "host_setup_shim.cpp"),
                    os.path.join(REPO, "mpi_b200", "csrc", "helm_setup.cpp")], check=True)
    lib = ctypes.CDLL(so)
    lib.t_gll_setup.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, P, P, P]
    lib.t_lu.argtypes = [ctypes.c_int, P, ctypes.POINTER(ctypes.c_int), P]
    lib.t_eig.argtypes = [ctypes.c_int, P, P, P, P]
    return lib


def _p(a):
    return a.ctypes.data_as(P)


@pytest.mark.parametrize("N,Ns,L", [(5, 1, 2.0), (33, 1, 2.0), (65, 1, 2.0), (10, 4, 1.0), (129, 1, 1.0)])
def test_gll_setup_matches_oracle(shim, N, Ns, L):
    y = np.zeros(Ns * (N - 1) + 1); D = np.zeros((N, N)); D2 = np.zeros((N, N))
    shim.t_gll_setup(N, Ns, L, _p(y), _p(D), _p(D2))
    yo, Do, D2o = O.gll_grid(N, Ns, L)
    assert np.abs(y - yo).max() < 1e-14 * L
    assert np.abs(D - Do).max() < 1e-12 * np.abs(Do).max()
    assert np.abs(D2 - D2o).max() < 1e-11 * np.abs(D2o).max()


def test_lu_scaled_pivoting_solves(shim):
    rng = np.random.default_rng(0)
    for n in (3, 17, 63):
        A = rng.standard_normal((n, n)) * np.exp(rng.standard_normal((n, 1)) * 3)
        b = rng.standard_normal(n)
        LU = A.copy(); x = b.copy(); perm = (ctypes.c_int * n)()
        assert shim.t_lu(n, _p(LU), perm, _p(x)) == 0
        assert np.linalg.norm(A @ x - b) < 1e-10 * np.linalg.norm(b) * np.linalg.cond(A) ** 0.5


def test_lu_singular(shim):
    A = np.ones((4, 4)); x = np.ones(4); perm = (ctypes.c_int * 4)()
    assert shim.t_lu(4, _p(A), perm, _p(x)) == 1


@pytest.mark.parametrize("N", [5, 17, 33, 65])
def test_interior_gll_operator_eigen(shim, N):
    y, D, D2 = O.gll_grid(N, 1, 2.0)
    n = N - 2
    A = np.ascontiguousarray(D2[1:-1, 1:-1])
    lam = np.zeros(n); V = np.zeros((n, n)); Vi = np.zeros((n, n))
    assert shim.t_eig(n, _p(A), _p(lam), _p(V), _p(Vi)) == 0
    assert np.abs(V @ np.diag(lam) @ Vi - A).max() < 1e-13 * np.abs(A).max()
    assert np.abs(V @ Vi - np.eye(n)).max() < 1e-13
    assert np.all(lam < 0)
    if N >= 17:  # spectral accuracy: smallest |eigenvalue| -> pi^2/4 on [-1, 1]
        assert abs(lam.max() + math_pi2_4()) < 1e-9


def math_pi2_4():
    return np.pi ** 2 / 4
