"""The C ABI: the library loads, exports every function include/helm_b200.h
declares, and rejects bad plans with the documented status codes before it
touches a device (CPU)."""
import ctypes
import os
import re
import subprocess

import pytest

from mpi_b200 import _lib as L

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def lib():
    from mpi_b200 import build

    build.build()
    return L.lib()


def _declared():
    names = set()
    for h in os.listdir(os.path.join(REPO, "include")):
        if h.endswith(".h"):
            txt = open(os.path.join(REPO, "include", h)).read()
            txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
            names |= set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(helm\w+)\s*\(", txt, flags=re.M))
    return names


def test_exports_every_declared_symbol(lib):
    declared = _declared()
    assert declared, "no declarations parsed"
    out = subprocess.run(["nm", "-D", "--defined-only", L.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (\w+)", out))
    missing = declared - exported
    assert not missing, f"declared but not exported: {sorted(missing)}"
    for n in declared:
        assert hasattr(lib, n)
    assert set(L.EXPORTS) <= declared


def _create2d(lib, Nx, Ny, N, prec=0, method=0, xr=1.0):
    p = ctypes.c_void_p()
    st = lib.helm2d_plan_create(Nx, Ny, N, 0.0, xr, 0.0, 1.0, None, 1.0, prec, method, ctypes.byref(p))
    if st == 0:
        lib.helm_plan_destroy(p)
    return st


def test_rejects_non_power_of_two(lib):
    assert _create2d(lib, 48, 9, 9) == L.HELM_ERR_NOT_POW2


def test_rejects_bad_sizes(lib):
    assert _create2d(lib, 64, 2, 2) == L.HELM_ERR_INVALID
    assert _create2d(lib, 64, 200, 200) == L.HELM_ERR_INVALID
    assert _create2d(lib, 2048, 9, 9) == L.HELM_ERR_UNSUPPORTED
    assert _create2d(lib, 64, 9, 9, prec=7) == L.HELM_ERR_INVALID
    assert _create2d(lib, 64, 9, 9, xr=0.0) == L.HELM_ERR_INVALID


def test_null_arguments(lib):
    assert lib.helm_solve(None, None, None, None, None, None) == L.HELM_ERR_INVALID
    assert lib.helm_plan_destroy(None) == L.HELM_OK
    assert lib.helm2d_plan_create(8, 9, 9, 0.0, 1.0, 0.0, 1.0, None, 1.0, 0, 0, None) == L.HELM_ERR_INVALID


def test_status_strings(lib):
    for s in range(8):
        assert lib.helm_status_string(s)


def _create_batch(lib, Nx, N, lam, prec=0, xr=1.0):
    n = len(Nx)
    b = ctypes.c_void_p()
    st = lib.helm2d_batch_create(n, (ctypes.c_int * max(n, 1))(*Nx), (ctypes.c_int * max(n, 1))(*N),
                                 (ctypes.c_double * max(n, 1))(*lam), 0.0, xr, -1.0, 1.0, prec, ctypes.byref(b))
    if st == 0:
        lib.helm_batch_destroy(b)
    return st


def test_batch_rejects_bad_input(lib):
    assert _create_batch(lib, [], [], []) == L.HELM_ERR_INVALID
    assert _create_batch(lib, [32, 48], [9, 9], [1.0, 1.0]) == L.HELM_ERR_NOT_POW2
    assert _create_batch(lib, [32, 2048], [9, 9], [1.0, 1.0]) == L.HELM_ERR_UNSUPPORTED
    assert _create_batch(lib, [32], [2], [1.0]) == L.HELM_ERR_INVALID
    assert _create_batch(lib, [32], [130], [1.0]) == L.HELM_ERR_INVALID
    assert _create_batch(lib, [32], [9], [float("nan")]) == L.HELM_ERR_INVALID
    assert _create_batch(lib, [32], [9], [1.0], prec=5) == L.HELM_ERR_INVALID
    assert _create_batch(lib, [32], [9], [1.0], xr=0.0) == L.HELM_ERR_INVALID
    assert lib.helm_batch_solve(None, None, None, None) == L.HELM_ERR_INVALID
    assert lib.helm_batch_destroy(None) == L.HELM_OK
