"""User operators through the C ABI (helm_plan_set_operator_callback), the
replacement of the reference's ConstructOperator callback
(SolvePDE(FieldVariable U[], void (*ConstructOperator)(const int)),
DPS/include/NonPeriodic2D_MPI.h:37; (int, int) in NonPeriodic3D_MPI.h:37).

* The stock operator handed over as a callback reproduces the stock plan (the
  same LU factors, so the same solution to rounding).
* A caller's own operator -- the stock one minus a coefficient c(y) varying
  along the GLL direction -- matches the reference's own SolvePDE run with that
  ConstructOperator (golden fixture tests/golden/user_operator.npz, written by
  tests/golden/make_golden.py).
* Refined plans, singular operators and the adjoint are declined with their
  status codes; a declined or failed call leaves the plan usable.
"""
import math

import numpy as np
import pytest
import torch

from mpi_b200 import NonPeriodic2D, NonPeriodic3D, Periodic2D
from mpi_b200._lib import HelmError
from tests.helpers import golden, max_rel

pytestmark = pytest.mark.gpu

PI = 3.1415926535897932  # the reference's constant (General.h:14)


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()


def _interior_d2(plan):
    _, _, D2 = plan.grid()
    return D2.numpy()[1:-1, 1:-1].copy()


def _shifted(A, lam, Lx, Ly=None, c=None):
    """The reference tests' ConstructOperator (TestNonPeriodic2D_MPI.cpp:67-74,
    TestNonPeriodic3D_MPI.cpp:71-79), optionally minus diag(c)."""
    n = A.shape[0]
    extra = np.zeros(n) if c is None else np.asarray(c)

    def op(iw, jw):
        s = lam + 4.0 * PI * PI * iw * iw / (Lx * Lx)
        if Ly is not None:
            s = s + 4.0 * PI * PI * jw * jw / (Ly * Ly)
        M = A.copy()
        for i in range(n):
            M[i, i] -= s
            M[i, i] -= extra[i]
        return M

    return op


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_stock_operator_as_callback_2d(cuda, precision):
    rng = np.random.default_rng(11)
    Nx, N, Ns, lam, bc = 32, 9, 3, 2.0, (1.0, 0.5, 0.7, 2.0)
    f = rng.standard_normal((Ns, Nx, N))
    gl, gr = rng.standard_normal(Nx), rng.standard_normal(Nx)
    kw = dict(Lambda=lam, bc=bc, precision=precision, method="lu")
    ref = NonPeriodic2D(Nx, Ns * N, N, 0.1, 1.4, 0.0, 0.9, **kw)
    p = NonPeriodic2D(Nx, Ns * N, N, 0.1, 1.4, 0.0, 0.9, **kw)
    calls = []
    op = _shifted(_interior_d2(p), lam, 1.3)
    p.SetOperator(lambda iw, jw: (calls.append((iw, jw)), op(iw, jw))[1])
    # once per |iw| = 0 .. Nx/2, as the reference's loop (NonPeriodic2D_MPI.cpp:239-241)
    assert sorted(calls) == [(iw, 0) for iw in range(Nx // 2 + 1)]
    assert p.info()["method"] == "lu"
    a = p.SolvePDE(_dev(f), _dev(gl), _dev(gr)).cpu().numpy()
    b = ref.SolvePDE(_dev(f), _dev(gl), _dev(gr)).cpu().numpy()
    assert max_rel(a, b) < (1e-13 if precision == "fp64" else 1e-6)


def test_stock_operator_as_callback_3d(cuda):
    rng = np.random.default_rng(12)
    Nx, Ny, N, lam = 16, 8, 17, 3.0
    f = rng.standard_normal((Nx, Ny, N))
    gl, gr = rng.standard_normal((Nx, Ny)), rng.standard_normal((Nx, Ny))
    ref = NonPeriodic3D(Nx, Ny, N, N, 0.0, 1.0, 0.0, 0.7, 0.0, 2.0, Lambda=lam, method="lu")
    p = NonPeriodic3D(Nx, Ny, N, N, 0.0, 1.0, 0.0, 0.7, 0.0, 2.0, Lambda=lam)
    calls = set()
    op = _shifted(_interior_d2(p), lam, 1.0, 0.7)
    p.SetOperator(lambda iw, jw: (calls.add((iw, jw)), op(iw, jw))[1])
    # once per (|iw|, |jw|) pair (NonPeriodic3D_MPI.cpp:248-253)
    assert calls == {(i, j) for i in range(Nx // 2 + 1) for j in range(Ny // 2 + 1)}
    a = p.SolvePDE(_dev(f), _dev(gl), _dev(gr)).cpu().numpy()
    b = ref.SolvePDE(_dev(f), _dev(gl), _dev(gr)).cpu().numpy()
    assert max_rel(a, b) < 1e-13


def test_user_operator_vs_reference_2d(cuda):
    g = golden("user_operator")
    xl, xr, yl, yr = [float(v) for v in g["dom2"]]
    Ns, Nx, N = g["f2"].shape
    lam = float(g["lam2"])
    p = NonPeriodic2D(Nx, Ns * N, N, xl, xr, yl, yr, Lambda=lam, bc=tuple(g["bc2"]))
    p.SetOperator(_shifted(_interior_d2(p), lam, xr - xl, c=g["c2"]))
    u = p.SolvePDE(_dev(g["f2"]), _dev(g["gl2"]), _dev(g["gr2"])).cpu().numpy()
    assert max_rel(u, g["u2"]) < 1e-12
    # the operator really is not the stock one
    stock = NonPeriodic2D(Nx, Ns * N, N, xl, xr, yl, yr, Lambda=lam, bc=tuple(g["bc2"]))
    us = stock.SolvePDE(_dev(g["f2"]), _dev(g["gl2"]), _dev(g["gr2"])).cpu().numpy()
    assert max_rel(us, g["u2"]) > 1e-3


def test_user_operator_vs_reference_3d(cuda):
    g = golden("user_operator")
    xl, xr, yl, yr, zl, zr = [float(v) for v in g["dom3"]]
    Nx, Ny, N = g["f3"].shape
    lam = float(g["lam3"])
    p = NonPeriodic3D(Nx, Ny, N, N, xl, xr, yl, yr, zl, zr, Lambda=lam)
    p.SetOperator(_shifted(_interior_d2(p), lam, xr - xl, yr - yl, c=g["c3"]))
    u = p.SolvePDE(_dev(g["f3"]), _dev(g["gl3"]), _dev(g["gr3"])).cpu().numpy()
    assert max_rel(u, g["u3"]) < 1e-12


def test_periodic_plan_takes_a_user_operator(cuda):
    """The periodic solvers pass ConstructOperator too (Periodic2D_MPI.h:35): the
    stock operator as a callback reproduces the stock periodic plan."""
    rng = np.random.default_rng(13)
    Nx, N, Ns, lam = 16, 9, 3, 0.8
    f = rng.standard_normal((Ns, Nx, N))
    ref = Periodic2D(Nx, Ns * N, N, 0.0, 1.0, 0.0, 2.0, Lambda=lam, method="lu")
    p = Periodic2D(Nx, Ns * N, N, 0.0, 1.0, 0.0, 2.0, Lambda=lam)
    p.SetOperator(_shifted(_interior_d2(p), lam, 1.0))
    assert max_rel(p.SolvePDE(_dev(f)).cpu().numpy(), ref.SolvePDE(_dev(f)).cpu().numpy()) < 1e-13


def test_layout_survives_the_rebuild(cuda):
    """The plan is rebuilt in place: a layout set before the callback stays."""
    rng = np.random.default_rng(14)
    Nx, N, lam = 16, 9, 1.0
    f = rng.standard_normal((Nx, N))
    p = NonPeriodic2D(Nx, N, N, 0.0, 1.0, 0.0, 1.0, Lambda=lam)
    p.set_layout(x_stride=N, elem_stride=2 * Nx * N)  # the reference's [2Nx][N] arrays
    p.SetOperator(_shifted(_interior_d2(p), lam, 1.0))
    F = np.zeros((2 * Nx, N)); F[:Nx] = f
    U = torch.full((2 * Nx, N), 5.0, dtype=torch.float64, device="cuda")
    z = torch.zeros(Nx, dtype=torch.float64, device="cuda")
    st = p._lib.helm_solve(p._plan, _dev(F).data_ptr(), z.data_ptr(), z.data_ptr(), U.data_ptr(),
                           torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert st == 0
    ref = NonPeriodic2D(Nx, N, N, 0.0, 1.0, 0.0, 1.0, Lambda=lam, method="lu").SolvePDE(_dev(f)).cpu().numpy()
    Uc = U.cpu().numpy()
    assert max_rel(Uc[:Nx], ref) < 1e-13
    assert np.all(Uc[Nx:] == 5.0)


def test_declined_cases(cuda):
    p = NonPeriodic2D(16, 9, 9, 0.0, 1.0, 0.0, 1.0, Lambda=1.0, precision="fp32_refine")
    with pytest.raises(HelmError):
        p.SetOperator(lambda iw, jw: np.eye(7))
    # a singular operator: HELM_ERR_SINGULAR, and the plan keeps its stock operator
    p = NonPeriodic2D(16, 9, 9, 0.0, 1.0, 0.0, 1.0, Lambda=1.0)
    rng = np.random.default_rng(15)
    f = _dev(rng.standard_normal((16, 9)))
    before = p.SolvePDE(f).cpu().numpy()
    with pytest.raises(HelmError):
        p.SetOperator(lambda iw, jw: np.zeros((7, 7)))
    assert np.array_equal(p.SolvePDE(f).cpu().numpy(), before)
    # the adjoint has no transposed user operator
    p.SetOperator(_shifted(_interior_d2(p), 1.0, 1.0))
    with pytest.raises(HelmError):
        p.SolveAdjoint(f)
    # an exception inside the callback reaches the caller
    def bad(iw, jw):
        raise ValueError("operator failed")
    with pytest.raises(ValueError):
        p.SetOperator(bad)
