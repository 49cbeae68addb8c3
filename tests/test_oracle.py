"""The oracle is pinned before it is trusted: the C restatement against the
reference's own solver (compiled from its sources), against the golden vectors
generated from it, and against the reference tests' manufactured solutions."""
import math

import numpy as np
import pytest

from oracle import oracle as O
from mpi_b200 import workloads as W
from tests.helpers import golden, max_rel


@pytest.fixture(scope="module", autouse=True)
def _build():
    O.build()


def _solve_golden_2d(g):
    xl, xr, yl, yr = g["dom"]
    return O.solve2d(g["f"], g.get("gl", np.zeros(int(g["Nx"]))), g.get("gr", np.zeros(int(g["Nx"]))),
                     Lx=xr - xl, Ly=yr - yl, lam=float(g["lam"]), bc=tuple(g["bc"]))


def _solve_golden_3d(g):
    xl, xr, yl, yr, zl, zr = g["dom"]
    nb = (int(g["Nx"]), int(g["Ny"]))
    return O.solve3d(g["f"], g.get("gl", np.zeros(nb)), g.get("gr", np.zeros(nb)), Lx=xr - xl, Ly=yr - yl,
                     Lz=zr - zl, lam=float(g["lam"]), bc=tuple(g["bc"]))


@pytest.mark.parametrize("name", ["cfg1_2d", "robin_2d_ns3"])
def test_restatement_matches_golden_2d(name):
    g = golden(name)
    assert max_rel(_solve_golden_2d(g), g["u"]) < 1e-12


@pytest.mark.parametrize("name", ["robin_3d", "robin_3d_ns2", "smooth_3d"])
def test_restatement_matches_golden_3d(name):
    g = golden(name)
    assert max_rel(_solve_golden_3d(g), g["u"]) < 1e-12


def test_cfg1_known_answer():
    g = golden("cfg1_2d")
    assert np.abs(g["u"] - g["u_exact"]).max() < 1e-13  # the reference's own solve
    assert np.abs(_solve_golden_2d(g) - g["u_exact"]).max() < 1e-13


def test_reference_stock_2d_known_answer():
    """TestNonPeriodic2D_MPI.cpp: 512 x 512, N = 10 (Ns = 52), Neumann/Dirichlet;
    the reference reaches 1.67e-13."""
    f, gl, gr, ue, bc = W.stock_2d()
    u = O.solve2d(f, gl, gr, Lx=1.0, Ly=1.0, lam=1.0, bc=bc)
    assert np.abs(u - ue).max() < 1e-12


def test_reference_stock_3d_known_answer():
    f, gl, gr, ue, bc = W.stock_3d()
    u = O.solve3d(f, gl, gr, Lx=1.0, Ly=1.0, Lz=1.0, lam=1.0, bc=bc)
    assert np.abs(u - ue).max() < 1e-12


@pytest.mark.parametrize("name", ["periodic_2d", "periodic_2d_ns4"])
def test_periodic_restatement_matches_golden_2d(name):
    g = golden(name)
    xl, xr, yl, yr = g["dom"]
    u = O.psolve2d(g["f"], Lx=xr - xl, Ly=yr - yl, lam=float(g["lam"]))
    assert max_rel(u, g["u"]) < 1e-12


@pytest.mark.parametrize("name", ["periodic_3d", "periodic_3d_ns3"])
def test_periodic_restatement_matches_golden_3d(name):
    g = golden(name)
    xl, xr, yl, yr, zl, zr = g["dom"]
    u = O.psolve3d(g["f"], Lx=xr - xl, Ly=yr - yl, Lz=zr - zl, lam=float(g["lam"]))
    assert max_rel(u, g["u"]) < 1e-12


def test_reference_stock_periodic_2d_known_answer():
    """TestPeriodic2D_MPI.cpp: 512 x 512, N = 10 (Ns = 52), periodic in y."""
    f, ue = W.stock_periodic_2d()
    u = O.psolve2d(f, Lx=1.0, Ly=1.0, lam=1.0)
    assert np.abs(u - ue).max() < 1e-11


def test_reference_stock_periodic_3d_known_answer():
    """TestPeriodic3D_MPI.cpp: 64 x 32 x 250, N = 10 (Ns = 25), periodic in z."""
    f, ue = W.stock_periodic_3d()
    u = O.psolve3d(f, Lx=1.0, Ly=1.0, Lz=1.0, lam=1.0)
    assert np.abs(u - ue).max() < 1e-11


@pytest.mark.skipif(not O.have_reference(), reason="reference sources were not available at build time")
def test_periodic_restatement_matches_reference_random():
    rng = np.random.default_rng(6)
    for Ns, N, Nx in [(1, 17, 16), (2, 9, 8), (5, 10, 32)]:
        f = rng.standard_normal((Ns, Nx, N))
        a = O.psolve2d(f, Lx=2 * math.pi, Ly=2.0, lam=1.5)
        b = O.ref_psolve2d(f, xl=0.0, xr=2 * math.pi, yl=0.0, yr=2.0, lam=1.5)
        assert max_rel(a, b) < 1e-11
    f = rng.standard_normal((4, 4, 8, 8))
    a = O.psolve3d(f, Lx=1.0, Ly=2.0, Lz=3.0, lam=0.7)
    b = O.ref_psolve3d(f, xl=0.0, xr=1.0, yl=0.0, yr=2.0, zl=0.0, zr=3.0, lam=0.7)
    assert max_rel(a, b) < 1e-11


@pytest.mark.parametrize("order", [1, 2])
def test_derivative_restatement_matches_golden(order):
    """Spectral (Fourier_Quadrature.cpp:1387-1834) and GLL (NonPeriodic2D_MPI.cpp:497-542,
    NonPeriodic3D_MPI.cpp:632-683) derivatives of the reference on seeded arrays."""
    g = golden("derivatives")
    L2, L3x, L3y = float(g["L2"]), float(g["L3x"]), float(g["L3y"])
    assert max_rel(O.fourier_deriv(g["u2"], axis=0, order=order, L=L2), g[f"fx2_{order}"]) < 1e-13
    assert max_rel(O.fourier_deriv(g["u3"], axis=0, order=order, L=L3x), g[f"fx3_{order}"]) < 1e-13
    assert max_rel(O.fourier_deriv(g["u3"], axis=1, order=order, L=L3y), g[f"fy3_{order}"]) < 1e-13
    assert max_rel(O.gll_deriv(g["ug2"], N=9, Ns=3, L=2.0, order=order), g[f"gy2_{order}"]) < 1e-13
    assert max_rel(O.gll_deriv(g["ug3"], N=7, Ns=2, L=1.5, order=order), g[f"gz3_{order}"]) < 1e-13


def test_collocation_residual_3d():
    g = golden("robin_3d")
    xl, xr, yl, yr, zl, zr = g["dom"]
    r = O.residual3d(g["u"], g["f"], g["gl"], g["gr"], Lx=xr - xl, Ly=yr - yl, Lz=zr - zl, lam=float(g["lam"]),
                     bc=tuple(g["bc"]))
    assert r < 1e-10 * np.abs(g["f"]).max() * 100


@pytest.mark.skipif(not O.have_reference(), reason="reference sources were not available at build time")
def test_restatement_matches_reference_random():
    rng = np.random.default_rng(5)
    for Ns, N, Nx in [(1, 5, 8), (2, 11, 32), (4, 6, 4)]:
        f = rng.standard_normal((Ns, Nx, N)); gl = rng.standard_normal(Nx); gr = rng.standard_normal(Nx)
        bc = (0.3, 1.0, 1.2, 0.4)
        a = O.solve2d(f, gl, gr, Lx=2.0, Ly=3.0, lam=0.7, bc=bc)
        b = O.ref_solve2d(f, gl, gr, xl=-1.0, xr=1.0, yl=0.0, yr=3.0, lam=0.7, bc=bc)
        assert max_rel(a, b) < 1e-12


def test_gll_grid_places_nodes_from_zero():
    """Grid quirk of NonPeriodic2D_MPI.cpp:103-112: nodes start at 0, not at yl."""
    y, D, D2 = O.gll_grid(9, 2, 3.0)
    assert y[0] == 0.0 and abs(y[-1] - 3.0) < 1e-15
    assert np.allclose(D @ D, D2, rtol=0, atol=1e-9 * np.abs(D2).max())


def _fd_case(g, c):
    Lx, Ly, Lz = (float(v) for v in g[f"L{c}"])
    return dict(Lx=Lx, Ly=Ly, Lz=Lz, lam=float(g[f"lam{c}"]), bc=tuple(float(v) for v in g[f"bc{c}"]))


def test_fd_restatement_matches_reference_golden():
    """The FD restatement against the reference's own HypreFDM 3D assembly
    (Helmholtz3D_MPI.cpp SetA / Setb, captured through the HYPRE IJ stub and
    solved directly): Dirichlet, Robin and mixed ends, golden vectors in
    tests/golden/fd3d_reference.npz."""
    g = golden("fd3d_reference")
    for c in range(int(g["ncases"])):
        u = O.fd3d_solve(g[f"f{c}"], g[f"gb{c}"], g[f"gf{c}"], **_fd_case(g, c))
        assert max_rel(u, g[f"u{c}"]) < 1e-13, f"case {c}"


def test_fd_reference_adjoint_golden_is_the_transpose_of_the_restatement():
    """The golden FD cotangents (the transpose of the reference's own assembled
    matrix) against the restatement's forward map: <u(f, gb, gf), ubar> =
    <f, fbar> + <gb, gbbar> + <gf, gfbar> for random inputs."""
    g = golden("fd3d_reference")
    rng = np.random.default_rng(29)
    for c in range(int(g["ncases"])):
        shape = g[f"ubar{c}"].shape
        for _ in range(3):
            f = rng.standard_normal(shape); gb = rng.standard_normal(shape[:2]); gf = rng.standard_normal(shape[:2])
            u = O.fd3d_solve(f, gb, gf, **_fd_case(g, c))
            lhs = float((u * g[f"ubar{c}"]).sum())
            rhs = float((f * g[f"fbar{c}"]).sum() + (gb * g[f"gbbar{c}"]).sum() + (gf * g[f"gfbar{c}"]).sum())
            assert abs(lhs - rhs) < 1e-12 * max(1.0, abs(lhs)), f"case {c}: {lhs} vs {rhs}"


@pytest.mark.skipif(not O.have_reference_fd(), reason="reference HypreFDM library not built")
@pytest.mark.parametrize("bc", [(0.0, 1.0, 0.0, 1.0), (1.0, 0.5, 0.7, 2.0), (1.0, 0.0, 1.0, 0.0)])
def test_fd_restatement_matches_reference_random(bc):
    rng = np.random.default_rng(17)
    f = rng.standard_normal((8, 16, 10)); gb = rng.standard_normal((8, 16)); gf = rng.standard_normal((8, 16))
    kw = dict(Lx=1.1, Ly=2.3, Lz=0.9, lam=2.0, bc=bc)
    assert max_rel(O.fd3d_solve(f, gb, gf, **kw), O.ref_fd3d_solve(f, gb, gf, **kw)) < 1e-13


@pytest.mark.parametrize("bc", [(0.0, 1.0, 0.0, 1.0), (1.0, 0.5, 0.7, 2.0)])
def test_fd_oracle_stencil_residual(bc):
    """Size-independent check of the FD restatement: the FP64 residual of the
    HypreFDM stencil."""
    rng = np.random.default_rng(3)
    f = rng.standard_normal((16, 8, 12)); gb = rng.standard_normal((16, 8)); gf = rng.standard_normal((16, 8))
    u = O.fd3d_solve(f, gb, gf, Lx=1.0, Ly=2.0, Lz=1.5, lam=1.0, bc=bc)
    assert O.fd3d_residual(u, f, gb, gf, Lx=1.0, Ly=2.0, Lz=1.5, lam=1.0, bc=bc) < 1e-11


def test_lu_restatement_solves():
    rng = np.random.default_rng(1)
    n = 12
    A = rng.standard_normal((n, n)) + 3 * np.eye(n)
    b = rng.standard_normal(n)
    LU = np.ascontiguousarray(A.copy())
    import ctypes
    piv = (ctypes.c_int * n)()
    assert O.lib().orc_lu_decompose(n, LU.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), piv) == 0
    x = b.copy()
    O.lib().orc_lu_solve(n, LU.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), piv,
                         x.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    assert np.allclose(A @ x, b, atol=1e-12)
