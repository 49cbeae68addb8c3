"""Parity of the CUDA solve with the oracle (GPU).

Golden vectors come from the reference's own SolvePDE (tests/golden); larger
cases are checked against the C restatement (oracle/helm_oracle.c), which
tests/test_oracle.py pins to the reference.  Tolerances: FP64 plans 1e-12
relative (max-norm); FP32 plans 1e-5 relative L2; FP32 plans with FP64-residual
refinement 1e-10 relative L2 (the accuracy target of the mixed-precision solve).
"""
import math

import numpy as np
import pytest
import torch

from mpi_b200 import NonPeriodic2D, NonPeriodic3D
from mpi_b200 import workloads as W
from mpi_b200._lib import HelmError
from oracle import oracle as O
from tests.helpers import golden, max_rel, rel_l2

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-12, "fp32": 1e-5, "fp32_refine": 1e-10}


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()


def _plan2d(g, precision="fp64", method="auto"):
    xl, xr, yl, yr = [float(v) for v in g["dom"]]
    return NonPeriodic2D(int(g["Nx"]), int(g["Ns"]) * int(g["N"]), int(g["N"]), xl, xr, yl, yr,
                         Lambda=float(g["lam"]), bc=tuple(g["bc"]), precision=precision, method=method)


def _plan3d(g, precision="fp64", method="auto"):
    xl, xr, yl, yr, zl, zr = [float(v) for v in g["dom"]]
    return NonPeriodic3D(int(g["Nx"]), int(g["Ny"]), int(g["Ns"]) * int(g["N"]), int(g["N"]), xl, xr, yl, yr, zl, zr,
                         Lambda=float(g["lam"]), bc=tuple(g["bc"]), precision=precision, method=method)


def _solve(plan, g):
    gl = _dev(g["gl"]) if "gl" in g else None
    gr = _dev(g["gr"]) if "gr" in g else None
    u = plan.SolvePDE(_dev(g["f"]), gl, gr)
    torch.cuda.synchronize()
    return u.cpu().numpy()


def _check(u, ref, precision):
    if precision == "fp64":
        assert max_rel(u, ref) < TOL["fp64"]
    else:
        assert rel_l2(u, ref) < TOL[precision]


@pytest.mark.parametrize("method", ["lu", "fdm"])
@pytest.mark.parametrize("precision", ["fp64", "fp32", "fp32_refine"])
@pytest.mark.parametrize("name", ["cfg1_2d", "robin_2d_ns3"])
def test_golden_2d(cuda, name, precision, method):
    g = golden(name)
    p = _plan2d(g, precision, method)
    assert p.info()["method"] == method
    _check(_solve(p, g), g["u"], precision)


@pytest.mark.parametrize("method", ["lu", "fdm"])
@pytest.mark.parametrize("precision", ["fp64", "fp32", "fp32_refine"])
@pytest.mark.parametrize("name", ["robin_3d", "robin_3d_ns2", "smooth_3d"])
def test_golden_3d(cuda, name, precision, method):
    g = golden(name)
    p = _plan3d(g, precision, method)
    _check(_solve(p, g), g["u"], precision)


@pytest.mark.parametrize("method", ["lu", "fdm"])
def test_cfg1_exact_solution(cuda, method):
    f, ue = W.manufactured_2d(64, 33, 1.0)
    p = NonPeriodic2D(64, 33, 33, 0.0, 2 * math.pi, -1.0, 1.0, Lambda=1.0, method=method)
    u = p.SolvePDE(_dev(f)).cpu().numpy()
    assert np.abs(u - ue).max() < 1e-13


@pytest.mark.parametrize("method", ["lu", "fdm"])
def test_reference_stock_2d(cuda, method):
    """The reference's NonPeriodic2D test (Ns = 52 elements, Neumann/Dirichlet)."""
    f, gl, gr, ue, bc = W.stock_2d()
    p = NonPeriodic2D(512, 512, 10, 0.0, 1.0, 0.0, 1.0, Lambda=1.0, bc=bc, method=method)
    assert p.Ns == 52
    u = p.SolvePDE(_dev(f), _dev(gl), _dev(gr)).cpu().numpy()
    assert np.abs(u - ue).max() < 1e-12


@pytest.mark.parametrize("method", ["lu", "fdm"])
def test_reference_stock_3d(cuda, method):
    """The reference's NonPeriodic3D test (64 x 32 x 250, N = 10, Ns = 25)."""
    f, gl, gr, ue, bc = W.stock_3d()
    p = NonPeriodic3D(64, 32, 250, 10, 0.0, 1.0, 0.0, 1.0, 0.0, 1.0, Lambda=1.0, bc=bc, method=method)
    u = p.SolvePDE(_dev(f), _dev(gl), _dev(gr)).cpu().numpy()
    assert np.abs(u - ue).max() < 1e-12


@pytest.mark.parametrize("Nx,N,lam", [(128, 65, 5.0), (256, 65, 10.0)])
@pytest.mark.parametrize("precision,method", [("fp64", "lu"), ("fp64", "fdm"), ("fp32", "fdm"),
                                              ("fp32_refine", "fdm"), ("fp32_refine", "lu")])
def test_full_size_3d_vs_oracle(cuda, Nx, N, lam, precision, method):
    """The 3D workloads at full size (128^2 x 65, lambda 5; 256^2 x 65, lambda 10)."""
    f = W.smooth_field_3d(Nx, Nx, N, seed=1236)
    z = np.zeros((Nx, Nx))
    ref = O.solve3d(f, z, z, Lx=2 * math.pi, Ly=2 * math.pi, Lz=2.0, lam=lam)
    p = NonPeriodic3D(Nx, Nx, N, N, 0.0, 2 * math.pi, 0.0, 2 * math.pi, 0.0, 2.0, Lambda=lam,
                      precision=precision, method=method)
    u = p.SolvePDE(_dev(f)).cpu().numpy()
    if precision == "fp64":
        assert rel_l2(u, ref) < 1e-12
    else:
        assert rel_l2(u, ref) < TOL[precision]


def test_reference_array_layout_3d(cuda):
    """The reference's own arrays: rhsPDE[2Nx][2Ny][N] and leftBC[2Nx][2Ny]."""
    g = golden("robin_3d")
    Nx, Ny, N = int(g["Nx"]), int(g["Ny"]), int(g["N"])
    F = np.zeros((2 * Nx, 2 * Ny, N)); F[:Nx, :Ny] = g["f"]
    GL = np.zeros((2 * Nx, 2 * Ny)); GL[:Nx, :Ny] = g["gl"]
    GR = np.zeros((2 * Nx, 2 * Ny)); GR[:Nx, :Ny] = g["gr"]
    p = _plan3d(g)
    p.set_layout(x_stride=2 * Ny * N, elem_stride=2 * Nx * 2 * Ny * N, bc_x_stride=2 * Ny)
    fd, ud = _dev(F), torch.full((2 * Nx, 2 * Ny, N), 7.0, dtype=torch.float64, device="cuda")
    gld, grd = _dev(GL), _dev(GR)  # keep the device buffers alive across the asynchronous solve
    st = p._lib.helm_solve(p._plan, fd.data_ptr(), gld.data_ptr(), grd.data_ptr(), ud.data_ptr(),
                           torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert st == 0
    U = ud.cpu().numpy()
    assert max_rel(U[:Nx, :Ny], g["u"]) < 1e-12
    assert np.all(U[Nx:] == 7.0) and np.all(U[:, Ny:] == 7.0)  # padding untouched


def test_fp32_io(cuda):
    g = golden("smooth_3d")
    p = _plan3d(g, "fp32")
    p.set_io_bytes(4)
    u = p.SolvePDE(torch.from_numpy(g["f"].astype(np.float32)).cuda()).cpu().numpy()
    assert rel_l2(u, g["u"]) < 1e-5


def test_repeated_solves_and_streams(cuda):
    """Plan reuse on a side stream, the input left untouched (the reference
    overwrites rhsPDE with its spectrum; this solver does not)."""
    g = golden("robin_2d_ns3")
    p = _plan2d(g)
    f = _dev(g["f"])
    f0 = f.clone()
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        for _ in range(3):
            u = p.SolvePDE(f, _dev(g["gl"]), _dev(g["gr"]), stream=s)
    s.synchronize()
    assert torch.equal(f, f0)
    assert max_rel(u.cpu().numpy(), g["u"]) < 1e-12


def test_linearity_full_size(cuda):
    """Size-independent property at the 256^2 x 65 size: S(a f1 + b f2) = a S f1 + b S f2."""
    Nx, N = 256, 65
    f1 = _dev(W.smooth_field_3d(Nx, Nx, N, seed=1))
    f2 = _dev(W.smooth_field_3d(Nx, Nx, N, seed=2))
    p = NonPeriodic3D(Nx, Nx, N, N, 0.0, 2 * math.pi, 0.0, 2 * math.pi, 0.0, 2.0, Lambda=10.0)
    u1, u2 = p.SolvePDE(f1), p.SolvePDE(f2)
    u12 = p.SolvePDE(2.0 * f1 - 3.0 * f2)
    err = (u12 - (2.0 * u1 - 3.0 * u2)).norm() / u12.norm()
    assert err.item() < 1e-13


@pytest.mark.parametrize("N", [33, 65, 129])
@pytest.mark.parametrize("precision", ["fp64", "fp32_refine"])
def test_every_launch_variant(cuda, N, precision):
    """Every FFT launch variant (0..7) and every row-solve variant (including the
    fused y-FFT / row / inverse-y slab kernel of FP64 plans) compute the same
    solve: each pinned combination against the oracle (Robin ends, so the
    boundary epilogue runs too)."""
    rng = np.random.default_rng(N)
    Nx, Ny, lam, bc = 16, 64, 3.0, (0.4, 1.0, 0.3, 2.0)
    f = rng.standard_normal((Nx, Ny, N))
    gl, gr = rng.standard_normal((Nx, Ny)), rng.standard_normal((Nx, Ny))
    ref = O.solve3d(f, gl, gr, Lx=1.0, Ly=1.5, Lz=2.0, lam=lam, bc=bc)
    p = NonPeriodic3D(Nx, Ny, N, N, 0.0, 1.0, 0.0, 1.5, 0.0, 2.0, Lambda=lam, bc=bc, precision=precision)
    fd, gld, grd = _dev(f), _dev(gl), _dev(gr)
    # row variant 2 (the fused slab kernel) exists for FP64 plans with <= 65 points
    rows = (0, 1, 2) if (precision == "fp64" and N <= 65) else (0, 1)
    for fv in range(8):
        for rv in rows:
            p.set_launch_variants([fv] * 4, rv)
            u = p.SolvePDE(fd, gld, grd).cpu().numpy()
            err = max_rel(u, ref) if precision == "fp64" else rel_l2(u, ref)
            assert err < TOL[precision], (fv, rv, err)


@pytest.mark.parametrize("precision", ["fp64", "fp32_refine"])
def test_maximum_sizes(cuda, precision):
    """The largest sizes the plan accepts: Nx = 1024 Fourier modes with N = 129 GLL
    points (2D), 64 elements (2D, Robin ends), and a 1024 x 8 x 17 3D plan; one
    past each limit is rejected."""
    rng = np.random.default_rng(17)
    tol = 1e-12 if precision == "fp64" else 1e-10
    f = rng.standard_normal((1024, 129))
    p = NonPeriodic2D(1024, 129, 129, 0.0, 2 * math.pi, -1.0, 1.0, Lambda=2.0, precision=precision)
    u = p.SolvePDE(_dev(f)).cpu().numpy()
    ref = O.solve2d(f, np.zeros(1024), np.zeros(1024), Lx=2 * math.pi, Ly=2.0, lam=2.0)
    assert rel_l2(u, ref) < tol
    bc = (0.4, 1.0, 0.3, 2.0)
    f = rng.standard_normal((64, 32, 6))
    gl, gr = rng.standard_normal(32), rng.standard_normal(32)
    p = NonPeriodic2D(32, 64 * 6, 6, 0.0, 1.0, 0.0, 3.0, Lambda=1.5, bc=bc, precision=precision)
    assert p.Ns == 64
    u = p.SolvePDE(_dev(f), _dev(gl), _dev(gr)).cpu().numpy()
    assert rel_l2(u, O.solve2d(f, gl, gr, Lx=1.0, Ly=3.0, lam=1.5, bc=bc)) < tol
    f = rng.standard_normal((1024, 8, 17))
    p = NonPeriodic3D(1024, 8, 17, 17, 0.0, 1.0, 0.0, 1.0, 0.0, 1.0, Lambda=1.0, precision=precision)
    u = p.SolvePDE(_dev(f)).cpu().numpy()
    z = np.zeros((1024, 8))
    assert rel_l2(u, O.solve3d(f, z, z, Lx=1.0, Ly=1.0, Lz=1.0, lam=1.0)) < tol
    for args in ((2048, 33, 33), (64, 130, 130), (64, 65 * 6, 6)):
        with pytest.raises(HelmError):
            NonPeriodic2D(*args, 0.0, 1.0, 0.0, 1.0, Lambda=1.0, precision=precision)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_long_pass_launch_variants(cuda, precision):
    """FFT variants 8..11 (512-thread CTAs, lengths 512 and 1024) against the
    oracle on 2D plans with Nx = 512 and 1024; 12..15 (pipelined, too large a
    tile) fail cleanly and leave the plan usable."""
    rng = np.random.default_rng(5)
    for Nx in (512, 1024):
        f = rng.standard_normal((Nx, 17))
        ref = O.solve2d(f, np.zeros(Nx), np.zeros(Nx), Lx=1.0, Ly=2.0, lam=1.0)
        p = NonPeriodic2D(Nx, 17, 17, 0.0, 1.0, -1.0, 1.0, Lambda=1.0, precision=precision)
        for fv in range(8, 16):
            p.set_launch_variants([fv] * 4, 0)
            try:
                u = p.SolvePDE(_dev(f)).cpu().numpy()
            except HelmError as e:
                assert fv & 4 and e.status == 5, (Nx, fv, e)
                continue
            err = max_rel(u, ref) if precision == "fp64" else rel_l2(u, ref)
            assert err < TOL[precision], (Nx, fv, err)
