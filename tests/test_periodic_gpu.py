"""Parity of the solvers periodic in the GLL direction (GPU).

Golden vectors come from the reference's own Periodic2D / Periodic3D SolvePDE
(tests/golden/periodic_*.npz); larger cases are checked against the C
restatement (orc_psolve2d / orc_psolve3d), which tests/test_oracle.py pins to
the reference.  Covers one element (the folded fast-diagonalisation kernels and
the fused slab kernel) and several elements (the cyclic interface sweep with
its rank-one correction in the row kernel).  Tolerances as the non-periodic
tests: FP64 1e-12 relative (max-norm; 1e-11 where the reference's own FFT
rounding dominates), FP32 1e-5 relative L2 (5e-5 for the 64-element chain,
whose sequential FP32 sweep carries 64 rounding steps), refined FP32 1e-10
relative L2; adjoint 1e-10 against the transposed dense map of the oracle.
"""
import math

import numpy as np
import pytest
import torch

from mpi_b200 import Periodic2D, Periodic3D
from mpi_b200 import workloads as W
from mpi_b200._lib import HelmError
from oracle import oracle as O
from tests.helpers import golden, max_rel, rel_l2

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-11, "fp32": 1e-5, "fp32_refine": 1e-10}


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()


def _check(u, ref, precision, Ns=1):
    if precision == "fp64":
        assert max_rel(u, ref) < TOL["fp64"]
    elif precision == "fp32" and Ns > 8:
        assert rel_l2(u, ref) < 5e-5
    else:
        assert rel_l2(u, ref) < TOL[precision]


def _plan2d(g, precision="fp64", method="auto"):
    xl, xr, yl, yr = [float(v) for v in g["dom"]]
    return Periodic2D(int(g["Nx"]), int(g["Ns"]) * int(g["N"]), int(g["N"]), xl, xr, yl, yr, Lambda=float(g["lam"]),
                      precision=precision, method=method)


def _plan3d(g, precision="fp64", method="auto"):
    xl, xr, yl, yr, zl, zr = [float(v) for v in g["dom"]]
    return Periodic3D(int(g["Nx"]), int(g["Ny"]), int(g["Ns"]) * int(g["N"]), int(g["N"]), xl, xr, yl, yr, zl, zr,
                      Lambda=float(g["lam"]), precision=precision, method=method)


@pytest.mark.parametrize("method", ["lu", "fdm"])
@pytest.mark.parametrize("precision", ["fp64", "fp32", "fp32_refine"])
@pytest.mark.parametrize("name", ["periodic_2d", "periodic_2d_ns4"])
def test_golden_periodic_2d(cuda, name, precision, method):
    g = golden(name)
    p = _plan2d(g, precision, method)
    u = p.SolvePDE(_dev(g["f"])).cpu().numpy()
    _check(u, g["u"], precision)


@pytest.mark.parametrize("method", ["lu", "fdm"])
@pytest.mark.parametrize("precision", ["fp64", "fp32", "fp32_refine"])
@pytest.mark.parametrize("name", ["periodic_3d", "periodic_3d_ns3"])
def test_golden_periodic_3d(cuda, name, precision, method):
    g = golden(name)
    p = _plan3d(g, precision, method)
    u = p.SolvePDE(_dev(g["f"])).cpu().numpy()
    _check(u, g["u"], precision)


@pytest.mark.parametrize("precision", ["fp64", "fp32", "fp32_refine"])
@pytest.mark.parametrize("Nx,N,Ns", [(64, 33, 1), (32, 65, 1), (16, 129, 1), (32, 17, 5), (16, 12, 64)])
def test_periodic_2d_vs_oracle(cuda, Nx, N, Ns, precision):
    rng = np.random.default_rng(Nx + N + Ns)
    f = rng.standard_normal((Ns, Nx, N))
    p = Periodic2D(Nx, Ns * N, N, 0.0, 2 * math.pi, 0.0, 1.7, Lambda=2.5, precision=precision)
    u = p.SolvePDE(_dev(f)).cpu().numpy()
    _check(u, O.psolve2d(f, Lx=2 * math.pi, Ly=1.7, lam=2.5), precision, Ns)


@pytest.mark.parametrize("precision", ["fp64", "fp32_refine"])
@pytest.mark.parametrize("Nx,Ny,N,Ns", [(16, 64, 33, 1), (32, 32, 65, 1), (8, 16, 17, 3)])
def test_periodic_3d_vs_oracle(cuda, Nx, Ny, N, Ns, precision):
    rng = np.random.default_rng(Nx * Ny + N + Ns)
    f = rng.standard_normal((Ns, Nx, Ny, N))
    p = Periodic3D(Nx, Ny, Ns * N, N, 0.0, 1.0, 0.0, 2.0, 0.0, 1.5, Lambda=0.8, precision=precision)
    u = p.SolvePDE(_dev(f)).cpu().numpy()
    _check(u, O.psolve3d(f, Lx=1.0, Ly=2.0, Lz=1.5, lam=0.8), precision)


def test_periodic_3d_every_launch_variant(cuda):
    """Row variants 0, 1 and the fused slab kernel (2) of an FP64 plan agree."""
    rng = np.random.default_rng(9)
    Nx, Ny, N = 16, 64, 33
    f = _dev(rng.standard_normal((Nx, Ny, N)))
    p = Periodic3D(Nx, Ny, N, N, 0.0, 1.0, 0.0, 2.0, 0.0, 1.5, Lambda=0.8)
    fft = p.launch_variants()["fft"]
    ref = O.psolve3d(f.cpu().numpy(), Lx=1.0, Ly=2.0, Lz=1.5, lam=0.8)
    ub = _dev(rng.standard_normal((Nx, Ny, N)))
    outs = []
    for rv in (0, 1, 2):
        p.set_launch_variants(fft, rv)
        u = p.SolvePDE(f)
        assert max_rel(u.cpu().numpy(), ref) < 1e-12
        fb, lb, _, _ = p.SolveAdjoint(ub, u=u)
        outs.append((fb.cpu().numpy(), lb.item()))
    for fb, lb in outs[1:]:
        assert rel_l2(fb, outs[0][0]) < 1e-12 and abs(lb - outs[0][1]) < 1e-11 * abs(outs[0][1])


def test_stock_periodic_2d_known_answer(cuda):
    """TestPeriodic2D_MPI.cpp: 512 x 512, N = 10 (Ns = 52 elements)."""
    f, ue = W.stock_periodic_2d()
    p = Periodic2D(512, 512, 10, 0.0, 1.0, 0.0, 1.0, Lambda=1.0)
    assert p.Ns == 52
    u = p.SolvePDE(_dev(f)).cpu().numpy()
    assert np.abs(u - ue).max() < 1e-11


def test_stock_periodic_3d_known_answer(cuda):
    """TestPeriodic3D_MPI.cpp: 64 x 32 x 250, N = 10 (Ns = 25 elements)."""
    f, ue = W.stock_periodic_3d()
    p = Periodic3D(64, 32, 250, 10, 0.0, 1.0, 0.0, 1.0, 0.0, 1.0, Lambda=1.0)
    assert p.Ns == 25
    u = p.SolvePDE(_dev(f)).cpu().numpy()
    assert np.abs(u - ue).max() < 1e-11


def _dense_map_2d(Nx, N, Lx, Ly, lam):
    nf = Nx * N
    S = np.zeros((nf, nf))
    for e in range(nf):
        f = np.zeros(nf)
        f[e] = 1.0
        S[:, e] = O.psolve2d(f.reshape(Nx, N), Lx=Lx, Ly=Ly, lam=lam).ravel()
    return S


def _dense_map_3d(Nx, Ny, N, Lx, Ly, Lz, lam):
    nf = Nx * Ny * N
    S = np.zeros((nf, nf))
    for e in range(nf):
        f = np.zeros(nf)
        f[e] = 1.0
        S[:, e] = O.psolve3d(f.reshape(Nx, Ny, N), Lx=Lx, Ly=Ly, Lz=Lz, lam=lam).ravel()
    return S


@pytest.mark.parametrize("precision", ["fp64", "fp32_refine"])
def test_periodic_adjoint_2d_dense(cuda, precision):
    """fbar = S^T ubar with S the oracle's forward map, and dL/dlambda = ubar . du/dlambda
    by central differences of oracle solves."""
    rng = np.random.default_rng(3)
    Nx, N, lam, Lx, Ly = 8, 9, 1.3, 2 * math.pi, 1.5
    S = _dense_map_2d(Nx, N, Lx, Ly, lam)
    ub = rng.standard_normal((Nx, N))
    f = rng.standard_normal((Nx, N))
    p = Periodic2D(Nx, N, N, 0.0, Lx, 0.0, Ly, Lambda=lam, precision=precision)
    u = p.SolvePDE(_dev(f))
    fb, lb, _, _ = p.SolveAdjoint(_dev(ub), u=u)
    fb_ref = (S.T @ ub.ravel()).reshape(Nx, N)
    assert rel_l2(fb.cpu().numpy(), fb_ref) < 1e-10
    assert np.abs(fb.cpu().numpy()[:, [0, N - 1]]).max() == 0.0
    h = 1e-6
    Lp = float(np.sum(ub * O.psolve2d(f, Lx=Lx, Ly=Ly, lam=lam + h)))
    Lm = float(np.sum(ub * O.psolve2d(f, Lx=Lx, Ly=Ly, lam=lam - h)))
    assert abs(lb.item() - (Lp - Lm) / (2 * h)) < 1e-6 * max(1.0, abs(lb.item()))


@pytest.mark.parametrize("precision", ["fp64", "fp32_refine"])
def test_periodic_adjoint_3d_dense(cuda, precision):
    rng = np.random.default_rng(4)
    Nx, Ny, N, lam, Lx, Ly, Lz = 8, 8, 9, 0.9, 1.0, 2.0, 1.5
    S = _dense_map_3d(Nx, Ny, N, Lx, Ly, Lz, lam)
    ub = rng.standard_normal((Nx, Ny, N))
    p = Periodic3D(Nx, Ny, N, N, 0.0, Lx, 0.0, Ly, 0.0, Lz, Lambda=lam, precision=precision)
    fb, _, _, _ = p.SolveAdjoint(_dev(ub))
    fb_ref = (S.T @ ub.ravel()).reshape(Nx, Ny, N)
    assert rel_l2(fb.cpu().numpy(), fb_ref) < 1e-10


def test_periodic_rejects_boundary_data_and_singular_lambda(cuda):
    p = Periodic2D(16, 9, 9, 0.0, 1.0, 0.0, 1.0, Lambda=1.0)
    f = torch.zeros(16, 9, dtype=torch.float64, device="cuda")
    with pytest.raises(ValueError):
        p.SolvePDE(f, torch.zeros(16, dtype=torch.float64, device="cuda"))
    with pytest.raises(HelmError) as e:
        Periodic2D(16, 9, 9, 0.0, 1.0, 0.0, 1.0, Lambda=0.0)
    assert e.value.status == 3
    with pytest.raises(HelmError):
        Periodic2D(16, 27, 9, 0.0, 1.0, 0.0, 1.0, Lambda=0.0)
