"""The finite-difference FFT/Thomas variant on the GPU (the HypreFDM stencil with
periodic x, y and Robin rows in z).  Parity against the reference's own
HypreFDM 3D assembly (Helmholtz3D_MPI.cpp SetA / Setb with the assembled system
solved directly: tests/golden/fd3d_reference.npz), against the C restatement
(oracle/helm_oracle.c: orc_fd3d_solve, itself pinned to those goldens) and, at
the 1024 x 1024 x 256 size, through the stencil residual of the GPU solution
itself.  Tolerances: FP64 1e-12 relative; FP32 eps_32 times the condition
number of the worst spectrum row."""
import math

import numpy as np
import pytest
import torch

from mpi_b200 import Helmholtz3DFD
from mpi_b200 import workloads as W
from oracle import oracle as O
from tests.helpers import max_rel, rel_l2

pytestmark = pytest.mark.gpu


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()


def _stencil_residual(u, f, gb, gf, Lx, Ly, Lz, lam, bc):
    """||f - A_h u|| / ||f|| of the HypreFDM stencil, evaluated on the GPU (FP64)."""
    Nx, Ny, Nz = u.shape
    dx, dy, dz = Lx / Nx, Ly / Ny, Lz / (Nz + 1)
    cx1, cy1, cz0, cz1 = 1 / dx**2, 1 / dy**2, 1 / dz, 1 / dz**2
    ab, bb, af, bf = bc
    a0, a1, a2 = 1.5 * ab * cz0 + bb, -2 * ab * cz0, 0.5 * ab * cz0
    e0, e1, e2 = 1.5 * af * cz0 + bf, -2 * af * cz0, 0.5 * af * cz0
    u0 = (gb - a1 * u[:, :, 0] - a2 * u[:, :, 1]) / a0
    uN = (gf - e1 * u[:, :, -1] - e2 * u[:, :, -2]) / e0
    um = torch.cat([u0[:, :, None], u[:, :, :-1]], dim=2)
    up = torch.cat([u[:, :, 1:], uN[:, :, None]], dim=2)
    au = (cx1 * (torch.roll(u, 1, 0) + torch.roll(u, -1, 0)) + cy1 * (torch.roll(u, 1, 1) + torch.roll(u, -1, 1))
          + cz1 * (um + up) + (-2 * (cx1 + cy1 + cz1) - lam) * u)
    return ((f - au).norm() / f.norm()).item()


@pytest.mark.parametrize("precision", ["fp64", "fp32_refine"])
def test_fd_matches_reference_golden(cuda, precision):
    """The GPU FD solve against the reference's own discretisation: Dirichlet,
    Robin and mixed ends (FP64 1e-12, refined 1e-10 relative, max-norm)."""
    from tests.helpers import golden
    g = golden("fd3d_reference")
    for c in range(int(g["ncases"])):
        f = g[f"f{c}"]
        Nx, Ny, Nz = f.shape
        Lx, Ly, Lz = (float(v) for v in g[f"L{c}"])
        bc = tuple(float(v) for v in g[f"bc{c}"])
        p = Helmholtz3DFD(Nx, Ny, Nz, 0.0, Lx, 0.0, Ly, 0.0, Lz, Lambda=float(g[f"lam{c}"]), bc=bc,
                          precision=precision)
        u = p.SolvePDE(_dev(f), _dev(g[f"gb{c}"]), _dev(g[f"gf{c}"])).double().cpu().numpy()
        err = max_rel(u, g[f"u{c}"])
        assert err < (1e-12 if precision == "fp64" else 1e-10), f"case {c}: {err:.3e}"


@pytest.mark.parametrize("precision", ["fp64", "fp32_refine"])
def test_fd_adjoint_matches_reference_golden(cuda, precision):
    """The GPU FD adjoint (fbar and both Robin-data cotangents) against the
    transpose of the reference's own assembled matrix (FP64 1e-12, refined
    1e-10 relative, max-norm)."""
    from tests.helpers import golden
    g = golden("fd3d_reference")
    for c in range(int(g["ncases"])):
        ub = g[f"ubar{c}"]
        Nx, Ny, Nz = ub.shape
        Lx, Ly, Lz = (float(v) for v in g[f"L{c}"])
        bc = tuple(float(v) for v in g[f"bc{c}"])
        p = Helmholtz3DFD(Nx, Ny, Nz, 0.0, Lx, 0.0, Ly, 0.0, Lz, Lambda=float(g[f"lam{c}"]), bc=bc,
                          precision=precision)
        fb, _, gbb, gfb = p.SolveAdjoint(_dev(ub), want_bc=True)
        tol = 1e-12 if precision == "fp64" else 1e-10
        for name, got, want in (("fbar", fb, g[f"fbar{c}"]), ("gbbar", gbb, g[f"gbbar{c}"]),
                                ("gfbar", gfb, g[f"gfbar{c}"])):
            err = max_rel(got.cpu().numpy(), want)
            assert err < tol, f"case {c} {name}: {err:.3e}"


@pytest.mark.parametrize("rows", [0, 1])
@pytest.mark.parametrize("bc", [(0.0, 1.0, 0.0, 1.0), (1.0, 0.5, 0.7, 2.0)])
@pytest.mark.parametrize("shape", [(16, 8, 12), (8, 32, 2), (64, 64, 33), (8, 8, 100), (8, 4, 300), (4, 4, 600),
                                   (8, 4, 256)])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_fd_matches_oracle(cuda, bc, shape, precision, rows):
    """Both tridiagonal shapes (row variant 0: a row per warp; 1: a row per
    half-warp for Nz <= 256, ignored above)."""
    rng = np.random.default_rng(hash((shape, bc)) % 2**32)
    Nx, Ny, Nz = shape
    f = rng.standard_normal(shape); gb = rng.standard_normal((Nx, Ny)); gf = rng.standard_normal((Nx, Ny))
    ref = O.fd3d_solve(f, gb, gf, Lx=1.0, Ly=2.0, Lz=1.5, lam=1.0, bc=bc)
    p = Helmholtz3DFD(Nx, Ny, Nz, 0.0, 1.0, 0.0, 2.0, 0.0, 1.5, Lambda=1.0, bc=bc, precision=precision)
    p.set_launch_variants(p.launch_variants()["fft"], rows)
    u = p.SolvePDE(_dev(f), _dev(gb), _dev(gf)).cpu().numpy()
    if precision == "fp64":
        assert max_rel(u, ref) < 1e-12
    else:
        # FP32 bound: eps_32 times the condition of the worst row, the kx = ky = 0
        # one, ~(4 cz1 + lambda) / lambda with cz1 = ((Nz + 1) / Lz)^2
        kappa = (4.0 * ((Nz + 1) / 1.5) ** 2 + 1.0) / 1.0
        assert rel_l2(u, ref) < 6e-8 * kappa


def test_fd_full_size_residual(cuda):
    """1024 x 1024 periodic x 256 interior points, Dirichlet, lambda = 1: the GPU
    solution satisfies the stencil to rounding, and FP32 agrees with FP64."""
    Nx, Ny, Nz = 1024, 1024, 256
    f = _dev(W.smooth_field_fd(Nx, Ny, Nz, seed=1239))
    z = torch.zeros((Nx, Ny), dtype=torch.float64, device="cuda")
    p64 = Helmholtz3DFD(Nx, Ny, Nz, 0.0, 1.0, 0.0, 1.0, 0.0, 1.0, Lambda=1.0)
    u = p64.SolvePDE(f)
    # floor of an FP64 residual: eps * ||A|| ||u|| / ||f|| with ||A|| ~ 8.6e6 (cx1 = cy1 =
    # 1024^2, cz1 = 257^2) and ||u|| / ||f|| ~ 6e-4 is ~1e-12 before the FFT's log factors
    assert _stencil_residual(u, f, z, z, 1.0, 1.0, 1.0, 1.0, (0.0, 1.0, 0.0, 1.0)) < 1e-10
    p64.DestroyPDEPlan()
    p32 = Helmholtz3DFD(Nx, Ny, Nz, 0.0, 1.0, 0.0, 1.0, 0.0, 1.0, Lambda=1.0, precision="fp32")
    u32 = p32.SolvePDE(f)
    # FP32 Thomas on the lowest modes: diagonal -2 cz1 - 1 against cz1 = 257^2, a
    # conditioning of ~2.4e4, so ~1e-4 is the FP32 accuracy of this stencil
    assert ((u32 - u).norm() / u.norm()).item() < 1e-3


def test_fd_robin_residual_midsize(cuda):
    Nx, Ny, Nz = 128, 64, 100
    rng = np.random.default_rng(4)
    bc = (1.0, 0.5, 0.7, 2.0)
    f = _dev(W.smooth_field_fd(Nx, Ny, Nz, seed=7))
    gb, gf = _dev(rng.standard_normal((Nx, Ny))), _dev(rng.standard_normal((Nx, Ny)))
    p = Helmholtz3DFD(Nx, Ny, Nz, 0.0, 1.0, 0.0, 2.0, 0.0, 1.5, Lambda=1.0, bc=bc)
    u = p.SolvePDE(f, gb, gf)
    assert _stencil_residual(u, f, gb, gf, 1.0, 2.0, 1.5, 1.0, bc) < 1e-11


@pytest.mark.parametrize("bc", [(0.0, 1.0, 0.0, 1.0), (1.0, 0.5, 0.7, 2.0)])
@pytest.mark.parametrize("rows", [0, 1])
def test_fd_adjoint_dense(cuda, bc, rows):
    Nx, Ny, Nz, lam = 8, 4, 5, 2.0
    nf, nb = Nx * Ny * Nz, Nx * Ny
    cols = []
    for e in range(nf + 2 * nb):
        f = np.zeros(nf); gb = np.zeros(nb); gf = np.zeros(nb)
        if e < nf:
            f[e] = 1
        elif e < nf + nb:
            gb[e - nf] = 1
        else:
            gf[e - nf - nb] = 1
        cols.append(O.fd3d_solve(f.reshape(Nx, Ny, Nz), gb.reshape(Nx, Ny), gf.reshape(Nx, Ny), Lx=1.0, Ly=1.3,
                                 Lz=0.8, lam=lam, bc=bc).ravel())
    S = np.stack(cols, axis=1)
    ubar = np.random.default_rng(9).standard_normal((Nx, Ny, Nz))
    g = S.T @ ubar.ravel()
    p = Helmholtz3DFD(Nx, Ny, Nz, 0.0, 1.0, 0.0, 1.3, 0.0, 0.8, Lambda=lam, bc=bc)
    p.set_launch_variants(p.launch_variants()["fft"], rows)
    fbar, _, glb, grb = p.SolveAdjoint(_dev(ubar), want_bc=True)
    assert rel_l2(fbar.cpu().numpy().ravel(), g[:nf]) < 1e-10
    assert rel_l2(glb.cpu().numpy().ravel(), g[nf:nf + nb]) < 1e-10
    assert rel_l2(grb.cpu().numpy().ravel(), g[nf + nb:]) < 1e-10


def test_fd_lambda_gradient(cuda):
    # h = 1e-4: with a loss of ~3e3, h = 1e-6 leaves only ~6 digits of the difference
    Nx, Ny, Nz, lam, h = 32, 32, 40, 1.0, 1e-4
    f = _dev(W.smooth_field_fd(Nx, Ny, Nz, seed=3))
    uobs = _dev(W.smooth_field_fd(Nx, Ny, Nz, seed=5))
    mk = lambda L: Helmholtz3DFD(Nx, Ny, Nz, 0.0, 1.0, 0.0, 1.0, 0.0, 1.0, Lambda=L)  # noqa: E731
    p = mk(lam)
    u = p.SolvePDE(f)
    _, lbar, _, _ = p.SolveAdjoint(u - uobs, u=u)
    loss = lambda q: 0.5 * float(((q.SolvePDE(f) - uobs) ** 2).sum())  # noqa: E731
    fd = (loss(mk(lam + h)) - loss(mk(lam - h))) / (2 * h)
    assert abs(fd - float(lbar)) < 1e-6 * abs(float(lbar))


@pytest.mark.parametrize("bc", [(0.0, 1.0, 0.0, 1.0), (1.0, 0.5, 0.7, 2.0)])
@pytest.mark.parametrize("shape", [(16, 8, 12), (8, 32, 2), (64, 64, 33), (4, 4, 600)])
def test_fd_refined_matches_oracle(cuda, bc, shape):
    """FP32 solves with two FP64-residual refinement sweeps reach FP64 accuracy
    (1e-10 relative) against the restatement, forward and adjoint (fbar, the
    boundary cotangents, lambda_bar) against the FP64 plan."""
    rng = np.random.default_rng(hash((shape, bc, 1)) % 2**32)
    Nx, Ny, Nz = shape
    f = rng.standard_normal(shape); gb = rng.standard_normal((Nx, Ny)); gf = rng.standard_normal((Nx, Ny))
    ref = O.fd3d_solve(f, gb, gf, Lx=1.0, Ly=2.0, Lz=1.5, lam=1.0, bc=bc)
    pr = Helmholtz3DFD(Nx, Ny, Nz, 0.0, 1.0, 0.0, 2.0, 0.0, 1.5, Lambda=1.0, bc=bc, precision="fp32_refine")
    assert pr.kernels().count("fd_residual_kernel") == 2
    u = pr.SolvePDE(_dev(f), _dev(gb), _dev(gf))
    assert rel_l2(u.cpu().numpy(), ref) < 1e-10
    p64 = Helmholtz3DFD(Nx, Ny, Nz, 0.0, 1.0, 0.0, 2.0, 0.0, 1.5, Lambda=1.0, bc=bc)
    u64 = p64.SolvePDE(_dev(f), _dev(gb), _dev(gf))
    ubar = _dev(rng.standard_normal(shape))
    got = pr.SolveAdjoint(ubar, u=u64, want_bc=True)
    want = p64.SolveAdjoint(ubar, u=u64, want_bc=True)
    for a, b in zip(got, want):
        assert rel_l2(a.cpu().numpy(), b.cpu().numpy()) < 1e-10
    uobs = _dev(rng.standard_normal(shape))
    got = pr.SolveAdjointMisfit(u64, uobs, want_bc=True)
    want = p64.SolveAdjointMisfit(u64, uobs, want_bc=True)
    for a, b in zip(got, want):
        assert rel_l2(a.cpu().numpy(), b.cpu().numpy()) < 1e-10


def test_fd_refined_full_size(cuda):
    """1024 x 1024 x 256: the refined solve against the FP64 solve, and the
    sweeps' effect (one sweep is not enough at this conditioning, two are)."""
    Nx, Ny, Nz = 1024, 1024, 256
    f = _dev(W.smooth_field_fd(Nx, Ny, Nz, seed=1239))
    p64 = Helmholtz3DFD(Nx, Ny, Nz, 0.0, 1.0, 0.0, 1.0, 0.0, 1.0, Lambda=1.0)
    u64 = p64.SolvePDE(f)
    p64.DestroyPDEPlan()
    pr = Helmholtz3DFD(Nx, Ny, Nz, 0.0, 1.0, 0.0, 1.0, 0.0, 1.0, Lambda=1.0, precision="fp32_refine")
    errs = []
    for sweeps in (0, 1, 2):
        pr.set_refine_sweeps(sweeps)
        u = pr.SolvePDE(f)
        errs.append(((u - u64).norm() / u64.norm()).item())
    assert errs[0] > 1e-6 and errs[1] < errs[0] * 1e-2 and errs[2] < 1e-10, errs
