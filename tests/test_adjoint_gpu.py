"""The adjoint solve and the autograd wrapper (GPU).

* A dense FP64 reference gradient: the forward map (f, gl, gr) -> u of the
  oracle assembled column by column at Nx = Ny = 16, N = 17 (and a Robin case
  at 8 x 8 x 9; several GLL elements at 2D 8 x 3*7, 3D 4 x 4 x 2*7), then
  dL/d(.) = S^T ubar, compared with helm_solve_adjoint.
* Central finite differences (h = 1e-6, FP64 forward solves) of
  L = 1/2 ||u - u_obs||^2 at the 128 x 128 x 65, lambda = 5 workload for
  dL/df (directional) and dL/dlambda.
Tolerances: FP64 plans 1e-10 relative; the FP32 plan's adjoint 1e-5.
"""
import math

import numpy as np
import pytest
import torch

from mpi_b200 import NonPeriodic3D, NonPeriodic2D
from mpi_b200 import workloads as W
from mpi_b200.autograd import helmholtz_solve
from oracle import oracle as O
from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu

DOM = (0.0, 2 * math.pi, 0.0, 2 * math.pi, 0.0, 2.0)


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()


def _dense_map_3d(Nx, Ny, N, lam, bc, dom):
    """Columns of the oracle's linear map from (f, gl, gr) to u."""
    Lx, Ly, Lz = dom[1] - dom[0], dom[3] - dom[2], dom[5] - dom[4]
    nf, nb = Nx * Ny * N, Nx * Ny
    cols = []
    z = np.zeros((Nx, Ny))
    for e in range(nf + 2 * nb):
        f = np.zeros(nf); gl = np.zeros(nb); gr = np.zeros(nb)
        if e < nf:
            f[e] = 1.0
        elif e < nf + nb:
            gl[e - nf] = 1.0
        else:
            gr[e - nf - nb] = 1.0
        u = O.solve3d(f.reshape(Nx, Ny, N), gl.reshape(Nx, Ny), gr.reshape(Nx, Ny), Lx=Lx, Ly=Ly, Lz=Lz, lam=lam,
                      bc=bc)
        cols.append(u.ravel())
    return np.stack(cols, axis=1)  # [nu, nf + 2 nb]


@pytest.mark.parametrize("Nx,N,bc,lam", [(16, 17, (0.0, 1.0, 0.0, 1.0), 5.0), (8, 9, (1.0, 0.5, 0.7, 2.0), 2.0)])
def test_adjoint_matches_dense_fp64_gradient(cuda, Nx, N, bc, lam):
    Ny = Nx
    S = _dense_map_3d(Nx, Ny, N, lam, bc, DOM)
    rng = np.random.default_rng(11)
    ubar = rng.standard_normal((Nx, Ny, N))
    g = S.T @ ubar.ravel()
    nf, nb = Nx * Ny * N, Nx * Ny
    p = NonPeriodic3D(Nx, Ny, N, N, *DOM, Lambda=lam, bc=bc, precision="fp64")
    fbar, _, glb, grb = p.SolveAdjoint(_dev(ubar), want_bc=True)
    assert rel_l2(fbar.cpu().numpy().ravel(), g[:nf]) < 1e-10
    assert rel_l2(glb.cpu().numpy().ravel(), g[nf:nf + nb]) < 1e-10
    assert rel_l2(grb.cpu().numpy().ravel(), g[nf + nb:]) < 1e-10
    assert np.all(fbar.cpu().numpy()[..., 0] == 0) and np.all(fbar.cpu().numpy()[..., -1] == 0)


def _loss(plan, f, uobs):
    u = plan.SolvePDE(f)
    return 0.5 * float(((u - uobs) ** 2).sum())


def test_adjoint_central_differences_cfg4(cuda):
    """128 x 128 x 65, lambda = 5: dL/df along a smooth direction and dL/dlambda."""
    Nx, N, lam, h = 128, 65, 5.0, 1e-6
    f = _dev(W.smooth_field_3d(Nx, Nx, N, seed=1237))
    uobs = _dev(W.smooth_field_3d(Nx, Nx, N, seed=4321))
    d = _dev(W.smooth_field_3d(Nx, Nx, N, seed=99))
    p = NonPeriodic3D(Nx, Nx, N, N, *DOM, Lambda=lam, precision="fp64")
    u = p.SolvePDE(f)
    fbar, lbar, _, _ = p.SolveAdjoint(u - uobs, u=u)
    fd = (_loss(p, f + h * d, uobs) - _loss(p, f - h * d, uobs)) / (2 * h)
    ad = float((fbar * d).sum())
    assert abs(fd - ad) < 1e-6 * abs(ad)
    pp = NonPeriodic3D(Nx, Nx, N, N, *DOM, Lambda=lam + h, precision="fp64")
    pm = NonPeriodic3D(Nx, Nx, N, N, *DOM, Lambda=lam - h, precision="fp64")
    fdl = (_loss(pp, f, uobs) - _loss(pm, f, uobs)) / (2 * h)
    assert abs(fdl - float(lbar)) < 1e-6 * abs(float(lbar))


@pytest.mark.parametrize("precision", ["fp64", "fp32", "fp32_refine"])
def test_autograd_function(cuda, precision):
    Nx, N, lam = 32, 17, 5.0
    p = NonPeriodic3D(Nx, Nx, N, N, *DOM, Lambda=lam, precision=precision)
    p64 = NonPeriodic3D(Nx, Nx, N, N, *DOM, Lambda=lam, precision="fp64")
    f = _dev(W.smooth_field_3d(Nx, Nx, N, seed=5)).requires_grad_(True)
    lamt = torch.tensor(lam, dtype=torch.float64, device="cuda", requires_grad=True)
    uobs = _dev(W.smooth_field_3d(Nx, Nx, N, seed=6))
    u = helmholtz_solve(p, f, lamt)
    loss = 0.5 * ((u - uobs) ** 2).sum()
    loss.backward()
    u64 = p64.SolvePDE(f.detach())
    fbar, lbar, _, _ = p64.SolveAdjoint(u64 - uobs, u=u64)
    tol = 1e-5 if precision == "fp32" else 1e-10
    assert rel_l2(f.grad.cpu().numpy(), fbar.cpu().numpy()) < tol
    assert abs(lamt.grad.item() - lbar.item()) < tol * abs(lbar.item())


def test_adjoint_2d(cuda):
    """2D plans share the adjoint path (one Fourier direction)."""
    Nx, N, lam = 16, 9, 2.0
    bc = (1.0, 0.5, 0.7, 2.0)
    nf = Nx * N
    cols = []
    for e in range(nf + 2 * Nx):
        f = np.zeros(nf); gl = np.zeros(Nx); gr = np.zeros(Nx)
        if e < nf:
            f[e] = 1
        elif e < nf + Nx:
            gl[e - nf] = 1
        else:
            gr[e - nf - Nx] = 1
        cols.append(O.solve2d(f.reshape(Nx, N), gl, gr, Lx=1.3, Ly=0.9, lam=lam, bc=bc).ravel())
    S = np.stack(cols, axis=1)
    ubar = np.random.default_rng(3).standard_normal((Nx, N))
    g = S.T @ ubar.ravel()
    p = NonPeriodic2D(Nx, N, N, 0.0, 1.3, 0.0, 0.9, Lambda=lam, bc=bc)
    fbar, _, glb, grb = p.SolveAdjoint(_dev(ubar[None]), want_bc=True)
    assert rel_l2(fbar.cpu().numpy().ravel(), g[:nf]) < 1e-10
    assert rel_l2(glb.cpu().numpy(), g[nf:nf + Nx]) < 1e-10
    assert rel_l2(grb.cpu().numpy(), g[nf + Nx:]) < 1e-10


def _dense_map_elems(dim, Nx, N, Ns, lam, bc, lengths):
    """Columns of the oracle's map (f [Ns, Nx, (Ny,) N], gl, gr) -> u with
    several GLL elements (the interface system of the reference's solver)."""
    fshape = (Ns, Nx, N) if dim == 2 else (Ns, Nx, Nx, N)
    bshape = (Nx,) if dim == 2 else (Nx, Nx)
    nf, nb = int(np.prod(fshape)), int(np.prod(bshape))
    cols = []
    for e in range(nf + 2 * nb):
        v = np.zeros(nf + 2 * nb)
        v[e] = 1.0
        f, gl, gr = v[:nf].reshape(fshape), v[nf:nf + nb].reshape(bshape), v[nf + nb:].reshape(bshape)
        if dim == 2:
            u = O.solve2d(f, gl, gr, Lx=lengths[0], Ly=lengths[1], lam=lam, bc=bc)
        else:
            u = O.solve3d(f, gl, gr, Lx=lengths[0], Ly=lengths[1], Lz=lengths[2], lam=lam, bc=bc)
        cols.append(u.ravel())
    return np.stack(cols, axis=1), fshape, bshape


@pytest.mark.parametrize("dim,Nx,N,Ns,bc,precision", [
    (2, 8, 7, 3, (1.0, 0.5, 0.7, 2.0), "fp64"),
    (2, 8, 9, 3, (0.0, 1.0, 0.0, 1.0), "fp32_refine"),
    (2, 8, 7, 3, (1.0, 0.5, 0.7, 2.0), "fp32"),
    (3, 4, 7, 2, (0.4, 1.0, 0.3, 2.0), "fp64"),
    (3, 4, 9, 2, (0.0, 1.0, 0.0, 1.0), "fp32_refine"),
])
def test_adjoint_several_elements_dense(cuda, dim, Nx, N, Ns, bc, precision):
    """The transposed interface system: S^T ubar of the oracle's dense map,
    and lambda_bar against central differences of the oracle's forward solve."""
    lam = 2.0
    lengths = (1.3, 0.9) if dim == 2 else (1.3, 1.1, 0.9)
    S, fshape, bshape = _dense_map_elems(dim, Nx, N, Ns, lam, bc, lengths)
    rng = np.random.default_rng(17 + dim)
    ubar = rng.standard_normal(fshape)
    g = S.T @ ubar.ravel()
    nf, nb = int(np.prod(fshape)), int(np.prod(bshape))
    if dim == 2:
        p = NonPeriodic2D(Nx, Ns * N, N, 0.0, lengths[0], 0.0, lengths[1], Lambda=lam, bc=bc, precision=precision)
    else:
        p = NonPeriodic3D(Nx, Nx, Ns * N, N, 0.0, lengths[0], 0.0, lengths[1], 0.0, lengths[2], Lambda=lam, bc=bc,
                          precision=precision)
    f = rng.standard_normal(fshape)
    if dim == 2:
        solve = lambda lm: O.solve2d(f, np.zeros(bshape), np.zeros(bshape), Lx=lengths[0], Ly=lengths[1], lam=lm,
                                     bc=bc)
    else:
        solve = lambda lm: O.solve3d(f, np.zeros(bshape), np.zeros(bshape), Lx=lengths[0], Ly=lengths[1],
                                     Lz=lengths[2], lam=lm, bc=bc)
    h = 1e-5
    dlam = float((solve(lam + h) - solve(lam - h)).ravel() @ ubar.ravel()) / (2 * h)
    u = solve(lam)
    fbar, lbar, glb, grb = p.SolveAdjoint(_dev(ubar), u=_dev(u), want_bc=True)
    tol = 1e-4 if precision == "fp32" else 1e-10
    assert rel_l2(fbar.cpu().numpy().ravel(), g[:nf]) < tol
    assert rel_l2(glb.cpu().numpy().ravel(), g[nf:nf + nb]) < tol
    assert rel_l2(grb.cpu().numpy().ravel(), g[nf + nb:]) < tol
    fb = fbar.cpu().numpy()
    assert np.all(fb[..., 0] == 0) and np.all(fb[..., -1] == 0)
    # central differences carry ~1e-9 of their own
    assert abs(lbar.item() - dlam) < max(tol, 1e-7) * abs(dlam)


@pytest.mark.parametrize("bc", [(0.0, 1.0, 0.0, 1.0), (0.4, 1.0, 0.3, 2.0)])
def test_adjoint_slab_variant(cuda, bc):
    """The fused slab kernel (row variant 2 of FP64 3D plans) in the adjoint
    solve gives the same fbar, glbar, grbar and lambda_bar as the separate passes."""
    rng = np.random.default_rng(21)
    Nx, Ny, N, lam = 16, 64, 33, 4.0
    p = NonPeriodic3D(Nx, Ny, N, N, *DOM, Lambda=lam, bc=bc, precision="fp64")
    f = _dev(rng.standard_normal((Nx, Ny, N)))
    ubar = _dev(rng.standard_normal((Nx, Ny, N)))
    outs = []
    for rv in (0, 2):
        p.set_launch_variants([0, 0, 0, 0], rv)
        u = p.SolvePDE(f)
        fb, lb, glb, grb = p.SolveAdjoint(ubar, u=u, want_bc=True)
        outs.append([x.cpu().numpy() for x in (u, fb, lb, glb, grb)])
    for a, b in zip(outs[0], outs[1]):
        assert rel_l2(b, a) < 1e-12


@pytest.mark.parametrize("kind", ["fp64", "fp32_refine", "fp32", "fd", "periodic"])
def test_misfit_adjoint_matches_explicit_ubar(cuda, kind):
    """helm_solve_adjoint_misfit (ubar = u - u_obs formed in the first pass) gives the
    gradients of helm_solve_adjoint on an explicit ubar."""
    from mpi_b200 import Helmholtz3DFD, Periodic3D

    rng = np.random.default_rng(31)
    bc = (0.4, 1.0, 0.3, 2.0)
    if kind == "fd":
        p = Helmholtz3DFD(16, 8, 12, 0.0, 1.0, 0.0, 2.0, 0.0, 1.5, Lambda=1.0, bc=bc)
        shape, want_bc = (16, 8, 12), True
    elif kind == "periodic":
        p = Periodic3D(16, 8, 17, 17, 0.0, 1.0, 0.0, 2.0, 0.0, 1.5, Lambda=1.0)
        shape, want_bc = (16, 8, 17), False
    else:
        p = NonPeriodic3D(16, 8, 17, 17, 0.0, 1.0, 0.0, 2.0, 0.0, 1.5, Lambda=1.0, bc=bc, precision=kind)
        shape, want_bc = (16, 8, 17), True
    f = _dev(rng.standard_normal(shape))
    uobs = _dev(rng.standard_normal(shape))
    u = p.SolvePDE(f).double()
    if kind == "fp32":
        uobs = uobs.float().double()
    a = p.SolveAdjoint((u - uobs).contiguous(), u=u, want_bc=want_bc)
    b = p.SolveAdjointMisfit(u, uobs, want_bc=want_bc)
    tol = 1e-5 if kind == "fp32" else 1e-13
    assert rel_l2(b[0].cpu().numpy(), a[0].cpu().numpy()) < tol
    assert abs(b[1].item() - a[1].item()) <= tol * abs(a[1].item())
    if want_bc:
        for x, y in zip(b[2:], a[2:]):
            assert rel_l2(x.cpu().numpy(), y.cpu().numpy()) < tol
