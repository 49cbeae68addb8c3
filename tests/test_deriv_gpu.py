"""The derivative helpers on the solver's arrays (GPU).

helm_gll_derivative (du = Dy u / Dyy u element by element: the reference's
FirstDerivativeY/Z, SecondDerivativeY/Z) and helm_fourier_derivative (spectral
d/dx, d/dy: FirstDerivativeFourierX/Y, SecondDerivativeFourierX/Y) against the
reference's own outputs (tests/golden/derivatives.npz) and the oracle's
restatement at larger sizes.  Tolerances: FP64 1e-12 relative (max-norm), FP32
(float arrays) 1e-5 relative L2.
"""
import math

import numpy as np
import pytest
import torch

from mpi_b200 import NonPeriodic2D, NonPeriodic3D, Periodic3D
from oracle import oracle as O
from tests.helpers import golden, max_rel, rel_l2

pytestmark = pytest.mark.gpu


def _dev(a, dtype=torch.float64):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to("cuda", dtype)


@pytest.mark.parametrize("order", [1, 2])
def test_golden_derivatives(cuda, order):
    g = golden("derivatives")
    first = order == 1
    # 2D Fourier x, one element
    p = NonPeriodic2D(16, 9, 9, 0.0, float(g["L2"]), -1.0, 1.0, Lambda=1.0)
    d = (p.FirstDerivativeX if first else p.SecondDerivativeX)(_dev(g["u2"]))
    assert max_rel(d.cpu().numpy(), g[f"fx2_{order}"]) < 1e-12
    # 2D GLL y, three elements
    p = NonPeriodic2D(8, 27, 9, 0.0, 1.0, float(g["yl"]), float(g["yr"]), Lambda=1.0)
    d = (p.FirstDerivativeY if first else p.SecondDerivativeY)(_dev(g["ug2"]))
    assert max_rel(d.cpu().numpy(), g[f"gy2_{order}"]) < 1e-12
    # 3D Fourier x and y
    p = NonPeriodic3D(8, 16, 5, 5, 0.0, float(g["L3x"]), 0.0, float(g["L3y"]), 0.0, 1.0, Lambda=1.0)
    u3 = _dev(g["u3"])
    d = (p.FirstDerivativeX if first else p.SecondDerivativeX)(u3)
    assert max_rel(d.cpu().numpy(), g[f"fx3_{order}"]) < 1e-12
    d = (p.FirstDerivativeY if first else p.SecondDerivativeY)(u3)
    assert max_rel(d.cpu().numpy(), g[f"fy3_{order}"]) < 1e-12
    # 3D GLL z, two elements
    p = NonPeriodic3D(4, 8, 14, 7, 0.0, 1.0, 0.0, 1.0, float(g["zl"]), float(g["zr"]), Lambda=1.0)
    d = (p.FirstDerivativeZ if first else p.SecondDerivativeZ)(_dev(g["ug3"]))
    assert max_rel(d.cpu().numpy(), g[f"gz3_{order}"]) < 1e-12


@pytest.mark.parametrize("order", [1, 2])
@pytest.mark.parametrize("Nx,Ny,N,Ns", [(64, 64, 65, 1), (64, 16, 33, 1), (16, 32, 129, 1), (32, 8, 10, 3),
                                        (8, 4, 64, 1)])
def test_derivatives_3d_vs_oracle(cuda, Nx, Ny, N, Ns, order):
    rng = np.random.default_rng(Nx + Ny + N + order)
    Lx, Ly, Lz = 2 * math.pi, 1.5, 2.0
    u = rng.standard_normal((Ns, Nx, Ny, N))
    p = NonPeriodic3D(Nx, Ny, Ns * N, N, 0.0, Lx, 0.0, Ly, 0.0, Lz, Lambda=1.0)
    ud = _dev(u)
    for axis, L in ((0, Lx), (1, Ly)):
        d = p._derivative(axis, order, ud, None, None).cpu().numpy()
        ref = np.stack([O.fourier_deriv(u[e], axis=axis, order=order, L=L) for e in range(Ns)])
        assert max_rel(d, ref) < 1e-12
    d = p._derivative(2, order, ud, None, None).cpu().numpy()
    assert max_rel(d, O.gll_deriv(u, N=N, Ns=Ns, L=Lz, order=order)) < 1e-12


def test_gll_derivative_in_place_and_float_io(cuda):
    rng = np.random.default_rng(7)
    Nx, Ny, N = 32, 32, 65
    u = rng.standard_normal((Nx, Ny, N))
    ref = O.gll_deriv(u, N=N, Ns=1, L=2.0, order=1)
    p = NonPeriodic3D(Nx, Ny, N, N, 0.0, 1.0, 0.0, 1.0, 0.0, 2.0, Lambda=1.0)
    ud = _dev(u)
    p.FirstDerivativeZ(ud, out=ud)
    assert max_rel(ud.cpu().numpy(), ref) < 1e-12
    q = NonPeriodic3D(Nx, Ny, N, N, 0.0, 1.0, 0.0, 1.0, 0.0, 2.0, Lambda=1.0, precision="fp32")
    q.set_io_bytes(4)
    uf = _dev(u, torch.float32)
    assert rel_l2(q.FirstDerivativeZ(uf).double().cpu().numpy(), ref) < 1e-5
    fx = O.fourier_deriv(u, axis=0, order=1, L=1.0)
    assert rel_l2(q.FirstDerivativeX(uf).double().cpu().numpy(), fx) < 1e-5


def test_derivative_of_solution_closes_the_equation(cuda):
    """u_xx + u_yy + u_zz - lambda u = f at the interior GLL nodes, with every
    second derivative taken by the helpers on the solver's own output."""
    rng = np.random.default_rng(11)
    Nx, Ny, N, lam = 32, 32, 33, 3.0
    f = rng.standard_normal((Nx, Ny, N))
    p = Periodic3D(Nx, Ny, N, N, 0.0, 2 * math.pi, 0.0, 2 * math.pi, 0.0, 2.0, Lambda=lam)
    fd = _dev(f)
    u = p.SolvePDE(fd)
    r = p.SecondDerivativeX(u) + p.SecondDerivativeY(u) + p.SecondDerivativeZ(u) - lam * u - fd
    # the discrete spectrum keeps the Nyquist modes of f that the solution cannot
    # represent in a first derivative; the second-derivative residual is exact
    assert r[:, :, 1:N - 1].abs().max().item() < 1e-9 * fd.abs().max().item()


def test_derivative_rejects_bad_axis(cuda):
    p = NonPeriodic2D(16, 9, 9, 0.0, 1.0, 0.0, 1.0, Lambda=1.0)
    u = torch.zeros(16, 9, dtype=torch.float64, device="cuda")
    with pytest.raises(ValueError):
        p.FirstDerivativeZ(u)
    from mpi_b200._lib import HelmError
    with pytest.raises(HelmError):
        p._derivative(1, 3, u, None, None)


def test_derivatives_in_the_reference_array_layout(cuda):
    """Padded reference arrays (U.phi[2Nx][2Ny][N] per element, two elements): the
    derivatives read and write only the solution rows, per element, through the
    plan's strides; the padding is left untouched."""
    rng = np.random.default_rng(23)
    Nx, Ny, N, Ns = 8, 16, 9, 2
    u = rng.standard_normal((Ns, Nx, Ny, N))
    p = NonPeriodic3D(Nx, Ny, Ns * N, N, 0.0, 1.0, 0.0, 2.0, 0.0, 3.0, Lambda=1.0)
    p.set_layout(x_stride=2 * Ny * N, elem_stride=2 * Nx * 2 * Ny * N, bc_x_stride=2 * Ny)
    U = np.zeros((Ns, 2 * Nx, 2 * Ny, N))
    U[:, :Nx, :Ny] = u
    ud = _dev(U)
    stream = torch.cuda.current_stream().cuda_stream
    cases = [(lambda o: p._lib.helm_fourier_derivative(p._plan, 0, 1, ud.data_ptr(), o.data_ptr(), stream),
              np.stack([O.fourier_deriv(u[e], axis=0, order=1, L=1.0) for e in range(Ns)])),
             (lambda o: p._lib.helm_fourier_derivative(p._plan, 1, 2, ud.data_ptr(), o.data_ptr(), stream),
              np.stack([O.fourier_deriv(u[e], axis=1, order=2, L=2.0) for e in range(Ns)])),
             (lambda o: p._lib.helm_gll_derivative(p._plan, 1, ud.data_ptr(), o.data_ptr(), stream),
              O.gll_deriv(u, N=N, Ns=Ns, L=3.0, order=1))]
    for run, ref in cases:
        od = torch.full(U.shape, 5.0, dtype=torch.float64, device="cuda")
        assert run(od) == 0
        torch.cuda.synchronize()
        D = od.cpu().numpy()
        assert max_rel(D[:, :Nx, :Ny], ref) < 1e-12
        assert np.all(D[:, Nx:] == 5.0) and np.all(D[:, :, Ny:] == 5.0)


@pytest.mark.parametrize("Nx,Ny,N,prec", [(256, 64, 33, "fp64"), (1024, 8, 9, "fp64"), (32, 512, 5, "fp64"),
                                          (4, 16, 7, "fp64"), (256, 32, 17, "fp32"), (1024, 4, 9, "fp32")])
def test_fourier_derivative_every_launch_variant(cuda, Nx, Ny, N, prec):
    """Every launch shape of the spectral derivative (plain and persistent
    pipelined kernels, 128/256/512/1024-thread CTAs, radix-8 and radix-16
    schedules) against the oracle, with odd column counts (a lone last column)
    and, at 256 x 64 x 33, more tiles than the persistent grid has CTAs.
    Pipelined shapes whose two tile buffers exceed shared memory are refused
    with an error, not run."""
    from mpi_b200._lib import HelmError
    rng = np.random.default_rng(Nx * 7 + Ny + N)
    Lx, Ly = 2 * math.pi, 1.5
    u = rng.standard_normal((Nx, Ny, N))
    p = NonPeriodic3D(Nx, Ny, N, N, 0.0, Lx, 0.0, Ly, 0.0, 2.0, Lambda=1.0, precision=prec)
    fp32 = prec == "fp32"
    if fp32:
        p.set_io_bytes(4)
    ud = _dev(u, torch.float32 if fp32 else torch.float64)
    refs = {(a, o): O.fourier_deriv(u, axis=a, order=o, L=(Lx, Ly)[a]) for a in (0, 1) for o in (1, 2)}
    assert p.derivative_variant() == -1
    for v in [-1] + list(range(16)):
        p.set_derivative_variant(v)
        for (axis, order), ref in refs.items():
            L_ax = (Nx, Ny)[axis]
            try:
                d = p._derivative(axis, order, ud, None, None).double().cpu().numpy()
            except HelmError:
                assert v & 4 and L_ax >= 512, f"variant {v} refused on length {L_ax}"
                continue
            err = rel_l2(d, ref) if fp32 else max_rel(d, ref)
            assert err < (1e-5 if fp32 else 1e-12), f"variant {v}, axis {axis}, order {order}: {err:.3e}"
    with pytest.raises(HelmError):
        p.set_derivative_variant(16)
