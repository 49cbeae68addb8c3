"""The eigen-basis pipeline (row variant 4, helm_eig.cu) and the FP64 row kernel
of refined plans (row variant 3) against the oracle.

The pipeline applies the GLL eigen-transform before the x FFT and its inverse
after the inverse x FFT, so every shape, boundary datum and layout it accepts
is checked here with the variant pinned: 2D (one fused launch) and 3D (three
launches), Dirichlet data with beta != 1, sizes from the smallest transform
lengths to the full 256 x 256 x 65 workload, the reference's padded array
layout, and the cases it must decline (Robin ends, several elements, periodic
plans).  Tolerances: 1e-12 relative (max-norm) for FP64 arithmetic, which both
FP64 plans and refined plans running these variants use.
"""
import math

import numpy as np
import pytest
import torch

from mpi_b200 import NonPeriodic2D, NonPeriodic3D, Periodic3D
from mpi_b200 import workloads as W
from mpi_b200._lib import HelmError
from oracle import oracle as O
from tests.helpers import golden, max_rel, rel_l2

pytestmark = pytest.mark.gpu

BC_DIR = (0.0, 0.5, 0.0, 2.0)  # Dirichlet ends with beta_l = 0.5, beta_r = 2
KERNELS3 = {4: "eig_fwd_kernel eig_conv_kernel eig_inv_kernel"}
KERNELS3_SPLIT = "eig_fwd_split_kernel eig_conv_kernel eig_inv_split_kernel"


def _status_ok(p):
    """No bounded wait on a TMA copy ran out (device status word 0)."""
    assert p.device_status() == 0


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()


def _pin(p, rows, conv=None):
    """Pins the row variant (and, given conv, bits 0-1 of the y-pass variant:
    bit 0 the CTA shape of the 3D second pass, 0 = 16 columns x 256 threads,
    1 = 8 x 128; bit 1 the pair-split first and third passes, Nx >= 64)."""
    fft = p.launch_variants()["fft"]
    if conv is not None:
        fft[1] = (fft[1] & ~3) | conv
    p.set_launch_variants(fft, rows)
    assert p.launch_variants()["rows"] == rows


@pytest.mark.parametrize("conv", [0, 1, 2, 3])
@pytest.mark.parametrize("rv", [4])
@pytest.mark.parametrize("precision", ["fp64", "fp32_refine"])
@pytest.mark.parametrize("Nx,Ny,N", [(8, 4, 5), (16, 8, 9), (32, 16, 17), (64, 32, 33), (128, 64, 65),
                                     (32, 512, 9), (256, 16, 66), (16, 128, 40), (256, 8, 64)])
def test_eig_3d_vs_oracle(cuda, Nx, Ny, N, precision, rv, conv):
    rng = np.random.default_rng(Nx * 1000 + Ny + N)
    f = rng.standard_normal((Nx, Ny, N))
    gl, gr = rng.standard_normal((Nx, Ny)), rng.standard_normal((Nx, Ny))
    lam = 3.0
    ref = O.solve3d(f, gl, gr, Lx=1.3, Ly=0.7, Lz=0.9, lam=lam, bc=BC_DIR)
    p = NonPeriodic3D(Nx, Ny, N, N, 0.0, 1.3, 0.0, 0.7, 0.0, 0.9, Lambda=lam, bc=BC_DIR, precision=precision)
    _pin(p, rv, conv)
    assert p.kernels() == (KERNELS3_SPLIT if (conv & 2 and Nx >= 64) else KERNELS3[rv])
    fd, gld, grd = _dev(f), _dev(gl), _dev(gr)
    for _ in range(2):  # the spectrum scratch is reused: two solves in a row
        u = p.SolvePDE(fd, gld, grd).cpu().numpy()
        assert max_rel(u, ref) < 1e-12
    # without boundary data: homogeneous Dirichlet rows
    ref0 = O.solve3d(f, 0 * gl, 0 * gr, Lx=1.3, Ly=0.7, Lz=0.9, lam=lam, bc=BC_DIR)
    assert max_rel(p.SolvePDE(fd).cpu().numpy(), ref0) < 1e-12
    _status_ok(p)


@pytest.mark.parametrize("precision", ["fp64", "fp32_refine"])
@pytest.mark.parametrize("Nx,N", [(8, 4), (16, 9), (32, 17), (64, 33), (128, 65), (256, 66), (256, 33)])
def test_eig_2d_vs_oracle(cuda, Nx, N, precision):
    rng = np.random.default_rng(Nx + N)
    f = rng.standard_normal((Nx, N))
    gl, gr = rng.standard_normal(Nx), rng.standard_normal(Nx)
    ref = O.solve2d(f, gl, gr, Lx=2.0, Ly=1.5, lam=0.7, bc=BC_DIR)
    p = NonPeriodic2D(Nx, N, N, 0.0, 2.0, 0.0, 1.5, Lambda=0.7, bc=BC_DIR, precision=precision)
    _pin(p, 4)
    assert p.kernels() == "eig_solve2d_kernel"
    u = p.SolvePDE(_dev(f), _dev(gl), _dev(gr)).cpu().numpy()
    assert max_rel(u, ref) < 1e-12


def test_eig_config1_golden_and_exact(cuda):
    """The 2D problem of config 1 (64 x 33, lambda 1) through the fused kernel:
    the reference's own solution and the manufactured exact one."""
    g = golden("cfg1_2d")
    xl, xr, yl, yr = [float(v) for v in g["dom"]]
    p = NonPeriodic2D(64, 33, 33, xl, xr, yl, yr, Lambda=1.0, bc=tuple(g["bc"]))
    _pin(p, 4)
    u = p.SolvePDE(_dev(g["f"])).cpu().numpy()
    assert max_rel(u, g["u"]) < 1e-12
    assert np.abs(u - g["u_exact"]).max() < 1e-13


@pytest.mark.parametrize("rv", [4])
def test_eig_golden_3d(cuda, rv):
    g = golden("smooth_3d")
    xl, xr, yl, yr, zl, zr = [float(v) for v in g["dom"]]
    assert float(g["bc"][0]) == 0.0 and float(g["bc"][2]) == 0.0
    p = NonPeriodic3D(16, 16, 17, 17, xl, xr, yl, yr, zl, zr, Lambda=float(g["lam"]), bc=tuple(g["bc"]))
    _pin(p, rv)
    assert max_rel(p.SolvePDE(_dev(g["f"])).cpu().numpy(), g["u"]) < 1e-12


@pytest.mark.parametrize("conv", [0, 1, 2, 3])
@pytest.mark.parametrize("rv", [4])
@pytest.mark.parametrize("precision", ["fp64", "fp32_refine"])
def test_eig_full_size_vs_oracle(cuda, precision, rv, conv):
    """256 x 256 x 65, lambda 10 (the headline workload) with the pipeline pinned."""
    Nx, N = 256, 65
    f = W.smooth_field_3d(Nx, Nx, N, seed=1236)
    z = np.zeros((Nx, Nx))
    ref = O.solve3d(f, z, z, Lx=2 * math.pi, Ly=2 * math.pi, Lz=2.0, lam=10.0)
    p = NonPeriodic3D(Nx, Nx, N, N, 0.0, 2 * math.pi, 0.0, 2 * math.pi, 0.0, 2.0, Lambda=10.0, precision=precision)
    _pin(p, rv, conv)
    u = p.SolvePDE(_dev(f)).cpu().numpy()
    assert rel_l2(u, ref) < 1e-12
    _status_ok(p)


@pytest.mark.parametrize("Nx,split", [(32, 0), (64, 0), (64, 2)])
@pytest.mark.parametrize("rv", [4])
def test_eig_reference_layout(cuda, rv, Nx, split):
    """The reference's padded arrays rhsPDE[2Nx][2Ny][N], leftBC[2Nx][2Ny]:
    results in the [Nx][Ny] corner, padding untouched."""
    rng = np.random.default_rng(5)
    Ny, N = 16, 17
    f, gl, gr = rng.standard_normal((Nx, Ny, N)), rng.standard_normal((Nx, Ny)), rng.standard_normal((Nx, Ny))
    ref = O.solve3d(f, gl, gr, Lx=1.0, Ly=2.0, Lz=1.5, lam=2.0, bc=BC_DIR)
    F = np.zeros((2 * Nx, 2 * Ny, N)); F[:Nx, :Ny] = f
    GL = np.zeros((2 * Nx, 2 * Ny)); GL[:Nx, :Ny] = gl
    GR = np.zeros((2 * Nx, 2 * Ny)); GR[:Nx, :Ny] = gr
    p = NonPeriodic3D(Nx, Ny, N, N, 0.0, 1.0, 0.0, 2.0, 0.0, 1.5, Lambda=2.0, bc=BC_DIR)
    _pin(p, rv, split)
    p.set_layout(x_stride=2 * Ny * N, elem_stride=2 * Nx * 2 * Ny * N, bc_x_stride=2 * Ny)
    fd, gld, grd = _dev(F), _dev(GL), _dev(GR)
    ud = torch.full((2 * Nx, 2 * Ny, N), 7.0, dtype=torch.float64, device="cuda")
    st = p._lib.helm_solve(p._plan, fd.data_ptr(), gld.data_ptr(), grd.data_ptr(), ud.data_ptr(),
                           torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert st == 0
    U = ud.cpu().numpy()
    assert max_rel(U[:Nx, :Ny], ref) < 1e-12
    assert np.all(U[Nx:] == 7.0) and np.all(U[:, Ny:] == 7.0)


def test_eig_declines_other_plans(cuda):
    """Robin ends, several elements and periodic plans have no eigen-basis
    pipeline: pinning it is an error, and the autotuned plan runs another path."""
    p = NonPeriodic3D(32, 16, 17, 17, 0.0, 1.0, 0.0, 1.0, 0.0, 1.0, Lambda=1.0, bc=(0.4, 1.0, 0.3, 2.0))
    with pytest.raises(HelmError):
        _pin(p, 4)
    assert "eig" not in p.kernels()
    p = NonPeriodic3D(32, 16, 34, 17, 0.0, 1.0, 0.0, 1.0, 0.0, 1.0, Lambda=1.0)  # two elements
    with pytest.raises(HelmError):
        _pin(p, 4)
    p = Periodic3D(32, 16, 17, 17, 0.0, 1.0, 0.0, 1.0, 0.0, 1.0, Lambda=1.0)
    with pytest.raises(HelmError):
        _pin(p, 4)
    p = NonPeriodic3D(32, 16, 17, 17, 0.0, 1.0, 0.0, 1.0, 0.0, 1.0, Lambda=1.0, precision="fp32")
    with pytest.raises(HelmError):
        _pin(p, 4)


@pytest.mark.parametrize("dim,shape,rv,split", [(3, (8, 4, 5), 4, 0), (3, (32, 16, 17), 4, 0),
                                                (3, (128, 64, 65), 4, 0), (3, (128, 64, 65), 4, 2),
                                                (3, (256, 8, 66), 4, 0), (3, (256, 8, 66), 4, 2),
                                                (3, (64, 16, 33), 4, 2), (2, (64, 33), 4, 0), (2, (256, 66), 4, 0)])
@pytest.mark.parametrize("precision", ["fp64", "fp32_refine"])
def test_eig_adjoint_matches_row_kernel_adjoint(cuda, dim, shape, rv, split, precision):
    """The transposed pipeline (row variant 4) against the transposed row-kernel
    pipeline (variant 0; checked against dense adjoint maps in
    test_adjoint_gpu.py): fbar, the boundary cotangents (beta != 1) and
    lambda_bar, plain and in the misfit form."""
    rng = np.random.default_rng(sum(shape))
    if dim == 3:
        Nx, Ny, N = shape
        p = NonPeriodic3D(Nx, Ny, N, N, 0.0, 1.0, 0.0, 2.0, 0.0, 1.5, Lambda=1.3, bc=BC_DIR, precision=precision)
    else:
        Nx, N = shape
        p = NonPeriodic2D(Nx, N, N, 0.0, 1.0, 0.0, 1.5, Lambda=1.3, bc=BC_DIR, precision=precision)
    f = _dev(rng.standard_normal(shape))
    ubar = _dev(rng.standard_normal(shape))
    uobs = _dev(rng.standard_normal(shape))
    out = {}
    for v in (0, rv):
        _pin(p, v, split if v == rv and dim == 3 else None)
        u = p.SolvePDE(f)
        fb, lb, glb, grb = p.SolveAdjoint(ubar, u=u, want_bc=True)
        mfb, mlb, mglb, mgrb = p.SolveAdjointMisfit(u, uobs, want_bc=True)
        torch.cuda.synchronize()
        out[v] = [t.cpu().numpy() for t in (u, fb, lb, glb, grb, mfb, mlb, mglb, mgrb)]
    names = ("u", "fbar", "lambda_bar", "glbar", "grbar", "misfit fbar", "misfit lambda_bar", "misfit glbar",
             "misfit grbar")
    tol = 1e-12 if precision == "fp64" else 1e-10
    for nm, a, b in zip(names, out[rv], out[0]):
        assert max_rel(a, b) < tol, (nm, max_rel(a, b))
    _status_ok(p)
    # boundary slots of fbar are zero (f is read at interior nodes only)
    assert np.all(out[rv][1][..., 0] == 0.0) and np.all(out[rv][1][..., -1] == 0.0)


@pytest.mark.parametrize("N", [17, 65])
def test_refined_plan_fp64_rows(cuda, N):
    """Row variant 3: a refined plan solving its FP64 spectrum with the FP64
    tensor-core row kernel (Robin ends, so the boundary epilogue runs)."""
    rng = np.random.default_rng(N)
    Nx, Ny, bc = 16, 32, (0.4, 1.0, 0.3, 2.0)
    f = rng.standard_normal((Nx, Ny, N))
    gl, gr = rng.standard_normal((Nx, Ny)), rng.standard_normal((Nx, Ny))
    ref = O.solve3d(f, gl, gr, Lx=1.0, Ly=1.5, Lz=2.0, lam=3.0, bc=bc)
    p = NonPeriodic3D(Nx, Ny, N, N, 0.0, 1.0, 0.0, 1.5, 0.0, 2.0, Lambda=3.0, bc=bc, precision="fp32_refine")
    _pin(p, 3)
    assert "fdm_mma16_kernel" in p.kernels()
    u = p.SolvePDE(_dev(f), _dev(gl), _dev(gr)).cpu().numpy()
    assert max_rel(u, ref) < 1e-12


def test_autotuned_refined_plan_accuracy(cuda):
    """Whatever the autotuner picks for the refined plan at 128 x 128 x 65
    (lambda 5), the solve meets the refined target of 1e-10 against the oracle."""
    Nx, N = 128, 65
    f = W.smooth_field_3d(Nx, Nx, N, seed=1235)
    z = np.zeros((Nx, Nx))
    ref = O.solve3d(f, z, z, Lx=2 * math.pi, Ly=2 * math.pi, Lz=2.0, lam=5.0)
    p = NonPeriodic3D(Nx, Nx, N, N, 0.0, 2 * math.pi, 0.0, 2 * math.pi, 0.0, 2.0, Lambda=5.0,
                      precision="fp32_refine")
    assert p.kernels()
    assert rel_l2(p.SolvePDE(_dev(f)).cpu().numpy(), ref) < 1e-10


def test_eig_unaligned_input_takes_elementwise_loads(cuda):
    """f starting 8 bytes past a 16-byte boundary cannot be described to the TMA
    unit; the first pass then loads element-wise, with the same result."""
    rng = np.random.default_rng(21)
    Nx, Ny, N = 32, 16, 17
    f = rng.standard_normal((Nx, Ny, N))
    gl, gr = rng.standard_normal((Nx, Ny)), rng.standard_normal((Nx, Ny))
    ref = O.solve3d(f, gl, gr, Lx=1.0, Ly=2.0, Lz=1.5, lam=2.0, bc=BC_DIR)
    p = NonPeriodic3D(Nx, Ny, N, N, 0.0, 1.0, 0.0, 2.0, 0.0, 1.5, Lambda=2.0, bc=BC_DIR)
    _pin(p, 4)
    buf = torch.zeros(f.size + 1, dtype=torch.float64, device="cuda")
    buf[1:] = _dev(f).reshape(-1)
    u = torch.empty(f.shape, dtype=torch.float64, device="cuda")
    gld, grd = _dev(gl), _dev(gr)  # held until the asynchronous solve has run
    st = p._lib.helm_solve(p._plan, buf[1:].data_ptr(), gld.data_ptr(), grd.data_ptr(), u.data_ptr(),
                           torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert st == 0 and buf[1:].data_ptr() % 16 == 8
    assert max_rel(u.cpu().numpy(), ref) < 1e-12
    aligned = p.SolvePDE(_dev(f), _dev(gl), _dev(gr)).cpu().numpy()
    assert max_rel(aligned, ref) < 1e-12
    _status_ok(p)
