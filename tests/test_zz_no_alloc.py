"""helm_solve_static_scratch: the solve for callers that cannot allocate
device memory at call time (their own memory manager owns the device, or their
device footprint must stay fixed after start-up).  Checked through the C ABI
against helm_solve on two calls in a row -- non-periodic 2D and 3D plans, a
plan periodic in the GLL direction, finite-difference plans (one of them long
enough in z to need the elimination scratch) and the fused slab row variant --
plus the size limit (16 MiB) rejected with HELM_ERR_UNSUPPORTED, boundary data
on a periodic plan rejected with HELM_ERR_INVALID, and helm_solve running on
the same plan from another host thread at the same time.  Collected last so
that a run stopping at its first failure has already run every other test."""
import ctypes
import math
import threading

import numpy as np
import pytest
import torch

from mpi_b200 import Helmholtz3DFD, NonPeriodic2D, NonPeriodic3D, Periodic3D
from mpi_b200 import _lib as L
from mpi_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _entry():
    lib = L.lib()
    fn = lib.helm_solve_static_scratch
    fn.argtypes = [ctypes.c_void_p] * 6
    fn.restype = ctypes.c_int
    return fn


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()


def _call(fn, plan, f, gl, gr, u):
    stream = torch.cuda.current_stream().cuda_stream
    return fn(plan.handle, f.data_ptr(), gl.data_ptr() if gl is not None else None,
              gr.data_ptr() if gr is not None else None, u.data_ptr(), stream)


@pytest.mark.parametrize("precision", ["fp64", "fp32", "fp32_refine"])
def test_static_scratch_matches_solve_3d(cuda, precision):
    fn = _entry()
    rng = np.random.default_rng(8)
    Nx, Ny, N = 64, 32, 33
    bc = (1.0, 0.5, 0.7, 2.0)
    p = NonPeriodic3D(Nx, Ny, N, N, 0.0, 1.3, 0.0, 0.7, 0.0, 0.9, Lambda=2.0, bc=bc, precision=precision)
    gl, gr = _dev(rng.standard_normal((Nx, Ny))), _dev(rng.standard_normal((Nx, Ny)))
    tol = 1e-5 if precision == "fp32" else 1e-12
    for seed in (1, 2):  # two calls in a row, different inputs
        f = _dev(W.smooth_field_3d(Nx, Ny, N, seed=seed))
        ref = p.SolvePDE(f, gl, gr)
        u = torch.full_like(f, np.nan)
        assert _call(fn, p, f, gl, gr, u) == L.HELM_OK
        torch.cuda.synchronize()
        err = ((u - ref).norm() / ref.norm()).item()
        assert err < tol, f"call with seed {seed}: relative difference {err:.3e}"


def test_static_scratch_matches_solve_2d(cuda):
    fn = _entry()
    f0, _ = W.manufactured_2d(64, 33, 1.0)
    p = NonPeriodic2D(64, 33, 33, 0.0, 2 * math.pi, -1.0, 1.0, Lambda=1.0)
    for scale in (1.0, -2.5):
        f = _dev(scale * f0)
        ref = p.SolvePDE(f)
        u = torch.empty_like(f)
        assert _call(fn, p, f, None, None, u) == L.HELM_OK
        torch.cuda.synchronize()
        assert ((u - ref).norm() / ref.norm()).item() < 1e-12


def test_static_scratch_rejects_large_plan(cuda):
    fn = _entry()
    p = NonPeriodic3D(256, 256, 65, 65, 0.0, 2 * math.pi, 0.0, 2 * math.pi, 0.0, 2.0, Lambda=10.0)  # 34 MB spectrum
    f = torch.zeros((256, 256, 65), dtype=torch.float64, device="cuda")
    u = torch.zeros_like(f)
    assert _call(fn, p, f, None, None, u) == L.HELM_ERR_UNSUPPORTED


def _twice(fn, plan, make_f, gl=None, gr=None, tol=1e-12):
    """Two calls in a row with different inputs, each against helm_solve."""
    for seed in (1, 2):
        f = make_f(seed)
        ref = plan.SolvePDE(f, gl, gr)
        u = torch.full_like(f, np.nan)
        assert _call(fn, plan, f, gl, gr, u) == L.HELM_OK
        torch.cuda.synchronize()
        err = ((u - ref).norm() / ref.norm()).item()
        assert err < tol, f"call with seed {seed}: relative difference {err:.3e}"


@pytest.mark.parametrize("precision", ["fp64", "fp32_refine"])
def test_static_scratch_periodic_3d(cuda, precision):
    fn = _entry()
    p = Periodic3D(16, 8, 9, 9, 0.0, 1.0, 0.0, 2.0, 0.0, 1.5, Lambda=0.5, precision=precision)
    rng = np.random.default_rng(3)
    _twice(fn, p, lambda s: _dev(rng.standard_normal((16, 8, 9)) * s))
    # boundary data on a plan periodic in the GLL direction is an argument error,
    # as in helm_solve
    f = _dev(rng.standard_normal((16, 8, 9)))
    g = _dev(rng.standard_normal((16, 8)))
    u = torch.zeros_like(f)
    assert _call(fn, p, f, g, None, u) == L.HELM_ERR_INVALID
    assert "periodic" in L.lib().helm_last_error().decode()


@pytest.mark.parametrize("shape", [(16, 8, 12), (4, 4, 600)])
def test_static_scratch_fd(cuda, shape):
    fn = _entry()
    Nx, Ny, Nz = shape
    bc = (1.0, 0.5, 0.7, 2.0)
    p = Helmholtz3DFD(Nx, Ny, Nz, 0.0, 1.0, 0.0, 2.0, 0.0, 1.5, Lambda=1.0, bc=bc)
    rng = np.random.default_rng(4)
    gl, gr = _dev(rng.standard_normal((Nx, Ny))), _dev(rng.standard_normal((Nx, Ny)))
    _twice(fn, p, lambda s: _dev(rng.standard_normal(shape)), gl, gr)


def test_static_scratch_slab_variant(cuda):
    fn = _entry()
    Nx, Ny, N = 32, 64, 33
    p = NonPeriodic3D(Nx, Ny, N, N, 0.0, 1.0, 0.0, 2.0, 0.0, 1.5, Lambda=3.0)
    p.set_launch_variants(p.launch_variants()["fft"], 2)  # the fused y-FFT / rows / inverse-y slab kernel
    assert p.launch_variants()["rows"] == 2
    _twice(fn, p, lambda s: _dev(W.smooth_field_3d(Nx, Ny, N, seed=s)))


def test_static_scratch_beside_helm_solve_on_another_thread(cuda):
    """The entry point only reads the plan: helm_solve on the same plan from a
    second host thread, on its own stream, keeps using the plan's workspace."""
    fn = _entry()
    Nx, Ny, N = 32, 16, 17
    p = NonPeriodic3D(Nx, Ny, N, N, 0.0, 1.0, 0.0, 2.0, 0.0, 1.5, Lambda=2.0)
    fa = _dev(W.smooth_field_3d(Nx, Ny, N, seed=5))
    fb = _dev(W.smooth_field_3d(Nx, Ny, N, seed=6))
    ref_a, ref_b = p.SolvePDE(fa), p.SolvePDE(fb)
    torch.cuda.synchronize()
    errs = []

    def other():
        s = torch.cuda.Stream()
        with torch.cuda.stream(s):
            for _ in range(50):
                u = p.SolvePDE(fb)
                s.synchronize()
                errs.append(((u - ref_b).norm() / ref_b.norm()).item())

    t = threading.Thread(target=other)
    t.start()
    for _ in range(50):
        u = torch.empty_like(fa)
        assert _call(fn, p, fa, None, None, u) == L.HELM_OK
        torch.cuda.current_stream().synchronize()
        errs.append(((u - ref_a).norm() / ref_a.norm()).item())
    t.join()
    assert len(errs) == 100 and max(errs) < 1e-12
