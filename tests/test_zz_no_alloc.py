"""helm_solve_static_scratch: the solve for callers that cannot allocate
device memory at call time (their own memory manager owns the device, or their
device footprint must stay fixed after start-up).  Checked through the C ABI
against helm_solve on two calls in a row, and the size limit (16 MiB of
spectrum) rejected with HELM_ERR_UNSUPPORTED.  Collected last so that a run
stopping at its first failure has already run every other test."""
import ctypes
import math

import numpy as np
import pytest
import torch

from mpi_b200 import NonPeriodic2D, NonPeriodic3D
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
