"""Host-side mirror of the reference's solver interface over the C ABI.

The reference (HelmholtzSolvers/DirectPseudoSpectral) exposes, per solver
family, ``CreatePDEPlan(...)`` / ``SolvePDE(U, ConstructOperator)`` /
``DestroyPDEPlan()`` over global arrays (NonPeriodic2D_MPI.h:33-37,
NonPeriodic3D_MPI.h:33-37).  Here each family is a class whose constructor is
CreatePDEPlan (plus the Lambda / alpha / beta globals and the shifted-Laplacian
ConstructOperator of the reference's tests), whose ``SolvePDE`` runs the solve on
the GPU, and whose ``DestroyPDEPlan`` frees it.  Arrays are torch CUDA tensors
in the reference's index order (GLL index fastest):

* ``NonPeriodic2D``: f, u ``[Ns, Nx, N]`` (or ``[Nx, N]`` when Ns == 1), gl/gr ``[Nx]``
* ``NonPeriodic3D``: f, u ``[Ns, Nx, Ny, N]`` (or ``[Nx, Ny, N]``), gl/gr ``[Nx, Ny]``
* ``Periodic2D`` / ``Periodic3D`` (periodic in the GLL direction too,
  Periodic2D_MPI.h / Periodic3D_MPI.h): the same f, u shapes and no boundary data

Errors raise :class:`mpi_b200._lib.HelmError` with the C status code (the
reference prints a message and exits).
"""
from __future__ import annotations

import ctypes
import math
from typing import Optional, Sequence

import torch

from . import _lib as L

_PREC = {"fp64": L.HELM_FP64, "fp32": L.HELM_FP32, "fp32_refine": L.HELM_FP32_REFINE}
_METHOD = {"auto": L.HELM_METHOD_AUTO, "lu": L.HELM_METHOD_LU, "fdm": L.HELM_METHOD_FDM}
_METHOD_NAME = {v: k for k, v in _METHOD.items()}


def _stream_ptr(stream) -> int:
    if stream is None:
        stream = torch.cuda.current_stream()
    return int(stream.cuda_stream) if hasattr(stream, "cuda_stream") else int(stream)


class _PlanBase:
    dim = 0

    def __init__(self):
        self._plan = ctypes.c_void_p()
        self._lib = L.lib()

    # -------------------------------------------------------------- info --
    @property
    def handle(self) -> int:
        return self._plan.value or 0

    def info(self) -> dict:
        ns, nop, meth = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        nb = ctypes.c_longlong()
        L.check(self._lib.helm_plan_info(self._plan, ctypes.byref(ns), ctypes.byref(nop), ctypes.byref(meth),
                                         ctypes.byref(nb)), "helm_plan_info")
        return {"Ns": ns.value, "n_operators": nop.value, "method": _METHOD_NAME[meth.value],
                "device_bytes": nb.value}

    @property
    def Ns(self) -> int:
        return self.info()["Ns"]

    def grid(self):
        """(nodes, D, D2) of the GLL direction as float64 CPU tensors (the
        reference's y/z, Dy/Dz and Dyy/Dzz globals)."""
        ns = self.Ns
        N = self.N
        nodes = torch.zeros(ns * (N - 1) + 1, dtype=torch.float64)
        D = torch.zeros(N, N, dtype=torch.float64)
        D2 = torch.zeros(N, N, dtype=torch.float64)
        L.check(self._lib.helm_plan_get_grid(self._plan, nodes.data_ptr(), D.data_ptr(), D2.data_ptr()),
                "helm_plan_get_grid")
        return nodes, D, D2

    def set_layout(self, x_stride: int = 0, elem_stride: int = 0, bc_x_stride: int = 0) -> None:
        L.check(self._lib.helm_plan_set_layout(self._plan, x_stride, elem_stride, bc_x_stride), "helm_plan_set_layout")

    def set_refine_sweeps(self, sweeps: int) -> None:
        L.check(self._lib.helm_plan_set_refine_sweeps(self._plan, sweeps), "helm_plan_set_refine_sweeps")

    def SetOperator(self, construct_operator) -> None:
        """The reference's ConstructOperator callback (SolvePDE(U,
        ConstructOperator), NonPeriodic2D_MPI.h:37 / NonPeriodic3D_MPI.h:37):
        ``construct_operator(iw, jw)`` returns the (N-2) x (N-2) interior
        operator of the wavenumber pair (|iw|, |jw|) (2D: jw = 0) as an array.
        It is called once per pair now; later solves use those operators."""
        import numpy as np

        err = []

        def cb(iw, jw, op, ld, user):
            try:
                a = np.asarray(construct_operator(iw, jw), dtype=np.float64)
                n = a.shape[0]
                dst = np.ctypeslib.as_array(op, shape=(n * ld,)).reshape(n, ld)
                dst[:, :n] = a
            except Exception as e:  # an exception cannot cross the C callback
                err.append(e)

        fn = L.OPERATOR_FN(cb)
        st = self._lib.helm_plan_set_operator_callback(self._plan, fn, None)
        if err:
            raise err[0]
        L.check(st, "helm_plan_set_operator_callback")

    def set_io_bytes(self, nbytes: int) -> None:
        L.check(self._lib.helm_plan_set_io_bytes(self._plan, nbytes), "helm_plan_set_io_bytes")
        self.io_dtype = torch.float32 if nbytes == 4 else torch.float64

    # ------------------------------------------------------------- solve --
    def _shape(self, Ns: int):
        raise NotImplementedError

    def _bc_shape(self):
        raise NotImplementedError

    def SolvePDE(self, f: torch.Tensor, gl: Optional[torch.Tensor] = None, gr: Optional[torch.Tensor] = None,
                 out: Optional[torch.Tensor] = None, stream=None) -> torch.Tensor:
        """u = solution of (lap - lambda) u = f with the plan's Robin data gl/gr
        (None: zero).  f, gl, gr, out: contiguous CUDA tensors."""
        ns = self.Ns
        full = self._shape(ns)
        if f.dim() == len(full) - 1 and ns == 1:
            fv = f.unsqueeze(0)
        else:
            fv = f
        if tuple(fv.shape) != full:
            raise ValueError(f"f has shape {tuple(f.shape)}, expected {full}")
        if not fv.is_cuda or fv.dtype != self.io_dtype or not fv.is_contiguous():
            raise ValueError(f"f must be a contiguous CUDA {self.io_dtype} tensor")
        bshape = self._bc_shape()
        for g, nm in ((gl, "gl"), (gr, "gr")):
            if g is not None and (tuple(g.shape) != bshape or g.dtype != torch.float64 or not g.is_cuda
                                  or not g.is_contiguous()):
                raise ValueError(f"{nm} must be a contiguous CUDA float64 tensor of shape {bshape}")
        if out is None:
            out = torch.empty(f.shape, dtype=self.io_dtype, device=f.device)
        elif tuple(out.shape) != tuple(f.shape) or out.dtype != self.io_dtype or not out.is_contiguous():
            raise ValueError("out does not match f")
        st = self._lib.helm_solve(self._plan, fv.data_ptr(), gl.data_ptr() if gl is not None else None,
                                  gr.data_ptr() if gr is not None else None, out.data_ptr(), _stream_ptr(stream))
        L.check(st, "helm_solve")
        return out

    solve = SolvePDE

    def SolveAdjoint(self, ubar: torch.Tensor, u: Optional[torch.Tensor] = None, want_bc: bool = False,
                     stream=None):
        """(fbar, lambda_bar, glbar, grbar) of the linear map (f, gl, gr) -> u
        for the cotangent ubar; lambda_bar needs the forward solution u."""
        fbar = torch.empty_like(ubar, dtype=torch.float64)
        lam = torch.zeros(1, dtype=torch.float64, device=ubar.device) if u is not None else None
        glb = torch.empty(self._bc_shape(), dtype=torch.float64, device=ubar.device) if want_bc else None
        grb = torch.empty(self._bc_shape(), dtype=torch.float64, device=ubar.device) if want_bc else None
        st = self._lib.helm_solve_adjoint(self._plan, ubar.data_ptr(), fbar.data_ptr(),
                                          glb.data_ptr() if glb is not None else None,
                                          grb.data_ptr() if grb is not None else None,
                                          u.data_ptr() if u is not None else None,
                                          lam.data_ptr() if lam is not None else None, _stream_ptr(stream))
        L.check(st, "helm_solve_adjoint")
        return fbar, lam, glb, grb

    # ------------------------------------------------------- derivatives --
    def _derivative(self, axis: int, order: int, u: torch.Tensor, out: Optional[torch.Tensor], stream) -> torch.Tensor:
        """axis: Fourier axes first (x; y in 3D), then the GLL axis."""
        ns = self.Ns
        full = self._shape(ns)
        uv = u.unsqueeze(0) if (u.dim() == len(full) - 1 and ns == 1) else u
        if tuple(uv.shape) != full or not u.is_cuda or u.dtype != self.io_dtype or not u.is_contiguous():
            raise ValueError(f"u must be a contiguous CUDA {self.io_dtype} tensor of shape {full}")
        if out is None:
            out = torch.empty_like(u)
        elif tuple(out.shape) != tuple(u.shape) or out.dtype != u.dtype or not out.is_contiguous():
            raise ValueError("out does not match u")
        if axis == self.dim - 1:
            st = self._lib.helm_gll_derivative(self._plan, order, u.data_ptr(), out.data_ptr(), _stream_ptr(stream))
            L.check(st, "helm_gll_derivative")
        else:
            if out.data_ptr() == u.data_ptr():
                raise ValueError("a Fourier derivative cannot run in place")
            st = self._lib.helm_fourier_derivative(self._plan, axis, order, u.data_ptr(), out.data_ptr(),
                                                   _stream_ptr(stream))
            L.check(st, "helm_fourier_derivative")
        return out

    def FirstDerivativeX(self, u, out=None, stream=None):
        """Spectral d/dx (Fourier_Quadrature.cpp FirstDerivativeFourierX)."""
        return self._derivative(0, 1, u, out, stream)

    def SecondDerivativeX(self, u, out=None, stream=None):
        return self._derivative(0, 2, u, out, stream)

    def FirstDerivativeY(self, u, out=None, stream=None):
        """2D: GLL d/dy per element (NonPeriodic2D_MPI.cpp:497-519); 3D: spectral d/dy."""
        return self._derivative(1, 1, u, out, stream)

    def SecondDerivativeY(self, u, out=None, stream=None):
        return self._derivative(1, 2, u, out, stream)

    def FirstDerivativeZ(self, u, out=None, stream=None):
        """3D: GLL d/dz per element (NonPeriodic3D_MPI.cpp:632-656)."""
        if self.dim != 3:
            raise ValueError("a 2D plan has no z direction")
        return self._derivative(2, 1, u, out, stream)

    def SecondDerivativeZ(self, u, out=None, stream=None):
        if self.dim != 3:
            raise ValueError("a 2D plan has no z direction")
        return self._derivative(2, 2, u, out, stream)

    # ------------------------------------------------------------ output --
    def WriteFile(self, u, path: str, exact=None, fmt: str = "tecplot") -> None:
        """The reference's WriteFile: u (any device, the plan's shape) written to
        `path` as a Tecplot point file (fmt "tecplot", with exact(x, y, z) beside
        it; 2D plans get z = 0) or a legacy-VTK structured grid (fmt "vtk")."""
        full = self._shape(self.Ns)
        uh = u.detach().to("cpu", torch.float64).contiguous().reshape(full)
        if fmt == "tecplot":
            cb = L.EXACT_FN(exact) if exact is not None else L.EXACT_FN()
            st = self._lib.helm_write_tecplot(self._plan, uh.data_ptr(), cb, path.encode())
        elif fmt == "vtk":
            st = self._lib.helm_write_vtk(self._plan, uh.data_ptr(), path.encode())
        else:
            raise ValueError("fmt must be 'tecplot' or 'vtk'")
        L.check(st, "helm_write_" + fmt)

    def SolveAdjointMisfit(self, u: torch.Tensor, u_obs: torch.Tensor, want_bc: bool = False, stream=None):
        """(fbar, lambda_bar, glbar, grbar) of L = 1/2 ||u - u_obs||^2, u the forward
        solution: SolveAdjoint with ubar = u - u_obs formed inside the adjoint's
        first pass (no ubar tensor)."""
        if u.shape != u_obs.shape or u.dtype != torch.float64 or u_obs.dtype != torch.float64:
            raise ValueError("u and u_obs must be float64 tensors of one shape")
        fbar = torch.empty_like(u)
        lam = torch.zeros(1, dtype=torch.float64, device=u.device)
        glb = torch.empty(self._bc_shape(), dtype=torch.float64, device=u.device) if want_bc else None
        grb = torch.empty(self._bc_shape(), dtype=torch.float64, device=u.device) if want_bc else None
        st = self._lib.helm_solve_adjoint_misfit(self._plan, u.data_ptr(), u_obs.data_ptr(), fbar.data_ptr(),
                                                 glb.data_ptr() if glb is not None else None,
                                                 grb.data_ptr() if grb is not None else None, lam.data_ptr(),
                                                 _stream_ptr(stream))
        L.check(st, "helm_solve_adjoint_misfit")
        return fbar, lam, glb, grb

    def enable_stage_timing(self, enable: bool = True) -> None:
        L.check(self._lib.helm_plan_set_stage_timing(self._plan, int(enable)), "helm_plan_set_stage_timing")

    STAGES = ("fft_x", "fft_y", "rows", "ifft_y", "ifft_x")

    def stage_times(self) -> dict:
        """Durations (ms) of the last solve's kernels, from CUDA events on its stream."""
        buf = (ctypes.c_float * 5)()
        L.check(self._lib.helm_plan_stage_times(self._plan, buf), "helm_plan_stage_times")
        return dict(zip(self.STAGES, [float(v) for v in buf]))

    def launch_variants(self) -> dict:
        """The autotuned (or pinned) kernel variants: FFT passes (x, y,
        inverse y, inverse x) and the row solve."""
        f4 = (ctypes.c_int * 4)()
        rv = ctypes.c_int()
        L.check(self._lib.helm_plan_get_launch_variants(self._plan, f4, ctypes.byref(rv)),
                "helm_plan_get_launch_variants")
        return {"fft": list(f4), "rows": rv.value}

    def set_launch_variants(self, fft: Sequence[int], rows: int) -> None:
        f4 = (ctypes.c_int * 4)(*fft)
        L.check(self._lib.helm_plan_set_launch_variants(self._plan, f4, int(rows)), "helm_plan_set_launch_variants")

    def derivative_variant(self) -> int:
        """Launch variant of the spectral derivatives (-1: chosen by length)."""
        v = ctypes.c_int()
        L.check(self._lib.helm_plan_get_derivative_variant(self._plan, ctypes.byref(v)),
                "helm_plan_get_derivative_variant")
        return v.value

    def set_derivative_variant(self, variant: int) -> None:
        L.check(self._lib.helm_plan_set_derivative_variant(self._plan, int(variant)),
                "helm_plan_set_derivative_variant")

    def device_status(self, reset: bool = True) -> int:
        """0, or the code of a tile-copy wait of the TMA-pipelined kernels that ran
        out of its iteration limit (waits for the device)."""
        code = ctypes.c_int()
        L.check(self._lib.helm_plan_device_status(self._plan, ctypes.byref(code), int(reset)),
                "helm_plan_device_status")
        return code.value

    def kernels(self) -> str:
        """Names of the kernels a forward solve launches, in launch order."""
        return self._lib.helm_plan_kernels(self._plan).decode()

    def DestroyPDEPlan(self) -> None:
        if self._plan.value:
            self._lib.helm_plan_destroy(self._plan)
            self._plan = ctypes.c_void_p()

    close = DestroyPDEPlan

    def __del__(self):
        try:
            self.DestroyPDEPlan()
        except Exception:
            pass


class NonPeriodic2D(_PlanBase):
    """2D Fourier (x) x GLL (y) solver: CreatePDEPlan(Nx, Ny, N, xl, xr, yl, yr)
    of NonPeriodic2D_MPI.cpp:40-126 with Lambda and the Robin coefficients
    (alphal, betal, alphar, betar) of NonPeriodic2D_MPI.h:27."""

    dim = 2

    def __init__(self, Nx: int, Ny: int, N: int, xl: float, xr: float, yl: float, yr: float, *,
                 Lambda: float, bc: Sequence[float] = (0.0, 1.0, 0.0, 1.0), precision: str = "fp64",
                 method: str = "auto"):
        super().__init__()
        self.Nx, self.N = Nx, N
        self.xl, self.xr, self.yl, self.yr = xl, xr, yl, yr
        self.Lambda = Lambda
        self.bc = tuple(float(b) for b in bc)
        self.precision = precision
        self.io_dtype = torch.float64
        r = L.robin_t(*self.bc)
        L.check(self._lib.helm2d_plan_create(Nx, Ny, N, xl, xr, yl, yr, ctypes.byref(r), Lambda, _PREC[precision],
                                             _METHOD[method], ctypes.byref(self._plan)), "helm2d_plan_create")

    def _shape(self, Ns):
        return (Ns, self.Nx, self.N)

    def _bc_shape(self):
        return (self.Nx,)


class NonPeriodic3D(_PlanBase):
    """3D Fourier (x, y) x GLL (z) solver: CreatePDEPlan(Nx, Ny, Nz, N, xl, xr,
    yl, yr, zl, zr) of NonPeriodic3D_MPI.cpp:40-134."""

    dim = 3

    def __init__(self, Nx: int, Ny: int, Nz: int, N: int, xl: float, xr: float, yl: float, yr: float, zl: float,
                 zr: float, *, Lambda: float, bc: Sequence[float] = (0.0, 1.0, 0.0, 1.0), precision: str = "fp64",
                 method: str = "auto"):
        super().__init__()
        self.Nx, self.Ny, self.N = Nx, Ny, N
        self.Lambda = Lambda
        self.bc = tuple(float(b) for b in bc)
        self.precision = precision
        self.io_dtype = torch.float64
        r = L.robin_t(*self.bc)
        L.check(self._lib.helm3d_plan_create(Nx, Ny, Nz, N, xl, xr, yl, yr, zl, zr, ctypes.byref(r), Lambda,
                                             _PREC[precision], _METHOD[method], ctypes.byref(self._plan)),
                "helm3d_plan_create")

    def _shape(self, Ns):
        return (Ns, self.Nx, self.Ny, self.N)

    def _bc_shape(self):
        return (self.Nx, self.Ny)


class _PeriodicMixin:
    """The GLL direction is periodic: no boundary data in or out."""

    def SolvePDE(self, f, gl=None, gr=None, out=None, stream=None):
        if gl is not None or gr is not None:
            raise ValueError("a solver periodic in the GLL direction takes no boundary data")
        return _PlanBase.SolvePDE(self, f, None, None, out=out, stream=stream)

    solve = SolvePDE

    def SolveAdjoint(self, ubar, u=None, want_bc: bool = False, stream=None):
        if want_bc:
            raise ValueError("a solver periodic in the GLL direction has no boundary data")
        return _PlanBase.SolveAdjoint(self, ubar, u=u, want_bc=False, stream=stream)


class Periodic2D(_PeriodicMixin, NonPeriodic2D):
    """2D Fourier (x) x GLL (y) solver periodic in y as well: CreatePDEPlan(Nx,
    Ny, N, xl, xr, yl, yr) of Periodic2D_MPI.cpp:36-125 with Lambda, solved by
    the cyclic interface sweep of Periodic2D_MPI.cpp:257-565."""

    def __init__(self, Nx: int, Ny: int, N: int, xl: float, xr: float, yl: float, yr: float, *, Lambda: float,
                 precision: str = "fp64", method: str = "auto"):
        _PlanBase.__init__(self)
        self.Nx, self.N = Nx, N
        self.xl, self.xr, self.yl, self.yr = xl, xr, yl, yr
        self.Lambda = Lambda
        self.bc = None
        self.precision = precision
        self.io_dtype = torch.float64
        L.check(self._lib.helm2d_periodic_plan_create(Nx, Ny, N, xl, xr, yl, yr, Lambda, _PREC[precision],
                                                      _METHOD[method], ctypes.byref(self._plan)),
                "helm2d_periodic_plan_create")


class Periodic3D(_PeriodicMixin, NonPeriodic3D):
    """3D Fourier (x, y) x GLL (z) solver periodic in z as well: CreatePDEPlan(Nx,
    Ny, Nz, N, xl, xr, yl, yr, zl, zr) of Periodic3D_MPI.cpp:36-133."""

    def __init__(self, Nx: int, Ny: int, Nz: int, N: int, xl: float, xr: float, yl: float, yr: float, zl: float,
                 zr: float, *, Lambda: float, precision: str = "fp64", method: str = "auto"):
        _PlanBase.__init__(self)
        self.Nx, self.Ny, self.N = Nx, Ny, N
        self.Lambda = Lambda
        self.bc = None
        self.precision = precision
        self.io_dtype = torch.float64
        L.check(self._lib.helm3d_periodic_plan_create(Nx, Ny, Nz, N, xl, xr, yl, yr, zl, zr, Lambda,
                                                      _PREC[precision], _METHOD[method], ctypes.byref(self._plan)),
                "helm3d_periodic_plan_create")


class Helmholtz3DFD(_PlanBase):
    """Second-order finite-difference solver on the HypreFDM stencil
    (HelmholtzSolvers/HypreFDM/src/Helmholtz3D_MPI.cpp, CreatePDEPlan 117-269,
    SetA 297-410) with x and y periodic and Nz interior points in z, solved
    directly by FFT + Thomas.  ``bc`` = (alpha_back, beta_back, alpha_front,
    beta_front) of the one-sided Robin rows at z = zl and z = zr.  Arrays:
    f, u ``[Nx, Ny, Nz]``; gl (back) and gr (front) ``[Nx, Ny]``."""

    dim = 3

    def __init__(self, Nx: int, Ny: int, Nz: int, xl: float, xr: float, yl: float, yr: float, zl: float, zr: float,
                 *, Lambda: float, bc: Sequence[float] = (0.0, 1.0, 0.0, 1.0), precision: str = "fp64"):
        super().__init__()
        self.Nx, self.Ny, self.N = Nx, Ny, Nz
        self.Lambda = Lambda
        self.bc = tuple(float(b) for b in bc)
        self.precision = precision
        self.io_dtype = torch.float64
        r = L.robin_t(*self.bc)
        L.check(self._lib.helm_fd3d_plan_create(Nx, Ny, Nz, xl, xr, yl, yr, zl, zr, ctypes.byref(r), Lambda,
                                                _PREC[precision], ctypes.byref(self._plan)), "helm_fd3d_plan_create")

    def _shape(self, Ns):
        return (Ns, self.Nx, self.Ny, self.N)

    def _bc_shape(self):
        return (self.Nx, self.Ny)


class BatchNonPeriodic2D:
    """Many independent 2D problems of uneven sizes solved together
    (helm2d_batch_*).  Problem p has ``Nx[p]`` Fourier modes, one GLL element of
    ``N[p]`` points, ``lambdas[p]`` and homogeneous Dirichlet rows in y, on the
    common domain.  ``f`` and ``u`` are packed 1-D float64 tensors: problem p is
    the ``[Nx[p], N[p]]`` block at ``offsets[p]``; :meth:`pack` / :meth:`unpack`
    convert from / to per-problem tensors.  One solve is one CUDA graph launch
    holding one persistent kernel (FP64 and refined batches of Nx 8..512 and
    4..129 GLL points) or the size classes' kernels (``graph=False``: launched
    directly)."""

    def __init__(self, Nx: Sequence[int], N: Sequence[int], lambdas: Sequence[float], xl: float, xr: float,
                 yl: float, yr: float, *, precision: str = "fp64"):
        self._lib = L.lib()
        self._batch = ctypes.c_void_p()
        n = len(Nx)
        if len(N) != n or len(lambdas) != n:
            raise ValueError("Nx, N and lambdas need one entry per problem")
        self.Nx, self.N, self.lambdas = list(Nx), list(N), [float(v) for v in lambdas]
        self.precision = precision
        ia = (ctypes.c_int * n)(*self.Nx)
        na = (ctypes.c_int * n)(*self.N)
        la = (ctypes.c_double * n)(*self.lambdas)
        L.check(self._lib.helm2d_batch_create(n, ia, na, la, xl, xr, yl, yr, _PREC[precision],
                                              ctypes.byref(self._batch)), "helm2d_batch_create")
        offs = (ctypes.c_longlong * n)()
        tot = ctypes.c_longlong()
        L.check(self._lib.helm_batch_offsets(self._batch, offs, ctypes.byref(tot)), "helm_batch_offsets")
        self.offsets = list(offs)
        self.total = tot.value

    def info(self) -> dict:
        nc, nk = ctypes.c_int(), ctypes.c_int()
        nb = ctypes.c_longlong()
        L.check(self._lib.helm_batch_info(self._batch, ctypes.byref(nc), ctypes.byref(nk), ctypes.byref(nb)),
                "helm_batch_info")
        return {"classes": nc.value, "kernels_per_solve": nk.value, "device_bytes": nb.value}

    def set_graph(self, enable: bool) -> None:
        L.check(self._lib.helm_batch_set_graph(self._batch, int(bool(enable))), "helm_batch_set_graph")

    def device_status(self, reset: bool = True) -> int:
        """0, or 7 when a dependency wait of the persistent kernel ran out."""
        code = ctypes.c_int()
        L.check(self._lib.helm_batch_device_status(self._batch, ctypes.byref(code), int(reset)),
                "helm_batch_device_status")
        return code.value

    def pack(self, fs: Sequence[torch.Tensor]) -> torch.Tensor:
        return torch.cat([f.reshape(-1).to(torch.float64) for f in fs]).contiguous()

    def unpack(self, u: torch.Tensor):
        return [u[o:o + a * b].view(a, b) for o, a, b in zip(self.offsets, self.Nx, self.N)]

    def solve(self, f: torch.Tensor, out: Optional[torch.Tensor] = None, stream=None) -> torch.Tensor:
        if f.dtype != torch.float64 or not f.is_cuda or not f.is_contiguous() or f.numel() != self.total:
            raise ValueError(f"f must be a contiguous CUDA float64 tensor of {self.total} elements")
        u = torch.empty_like(f) if out is None else out
        L.check(self._lib.helm_batch_solve(self._batch, ctypes.c_void_p(f.data_ptr()), ctypes.c_void_p(u.data_ptr()),
                                           ctypes.c_void_p(_stream_ptr(stream))), "helm_batch_solve")
        return u

    def destroy(self) -> None:
        if self._batch:
            self._lib.helm_batch_destroy(self._batch)
            self._batch = ctypes.c_void_p()

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


def gdof(Nx: int, Ny: int, N: int, Ns: int = 1) -> int:
    """Degrees of freedom of one solve: grid values of u (Ns elements of N GLL points)."""
    return Nx * Ny * N * Ns


__all__ = ["BatchNonPeriodic2D", "Helmholtz3DFD", "NonPeriodic2D", "NonPeriodic3D", "gdof", "math"]
