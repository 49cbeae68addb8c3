"""Python access to the CPU oracles (TEST INFRASTRUCTURE ONLY).

Two libraries, both built by ``oracle/Makefile``:

* ``liboracle.so`` -- the plain-C restatement (``helm_oracle.c``) of the
  reference's DirectPseudoSpectral solve and of the HypreFDM stencil solved by
  FFT/Thomas.  Always buildable (gcc only).
* ``_ref/libref2d.so`` / ``_ref/libref3d.so`` (and ``libref2dp.so`` /
  ``libref3dp.so``, the solvers periodic in the GLL direction) -- the
  reference's own C++ sources compiled unchanged, wrapped by
  ``ref_driver2d.cpp`` / ``ref_driver3d.cpp`` / ``ref_driver2dp.cpp`` /
  ``ref_driver3dp.cpp``.  Present only where the reference tree was available
  at build time; :func:`have_reference` says whether they were built.
* ``_ref/libreffd3d.so`` -- the reference's HypreFDM 3D solver
  (``Helmholtz3D_MPI.cpp``) compiled unchanged against an in-memory HYPRE IJ
  stub, its assembled system solved directly (``ref_driver_fd3d.cpp``);
  :func:`have_reference_fd`.

Only ``tests/``, ``__graft_entry__.smoke`` and the CPU-baseline leg of
``bench.py`` may import this module, and only as the checker.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_D = ctypes.c_double
_I = ctypes.c_int
_P = ctypes.POINTER(ctypes.c_double)

_lib = None
_ref2d = None
_ref3d = None
_refp = {}


def reference_root() -> str:
    """The reference checkout: $REF_ROOT, else a sibling of this repository
    (``<repo>/../reference``)."""
    return os.environ.get("REF_ROOT", os.path.abspath(os.path.join(_HERE, "..", "..", "reference")))


def build(quiet: bool = True) -> None:
    """Compile the C restatement (and the reference wrappers when the reference
    sources are present on this machine)."""
    out = subprocess.DEVNULL if quiet else None
    subprocess.run(["make", "-s", "-C", _HERE], check=True, stdout=out)
    ref_root = reference_root()
    if os.path.isdir(os.path.join(ref_root, "HelmholtzSolvers", "DirectPseudoSpectral")):
        subprocess.run(["make", "-s", "-C", _HERE, "ref", f"REF_ROOT={ref_root}"], check=True, stdout=out)
        if os.path.exists(os.path.join(_HERE, "..", "mpi_b200", "libhelm_b200.so")):
            subprocess.run(["make", "-s", "-C", _HERE, "shim", f"REF_ROOT={ref_root}"], check=True, stdout=out)


def _p(a: np.ndarray):
    return a.ctypes.data_as(_P)


def _c64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        _lib = ctypes.CDLL(path)
        _lib.orc_solve2d.restype = _I
        _lib.orc_solve2d.argtypes = [_I, _I, _I] + [_D] * 7 + [_P] * 4
        _lib.orc_solve3d.restype = _I
        _lib.orc_solve3d.argtypes = [_I, _I, _I, _I] + [_D] * 8 + [_P] * 4
        _lib.orc_gll_deriv.restype = None
        _lib.orc_gll_deriv.argtypes = [_I, _I, _D, _I, ctypes.c_long, _P, _P]
        _lib.orc_fourier_deriv.restype = None
        _lib.orc_fourier_deriv.argtypes = [_I] * 5 + [_D, _P, _P]
        _lib.orc_psolve2d.restype = _I
        _lib.orc_psolve2d.argtypes = [_I, _I, _I] + [_D] * 3 + [_P] * 2
        _lib.orc_psolve3d.restype = _I
        _lib.orc_psolve3d.argtypes = [_I, _I, _I, _I] + [_D] * 4 + [_P] * 2
        _lib.orc_residual3d.restype = _D
        _lib.orc_residual3d.argtypes = [_I, _I, _I] + [_D] * 8 + [_P] * 5
        _lib.orc_fd3d_solve.restype = _I
        _lib.orc_fd3d_solve.argtypes = [_I, _I, _I] + [_D] * 8 + [_P] * 4
        _lib.orc_fd3d_residual.restype = _D
        _lib.orc_fd3d_residual.argtypes = [_I, _I, _I] + [_D] * 8 + [_P] * 4
        _lib.orc_gll_setup.restype = None
        _lib.orc_gll_setup.argtypes = [_I, _I, _D, _P, _P, _P]
        _lib.orc_lu_decompose.restype = _I
        _lib.orc_lu_decompose.argtypes = [_I, _P, ctypes.POINTER(_I)]
        _lib.orc_lu_solve.restype = None
        _lib.orc_lu_solve.argtypes = [_I, _P, ctypes.POINTER(_I), _P]
    return _lib


def have_reference() -> bool:
    return all(os.path.exists(os.path.join(_HERE, "_ref", n))
               for n in ("libref2d.so", "libref3d.so", "libref2dp.so", "libref3dp.so"))


def _ref(which: int):
    global _ref2d, _ref3d
    if which == 2:
        if _ref2d is None:
            _ref2d = ctypes.CDLL(os.path.join(_HERE, "_ref", "libref2d.so"))
            _ref2d.oracle_ref2d_solve.restype = _I
            _ref2d.oracle_ref2d_solve.argtypes = [_I] * 3 + [_D] * 9 + [_P] * 6
        return _ref2d
    if _ref3d is None:
        _ref3d = ctypes.CDLL(os.path.join(_HERE, "_ref", "libref3d.so"))
        _ref3d.oracle_ref3d_solve.restype = _I
        _ref3d.oracle_ref3d_solve.argtypes = [_I] * 4 + [_D] * 11 + [_P] * 6
    return _ref3d


def _ref_periodic(which: int):
    if which not in _refp:
        lib_ = ctypes.CDLL(os.path.join(_HERE, "_ref", f"libref{which}dp.so"))
        if which == 2:
            lib_.oracle_ref2dp_solve.restype = _I
            lib_.oracle_ref2dp_solve.argtypes = [_I] * 3 + [_D] * 5 + [_P] * 4
        else:
            lib_.oracle_ref3dp_solve.restype = _I
            lib_.oracle_ref3dp_solve.argtypes = [_I] * 4 + [_D] * 7 + [_P] * 4
        _refp[which] = lib_
    return _refp[which]


# ------------------------------------------------------------------ grid --
def gll_grid(N: int, Ns: int, L: float):
    """(nodes[Ns*(N-1)+1], D[N,N], D2[N,N]) of one element of length L/Ns,
    nodes placed from 0 as the reference does."""
    y = np.zeros(Ns * (N - 1) + 1)
    D = np.zeros((N, N))
    D2 = np.zeros((N, N))
    lib().orc_gll_setup(N, Ns, L, _p(y), _p(D), _p(D2))
    return y, D, D2


# ------------------------------------------------------ restatement solves --
def solve2d(f, gl, gr, *, Lx, Ly, lam, bc=(0.0, 1.0, 0.0, 1.0)):
    """f: [Ns, Nx, N] or [Nx, N]; returns u of the same shape."""
    f = _c64(f)
    squeeze = f.ndim == 2
    if squeeze:
        f = f[None]
    Ns, Nx, N = f.shape
    u = np.zeros_like(f)
    st = lib().orc_solve2d(Nx, N, Ns, Lx, Ly, *bc, lam, _p(f), _p(_c64(gl)), _p(_c64(gr)), _p(u))
    if st:
        raise RuntimeError(f"orc_solve2d status {st}")
    return u[0] if squeeze else u


def solve3d(f, gl, gr, *, Lx, Ly, Lz, lam, bc=(0.0, 1.0, 0.0, 1.0)):
    """f: [Ns, Nx, Ny, N] or [Nx, Ny, N]; returns u of the same shape."""
    f = _c64(f)
    squeeze = f.ndim == 3
    if squeeze:
        f = f[None]
    Ns, Nx, Ny, N = f.shape
    u = np.zeros_like(f)
    st = lib().orc_solve3d(Nx, Ny, N, Ns, Lx, Ly, Lz, *bc, lam, _p(f), _p(_c64(gl)), _p(_c64(gr)), _p(u))
    if st:
        raise RuntimeError(f"orc_solve3d status {st}")
    return u[0] if squeeze else u


def psolve2d(f, *, Lx, Ly, lam):
    """Periodic in the GLL direction.  f: [Ns, Nx, N] or [Nx, N]."""
    f = _c64(f)
    squeeze = f.ndim == 2
    if squeeze:
        f = f[None]
    Ns, Nx, N = f.shape
    u = np.zeros_like(f)
    st = lib().orc_psolve2d(Nx, N, Ns, Lx, Ly, lam, _p(f), _p(u))
    if st:
        raise RuntimeError(f"orc_psolve2d status {st}")
    return u[0] if squeeze else u


def psolve3d(f, *, Lx, Ly, Lz, lam):
    """Periodic in the GLL direction.  f: [Ns, Nx, Ny, N] or [Nx, Ny, N]."""
    f = _c64(f)
    squeeze = f.ndim == 3
    if squeeze:
        f = f[None]
    Ns, Nx, Ny, N = f.shape
    u = np.zeros_like(f)
    st = lib().orc_psolve3d(Nx, Ny, N, Ns, Lx, Ly, Lz, lam, _p(f), _p(u))
    if st:
        raise RuntimeError(f"orc_psolve3d status {st}")
    return u[0] if squeeze else u


def gll_deriv(u, *, N, Ns, L, order):
    """du = D u (order 1) or D2 u (order 2) along the last axis (length N) of u,
    with the element matrices of an Ns-element GLL grid of total length L."""
    u = _c64(u)
    du = np.zeros_like(u)
    lib().orc_gll_deriv(N, Ns, L, order, u.size // N, _p(u), _p(du))
    return du


def fourier_deriv(u, *, axis, order, L):
    """Spectral derivative of a real [n0, n1(, n2)] array along axis 0 or 1."""
    u = _c64(u)
    shp = u.shape + (1,) * (3 - u.ndim)
    du = np.zeros_like(u)
    lib().orc_fourier_deriv(shp[0], shp[1], shp[2], axis, order, L, _p(u), _p(du))
    return du


def residual3d(u, f, gl, gr, *, Lx, Ly, Lz, lam, bc=(0.0, 1.0, 0.0, 1.0)):
    """Max-abs collocation residual (FP64) of a single-element 3D solution."""
    u = _c64(u)
    Nx, Ny, N = u.shape
    r = np.zeros_like(u)
    return lib().orc_residual3d(Nx, Ny, N, Lx, Ly, Lz, *bc, lam, _p(_c64(f)), _p(_c64(gl)), _p(_c64(gr)), _p(u), _p(r))


def fd3d_solve(f, gb, gf, *, Lx, Ly, Lz, lam, bc=(0.0, 1.0, 0.0, 1.0)):
    f = _c64(f)
    Nx, Ny, Nz = f.shape
    u = np.zeros_like(f)
    st = lib().orc_fd3d_solve(Nx, Ny, Nz, Lx, Ly, Lz, *bc, lam, _p(f), _p(_c64(gb)), _p(_c64(gf)), _p(u))
    if st:
        raise RuntimeError(f"orc_fd3d_solve status {st}")
    return u


def fd3d_residual(u, f, gb, gf, *, Lx, Ly, Lz, lam, bc=(0.0, 1.0, 0.0, 1.0)):
    u = _c64(u)
    Nx, Ny, Nz = u.shape
    return lib().orc_fd3d_residual(Nx, Ny, Nz, Lx, Ly, Lz, *bc, lam, _p(_c64(f)), _p(_c64(gb)), _p(_c64(gf)), _p(u))


# ------------------------------------------------------- the reference itself --
def ref_solve2d(f, gl, gr, *, xl, xr, yl, yr, lam, bc=(0.0, 1.0, 0.0, 1.0), return_time=False):
    """The reference's own SolvePDE (2D).  f: [Ns, Nx, N] or [Nx, N]."""
    f = _c64(f)
    squeeze = f.ndim == 2
    if squeeze:
        f = f[None]
    Ns, Nx, N = f.shape
    u = np.zeros_like(f)
    y = np.zeros(Ns * (N - 1) + 1)
    ms = np.zeros(1)
    ns = _ref(2).oracle_ref2d_solve(Nx, Ns * N, N, xl, xr, yl, yr, *bc, lam,
                                    _p(f), _p(_c64(gl)), _p(_c64(gr)), _p(u), _p(y), _p(ms))
    if ns != Ns:
        raise RuntimeError(f"reference chose Ns={ns}, expected {Ns}")
    out = u[0] if squeeze else u
    return (out, ms[0]) if return_time else out


def ref_solve3d(f, gl, gr, *, xl, xr, yl, yr, zl, zr, lam, bc=(0.0, 1.0, 0.0, 1.0), return_time=False):
    """The reference's own SolvePDE (3D).  f: [Ns, Nx, Ny, N] or [Nx, Ny, N]."""
    f = _c64(f)
    squeeze = f.ndim == 3
    if squeeze:
        f = f[None]
    Ns, Nx, Ny, N = f.shape
    u = np.zeros_like(f)
    z = np.zeros(Ns * (N - 1) + 1)
    ms = np.zeros(1)
    ns = _ref(3).oracle_ref3d_solve(Nx, Ny, Ns * N, N, xl, xr, yl, yr, zl, zr, *bc, lam,
                                    _p(f), _p(_c64(gl)), _p(_c64(gr)), _p(u), _p(z), _p(ms))
    if ns != Ns:
        raise RuntimeError(f"reference chose Ns={ns}, expected {Ns}")
    out = u[0] if squeeze else u
    return (out, ms[0]) if return_time else out


_reffd = None


def have_reference_fd() -> bool:
    return os.path.exists(os.path.join(_HERE, "_ref", "libreffd3d.so"))


def _ref_fd():
    global _reffd
    if _reffd is None:
        _reffd = ctypes.CDLL(os.path.join(_HERE, "_ref", "libreffd3d.so"))
        for fn in (_reffd.oracle_ref_fd3d_solve, _reffd.oracle_ref_fd3d_adjoint):
            fn.restype = _I
            fn.argtypes = [_I] * 3 + [_D] * 11 + [_P] * 4
    return _reffd


def ref_fd3d_adjoint(ubar, *, Lx, Ly, Lz, lam, bc=(0.0, 1.0, 0.0, 1.0)):
    """The transpose of ref_fd3d_solve's linear map (f, gb, gf) -> u, from the
    reference's own assembled matrix: (fbar, gbbar, gfbar) for the cotangent
    ubar [Nx, Ny, Nz]."""
    ubar = _c64(ubar)
    Nx, Ny, Nz = ubar.shape
    fbar = np.zeros_like(ubar)
    gbb = np.zeros((Nx, Ny)); gfb = np.zeros((Nx, Ny))
    st = _ref_fd().oracle_ref_fd3d_adjoint(Nx, Ny, Nz, 0.0, Lx, 0.0, Ly, 0.0, Lz, *bc, lam,
                                           _p(ubar), _p(fbar), _p(gbb), _p(gfb))
    if st:
        raise RuntimeError(f"oracle_ref_fd3d_adjoint status {st}")
    return fbar, gbb, gfb


def ref_fd3d_solve(f, gb, gf, *, Lx, Ly, Lz, lam, bc=(0.0, 1.0, 0.0, 1.0)):
    """The reference's own HypreFDM 3D solver (Helmholtz3D_MPI.cpp SetA / Setb
    assembly, x and y periodic, Robin ends in z) with the assembled system
    solved directly.  f: [Nx, Ny, Nz] interior points; gb, gf: [Nx, Ny] Robin
    data at z = 0 and z = Lz; bc = (alpha_back, beta_back, alpha_front,
    beta_front).  Returns the interior solution [Nx, Ny, Nz]."""
    f = _c64(f)
    Nx, Ny, Nz = f.shape
    u = np.zeros_like(f)
    st = _ref_fd().oracle_ref_fd3d_solve(Nx, Ny, Nz, 0.0, Lx, 0.0, Ly, 0.0, Lz, *bc, lam,
                                      _p(f), _p(_c64(gb)), _p(_c64(gf)), _p(u))
    if st:
        raise RuntimeError(f"oracle_ref_fd3d_solve status {st}")
    return u


def ref_set_cdiag(dim: int, c=None):
    """Extra diagonal c_i (interior GLL nodes) that the reference drivers'
    ConstructOperator subtracts from the stock operator; None restores it."""
    lib_ = _ref(dim)
    fn = lib_.oracle_ref2d_set_cdiag if dim == 2 else lib_.oracle_ref3d_set_cdiag
    fn.restype = None
    fn.argtypes = [_P, _I]
    if c is None:
        fn(None, 0)
    else:
        c = _c64(c)
        fn(_p(c), int(c.size))


def ref_psolve2d(f, *, xl, xr, yl, yr, lam, return_time=False):
    """The reference's own Periodic2D SolvePDE.  f: [Ns, Nx, N] or [Nx, N]."""
    f = _c64(f)
    squeeze = f.ndim == 2
    if squeeze:
        f = f[None]
    Ns, Nx, N = f.shape
    u = np.zeros_like(f)
    y = np.zeros(Ns * (N - 1) + 1)
    ms = np.zeros(1)
    ns = _ref_periodic(2).oracle_ref2dp_solve(Nx, Ns * N, N, xl, xr, yl, yr, lam, _p(f), _p(u), _p(y), _p(ms))
    if ns != Ns:
        raise RuntimeError(f"reference chose Ns={ns}, expected {Ns}")
    out = u[0] if squeeze else u
    return (out, ms[0]) if return_time else out


def ref_psolve3d(f, *, xl, xr, yl, yr, zl, zr, lam, return_time=False):
    """The reference's own Periodic3D SolvePDE.  f: [Ns, Nx, Ny, N] or [Nx, Ny, N]."""
    f = _c64(f)
    squeeze = f.ndim == 3
    if squeeze:
        f = f[None]
    Ns, Nx, Ny, N = f.shape
    u = np.zeros_like(f)
    z = np.zeros(Ns * (N - 1) + 1)
    ms = np.zeros(1)
    ns = _ref_periodic(3).oracle_ref3dp_solve(Nx, Ny, Ns * N, N, xl, xr, yl, yr, zl, zr, lam,
                                              _p(f), _p(u), _p(z), _p(ms))
    if ns != Ns:
        raise RuntimeError(f"reference chose Ns={ns}, expected {Ns}")
    out = u[0] if squeeze else u
    return (out, ms[0]) if return_time else out


def _ref_deriv(which: int):
    lib_ = _ref(which)
    if not hasattr(lib_, "_deriv_ready"):
        if which == 2:
            lib_.oracle_ref2d_deriv_y.restype = _I
            lib_.oracle_ref2d_deriv_y.argtypes = [_I] * 3 + [_D] * 2 + [_I] + [_P] * 2
            lib_.oracle_ref_fourier_deriv_2d.restype = None
            lib_.oracle_ref_fourier_deriv_2d.argtypes = [_I] * 4 + [_D] + [_P] * 2
        else:
            lib_.oracle_ref3d_deriv_z.restype = _I
            lib_.oracle_ref3d_deriv_z.argtypes = [_I] * 4 + [_D] * 2 + [_I] + [_P] * 2
            lib_.oracle_ref_fourier_deriv_3d.restype = None
            lib_.oracle_ref_fourier_deriv_3d.argtypes = [_I] * 5 + [_D] + [_P] * 2
        lib_._deriv_ready = True
    return lib_


def ref_gll_deriv_2d(u, *, yl, yr, order):
    """The reference's NonPeriodic2D FirstDerivativeY / SecondDerivativeY.  u: [Ns, Nx, N]."""
    u = _c64(u)
    Ns, Nx, N = u.shape
    du = np.zeros_like(u)
    ns = _ref_deriv(2).oracle_ref2d_deriv_y(Nx, Ns * N, N, yl, yr, order, _p(u), _p(du))
    if ns != Ns:
        raise RuntimeError(f"reference chose Ns={ns}, expected {Ns}")
    return du


def ref_gll_deriv_3d(u, *, zl, zr, order):
    """The reference's NonPeriodic3D FirstDerivativeZ / SecondDerivativeZ.  u: [Ns, Nx, Ny, N]."""
    u = _c64(u)
    Ns, Nx, Ny, N = u.shape
    du = np.zeros_like(u)
    ns = _ref_deriv(3).oracle_ref3d_deriv_z(Nx, Ny, Ns * N, N, zl, zr, order, _p(u), _p(du))
    if ns != Ns:
        raise RuntimeError(f"reference chose Ns={ns}, expected {Ns}")
    return du


def ref_fourier_deriv(u, *, axis, order, L):
    """The reference's FirstDerivativeFourierX/Y, SecondDerivativeFourierX/Y on a
    real [n0, n1] or [n0, n1, n2] array (Fourier_Quadrature.cpp:1387-1834)."""
    u = _c64(u)
    du = np.zeros_like(u)
    if u.ndim == 2:
        _ref_deriv(2).oracle_ref_fourier_deriv_2d(u.shape[0], u.shape[1], axis, order, L, _p(u), _p(du))
    else:
        _ref_deriv(3).oracle_ref_fourier_deriv_3d(u.shape[0], u.shape[1], u.shape[2], axis, order, L, _p(u), _p(du))
    return du


def ref_write_tecplot(u, dom, workdir):
    """The reference's WriteFile (TECPLOT) of u ([Ns, Nx, N] or [Ns, Nx, Ny, N]) on
    the domain `dom`; returns the text of Output/Solution-0000.tec written under
    `workdir` (exact = sin(x) cos(y) [* z])."""
    u = _c64(u)
    os.makedirs(os.path.join(workdir, "Output"), exist_ok=True)
    cwd = os.getcwd()
    os.chdir(workdir)
    try:
        if u.ndim == 3:
            Ns, Nx, N = u.shape
            lib_ = _ref(2)
            lib_.oracle_ref2d_write.restype = _I
            lib_.oracle_ref2d_write.argtypes = [_I] * 3 + [_D] * 4 + [_P]
            lib_.oracle_ref2d_write(Nx, Ns * N, N, *dom, _p(u))
        else:
            Ns, Nx, Ny, N = u.shape
            lib_ = _ref(3)
            lib_.oracle_ref3d_write.restype = _I
            lib_.oracle_ref3d_write.argtypes = [_I] * 4 + [_D] * 6 + [_P]
            lib_.oracle_ref3d_write(Nx, Ny, Ns * N, N, *dom, _p(u))
        with open(os.path.join("Output", "Solution-0000.tec")) as fh:
            return fh.read()
    finally:
        os.chdir(cwd)
