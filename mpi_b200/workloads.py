"""Seeded synthetic inputs for the solver's workloads (numpy, FP64).

* :func:`manufactured_2d` -- the 2D problem (d2/dx2 + d2/dy2 - lambda) u = f on
  [0, 2pi) x [-1, 1] with u = sin(3x) (1 - y^2) exp(y), Dirichlet in y, placed
  on the reference's GLL nodes (which start at 0, so the physical y is node - 1).
* :func:`smooth_field_3d` / :func:`smooth_field_2d` -- seeded complex Gaussian
  coefficients over Fourier x Legendre modes with amplitude (1 + |k|^2)^-1.5 and
  zero mean, synthesised on the grid.  |k|^2 counts the Fourier wavenumbers and
  the Legendre degree.
* :func:`stock_2d` / :func:`stock_3d` -- the reference's own manufactured tests
  (TestNonPeriodic2D_MPI.cpp:26-62, TestNonPeriodic3D_MPI.cpp:26-66).

No public dataset is involved; these stand in for the reference's inputs.
"""
from __future__ import annotations

import math

import numpy as np

REF_PI = 3.1415926535897932  # the reference's PI (General.h:15)


def gll_nodes_unit(N: int) -> np.ndarray:
    """GLL nodes on [-1, 1] (ascending)."""
    from numpy.polynomial import legendre as npl

    c = np.zeros(N)
    c[-1] = 1.0
    inner = np.sort(npl.legroots(npl.legder(c)).real)
    return np.concatenate(([-1.0], inner, [1.0]))


def element_nodes(N: int, Ns: int, L: float) -> np.ndarray:
    """[Ns, N] node coordinates, element jj on [jj L/Ns, (jj+1) L/Ns] from 0."""
    xi = gll_nodes_unit(N)
    out = np.zeros((Ns, N))
    for jj in range(Ns):
        a = jj * L / Ns
        out[jj] = 0.5 * (2 * a + L / Ns + (L / Ns) * xi)
    return out


def manufactured_2d(Nx: int = 64, N: int = 33, lam: float = 1.0):
    """(f, u_exact) [Nx, N] of the sin(3x)(1-y^2)e^y problem on the reference grid."""
    x = 2.0 * math.pi * np.arange(Nx) / Nx
    y = element_nodes(N, 1, 2.0)[0] - 1.0
    g = (1 - y**2) * np.exp(y)
    gpp = (-1 - 4 * y - y**2) * np.exp(y)
    f = np.sin(3 * x)[:, None] * (-9 * g + gpp - lam * g)[None, :]
    u = np.sin(3 * x)[:, None] * g[None, :]
    return np.ascontiguousarray(f), np.ascontiguousarray(u)


def _legendre_vandermonde(N: int) -> np.ndarray:
    from numpy.polynomial import legendre as npl

    xi = gll_nodes_unit(N)
    return np.stack([npl.legval(xi, np.eye(N)[l]) for l in range(N)], axis=1)  # [node, degree]


def smooth_field_3d(Nx: int, Ny: int, N: int, seed: int) -> np.ndarray:
    """f[Nx, Ny, N]: Re of sum c_{kx,ky,l} e^{i(kx x + ky y)} P_l(z), seeded."""
    rng = np.random.default_rng(seed)
    kx = np.fft.fftfreq(Nx, 1.0 / Nx)
    ky = np.fft.fftfreq(Ny, 1.0 / Ny)
    l = np.arange(N)
    k2 = kx[:, None, None] ** 2 + ky[None, :, None] ** 2 + l[None, None, :] ** 2
    amp = (1.0 + k2) ** -1.5
    c = (rng.standard_normal((Nx, Ny, N)) + 1j * rng.standard_normal((Nx, Ny, N))) * amp
    c[0, 0, 0] = 0.0
    spec_xy = np.fft.ifft2(c, axes=(0, 1)).real * (Nx * Ny)  # [Nx, Ny, l]
    V = _legendre_vandermonde(N)  # [k, l]
    f = spec_xy @ V.T
    f -= f.mean()
    return np.ascontiguousarray(f)


def smooth_field_2d(Nx: int, N: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    kx = np.fft.fftfreq(Nx, 1.0 / Nx)
    l = np.arange(N)
    amp = (1.0 + kx[:, None] ** 2 + l[None, :] ** 2) ** -1.5
    c = (rng.standard_normal((Nx, N)) + 1j * rng.standard_normal((Nx, N))) * amp
    c[0, 0] = 0.0
    spec = np.fft.ifft(c, axis=0).real * Nx
    f = spec @ _legendre_vandermonde(N).T
    f -= f.mean()
    return np.ascontiguousarray(f)


def stock_2d(Nx: int = 512, Ny: int = 512, N: int = 10, lam: float = 1.0, bc=(1.0, 0.0, 0.0, 1.0)):
    """The reference's NonPeriodic2D test on [0,1]^2: exact u = sin(8 pi x) cos(6 pi y),
    left Neumann / right Dirichlet.  Returns (f[Ns,Nx,N], gl, gr, u_exact, bc)."""
    Ns = math.ceil(Ny / N)
    Lx = Ly = 1.0
    al, bl, ar, br = bc
    x = np.arange(Nx) * Lx / Nx
    y = element_nodes(N, Ns, Ly)
    sx = np.sin(8 * REF_PI * x / Lx)
    f = -(64 * REF_PI**2 / Lx**2 + 36 * REF_PI**2 / Ly**2 + lam) * sx[None, :, None] * np.cos(6 * REF_PI * y / Ly)[:, None, :]
    u = sx[None, :, None] * np.cos(6 * REF_PI * y / Ly)[:, None, :]
    gl = (al * 6 * REF_PI * math.sin(0.0) / Ly + bl * math.cos(0.0)) * sx
    gr = (-ar * 6 * REF_PI * math.sin(6 * REF_PI) / Ly + br * math.cos(6 * REF_PI)) * sx
    return np.ascontiguousarray(f), gl, gr, np.ascontiguousarray(u), bc


def stock_3d(Nx: int = 64, Ny: int = 32, Nz: int = 250, N: int = 10, lam: float = 1.0, bc=(1.0, 0.0, 0.0, 1.0)):
    """The reference's NonPeriodic3D test on [0,1]^3: u = sin(8 pi x) cos(6 pi y) cos(4 pi z)."""
    Ns = math.ceil(Nz / N)
    al, bl, ar, br = bc
    x = np.arange(Nx) / Nx
    y = np.arange(Ny) / Ny
    z = element_nodes(N, Ns, 1.0)
    sxy = np.sin(8 * REF_PI * x)[:, None] * np.cos(6 * REF_PI * y)[None, :]
    cz = np.cos(4 * REF_PI * z)
    f = -(64 * REF_PI**2 + 36 * REF_PI**2 + 16 * REF_PI**2 + lam) * sxy[None, :, :, None] * cz[:, None, None, :]
    u = sxy[None, :, :, None] * cz[:, None, None, :]
    gl = (al * 4 * REF_PI * math.sin(0.0) + bl * math.cos(0.0)) * sxy
    gr = (-ar * 4 * REF_PI * math.sin(4 * REF_PI) + br * math.cos(4 * REF_PI)) * sxy
    return np.ascontiguousarray(f), gl, gr, np.ascontiguousarray(u), bc


def stock_periodic_2d(Nx: int = 512, Ny: int = 512, N: int = 10, lam: float = 1.0):
    """The reference's Periodic2D test on [0,1]^2 (periodic in both directions):
    exact u = sin(8 pi x) cos(6 pi y).  Returns (f[Ns,Nx,N], u_exact)."""
    Ns = math.ceil(Ny / N)
    x = np.arange(Nx) / Nx
    y = element_nodes(N, Ns, 1.0)
    sx = np.sin(8 * REF_PI * x)
    u = sx[None, :, None] * np.cos(6 * REF_PI * y)[:, None, :]
    f = -(64 * REF_PI**2 + 36 * REF_PI**2 + lam) * u
    return np.ascontiguousarray(f), np.ascontiguousarray(u)


def stock_periodic_3d(Nx: int = 64, Ny: int = 32, Nz: int = 250, N: int = 10, lam: float = 1.0):
    """The reference's Periodic3D test on [0,1]^3: u = sin(8 pi x) cos(6 pi y) cos(4 pi z)."""
    Ns = math.ceil(Nz / N)
    x = np.arange(Nx) / Nx
    y = np.arange(Ny) / Ny
    z = element_nodes(N, Ns, 1.0)
    sxy = np.sin(8 * REF_PI * x)[:, None] * np.cos(6 * REF_PI * y)[None, :]
    u = sxy[None, :, :, None] * np.cos(4 * REF_PI * z)[:, None, None, :]
    f = -(64 * REF_PI**2 + 36 * REF_PI**2 + 16 * REF_PI**2 + lam) * u
    return np.ascontiguousarray(f), np.ascontiguousarray(u)


def smooth_field_fd(Nx: int, Ny: int, Nz: int, seed: int, kmax: int = 64) -> np.ndarray:
    """f[Nx, Ny, Nz] on the interior points of the finite-difference grid:
    Re of sum c_{kx,ky,l} e^{i(kx x + ky y)} sin(pi l z / Lz), l = 1..Nz, with
    seeded complex Gaussian c of amplitude (1 + kx^2 + ky^2 + l^2)^-1.5 and zero
    mean; modes beyond |k| = kmax (amplitude < 4e-6 of the largest) are omitted."""
    rng = np.random.default_rng(seed)
    kx = np.fft.fftfreq(Nx, 1.0 / Nx)
    ky = np.fft.fftfreq(Ny, 1.0 / Ny)
    L = min(Nz, kmax)
    l = np.arange(1, L + 1)
    keepx = np.abs(kx) <= kmax
    keepy = np.abs(ky) <= kmax
    planes = np.empty((L, Nx, Ny))
    for li in range(L):
        c = np.zeros((Nx, Ny), dtype=np.complex128)
        sub = (rng.standard_normal((keepx.sum(), keepy.sum())) + 1j * rng.standard_normal((keepx.sum(), keepy.sum())))
        amp = (1.0 + kx[keepx][:, None] ** 2 + ky[keepy][None, :] ** 2 + l[li] ** 2) ** -1.5
        c[np.ix_(keepx, keepy)] = sub * amp
        planes[li] = np.fft.ifft2(c).real * (Nx * Ny)
    z = np.arange(1, Nz + 1) / (Nz + 1)
    S = np.sin(np.pi * l[:, None] * z[None, :])  # [L, Nz]
    f = planes.reshape(L, Nx * Ny).T @ S
    f -= f.mean()
    return np.ascontiguousarray(f.reshape(Nx, Ny, Nz))


BATCH_NX = (32, 64, 128, 256, 512)
BATCH_ORDER = (16, 32, 64, 128)  # GLL polynomial orders; N + 1 points


def batch_2d(nprob: int = 512, seed: int = 1237):
    """Uneven batch of independent 2D problems: per problem Nx drawn from
    {32, 64, 128, 256, 512}, GLL order from {16, 32, 64, 128} (order + 1
    points), lambda log-uniform in [1e-2, 1e4], and f / u_exact the
    manufactured sin(3x)(1-y^2)e^y problem of :func:`manufactured_2d` at that
    size and lambda.  Returns (Nx list, points list, lambda list, f list, u list)."""
    rng = np.random.default_rng(seed)
    Nx = [int(v) for v in rng.choice(BATCH_NX, nprob)]
    P = [int(v) + 1 for v in rng.choice(BATCH_ORDER, nprob)]
    lam = [float(v) for v in 10.0 ** rng.uniform(-2.0, 4.0, nprob)]
    fs, us = [], []
    for nx, p, la in zip(Nx, P, lam):
        f, u = manufactured_2d(nx, p, la)
        fs.append(f)
        us.append(u)
    return Nx, P, lam, fs, us
