"""Generate the golden vectors in tests/golden/ from the reference's own solver.

Runs the reference's DirectPseudoSpectral SolvePDE and its HypreFDM 3D
assembly (compiled from its sources by oracle/Makefile into oracle/_ref) on
small seeded problems and stores inputs and
outputs as compressed .npz files.  Needs the reference tree at build time; the
committed .npz files are what the tests read.

    python tests/golden/make_golden.py [fixture names]
"""
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from mpi_b200 import workloads as W  # noqa: E402
from oracle import oracle as O  # noqa: E402


def main():
    O.build()
    if not O.have_reference():
        raise SystemExit("reference oracle (oracle/_ref) not built: reference tree absent")
    rng = np.random.default_rng(20240601)
    out = {}

    # config-1 manufactured problem, Dirichlet
    f, ue = W.manufactured_2d(64, 33, 1.0)
    z = np.zeros(64)
    u = O.ref_solve2d(f, z, z, xl=0.0, xr=2 * math.pi, yl=-1.0, yr=1.0, lam=1.0)
    out["cfg1_2d"] = dict(f=f, u=u, u_exact=ue, Nx=64, N=33, Ns=1, dom=[0.0, 2 * math.pi, -1.0, 1.0], lam=1.0,
                          bc=[0.0, 1.0, 0.0, 1.0])

    # 2D Robin, three elements
    Nx, N, Ns = 16, 9, 3
    f = rng.standard_normal((Ns, Nx, N)); gl = rng.standard_normal(Nx); gr = rng.standard_normal(Nx)
    bc = [1.0, 0.5, 0.7, 2.0]
    u = O.ref_solve2d(f, gl, gr, xl=0.1, xr=1.4, yl=0.0, yr=0.9, lam=2.0, bc=tuple(bc))
    out["robin_2d_ns3"] = dict(f=f, gl=gl, gr=gr, u=u, Nx=Nx, N=N, Ns=Ns, dom=[0.1, 1.4, 0.0, 0.9], lam=2.0, bc=bc)

    # 3D Robin, one element, Lx != Ly
    Nx, Ny, N = 8, 16, 9
    f = rng.standard_normal((Nx, Ny, N)); gl = rng.standard_normal((Nx, Ny)); gr = rng.standard_normal((Nx, Ny))
    u = O.ref_solve3d(f, gl, gr, xl=0.0, xr=1.3, yl=0.0, yr=0.7, zl=0.0, zr=0.9, lam=2.0, bc=tuple(bc))
    out["robin_3d"] = dict(f=f, gl=gl, gr=gr, u=u, Nx=Nx, Ny=Ny, N=N, Ns=1,
                           dom=[0.0, 1.3, 0.0, 0.7, 0.0, 0.9], lam=2.0, bc=bc)

    # 3D Robin, two elements
    Nx, Ny, N, Ns = 8, 4, 7, 2
    f = rng.standard_normal((Ns, Nx, Ny, N)); gl = rng.standard_normal((Nx, Ny)); gr = rng.standard_normal((Nx, Ny))
    u = O.ref_solve3d(f, gl, gr, xl=0.0, xr=1.0, yl=0.0, yr=2.0, zl=0.0, zr=1.5, lam=0.5, bc=tuple(bc))
    out["robin_3d_ns2"] = dict(f=f, gl=gl, gr=gr, u=u, Nx=Nx, Ny=Ny, N=N, Ns=Ns,
                               dom=[0.0, 1.0, 0.0, 2.0, 0.0, 1.5], lam=0.5, bc=bc)

    # config-2 shape in miniature: smooth seeded field, Dirichlet, lambda = 10
    Nx = Ny = 16; N = 17
    f = W.smooth_field_3d(Nx, Ny, N, seed=1236)
    zb = np.zeros((Nx, Ny))
    u = O.ref_solve3d(f, zb, zb, xl=0.0, xr=2 * math.pi, yl=0.0, yr=2 * math.pi, zl=0.0, zr=2.0, lam=10.0)
    out["smooth_3d"] = dict(f=f, u=u, Nx=Nx, Ny=Ny, N=N, Ns=1, dom=[0.0, 2 * math.pi, 0.0, 2 * math.pi, 0.0, 2.0],
                            lam=10.0, bc=[0.0, 1.0, 0.0, 1.0])

    # solvers periodic in the GLL direction (Periodic2D_MPI.cpp, Periodic3D_MPI.cpp)
    prng = np.random.default_rng(20240602)
    Nx, N, Ns = 16, 9, 1
    f = prng.standard_normal((Ns, Nx, N))
    u = O.ref_psolve2d(f, xl=0.0, xr=1.3, yl=0.0, yr=0.8, lam=1.5)
    out["periodic_2d"] = dict(f=f, u=u, Nx=Nx, N=N, Ns=Ns, dom=[0.0, 1.3, 0.0, 0.8], lam=1.5)
    Nx, N, Ns = 16, 8, 4
    f = prng.standard_normal((Ns, Nx, N))
    u = O.ref_psolve2d(f, xl=0.0, xr=2.0, yl=0.0, yr=3.0, lam=0.6)
    out["periodic_2d_ns4"] = dict(f=f, u=u, Nx=Nx, N=N, Ns=Ns, dom=[0.0, 2.0, 0.0, 3.0], lam=0.6)
    Nx, Ny, N, Ns = 8, 16, 9, 1
    f = prng.standard_normal((Ns, Nx, Ny, N))
    u = O.ref_psolve3d(f, xl=0.0, xr=1.3, yl=0.0, yr=0.7, zl=0.0, zr=0.9, lam=2.0)
    out["periodic_3d"] = dict(f=f, u=u, Nx=Nx, Ny=Ny, N=N, Ns=Ns, dom=[0.0, 1.3, 0.0, 0.7, 0.0, 0.9], lam=2.0)
    Nx, Ny, N, Ns = 8, 4, 7, 3
    f = prng.standard_normal((Ns, Nx, Ny, N))
    u = O.ref_psolve3d(f, xl=0.0, xr=1.0, yl=0.0, yr=2.0, zl=0.0, zr=1.5, lam=0.5)
    out["periodic_3d_ns3"] = dict(f=f, u=u, Nx=Nx, Ny=Ny, N=N, Ns=Ns, dom=[0.0, 1.0, 0.0, 2.0, 0.0, 1.5], lam=0.5)

    # derivative helpers: the reference's spectral derivatives and GLL derivatives
    drng = np.random.default_rng(20240603)
    u2 = drng.standard_normal((16, 9))
    u3 = drng.standard_normal((8, 16, 5))
    ug2 = drng.standard_normal((3, 8, 9))
    ug3 = drng.standard_normal((2, 4, 8, 7))
    d = dict(u2=u2, u3=u3, ug2=ug2, ug3=ug3, L2=1.3, L3x=0.7, L3y=2.1, yl=-1.0, yr=1.0, zl=0.0, zr=1.5)
    for order in (1, 2):
        d[f"fx2_{order}"] = O.ref_fourier_deriv(u2, axis=0, order=order, L=1.3)
        d[f"fx3_{order}"] = O.ref_fourier_deriv(u3, axis=0, order=order, L=0.7)
        d[f"fy3_{order}"] = O.ref_fourier_deriv(u3, axis=1, order=order, L=2.1)
        d[f"gy2_{order}"] = O.ref_gll_deriv_2d(ug2, yl=-1.0, yr=1.0, order=order)
        d[f"gz3_{order}"] = O.ref_gll_deriv_3d(ug3, zl=0.0, zr=1.5, order=order)
    out["derivatives"] = d

    # the reference's Tecplot writer (WriteFile) on seeded small fields
    import tempfile
    wrng = np.random.default_rng(20240604)
    u2 = wrng.standard_normal((2, 8, 5))
    u3 = wrng.standard_normal((2, 4, 4, 4))
    with tempfile.TemporaryDirectory() as td:
        t2 = O.ref_write_tecplot(u2, (0.5, 2.0, -1.0, 1.0), td)
        t3 = O.ref_write_tecplot(u3, (0.0, 1.0, 0.5, 1.5, 0.0, 2.0), td)
    with open(os.path.join(HERE, "writer_2d.tec"), "w") as fh:
        fh.write(t2)
    with open(os.path.join(HERE, "writer_3d.tec"), "w") as fh:
        fh.write(t3)
    out["writer_fields"] = dict(u2=u2, u3=u3, dom2=[0.5, 2.0, -1.0, 1.0], dom3=[0.0, 1.0, 0.5, 1.5, 0.0, 2.0])

    # a caller's own operator through SolvePDE's ConstructOperator callback: the
    # stock operator minus a coefficient c(y) varying along the GLL direction
    # (Dyy_int - diag(lambda + k^2 + c_i)), 2D with two Robin elements, 3D with
    # one element and Lx = Ly
    orng = np.random.default_rng(20240605)
    d = {}
    Nx, N, Ns = 16, 9, 2
    c2 = 1.0 + orng.random(N - 2)
    f = orng.standard_normal((Ns, Nx, N)); gl = orng.standard_normal(Nx); gr = orng.standard_normal(Nx)
    O.ref_set_cdiag(2, c2)
    u = O.ref_solve2d(f, gl, gr, xl=0.0, xr=1.2, yl=0.0, yr=0.8, lam=1.5, bc=(1.0, 0.5, 0.7, 2.0))
    O.ref_set_cdiag(2, None)
    d.update(f2=f, gl2=gl, gr2=gr, u2=u, c2=c2, dom2=[0.0, 1.2, 0.0, 0.8], lam2=1.5, bc2=[1.0, 0.5, 0.7, 2.0])
    Nx, Ny, N = 8, 8, 9
    c3 = 2.0 * orng.random(N - 2)
    f = orng.standard_normal((Nx, Ny, N)); gl = orng.standard_normal((Nx, Ny)); gr = orng.standard_normal((Nx, Ny))
    O.ref_set_cdiag(3, c3)
    u = O.ref_solve3d(f, gl, gr, xl=0.0, xr=1.0, yl=0.0, yr=1.0, zl=0.0, zr=1.5, lam=0.5)
    O.ref_set_cdiag(3, None)
    d.update(f3=f, gl3=gl, gr3=gr, u3=u, c3=c3, dom3=[0.0, 1.0, 0.0, 1.0, 0.0, 1.5], lam3=0.5)
    out["user_operator"] = d

    # the reference's HypreFDM 3D solver (its own SetA / Setb assembly; the
    # assembled system solved directly, and its transpose for the adjoint):
    # x, y periodic, Robin ends in z
    if O.have_reference_fd():
        frng = np.random.default_rng(20241204)
        d = {}
        cases = [((8, 4, 6), (0.0, 1.0, 0.0, 1.0), 1.0, (1.0, 0.5, 1.5)),
                 ((16, 8, 12), (1.0, 0.5, 0.7, 2.0), 3.0, (1.3, 0.7, 1.9)),
                 ((4, 16, 9), (1.0, 0.3, 0.0, 1.0), 0.5, (2.0, 1.0, 0.8))]
        for c, (shape, bc, lam, (Lx, Ly, Lz)) in enumerate(cases):
            f = frng.standard_normal(shape)
            gb = frng.standard_normal(shape[:2]); gf = frng.standard_normal(shape[:2])
            u = O.ref_fd3d_solve(f, gb, gf, Lx=Lx, Ly=Ly, Lz=Lz, lam=lam, bc=bc)
            d.update({f"f{c}": f, f"gb{c}": gb, f"gf{c}": gf, f"u{c}": u, f"bc{c}": list(bc), f"lam{c}": lam,
                      f"L{c}": [Lx, Ly, Lz]})
        # the transpose of each map, from the reference's own assembled matrix
        arng = np.random.default_rng(20241205)
        for c, (shape, bc, lam, (Lx, Ly, Lz)) in enumerate(cases):
            ub = arng.standard_normal(shape)
            fb, gbb, gfb = O.ref_fd3d_adjoint(ub, Lx=Lx, Ly=Ly, Lz=Lz, lam=lam, bc=bc)
            d.update({f"ubar{c}": ub, f"fbar{c}": fb, f"gbbar{c}": gbb, f"gfbar{c}": gfb})
        d["ncases"] = len(cases)
        out["fd3d_reference"] = d

    only = sys.argv[1:]  # optional: names of the fixtures to (re)write
    for name, d in out.items():
        if only and name not in only:
            continue
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **{k: np.asarray(v) for k, v in d.items()})
        print(name, {k: np.asarray(v).shape for k, v in d.items()})


if __name__ == "__main__":
    main()
