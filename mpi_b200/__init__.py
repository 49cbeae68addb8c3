"""B200 (sm_100a) pseudo-spectral Helmholtz solver: the DirectPseudoSpectral
solve of gpritam/MPI (Fourier x GLL collocation, per-wavenumber LU, interface
sweep, inverse FFT) as CUDA kernels behind a C ABI (include/helm_b200.h).

The solver classes load on first use, so that `mpi_b200.workloads` (numpy only)
imports without torch, e.g. in CPU worker processes."""

_SOLVER_NAMES = ("BatchNonPeriodic2D", "Helmholtz3DFD", "NonPeriodic2D", "NonPeriodic3D", "Periodic2D", "Periodic3D",
                 "gdof")

__all__ = list(_SOLVER_NAMES)


def __getattr__(name):
    if name in _SOLVER_NAMES:
        from . import solver

        return getattr(solver, name)
    raise AttributeError(f"module 'mpi_b200' has no attribute {name!r}")
