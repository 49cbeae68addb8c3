"""B200 (sm_100a) pseudo-spectral Helmholtz solver: the DirectPseudoSpectral
solve of gpritam/MPI (Fourier x GLL collocation, per-wavenumber LU, interface
sweep, inverse FFT) as CUDA kernels behind a C ABI (include/helm_b200.h)."""
from .solver import BatchNonPeriodic2D, Helmholtz3DFD, NonPeriodic2D, NonPeriodic3D, gdof  # noqa: F401
