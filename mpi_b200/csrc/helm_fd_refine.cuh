// Residual of the finite-difference system for the refinement sweeps of
// HELM_FP32_REFINE finite-difference plans (helm_fd_refine.cu).
#pragma once
#include <cuda_runtime.h>

namespace helm {

struct FdResidualArgs {
    const double* rhs;  // f (forward) or ubar (adjoint)
    const double* sub;  // adjoint of a misfit: subtracted from rhs (NULL: none)
    const double* gl;   // forward boundary data (NULL: zero)
    const double* gr;
    const double* v;    // current u (forward) or fbar (adjoint)
    float* r;           // out: rhs - A v (forward) or rhs - A^T v (adjoint)
    int Nx, Ny, Nz, transpose;
    double cx1, cy1, cz1, lam;
    double dfirst, sfirst, dlast, slast, scale_l, scale_r;
};

int launch_fd_residual(const FdResidualArgs& a, cudaStream_t s);

}  // namespace helm
