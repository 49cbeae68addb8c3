// FP64 residual of the finite-difference system, the refinement step of FD
// plans created with HELM_FP32_REFINE: the solve runs in FP32 (FP32 spectrum,
// FP32 tridiagonal solves), the residual r = f - A_h u is formed here from the
// 7-point stencil in FP64 (HypreFDM/src/Helmholtz3D_MPI.cpp:387-403, x and y
// periodic, the Robin rows eliminated into the first and last z equations as
// the solve does), and an FP32 solve of A_h d = r is added to u.  The adjoint
// refines the same way with the transposed stencil.
#include <cuda_runtime.h>

#include "helm_device.cuh"
#include "helm_fd_refine.cuh"

namespace helm {

namespace {

// One thread per interior point (i, j, k), k fastest.  The z rows of A_h on
// the interior unknowns: diagonal dz = -2 cz1 (+ dfirst at k = 0, + dlast at
// k = Nz - 1), neighbours cz1, except A[0][1] = sfirst and A[Nz-1][Nz-2] =
// slast; forward data terms scale_l * gl at k = 0 and scale_r * gr at
// k = Nz - 1 on the right-hand side.
__global__ void fd_residual_kernel(FdResidualArgs a)
{
    pdl_enter();
    const long long nz = a.Nz, ny = a.Ny, plane = ny * nz, total = (long long)a.Nx * plane;
    const double cdiag = -2.0 * (a.cx1 + a.cy1 + a.cz1) - a.lam;
    for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < total;
         o += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(o % nz);
        const long long rj = o / nz;
        const int j = (int)(rj % ny), i = (int)(rj / ny);
        const double* v = a.v;
        const double vc = v[o];
        const double vx = v[i == 0 ? o + (long long)(a.Nx - 1) * plane : o - plane] +
                          v[i == a.Nx - 1 ? o - (long long)(a.Nx - 1) * plane : o + plane];
        const double vy = v[j == 0 ? o + (long long)(a.Ny - 1) * nz : o - nz] +
                          v[j == a.Ny - 1 ? o - (long long)(a.Ny - 1) * nz : o + nz];
        double az = (k == 0 ? a.dfirst : 0.0) + (k == a.Nz - 1 ? a.dlast : 0.0);
        az *= vc;
        if (!a.transpose) {
            if (k > 0) az += (k == a.Nz - 1 ? a.slast : a.cz1) * v[o - 1];
            if (k < a.Nz - 1) az += (k == 0 ? a.sfirst : a.cz1) * v[o + 1];
        } else {
            if (k > 0) az += (k == 1 ? a.sfirst : a.cz1) * v[o - 1];
            if (k < a.Nz - 1) az += (k == a.Nz - 2 ? a.slast : a.cz1) * v[o + 1];
        }
        const double av = a.cx1 * vx + a.cy1 * vy + cdiag * vc + az;
        double rhs = a.rhs[o];
        if (a.sub) rhs -= a.sub[o];
        if (k == 0 && a.gl) rhs += a.scale_l * a.gl[rj];
        if (k == a.Nz - 1 && a.gr) rhs += a.scale_r * a.gr[rj];
        a.r[o] = (float)(rhs - av);
    }
}

}  // namespace

int launch_fd_residual(const FdResidualArgs& a, cudaStream_t s)
{
    const long long total = (long long)a.Nx * a.Ny * a.Nz;
    const long long blocks = std::min<long long>((total + 255) / 256, 148LL * 16);
    return (int)launch_k(fd_residual_kernel, dim3((unsigned)blocks), dim3(256), 0, s, a);
}

}  // namespace helm
