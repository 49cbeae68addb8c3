// Host utilities of the C ABI that the reference's global-state interface
// needs from its own helpers (the GLL grid of CreatePDEPlan, LUDecomposition /
// LUSolve), and the device max-norm reduction behind ComputeError.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/helm_b200.h"
#include "helm_device.cuh"
#include "helm_plan.hpp"
#include "helm_setup.hpp"

namespace helm {

namespace {

// max |a - b| over the points of a plan's arrays: element e, x row, the Ny*P
// values of the row; non-negative doubles order as their bit patterns, so the
// maximum is one 64-bit atomicMax (a NaN, whose pattern is larger, wins).
__global__ void max_abs_diff_kernel(const double* a, const double* b, unsigned long long* out, long long nx,
                                    long long row, long long x_stride, long long elem_stride, long long total)
{
    pdl_enter();
    double m = 0.0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
        const long long k = t % row, r = t / row, x = r % nx, e = r / nx;
        const long long o = e * elem_stride + x * x_stride + k;
        const double d = fabs(a[o] - b[o]);
        m = (d > m || d != d) ? d : m;
    }
    for (int s = 16; s > 0; s >>= 1) {
        const double o = __shfl_xor_sync(0xffffffffu, m, s);
        m = (o > m || o != o) ? o : m;
    }
    if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

}  // namespace

}  // namespace helm

using helm::Plan;

extern "C" {

int helm_gll_grid(int N, int Ns, double L, double* nodes, double* D, double* D2)
{
    if (N < 2 || N > 1024 || Ns < 1 || !(L > 0.0)) return HELM_ERR_INVALID;
    const helm::GllSetup g = helm::build_gll_setup(N, Ns, L);
    if (nodes) std::memcpy(nodes, g.nodes.data(), g.nodes.size() * sizeof(double));
    if (D) std::memcpy(D, g.D.data(), g.D.size() * sizeof(double));
    if (D2) std::memcpy(D2, g.D2.data(), g.D2.size() * sizeof(double));
    return HELM_OK;
}

int helm_lu_factor(int n, double* A, int* perm, double* determinant)
{
    if (n < 1 || !A || !perm) return HELM_ERR_INVALID;
    if (!helm::lu_factor(n, A, perm)) {
        helm::set_last_error("matrix is singular (scaled pivot below 1e-12)");
        return HELM_ERR_SINGULAR;
    }
    if (determinant) {
        // product of U's diagonal times the sign of the row permutation
        double d = 1.0;
        for (int i = 0; i < n; ++i) d *= A[(size_t)i * n + i];
        std::vector<char> seen(n, 0);
        for (int i = 0; i < n; ++i) {
            if (seen[i]) continue;
            int len = 0;
            for (int j = i; !seen[j]; j = perm[j]) {
                seen[j] = 1;
                ++len;
            }
            if (len % 2 == 0) d = -d;
        }
        *determinant = d;
    }
    return HELM_OK;
}

int helm_lu_solve(int n, const double* LU, const int* perm, double* b)
{
    if (n < 1 || !LU || !perm || !b) return HELM_ERR_INVALID;
    helm::lu_solve(n, LU, perm, b);
    return HELM_OK;
}

int helm_max_abs_diff(helm_plan_t plan, const double* a, const double* b, double* result, void* stream)
{
    if (!plan || !a || !b || !result) return HELM_ERR_INVALID;
    const Plan& p = *reinterpret_cast<const Plan*>(plan);
    if (p.batch > 1) {
        helm::set_last_error("helm_max_abs_diff takes single-problem plans");
        return HELM_ERR_UNSUPPORTED;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != p.device) cudaSetDevice(p.device);
    const long long row = (long long)(p.dim == 3 ? p.Ny : 1) * p.N;
    const long long total = (long long)p.Ns * p.Nx * row;
    cudaError_t e = cudaMemsetAsync(result, 0, sizeof(double), s);
    if (e == cudaSuccess) {
        const long long blocks = std::min<long long>((total + 255) / 256, 4 * 148);
        e = helm::launch_k(helm::max_abs_diff_kernel, dim3((unsigned)std::max<long long>(blocks, 1)), dim3(256), 0,
                           s, a, b, reinterpret_cast<unsigned long long*>(result), (long long)p.Nx, row, p.x_stride,
                           p.elem_stride, total);
    }
    if (cur != p.device) cudaSetDevice(cur);
    if (e != cudaSuccess) {
        cudaGetLastError();
        helm::set_last_error(cudaGetErrorString(e));
        return HELM_ERR_CUDA;
    }
    return HELM_OK;
}

}  // extern "C"
