// Shared pieces of the reference-API shims (NonPeriodic2D_B200.cpp,
// NonPeriodic3D_B200.cpp): the reference's global-state solver interface
// re-implemented over the C ABI of libhelm_b200.  Host C++; the device work
// happens inside the library.
#pragma once
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "helm_b200.h"

namespace shim {

// Stops the program with the library's message, as the reference's
// ErrorMessage (General.cpp:6-11) does on its own failures.
inline void check(int st, const char* what)
{
    if (st != HELM_OK) {
        std::fprintf(stderr, "%s: %s [%s]\n", what, helm_status_string(st), helm_last_error());
        std::exit(1);
    }
}

inline void check_cuda(cudaError_t e, const char* what)
{
    if (e != cudaSuccess) {
        std::fprintf(stderr, "%s: %s\n", what, cudaGetErrorString(e));
        std::exit(1);
    }
}

// A device buffer of doubles that grows on demand.
struct DeviceBuf {
    double* p = nullptr;
    size_t n = 0;
    double* get(size_t count)
    {
        if (count > n) {
            if (p) cudaFree(p);
            p = nullptr;
            check_cuda(cudaMalloc(&p, count * sizeof(double)), "cudaMalloc");
            n = count;
        }
        return p;
    }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
};

// The operators one SolvePDE harvested from the caller's ConstructOperator,
// one n x n block per wavenumber pair, and the key they were harvested under.
struct OperatorSet {
    int n = 0;
    std::vector<int> iw, jw;
    std::vector<double> ops;
    const double* lookup(int i, int j) const
    {
        for (size_t k = 0; k < iw.size(); ++k)
            if (iw[k] == i && jw[k] == j) return &ops[k * (size_t)n * n];
        return nullptr;
    }
};

// Operator callback of helm_plan_set_operator_callback serving a harvested set.
inline void serve_operator(int iw, int jw, double* op, int ld, void* user)
{
    const OperatorSet* s = static_cast<const OperatorSet*>(user);
    const double* a = s->lookup(iw, jw);
    for (int i = 0; i < s->n; ++i)
        for (int j = 0; j < s->n; ++j) op[(size_t)i * ld + j] = a ? a[(size_t)i * s->n + j] : 0.0;
}

// The matrix most recently handed to LUDecomposition (LU_B200.cpp), which the
// reference's ConstructOperator callbacks call on their Operator before
// returning: the unfactored operator of that wavenumber pair.
bool take_captured(double* dst, int n);
void clear_captured();

// Device max |a - b| over a plan's solution points (helm_max_abs_diff), read back.
inline double max_abs_diff(helm_plan_t plan, const double* a, const double* b)
{
    double* d = nullptr;
    check_cuda(cudaMalloc(&d, sizeof(double)), "cudaMalloc");
    check(helm_max_abs_diff(plan, a, b, d, nullptr), "helm_max_abs_diff");
    double h = 0.0;
    check_cuda(cudaMemcpy(&h, d, sizeof(double), cudaMemcpyDeviceToHost), "cudaMemcpy");
    cudaFree(d);
    return h;
}

}  // namespace shim
