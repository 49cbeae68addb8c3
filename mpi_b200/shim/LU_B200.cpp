// LUDecomposition / LUSolve of the reference's LU_Decomposition.h, over the
// library's FP64 LU with scaled partial pivoting (helm_lu_factor /
// helm_lu_solve).  Both come from here, so the factor storage only has to
// agree between the two: P A = L U with whole rows swapped, npivot[i] the
// original row of position i (the reference keeps its own in-place
// convention; callers only hand the factors back to LUSolve).
//
// LUDecomposition also records the matrix it receives before factoring it:
// the reference's ConstructOperator callbacks fill the global Operator and
// call LUDecomposition on it (TestNonPeriodic2D_MPI.cpp:67-74), so the shims'
// SolvePDE reads each wavenumber's operator from here.
#include <cstring>
#include <vector>

#include "LU_Decomposition.h"
#include "shim_common.hpp"

namespace shim {

static std::vector<double> g_captured;
static int g_captured_n = 0;

bool take_captured(double* dst, int n)
{
    if (g_captured_n != n) return false;
    std::memcpy(dst, g_captured.data(), (size_t)n * n * sizeof(double));
    return true;
}

void clear_captured() { g_captured_n = 0; }

}  // namespace shim

void LUDecomposition(double**& A, int*& npivot, double& determinant, const int N)
{
    std::vector<double> a((size_t)N * N);
    for (int i = 0; i < N; ++i) std::memcpy(&a[(size_t)i * N], A[i], N * sizeof(double));
    shim::g_captured = a;
    shim::g_captured_n = N;
    shim::check(helm_lu_factor(N, a.data(), npivot, &determinant), "LUDecomposition");
    for (int i = 0; i < N; ++i) std::memcpy(A[i], &a[(size_t)i * N], N * sizeof(double));
}

void LUSolve(double** A, int* npivot, double*& b, const int N)
{
    std::vector<double> a((size_t)N * N);
    for (int i = 0; i < N; ++i) std::memcpy(&a[(size_t)i * N], A[i], N * sizeof(double));
    shim::check(helm_lu_solve(N, a.data(), npivot, b), "LUSolve");
}
