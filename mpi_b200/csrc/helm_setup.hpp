// Host-side FP64 setup of a Helmholtz plan: GLL nodes and derivative matrices,
// the shifted interior operators and their LU factors, the homogeneous
// solutions, the eigen-decomposition of the interior GLL operator, and the
// grouping of Fourier rows by shift.  Pure C++ (no CUDA).
#pragma once
#include <cstdint>
#include <vector>

namespace helm {

// N Gauss-Lobatto-Legendre nodes on [-1,1], ascending: the end points and the
// roots of P'_{N-1} (the nodes of GaussLobattoLegendrePoints,
// GLLQuadrature.cpp:78-128).  Newton iteration in long double.
void gll_nodes(int N, double* x);

// First-derivative collocation matrix on the GLL nodes, row-major N x N
// (FirstDerivativeMatrix, GLLQuadrature.cpp:198-213).
void gll_derivative(int N, const double* x, double* D);

// C = A B, N x N row-major.
void matmul(int N, const double* A, const double* B, double* C);

// LU with scaled partial pivoting on an n x n row-major matrix, pivot choice
// as in LUDecomposition (LU_Decomposition.cpp:7-72): row scales are the row
// max-abs of the input and stay with their row positions.  Unlike the
// reference's storage, whole rows (multipliers included) are swapped, so on
// return A holds L (unit, strictly lower) and U of P A = L U, and perm[i] is the
// original row of position i.  Returns false when a scaled pivot is <= 1e-12.
bool lu_factor(int n, double* A, int* perm);

// Solves (P A) x = P b with the factors of lu_factor, b overwritten by x.
void lu_solve(int n, const double* LU, const int* perm, double* b);

// Eigen-decomposition A = V diag(lam) V^-1 of a real n x n matrix whose
// eigenvalues are real and distinct (the interior GLL second-derivative
// operator).  Hessenberg reduction + shifted QR for the eigenvalues, inverse
// iteration for the eigenvectors, LU for V^-1; long double throughout.
// Returns false if it does not converge or the residual check fails.
bool real_eigen(int n, const double* A, double* lam, double* V, double* Vinv);

// The orthogonal even/odd fold of the n interior GLL nodes and the
// eigen-decompositions of the two blocks it makes of a centrosymmetric n x n
// operator A0 (the interior GLL second derivative): Q A0 Q^T = diag(Ms, Ma),
// Ms = Vs diag(ls) Vs^-1 (ms = ceil(n/2)), Ma = Va diag(la) Va^-1 (ma = n/2).
// Row k < m of Q is (e_k + e_{n-1-k}) / sqrt 2, row ms + k is
// (e_k - e_{n-1-k}) / sqrt 2, and row m is e_m when n is odd.
struct FoldedEigen {
    int n = 0, m = 0, ms = 0, ma = 0;
    std::vector<double> Q, Ms, Ma, ls, Vs, Vsi, la, Va, Vai;
};
// False when A0 is not centrosymmetric to rounding or a decomposition fails.
bool fold_eigen(int n, const std::vector<double>& A0, FoldedEigen& fe);

// Grid and operators of one plan, FP64, built by build_gll_setup.
struct GllSetup {
    int N = 0, Ns = 1;
    double L = 0;                 // extent of the GLL direction
    std::vector<double> nodes;    // Ns*(N-1)+1, placed from 0
    std::vector<double> D, D2;    // N*N scaled by 2Ns/L and 4Ns^2/L^2
};
GllSetup build_gll_setup(int N, int Ns, double L);

}  // namespace helm
