// Test-only C entry points over the product's host setup (helm_setup.cpp), so
// the CPU tests can check the FP64 setup math without a GPU.
#include "../mpi_b200/csrc/helm_setup.hpp"
#include <cstring>
extern "C" {
void t_gll_setup(int N, int Ns, double L, double* nodes, double* D, double* D2)
{
    helm::GllSetup s = helm::build_gll_setup(N, Ns, L);
    std::memcpy(nodes, s.nodes.data(), s.nodes.size() * sizeof(double));
    std::memcpy(D, s.D.data(), s.D.size() * sizeof(double));
    std::memcpy(D2, s.D2.data(), s.D2.size() * sizeof(double));
}
int t_lu(int n, double* A, int* perm, double* b)
{
    if (!helm::lu_factor(n, A, perm)) return 1;
    helm::lu_solve(n, A, perm, b);
    return 0;
}
int t_eig(int n, const double* A, double* lam, double* V, double* Vi) { return helm::real_eigen(n, A, lam, V, Vi) ? 0 : 1; }
}
