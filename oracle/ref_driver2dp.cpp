// Test infrastructure (oracle), never shipped: a C entry point around the
// reference's own 2D solver that is periodic in the GLL direction
// (Periodic2D_MPI.cpp, compiled unchanged by oracle/Makefile).
//
// Follows the reference's test driver TestPeriodic2D_MPI.cpp:71-89:
// CreatePDEPlan -> CreateFFTPlan -> fill rhsPDE -> SolvePDE with the
// shifted-Laplacian ConstructOperator (TestPeriodic2D_MPI.cpp:44-51) -> read U.
#include "Periodic2D_MPI.h"
#include <chrono>

static void oracle_construct_operator_2dp(const int iw)
{
    for (int i = 0; i < N - 2; ++i)
        for (int j = 0; j < N - 2; ++j)
            Operator[i][j] = Dyy[i + 1][j + 1] - (i == j ? (Lambda + 4.0 * PI * PI * iw * iw / (Lx * Lx)) : 0.0);
    LUDecomposition(Operator, npivot, determinant, N - 2);
}

// f, u: [Ns][Nx][N] (row-major, GLL index fastest); ygrid: Ns*(N-1)+1 nodes.
extern "C" int oracle_ref2dp_solve(int nx, int ny, int n, double xl_, double xr_, double yl_, double yr_,
                                   double lam, const double* f, double* u, double* ygrid, double* solve_ms)
{
    Rank = 0;
    size = 1;
    CreatePDEPlan(nx, ny, n, xl_, xr_, yl_, yr_);
    CreateFFTPlan(Nx);
    Lambda = lam;

    FieldVariable* V = new FieldVariable[Ns];
    for (int jj = 0; jj < Ns; ++jj) Allocate(V[jj].phi, NX, N);
    for (int jj = 0; jj < Ns; ++jj)
        for (int i = 0; i < Nx; ++i)
            for (int j = 0; j < N; ++j)
                rhsPDE[jj][i][j] = f[((size_t)jj * Nx + i) * N + j];

    auto t0 = std::chrono::steady_clock::now();
    SolvePDE(V, oracle_construct_operator_2dp);
    auto t1 = std::chrono::steady_clock::now();
    if (solve_ms) *solve_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();

    for (int jj = 0; jj < Ns; ++jj)
        for (int i = 0; i < Nx; ++i)
            for (int j = 0; j < N; ++j)
                u[((size_t)jj * Nx + i) * N + j] = V[jj].phi[i][j];
    if (ygrid)
        for (int j = 0; j < Ns * (N - 1) + 1; ++j) ygrid[j] = y[j];

    int ns = Ns;
    for (int jj = 0; jj < Ns; ++jj) Deallocate(V[jj].phi, NX, N);
    delete[] V;
    DestroyFFTPlan(Nx);
    DestroyPDEPlan();
    return ns;
}
