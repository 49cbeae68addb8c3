// Test infrastructure (oracle), never shipped: a C entry point around the
// reference's own 3D solver that is periodic in the GLL direction
// (Periodic3D_MPI.cpp, compiled unchanged by oracle/Makefile).
//
// Follows TestPeriodic3D_MPI.cpp:73-93 with the ConstructOperator of
// TestPeriodic3D_MPI.cpp:46-54.
#include "Periodic3D_MPI.h"
#include <chrono>

static void oracle_construct_operator_3dp(const int iw, const int jw)
{
    for (int i = 0; i < N - 2; ++i)
        for (int j = 0; j < N - 2; ++j)
            Operator[i][j] = Dzz[i + 1][j + 1] -
                (i == j ? (Lambda + 4.0 * PI * PI * iw * iw / (Lx * Lx) + 4.0 * PI * PI * jw * jw / (Ly * Ly)) : 0.0);
    LUDecomposition(Operator, npivot, determinant, N - 2);
}

// f, u: [Ns][Nx][Ny][N] (GLL index fastest); zgrid: Ns*(N-1)+1 nodes.
extern "C" int oracle_ref3dp_solve(int nx, int ny, int nz, int n, double xl_, double xr_, double yl_, double yr_,
                                   double zl_, double zr_, double lam, const double* f, double* u, double* zgrid,
                                   double* solve_ms)
{
    Rank = 0;
    size = 1;
    CreatePDEPlan(nx, ny, nz, n, xl_, xr_, yl_, yr_, zl_, zr_);
    CreateFFTPlan(Nx > Ny ? Nx : Ny);
    Lambda = lam;

    FieldVariable* V = new FieldVariable[Ns];
    for (int kk = 0; kk < Ns; ++kk) Allocate(V[kk].phi, 2 * Nx, NY, N);
    for (int kk = 0; kk < Ns; ++kk)
        for (int i = 0; i < Nx; ++i)
            for (int j = 0; j < Ny; ++j)
                for (int k = 0; k < N; ++k)
                    rhsPDE[kk][i][j][k] = f[(((size_t)kk * Nx + i) * Ny + j) * N + k];

    auto t0 = std::chrono::steady_clock::now();
    SolvePDE(V, oracle_construct_operator_3dp);
    auto t1 = std::chrono::steady_clock::now();
    if (solve_ms) *solve_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();

    for (int kk = 0; kk < Ns; ++kk)
        for (int i = 0; i < Nx; ++i)
            for (int j = 0; j < Ny; ++j)
                for (int k = 0; k < N; ++k)
                    u[(((size_t)kk * Nx + i) * Ny + j) * N + k] = V[kk].phi[i][j][k];
    if (zgrid)
        for (int k = 0; k < Ns * (N - 1) + 1; ++k) zgrid[k] = z[k];

    int ns = Ns;
    for (int kk = 0; kk < Ns; ++kk) Deallocate(V[kk].phi, 2 * Nx, NY, N);
    delete[] V;
    DestroyFFTPlan(Nx > Ny ? Nx : Ny);
    DestroyPDEPlan();
    return ns;
}
