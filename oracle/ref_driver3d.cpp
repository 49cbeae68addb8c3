// Test infrastructure (oracle), never shipped: a C entry point around the
// reference's own 3D Fourier x Fourier x GLL solver.  The reference sources are
// compiled unchanged from HelmholtzSolvers/DirectPseudoSpectral/src by oracle/Makefile.
//
// Follows TestNonPeriodic3D_MPI.cpp:84-160 with the ConstructOperator of
// TestNonPeriodic3D_MPI.cpp:71-79.
#include "NonPeriodic3D_MPI.h"
#include <chrono>
#include <vector>

// Extra diagonal of a user operator (empty: the stock operator); see
// oracle_ref2d_set_cdiag.
static std::vector<double> g_cdiag;

extern "C" void oracle_ref3d_set_cdiag(const double* c, int n) { g_cdiag.assign(c, c + (c ? n : 0)); }

static void oracle_construct_operator_3d(const int iw, const int jw)
{
    for (int i = 0; i < N - 2; ++i)
        for (int j = 0; j < N - 2; ++j)
            Operator[i][j] = Dzz[i + 1][j + 1] -
                (i == j ? (Lambda + 4.0 * PI * PI * iw * iw / (Lx * Lx) + 4.0 * PI * PI * jw * jw / (Ly * Ly)) : 0.0);
    if (!g_cdiag.empty())
        for (int i = 0; i < N - 2; ++i) Operator[i][i] -= g_cdiag[i];
    LUDecomposition(Operator, npivot, determinant, N - 2);
}

// f, u: [Ns][Nx][Ny][N] (GLL index fastest); gl, gr: [Nx][Ny]; zgrid: Ns*(N-1)+1.
extern "C" int oracle_ref3d_solve(int nx, int ny, int nz, int n,
                                  double xl_, double xr_, double yl_, double yr_, double zl_, double zr_,
                                  double al, double bl, double ar, double br_, double lam,
                                  const double* f, const double* gl, const double* gr,
                                  double* u, double* zgrid, double* solve_ms)
{
    Rank = 0;
    size = 1;
    CreatePDEPlan(nx, ny, nz, n, xl_, xr_, yl_, yr_, zl_, zr_);
    CreateFFTPlan(Nx > Ny ? Nx : Ny);
    alphal = al; betal = bl; alphar = ar; betar = br_; Lambda = lam;

    FieldVariable* V = new FieldVariable[Ns];
    for (int kk = 0; kk < Ns; ++kk) Allocate(V[kk].phi, 2 * Nx, NY, N);

    for (int kk = 0; kk < Ns; ++kk)
        for (int i = 0; i < Nx; ++i)
            for (int j = 0; j < Ny; ++j)
                for (int k = 0; k < N; ++k)
                    rhsPDE[kk][i][j][k] = f[(((size_t)kk * Nx + i) * Ny + j) * N + k];
    for (int i = 0; i < Nx; ++i)
        for (int j = 0; j < Ny; ++j) {
            leftBC[i][j] = gl[(size_t)i * Ny + j];
            rightBC[i][j] = gr[(size_t)i * Ny + j];
        }

    auto t0 = std::chrono::steady_clock::now();
    SolvePDE(V, oracle_construct_operator_3d);
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

// The reference's GLL derivative of a 3D field, FirstDerivativeZ / SecondDerivativeZ
// (NonPeriodic3D_MPI.cpp:632-683).  u, du: [Ns][Nx][Ny][N].
extern "C" int oracle_ref3d_deriv_z(int nx, int ny, int nz, int n, double zl_, double zr_, int order,
                                    const double* u, double* du)
{
    Rank = 0;
    size = 1;
    CreatePDEPlan(nx, ny, nz, n, 0.0, 1.0, 0.0, 1.0, zl_, zr_);
    FieldVariable* V = new FieldVariable[Ns];
    FieldVariable* W = new FieldVariable[Ns];
    for (int kk = 0; kk < Ns; ++kk) { Allocate(V[kk].phi, 2 * Nx, NY, N); Allocate(W[kk].phi, 2 * Nx, NY, N); }
    for (int kk = 0; kk < Ns; ++kk)
        for (int i = 0; i < Nx; ++i)
            for (int j = 0; j < Ny; ++j)
                for (int k = 0; k < N; ++k) V[kk].phi[i][j][k] = u[(((size_t)kk * Nx + i) * Ny + j) * N + k];
    if (order == 1) FirstDerivativeZ(W, V); else SecondDerivativeZ(W, V);
    for (int kk = 0; kk < Ns; ++kk)
        for (int i = 0; i < Nx; ++i)
            for (int j = 0; j < Ny; ++j)
                for (int k = 0; k < N; ++k) du[(((size_t)kk * Nx + i) * Ny + j) * N + k] = W[kk].phi[i][j][k];
    int ns = Ns;
    for (int kk = 0; kk < Ns; ++kk) { Deallocate(V[kk].phi, 2 * Nx, NY, N); Deallocate(W[kk].phi, 2 * Nx, NY, N); }
    delete[] V;
    delete[] W;
    DestroyPDEPlan();
    return ns;
}

// The reference's spectral derivatives of a real [n0][n1][n2] array along x or y
// (Fourier_Quadrature.cpp:1494-1575, 1721-1800).
extern "C" void oracle_ref_fourier_deriv_3d(int n0, int n1, int n2, int axis, int order, double L, const double* u,
                                            double* du)
{
    CreateFFTPlan(n0 > n1 ? n0 : n1);
    double ***F, ***G;
    Allocate(F, n0, n1, n2);
    Allocate(G, n0, n1, n2);
    for (int i = 0; i < n0; ++i)
        for (int j = 0; j < n1; ++j)
            for (int k = 0; k < n2; ++k) F[i][j][k] = u[((size_t)i * n1 + j) * n2 + k];
    if (axis == 0) {
        if (order == 1) FirstDerivativeFourierX(G, F, n0, n1, n2, L); else SecondDerivativeFourierX(G, F, n0, n1, n2, L);
    } else {
        if (order == 1) FirstDerivativeFourierY(G, F, n0, n1, n2, L); else SecondDerivativeFourierY(G, F, n0, n1, n2, L);
    }
    for (int i = 0; i < n0; ++i)
        for (int j = 0; j < n1; ++j)
            for (int k = 0; k < n2; ++k) du[((size_t)i * n1 + j) * n2 + k] = G[i][j][k];
    Deallocate(F, n0, n1, n2);
    Deallocate(G, n0, n1, n2);
    DestroyFFTPlan(n0 > n1 ? n0 : n1);
}

// The reference's WriteFile (NonPeriodic3D_MPI.cpp:713-741, TECPLOT branch) of u
// [Ns][Nx][Ny][N] with exact(x, y, z) = sin(x) cos(y) z; writes
// Output/Solution-0000.tec under the current directory.
static double oracle_exact_3d(const double x, const double y, const double zz) { return sin(x) * cos(y) * zz; }
extern "C" int oracle_ref3d_write(int nx, int ny, int nz, int n, double xl_, double xr_, double yl_, double yr_,
                                  double zl_, double zr_, const double* u)
{
    Rank = 0;
    size = 1;
    CreatePDEPlan(nx, ny, nz, n, xl_, xr_, yl_, yr_, zl_, zr_);
    FieldVariable* V = new FieldVariable[Ns];
    for (int kk = 0; kk < Ns; ++kk) Allocate(V[kk].phi, 2 * Nx, NY, N);
    for (int kk = 0; kk < Ns; ++kk)
        for (int i = 0; i < Nx; ++i)
            for (int j = 0; j < Ny; ++j)
                for (int k = 0; k < N; ++k) V[kk].phi[i][j][k] = u[(((size_t)kk * Nx + i) * Ny + j) * N + k];
    WriteFile(V, oracle_exact_3d);
    int ns = Ns;
    for (int kk = 0; kk < Ns; ++kk) Deallocate(V[kk].phi, 2 * Nx, NY, N);
    delete[] V;
    DestroyPDEPlan();
    return ns;
}
