// Test infrastructure (oracle), never shipped: a C entry point around the
// reference's own 2D Fourier x GLL solver so the tests can run it on the same
// inputs as the CUDA path.  The reference sources are compiled unchanged from
// HelmholtzSolvers/DirectPseudoSpectral/src by oracle/Makefile.
//
// Follows the reference's test driver TestNonPeriodic2D_MPI.cpp:79-142:
// CreatePDEPlan -> CreateFFTPlan -> fill rhsPDE/leftBC/rightBC -> SolvePDE with the
// shifted-Laplacian ConstructOperator (TestNonPeriodic2D_MPI.cpp:67-74) -> read U.
#include "NonPeriodic2D_MPI.h"
#include <chrono>
#include <vector>

// Extra diagonal of a user operator (empty: the stock operator), set by
// oracle_ref2d_set_cdiag: the callback below then builds
// Dyy_int - diag(lambda + (2 pi iw / Lx)^2 + c_i), the kind of operator a
// caller's own ConstructOperator passes (a coefficient varying along y).
static std::vector<double> g_cdiag;

extern "C" void oracle_ref2d_set_cdiag(const double* c, int n) { g_cdiag.assign(c, c + (c ? n : 0)); }

// The operator the reference's tests pass to SolvePDE: Dyy on the interior
// nodes minus (lambda + (2 pi iw / Lx)^2) on the diagonal, LU-factored in place.
static void oracle_construct_operator_2d(const int iw)
{
    for (int i = 0; i < N - 2; ++i)
        for (int j = 0; j < N - 2; ++j)
            Operator[i][j] = Dyy[i + 1][j + 1] - (i == j ? (Lambda + 4.0 * PI * PI * iw * iw / (Lx * Lx)) : 0.0);
    if (!g_cdiag.empty())
        for (int i = 0; i < N - 2; ++i) Operator[i][i] -= g_cdiag[i];
    LUDecomposition(Operator, npivot, determinant, N - 2);
}

// f, u: [Ns][Nx][N] (row-major, GLL index fastest); gl, gr: [Nx];
// ygrid: Ns*(N-1)+1 node coordinates.  Ns = ceil(ny / n) as in CreatePDEPlan.
extern "C" int oracle_ref2d_solve(int nx, int ny, int n,
                                  double xl_, double xr_, double yl_, double yr_,
                                  double al, double bl, double ar, double br_, double lam,
                                  const double* f, const double* gl, const double* gr,
                                  double* u, double* ygrid, double* solve_ms)
{
    Rank = 0;
    size = 1;
    CreatePDEPlan(nx, ny, n, xl_, xr_, yl_, yr_);
    CreateFFTPlan(Nx);
    alphal = al; betal = bl; alphar = ar; betar = br_; Lambda = lam;

    FieldVariable* V = new FieldVariable[Ns];
    for (int jj = 0; jj < Ns; ++jj) Allocate(V[jj].phi, NX, N);

    for (int jj = 0; jj < Ns; ++jj)
        for (int i = 0; i < Nx; ++i)
            for (int j = 0; j < N; ++j)
                rhsPDE[jj][i][j] = f[((size_t)jj * Nx + i) * N + j];
    for (int i = 0; i < Nx; ++i) { leftBC[i] = gl[i]; rightBC[i] = gr[i]; }

    auto t0 = std::chrono::steady_clock::now();
    SolvePDE(V, oracle_construct_operator_2d);
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

// The reference's GLL derivative of a 2D field, FirstDerivativeY / SecondDerivativeY
// (NonPeriodic2D_MPI.cpp:497-542) on the plan's grid.  u, du: [Ns][Nx][N].
extern "C" int oracle_ref2d_deriv_y(int nx, int ny, int n, double yl_, double yr_, int order, const double* u,
                                    double* du)
{
    Rank = 0;
    size = 1;
    CreatePDEPlan(nx, ny, n, 0.0, 1.0, yl_, yr_);
    FieldVariable* V = new FieldVariable[Ns];
    FieldVariable* W = new FieldVariable[Ns];
    for (int jj = 0; jj < Ns; ++jj) { Allocate(V[jj].phi, NX, N); Allocate(W[jj].phi, NX, N); }
    for (int jj = 0; jj < Ns; ++jj)
        for (int i = 0; i < Nx; ++i)
            for (int j = 0; j < N; ++j) V[jj].phi[i][j] = u[((size_t)jj * Nx + i) * N + j];
    if (order == 1) FirstDerivativeY(W, V); else SecondDerivativeY(W, V);
    for (int jj = 0; jj < Ns; ++jj)
        for (int i = 0; i < Nx; ++i)
            for (int j = 0; j < N; ++j) du[((size_t)jj * Nx + i) * N + j] = W[jj].phi[i][j];
    int ns = Ns;
    for (int jj = 0; jj < Ns; ++jj) { Deallocate(V[jj].phi, NX, N); Deallocate(W[jj].phi, NX, N); }
    delete[] V;
    delete[] W;
    DestroyPDEPlan();
    return ns;
}

// The reference's spectral derivatives of a real [n0][n1] array
// (FirstDerivativeFourierX / Y, SecondDerivativeFourierX / Y, Fourier_Quadrature.cpp:1420-1716).
extern "C" void oracle_ref_fourier_deriv_2d(int n0, int n1, int axis, int order, double L, const double* u, double* du)
{
    CreateFFTPlan(n0 > n1 ? n0 : n1);
    double **F, **G;
    Allocate(F, n0, n1);
    Allocate(G, n0, n1);
    for (int i = 0; i < n0; ++i)
        for (int j = 0; j < n1; ++j) F[i][j] = u[(size_t)i * n1 + j];
    if (axis == 0) {
        if (order == 1) FirstDerivativeFourierX(G, F, n0, n1, L); else SecondDerivativeFourierX(G, F, n0, n1, L);
    } else {
        if (order == 1) FirstDerivativeFourierY(G, F, n0, n1, L); else SecondDerivativeFourierY(G, F, n0, n1, L);
    }
    for (int i = 0; i < n0; ++i)
        for (int j = 0; j < n1; ++j) du[(size_t)i * n1 + j] = G[i][j];
    Deallocate(F, n0, n1);
    Deallocate(G, n0, n1);
    DestroyFFTPlan(n0 > n1 ? n0 : n1);
}

// The reference's WriteFile (NonPeriodic2D_MPI.cpp:571-598, TECPLOT branch) of u
// [Ns][Nx][N] with exact(x, y) = sin(x) cos(y); writes Output/Solution-0000.tec
// under the current directory.
static double oracle_exact_2d(const double x, const double y) { return sin(x) * cos(y); }
extern "C" int oracle_ref2d_write(int nx, int ny, int n, double xl_, double xr_, double yl_, double yr_,
                                  const double* u)
{
    Rank = 0;
    size = 1;
    CreatePDEPlan(nx, ny, n, xl_, xr_, yl_, yr_);
    FieldVariable* V = new FieldVariable[Ns];
    for (int jj = 0; jj < Ns; ++jj) Allocate(V[jj].phi, NX, N);
    for (int jj = 0; jj < Ns; ++jj)
        for (int i = 0; i < Nx; ++i)
            for (int j = 0; j < N; ++j) V[jj].phi[i][j] = u[((size_t)jj * Nx + i) * N + j];
    WriteFile(V, oracle_exact_2d);
    int ns = Ns;
    for (int jj = 0; jj < Ns; ++jj) Deallocate(V[jj].phi, NX, N);
    delete[] V;
    DestroyPDEPlan();
    return ns;
}
