// Test infrastructure (oracle), never shipped: a C entry point around the
// reference's own finite-difference 3D Helmholtz solver
// (HelmholtzSolvers/HypreFDM/src/Helmholtz3D_MPI.cpp), compiled unchanged by
// oracle/Makefile against the single-rank MPI stub (oracle/ref_stub) and the
// in-memory HYPRE IJ stub (oracle/ref_stub_hypre).
//
// Follows TestHelmholtz3D_MPI.cpp:119-182: CreatePDEPlan, Robin coefficients
// and lambda as globals, rhsPDE / backBC / frontBC filled, SolvePDE(V).  The
// reference's SetA and Setb (Helmholtz3D_MPI.cpp:296-492) assemble the
// 7-point operator and the Robin rows exactly as they do for HYPRE; only the
// Krylov solve (HypreSolvers.cpp, tolerance 1e-10) is replaced here by a direct
// solve of that assembled system, so the result is the reference
// discretisation's exact solution.  x and y are periodic (Nx, Ny points,
// dx = Lx/Nx), z has Robin ends (back at zl, front at zr) and nz interior
// points, i.e. nz + 2 reference points with dz = Lz/(nz + 1).
#include "Helmholtz3D_MPI.h"

#include <cmath>
#include <vector>

// Adjoint mode: HypreSolve solves A^T x = g_adj_rhs instead (the right-hand
// side assembled by Setb is ignored) and leaves x in g_adj_out.
static bool g_adjoint = false;
static std::vector<double> g_adj_rhs, g_adj_out;

// Dense LU with partial pivoting of the captured rows (of A, or of A^T in
// adjoint mode); solution into x.
void HypreSolve(HYPRE_ParCSRMatrix A, HYPRE_ParVector b, HYPRE_ParVector x, int& iterations, double& residual,
                const int, const double, const int, const bool)
{
    const int n = A->hi - A->lo + 1;
    std::vector<double> M((size_t)n * n, 0.0), r(g_adjoint ? g_adj_rhs : b->v);
    for (int i = 0; i < n; ++i)
        for (const auto& kv : A->rows[i]) {
            const int j = kv.first - A->lo;
            M[g_adjoint ? (size_t)j * n + i : (size_t)i * n + j] = kv.second;
        }
    std::vector<int> perm(n);
    for (int i = 0; i < n; ++i) perm[i] = i;
    for (int c = 0; c < n; ++c) {
        int p = c;
        for (int i = c + 1; i < n; ++i)
            if (std::fabs(M[(size_t)i * n + c]) > std::fabs(M[(size_t)p * n + c])) p = i;
        if (p != c) {
            for (int j = 0; j < n; ++j) std::swap(M[(size_t)c * n + j], M[(size_t)p * n + j]);
            std::swap(r[c], r[p]);
        }
        const double d = M[(size_t)c * n + c];
        for (int i = c + 1; i < n; ++i) {
            const double l = M[(size_t)i * n + c] / d;
            if (l == 0.0) continue;
            for (int j = c; j < n; ++j) M[(size_t)i * n + j] -= l * M[(size_t)c * n + j];
            r[i] -= l * r[c];
        }
    }
    for (int i = n - 1; i >= 0; --i) {
        double s = r[i];
        for (int j = i + 1; j < n; ++j) s -= M[(size_t)i * n + j] * x->v[j];
        x->v[i] = s / M[(size_t)i * n + i];
    }
    if (g_adjoint) g_adj_out = x->v;
    iterations = 0;
    residual = 0.0;
}

// f: [nx][ny][nz] interior right-hand side (z fastest); gback, gfront: [nx][ny]
// Robin data at zl and zr; u: [nx][ny][nz] the interior solution.
extern "C" int oracle_ref_fd3d_solve(int nx, int ny, int nz, double xl_, double xr_, double yl_, double yr_,
                                     double zl_, double zr_, double ab, double bb, double af, double bf, double lam,
                                     const double* f, const double* gback, const double* gfront, double* u)
{
    Rank = 0;
    size = 1;
    CreatePDEPlan(nx, ny, nz + 2, xl_, xr_, yl_, yr_, zl_, zr_, false, true, true);
    alphaback = ab;
    betaback = bb;
    alphaf = af;
    betaf = bf;
    Lambda = lam;
    double*** V;
    Allocate(V, Nx + 2 * offset, Ny + 2 * offset, Nz + 2 * offset, offset, offset, offset);
    for (int i = 0; i < Nx; ++i)
        for (int j = 0; j < Ny; ++j) {
            backBC[i][j] = gback[(size_t)i * ny + j];
            frontBC[i][j] = gfront[(size_t)i * ny + j];
            for (int k = 0; k < Nz; ++k) {
                V[i][j][k] = 0.0;
                rhsPDE[i][j][k] = (k >= 1 && k <= nz) ? f[((size_t)i * ny + j) * nz + (k - 1)] : 0.0;
            }
        }
    SolvePDE(V);
    for (int i = 0; i < Nx; ++i)
        for (int j = 0; j < Ny; ++j)
            for (int k = 0; k < nz; ++k) u[((size_t)i * ny + j) * nz + k] = V[i][j][k + 1];
    Deallocate(V, Nx + 2 * offset, Ny + 2 * offset, Nz + 2 * offset, offset, offset, offset);
    DestroyPDEPlan();
    return 0;
}

// The transpose of the same map (f, gback, gfront) -> u: for a cotangent ubar
// of the interior solution, fbar = (A^-T P^T ubar) at the interior rows and
// gbback / gbfront at the Robin rows (A: the reference's assembled system,
// P: the interior points).  Same arguments and layouts as the forward entry.
extern "C" int oracle_ref_fd3d_adjoint(int nx, int ny, int nz, double xl_, double xr_, double yl_, double yr_,
                                       double zl_, double zr_, double ab, double bb, double af, double bf, double lam,
                                       const double* ubar, double* fbar, double* gbback, double* gbfront)
{
    const int nzr = nz + 2;
    // global index of the reference: k Nx Ny + j Nx + i (one rank)
    g_adj_rhs.assign((size_t)nx * ny * nzr, 0.0);
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k)
                g_adj_rhs[(size_t)(k + 1) * nx * ny + (size_t)j * nx + i] = ubar[((size_t)i * ny + j) * nz + k];
    std::vector<double> zf((size_t)nx * ny * nz, 0.0), zb((size_t)nx * ny, 0.0), zu((size_t)nx * ny * nz);
    g_adjoint = true;
    oracle_ref_fd3d_solve(nx, ny, nz, xl_, xr_, yl_, yr_, zl_, zr_, ab, bb, af, bf, lam, zf.data(), zb.data(),
                          zb.data(), zu.data());
    g_adjoint = false;
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j) {
            gbback[(size_t)i * ny + j] = g_adj_out[(size_t)j * nx + i];
            gbfront[(size_t)i * ny + j] = g_adj_out[(size_t)(nzr - 1) * nx * ny + (size_t)j * nx + i];
            for (int k = 0; k < nz; ++k)
                fbar[((size_t)i * ny + j) * nz + k] = g_adj_out[(size_t)(k + 1) * nx * ny + (size_t)j * nx + i];
        }
    return 0;
}
