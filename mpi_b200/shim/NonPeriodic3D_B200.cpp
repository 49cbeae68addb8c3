// Drop-in replacement of the reference's 3D Fourier x Fourier x GLL solver
// (HelmholtzSolvers/DirectPseudoSpectral/src/NonPeriodic3D_MPI.cpp): the globals
// and entry points of include/NonPeriodic3D_MPI.h:21-51 over libhelm_b200, so
// the reference's TestNonPeriodic3D_MPI.cpp links against this file unchanged
// and solves on the GPU.  The same behaviour and differences as the 2D shim
// (NonPeriodic2D_B200.cpp): single rank; rhsPDE[Ns][2Nx][2Ny][N] and
// leftBC / rightBC[2Nx][2Ny] are read, not overwritten; ConstructOperator(iw,
// jw) runs for iw = 0 .. Nx/2, jw = 0 .. Ny/2 (NonPeriodic3D_MPI.cpp:248-253).
#include <cmath>
#include <cstring>
#include <iostream>
#include <vector>

#include "NonPeriodic3D_MPI.h"
#include "shim_common.hpp"

int Rank, size;
int Nx, Ny, Nz, NY, N, Ns;
double xl, xr, yl, yr, zl, zr, Lx, Ly, Lz, dx, dy;
double alphal, betal, alphar, betar, Lambda;
double **Dz, **Dzz, **Operator, *z, ****rhsPDE, **leftBC, **rightBC, determinant;
int* npivot;

namespace {

helm_plan_t g_plan = nullptr;
double g_key[5];
shim::OperatorSet g_ops;
shim::DeviceBuf g_f, g_u, g_gl, g_gr, g_a, g_b;

// elements of one U[kk].phi / rhsPDE[kk] block: [2Nx][2Ny][N]
size_t block() { return (size_t)2 * Nx * NY * N; }

void ensure_plan()
{
    const double key[5] = {alphal, betal, alphar, betar, Lambda};
    if (g_plan && std::memcmp(key, g_key, sizeof(key)) == 0) return;
    if (g_plan) helm_plan_destroy(g_plan);
    g_plan = nullptr;
    g_ops = shim::OperatorSet();
    const helm_robin_t bc{alphal, betal, alphar, betar};
    shim::check(helm3d_plan_create(Nx, Ny, Nz, N, xl, xr, yl, yr, zl, zr, &bc, Lambda, HELM_FP64, HELM_METHOD_LU,
                                   &g_plan),
                "CreatePDEPlan");
    // the reference's arrays: x rows of 2Ny * N, elements 2Nx * 2Ny * N apart,
    // boundary data rows of 2Ny
    shim::check(helm_plan_set_layout(g_plan, (long long)NY * N, (long long)block(), NY), "layout");
    std::memcpy(g_key, key, sizeof(key));
}

double* upload_field(FieldVariable U[], shim::DeviceBuf& buf)
{
    double* d = buf.get((size_t)Ns * block());
    for (int kk = 0; kk < Ns; ++kk)
        shim::check_cuda(cudaMemcpy(d + (size_t)kk * block(), U[kk].phi[0][0], block() * sizeof(double),
                                    cudaMemcpyHostToDevice),
                         "upload");
    return d;
}

// Copies x rows 0 .. rows-1 of each element's block back into U[kk].phi.
void download_field(const double* d, FieldVariable U[], int rows)
{
    for (int kk = 0; kk < Ns; ++kk)
        shim::check_cuda(cudaMemcpy(U[kk].phi[0][0], d + (size_t)kk * block(), (size_t)rows * NY * N * sizeof(double),
                                    cudaMemcpyDeviceToHost),
                         "download");
}

double (*g_exact)(const double, const double, const double) = nullptr;
double exact3(double x, double yy, double zz) { return g_exact(x, yy, zz); }

}  // namespace

void CreatePDEPlan(const int Nx_, const int Ny_, const int Nz_, const int N_, const double xl_, const double xr_,
                   const double yl_, const double yr_, const double zl_, const double zr_)
{
    ::Nx = Nx_;
    ::Ny = Ny_;
    ::Nz = Nz_;
    ::N = N_;
    ::xl = xl_;
    ::xr = xr_;
    ::yl = yl_;
    ::yr = yr_;
    ::zl = zl_;
    ::zr = zr_;
    NY = 2 * Ny;
    Lx = xr - xl;
    Ly = yr - yl;
    Lz = zr - zl;
    dx = Lx / Nx;
    dy = Ly / Ny;
    if (size < 1) size = 1;
    Ns = (int)std::ceil(((double)Nz) / (size * N));
    Allocate(z, Ns * (N - 1) + 1);
    Allocate(rhsPDE, Ns, 2 * Nx, NY, N);
    Allocate(leftBC, 2 * Nx, NY);
    Allocate(rightBC, 2 * Nx, NY);
    Allocate(Dz, N, N);
    Allocate(Dzz, N, N);
    Allocate(Operator, N - 2, N - 2);
    Allocate(npivot, N - 2);
    std::vector<double> D((size_t)N * N), D2((size_t)N * N);
    shim::check(helm_gll_grid(N, Ns, Lz, z, D.data(), D2.data()), "CreatePDEPlan");
    for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j) {
            Dz[i][j] = D[(size_t)i * N + j];
            Dzz[i][j] = D2[(size_t)i * N + j];
        }
}

void DestroyPDEPlan()
{
    if (g_plan) helm_plan_destroy(g_plan);
    g_plan = nullptr;
    g_ops = shim::OperatorSet();
    for (shim::DeviceBuf* b : {&g_f, &g_u, &g_gl, &g_gr, &g_a, &g_b}) b->release();
    Deallocate(z, Ns * (N - 1) + 1);
    Deallocate(rhsPDE, Ns, 2 * Nx, NY, N);
    Deallocate(leftBC, 2 * Nx, NY);
    Deallocate(rightBC, 2 * Nx, NY);
    Deallocate(Dz, N, N);
    Deallocate(Dzz, N, N);
    Deallocate(Operator, N - 2, N - 2);
    Deallocate(npivot, N - 2);
}

void CreateFFTPlan(const int) {}
void DestroyFFTPlan(const int) {}

void SolvePDE(FieldVariable U[], void (*ConstructOperator)(const int, const int))
{
    const int n = N - 2;
    shim::OperatorSet ops;
    ops.n = n;
    for (int iw = 0; iw <= Nx / 2; ++iw)
        for (int jw = 0; jw <= Ny / 2; ++jw) {
            shim::clear_captured();
            ConstructOperator(iw, jw);
            const size_t at = ops.ops.size();
            ops.ops.resize(at + (size_t)n * n);
            double* dst = &ops.ops[at];
            if (!shim::take_captured(dst, n))
                for (int i = 0; i < n; ++i) std::memcpy(dst + (size_t)i * n, Operator[i], n * sizeof(double));
            ops.iw.push_back(iw);
            ops.jw.push_back(jw);
        }
    ensure_plan();
    if (ops.ops != g_ops.ops) {
        g_ops = ops;
        shim::check(helm_plan_set_operator_callback(g_plan, shim::serve_operator, &g_ops), "SolvePDE");
    }
    const size_t cnt = (size_t)Ns * block();
    double* f = g_f.get(cnt);
    double* u = g_u.get(cnt);
    shim::check_cuda(cudaMemcpy(f, rhsPDE[0][0][0], cnt * sizeof(double), cudaMemcpyHostToDevice), "upload");
    shim::check_cuda(cudaMemset(u, 0, cnt * sizeof(double)), "memset");
    const size_t nb = (size_t)2 * Nx * NY;
    double* gl = g_gl.get(nb);
    double* gr = g_gr.get(nb);
    shim::check_cuda(cudaMemcpy(gl, leftBC[0], nb * sizeof(double), cudaMemcpyHostToDevice), "upload");
    shim::check_cuda(cudaMemcpy(gr, rightBC[0], nb * sizeof(double), cudaMemcpyHostToDevice), "upload");
    shim::check(helm_solve(g_plan, f, gl, gr, u, nullptr), "SolvePDE");
    download_field(u, U, 2 * Nx);
}

// x and y: the library's spectral derivatives (the reference's solver-level
// ones are empty stubs, NonPeriodic3D_MPI.cpp:598-630); z: the GLL derivative
// (NonPeriodic3D_MPI.cpp:632-683).
static void derivative(FieldVariable Ud[], FieldVariable U[], int axis, int order)
{
    ensure_plan();
    const double* a = upload_field(U, g_a);
    double* b = g_b.get((size_t)Ns * block());
    if (axis == 2)
        shim::check(helm_gll_derivative(g_plan, order, a, b, nullptr), "FirstDerivativeZ");
    else
        shim::check(helm_fourier_derivative(g_plan, axis, order, a, b, nullptr), "FirstDerivativeX");
    download_field(b, Ud, Nx);
}

void FirstDerivativeX(FieldVariable Ux[], FieldVariable U[]) { derivative(Ux, U, 0, 1); }
void SecondDerivativeX(FieldVariable Uxx[], FieldVariable U[]) { derivative(Uxx, U, 0, 2); }
void FirstDerivativeY(FieldVariable Uy[], FieldVariable U[]) { derivative(Uy, U, 1, 1); }
void SecondDerivativeY(FieldVariable Uyy[], FieldVariable U[]) { derivative(Uyy, U, 1, 2); }
void FirstDerivativeZ(FieldVariable Uz[], FieldVariable U[]) { derivative(Uz, U, 2, 1); }
void SecondDerivativeZ(FieldVariable Uzz[], FieldVariable U[]) { derivative(Uzz, U, 2, 2); }

// NonPeriodic3D_MPI.cpp:688-708 with the maximum taken on the device.
void ComputeError(FieldVariable U[], double (*ExactFunction)(const double, const double, const double))
{
    ensure_plan();
    const double* a = upload_field(U, g_a);
    std::vector<double> ex((size_t)Ns * block(), 0.0);
    for (int kk = 0; kk < Ns; ++kk)
        for (int i = 0; i < Nx; ++i)
            for (int j = 0; j < Ny; ++j)
                for (int k = 0; k < N; ++k)
                    ex[(size_t)kk * block() + ((size_t)i * NY + j) * N + k] =
                        ExactFunction((xl + i * dx), (yl + j * dy), z[kk * (N - 1) + k]);
    double* b = g_b.get(ex.size());
    shim::check_cuda(cudaMemcpy(b, ex.data(), ex.size() * sizeof(double), cudaMemcpyHostToDevice), "upload");
    const double Error = shim::max_abs_diff(g_plan, a, b);
    if (Rank == 0) std::cout << "Error = " << Error << std::endl << std::endl;
}

void WriteFile(FieldVariable U[], double (*ExactFunction)(const double, const double, const double))
{
    ensure_plan();
    std::vector<double> u((size_t)Ns * Nx * Ny * N);
    for (int kk = 0; kk < Ns; ++kk)
        for (int i = 0; i < Nx; ++i)
            for (int j = 0; j < Ny; ++j)
                std::memcpy(&u[(((size_t)kk * Nx + i) * Ny + j) * N], U[kk].phi[i][j], (size_t)N * sizeof(double));
    char path[64];
    std::snprintf(path, sizeof(path), "Output/Solution-%04d.tec", Rank);
    g_exact = ExactFunction;
    shim::check(helm_write_tecplot(g_plan, u.data(), exact3, path), "WriteFile");
}
