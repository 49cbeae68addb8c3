// Drop-in replacement of the reference's 2D Fourier x GLL solver
// (HelmholtzSolvers/DirectPseudoSpectral/src/NonPeriodic2D_MPI.cpp): the globals
// and entry points its header declares (include/NonPeriodic2D_MPI.h:21-47),
// re-implemented over libhelm_b200, so a program written against that header
// -- the reference's own TestNonPeriodic2D_MPI.cpp, unchanged -- links against
// this file instead of the reference's solver and solves on the GPU.
//
// Behaviour kept: the globals CreatePDEPlan sets and allocates (grid y, the
// scaled Dy / Dyy, rhsPDE[Ns][2Nx][N], leftBC / rightBC[2Nx], Operator,
// npivot), SolvePDE calling ConstructOperator(iw) for iw = 0 .. Nx/2 and
// solving with those operators, the solution's real part in U[jj].phi[i < Nx],
// ComputeError's "Error = " line and WriteFile's Output/Solution-%04d.tec.
// Differences: single rank (the reference's rank chain along y is not
// reproduced); SolvePDE leaves rhsPDE / leftBC / rightBC as the caller filled
// them (the reference overwrites them with their transforms,
// NonPeriodic2D_MPI.cpp:233-236); CreateFFTPlan / DestroyFFTPlan do nothing
// (the library's plans carry their own twiddles).  Errors print the library's
// message and exit(1), as the reference's ErrorMessage does.
#include <cmath>
#include <cstring>
#include <iostream>
#include <vector>

#include "NonPeriodic2D_MPI.h"
#include "shim_common.hpp"

int Rank, size;
int Nx, Ny, NX, N, Ns;
double xl, xr, yl, yr, Lx, Ly, dx;
double alphal, betal, alphar, betar, Lambda;
double **Dy, **Dyy, **Operator, *y, ***rhsPDE, *leftBC, *rightBC, determinant;
int* npivot;

namespace {

helm_plan_t g_plan = nullptr;
double g_key[5];              // alphal, betal, alphar, betar, Lambda of g_plan
shim::OperatorSet g_ops;      // the operators g_plan solves with
shim::DeviceBuf g_f, g_u, g_gl, g_gr, g_a, g_b;

// The plan for the current globals, created (or re-created) when they changed.
void ensure_plan()
{
    const double key[5] = {alphal, betal, alphar, betar, Lambda};
    if (g_plan && std::memcmp(key, g_key, sizeof(key)) == 0) return;
    if (g_plan) helm_plan_destroy(g_plan);
    g_plan = nullptr;
    g_ops = shim::OperatorSet();
    const helm_robin_t bc{alphal, betal, alphar, betar};
    shim::check(helm2d_plan_create(Nx, Ny, N, xl, xr, yl, yr, &bc, Lambda, HELM_FP64, HELM_METHOD_LU, &g_plan),
                "CreatePDEPlan");
    // the reference's arrays: rows of 2Nx, N per row, elements NX * N apart
    shim::check(helm_plan_set_layout(g_plan, N, (long long)NX * N, 0), "layout");
    std::memcpy(g_key, key, sizeof(key));
}

// Copies the caller's U[jj].phi (NX x N each) into one device array.
double* upload_field(FieldVariable U[], shim::DeviceBuf& buf)
{
    double* d = buf.get((size_t)Ns * NX * N);
    for (int jj = 0; jj < Ns; ++jj)
        shim::check_cuda(cudaMemcpy(d + (size_t)jj * NX * N, U[jj].phi[0], (size_t)NX * N * sizeof(double),
                                    cudaMemcpyHostToDevice),
                         "upload");
    return d;
}

// Copies rows 0 .. rows-1 of each element's NX x N block back into U[jj].phi.
void download_field(const double* d, FieldVariable U[], int rows)
{
    for (int jj = 0; jj < Ns; ++jj)
        shim::check_cuda(cudaMemcpy(U[jj].phi[0], d + (size_t)jj * NX * N, (size_t)rows * N * sizeof(double),
                                    cudaMemcpyDeviceToHost),
                         "download");
}

double (*g_exact)(const double, const double) = nullptr;
double exact3(double x, double yy, double) { return g_exact(x, yy); }

}  // namespace

void CreatePDEPlan(const int Nx_, const int Ny_, const int N_, const double xl_, const double xr_, const double yl_,
                   const double yr_)
{
    ::Nx = Nx_;
    ::Ny = Ny_;
    ::N = N_;
    ::xl = xl_;
    ::xr = xr_;
    ::yl = yl_;
    ::yr = yr_;
    NX = 2 * Nx;
    Lx = xr - xl;
    Ly = yr - yl;
    dx = Lx / Nx;
    if (size < 1) size = 1;
    Ns = (int)std::ceil(((double)Ny) / (size * N));
    Allocate(y, Ns * (N - 1) + 1);
    Allocate(rhsPDE, Ns, NX, N);
    Allocate(leftBC, NX);
    Allocate(rightBC, NX);
    Allocate(Dy, N, N);
    Allocate(Dyy, N, N);
    Allocate(Operator, N - 2, N - 2);
    Allocate(npivot, N - 2);
    std::vector<double> D((size_t)N * N), D2((size_t)N * N);
    shim::check(helm_gll_grid(N, Ns, Ly, y, D.data(), D2.data()), "CreatePDEPlan");
    for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j) {
            Dy[i][j] = D[(size_t)i * N + j];
            Dyy[i][j] = D2[(size_t)i * N + j];
        }
}

void DestroyPDEPlan()
{
    if (g_plan) helm_plan_destroy(g_plan);
    g_plan = nullptr;
    g_ops = shim::OperatorSet();
    for (shim::DeviceBuf* b : {&g_f, &g_u, &g_gl, &g_gr, &g_a, &g_b}) b->release();
    Deallocate(y, Ns * (N - 1) + 1);
    Deallocate(rhsPDE, Ns, NX, N);
    Deallocate(leftBC, NX);
    Deallocate(rightBC, NX);
    Deallocate(Dy, N, N);
    Deallocate(Dyy, N, N);
    Deallocate(Operator, N - 2, N - 2);
    Deallocate(npivot, N - 2);
}

void CreateFFTPlan(const int) {}
void DestroyFFTPlan(const int) {}

void SolvePDE(FieldVariable U[], void (*ConstructOperator)(const int))
{
    // the caller's operators, one per |iw| (NonPeriodic2D_MPI.cpp:239-241)
    const int n = N - 2;
    shim::OperatorSet ops;
    ops.n = n;
    ops.ops.resize((size_t)(Nx / 2 + 1) * n * n);
    for (int iw = 0; iw <= Nx / 2; ++iw) {
        shim::clear_captured();
        ConstructOperator(iw);
        double* dst = &ops.ops[(size_t)iw * n * n];
        if (!shim::take_captured(dst, n))  // a callback that did not factor its Operator
            for (int i = 0; i < n; ++i) std::memcpy(dst + (size_t)i * n, Operator[i], n * sizeof(double));
        ops.iw.push_back(iw);
        ops.jw.push_back(0);
    }
    ensure_plan();
    if (ops.ops != g_ops.ops) {
        g_ops = ops;
        shim::check(helm_plan_set_operator_callback(g_plan, shim::serve_operator, &g_ops), "SolvePDE");
    }
    const size_t cnt = (size_t)Ns * NX * N;
    double* f = g_f.get(cnt);
    double* u = g_u.get(cnt);
    shim::check_cuda(cudaMemcpy(f, rhsPDE[0][0], cnt * sizeof(double), cudaMemcpyHostToDevice), "upload");
    shim::check_cuda(cudaMemset(u, 0, cnt * sizeof(double)), "memset");
    double* gl = g_gl.get(NX);
    double* gr = g_gr.get(NX);
    shim::check_cuda(cudaMemcpy(gl, leftBC, NX * sizeof(double), cudaMemcpyHostToDevice), "upload");
    shim::check_cuda(cudaMemcpy(gr, rightBC, NX * sizeof(double), cudaMemcpyHostToDevice), "upload");
    shim::check(helm_solve(g_plan, f, gl, gr, u, nullptr), "SolvePDE");
    // the real part in rows 0 .. Nx-1; rows Nx .. 2Nx-1, the reference's
    // imaginary parts of the inverse transform, are zero
    download_field(u, U, NX);
}

// The reference's solver-level x derivatives are empty stubs
// (NonPeriodic2D_MPI.cpp:479-495); here they are the spectral derivatives of
// the library (helm_fourier_derivative), the same as its FirstDerivativeFourierX.
static void x_derivative(FieldVariable Ux[], FieldVariable U[], int order)
{
    ensure_plan();
    const double* a = upload_field(U, g_a);
    double* b = g_b.get((size_t)Ns * NX * N);
    shim::check(helm_fourier_derivative(g_plan, 0, order, a, b, nullptr), "FirstDerivativeX");
    download_field(b, Ux, Nx);
}

static void y_derivative(FieldVariable Uy[], FieldVariable U[], int order)
{
    ensure_plan();
    const double* a = upload_field(U, g_a);
    double* b = g_b.get((size_t)Ns * NX * N);
    shim::check(helm_gll_derivative(g_plan, order, a, b, nullptr), "FirstDerivativeY");
    download_field(b, Uy, Nx);
}

void FirstDerivativeX(FieldVariable Ux[], FieldVariable U[]) { x_derivative(Ux, U, 1); }
void SecondDerivativeX(FieldVariable Uxx[], FieldVariable U[]) { x_derivative(Uxx, U, 2); }
void FirstDerivativeY(FieldVariable Uy[], FieldVariable U[]) { y_derivative(Uy, U, 1); }
void SecondDerivativeY(FieldVariable Uyy[], FieldVariable U[]) { y_derivative(Uyy, U, 2); }

// Maximum |U - exact| over the solution points (NonPeriodic2D_MPI.cpp:547-566),
// reduced on the device.
void ComputeError(FieldVariable U[], double (*ExactFunction)(const double, const double))
{
    ensure_plan();
    const double* a = upload_field(U, g_a);
    std::vector<double> ex((size_t)Ns * NX * N, 0.0);
    for (int jj = 0; jj < Ns; ++jj)
        for (int i = 0; i < Nx; ++i)
            for (int j = 0; j < N; ++j)
                ex[((size_t)jj * NX + i) * N + j] = ExactFunction((xl + i * dx), y[jj * (N - 1) + j]);
    double* b = g_b.get(ex.size());
    shim::check_cuda(cudaMemcpy(b, ex.data(), ex.size() * sizeof(double), cudaMemcpyHostToDevice), "upload");
    const double Error = shim::max_abs_diff(g_plan, a, b);
    if (Rank == 0) std::cout << "Error = " << Error << std::endl << std::endl;
}

// Tecplot file of the solution beside the exact function
// (NonPeriodic2D_MPI.cpp:571-600), written by helm_write_tecplot.
void WriteFile(FieldVariable U[], double (*ExactFunction)(const double, const double))
{
    ensure_plan();
    std::vector<double> u((size_t)Ns * Nx * N);
    for (int jj = 0; jj < Ns; ++jj)
        std::memcpy(&u[(size_t)jj * Nx * N], U[jj].phi[0], (size_t)Nx * N * sizeof(double));
    char path[64];
    std::snprintf(path, sizeof(path), "Output/Solution-%04d.tec", Rank);
    g_exact = ExactFunction;
    shim::check(helm_write_tecplot(g_plan, u.data(), exact3, path), "WriteFile");
}
