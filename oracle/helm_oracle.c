/*
 * helm_oracle.c -- CPU restatement of the reference's DirectPseudoSpectral
 * Helmholtz solve, (d2/dx2 + d2/dy2 [+ d2/dz2] - lambda) u = f, Fourier in the
 * periodic directions, Gauss-Lobatto-Legendre (GLL) collocation in the last
 * direction, plus a second-order finite-difference FFT/Thomas variant.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the oracle that the tests, the
 * smoke check and the CPU-baseline leg of bench.py use to check the CUDA
 * path.  Nothing in the product links, loads or calls it.
 *
 * Pinning: tests/test_oracle.py checks every function here against the
 * reference's own code compiled from its sources (oracle/_ref, built by
 * oracle/Makefile) and against the golden vectors in tests/golden/ that were
 * generated from it (tests/golden/make_golden.py), plus the reference's
 * manufactured-solution known answers (TestNonPeriodic2D_MPI.cpp,
 * TestNonPeriodic3D_MPI.cpp).  The finite-difference variant has no reference
 * implementation in the tree (DirectUniformFDM/ is absent); it restates the
 * HypreFDM stencil (HelmholtzSolvers/HypreFDM/src/Helmholtz3D_MPI.cpp:297-410)
 * and is pinned by its own FP64 stencil residual (orc_fd3d_residual).
 *
 * Array conventions (row-major, last index fastest):
 *   2D  f, u : [Ns][Nx][N]       gl, gr : [Nx]
 *   3D  f, u : [Ns][Nx][Ny][N]   gl, gr : [Nx][Ny]
 *   FD  f, u : [Nx][Ny][Nz]      gb, gf : [Nx][Ny]   (Nz interior points)
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define ORC_PI 3.1415926535897932 /* General.h:15 */

/* ------------------------------------------------------------------ GLL -- */

/* P_n(x) and P_n'(x) by the three-term recurrence (GLLQuadrature.cpp:7-40). */
static void orc_legendre(int n, double x, double* p, double* dp)
{
    double p0 = 1.0, p1 = x, pn = (n == 0 ? 1.0 : x);
    if (n == 0) { *p = 1.0; *dp = 0.0; return; }
    for (int i = 2; i <= n; ++i) {
        pn = ((2.0 * i - 1.0) * x * p1 - (i - 1.0) * p0) / i;
        p0 = p1;
        p1 = pn;
    }
    *p = pn;
    /* derivative from P_n and P_{n-1}; callers only ask for it at |x| < 1 */
    *dp = (n == 1) ? 1.0 : n * (x * pn - p0) / (x * x - 1.0);
}

/* N GLL nodes on [-1,1] in ascending order: the end points and the roots of
 * P'_{N-1}.  Same nodes as GaussLobattoLegendrePoints (GLLQuadrature.cpp:78-128),
 * computed by Newton's method instead of the tridiagonal eigenproblem. */
void orc_gll_nodes(int N, double* x)
{
    int n = N - 1;
    x[0] = -1.0;
    x[N - 1] = 1.0;
    for (int i = 1; i < N - 1; ++i) {
        double t = -cos(ORC_PI * i / n);
        for (int it = 0; it < 100; ++it) {
            double p, dp;
            orc_legendre(n, t, &p, &dp);
            double d2p = (2.0 * t * dp - n * (n + 1.0) * p) / (1.0 - t * t);
            double dt = dp / d2p;
            t -= dt;
            if (fabs(dt) < 1e-17) break;
        }
        x[i] = t;
    }
    for (int i = 0; i < N / 2; ++i) { /* exact symmetry about 0 */
        double s = 0.5 * (x[N - 1 - i] - x[i]);
        x[i] = -s;
        x[N - 1 - i] = s;
    }
    if (N % 2) x[N / 2] = 0.0;
}

/* First-derivative collocation matrix (GLLQuadrature.cpp:198-213), D[i*N+j]. */
void orc_deriv_matrix(int N, const double* x, double* D)
{
    double* P = (double*)malloc(sizeof(double) * N);
    for (int i = 0; i < N; ++i) { double dp; orc_legendre(N - 1, x[i], &P[i], &dp); }
    for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j)
            D[i * N + j] = (i == j) ? 0.0 : P[i] / (P[j] * (x[i] - x[j]));
    D[0] = -0.25 * N * (N - 1);
    D[N * N - 1] = 0.25 * N * (N - 1);
    free(P);
}

/* C = A * B for N x N row-major (SecondDerivativeMatrix, GLLQuadrature.cpp:250-262). */
static void orc_matmul(int N, const double* A, const double* B, double* C)
{
    for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j) {
            double s = 0.0;
            for (int k = 0; k < N; ++k) s += A[i * N + k] * B[k * N + j];
            C[i * N + j] = s;
        }
}

/* Scaled GLL grid for one element of length L/Ns placed from 0 (the
 * reference's node placement, NonPeriodic2D_MPI.cpp:95-123): y[Ns*(N-1)+1],
 * D and D2 scaled to the element. */
void orc_gll_setup(int N, int Ns, double L, double* y, double* D, double* D2)
{
    double* xi = (double*)malloc(sizeof(double) * N);
    double* Dr = (double*)malloc(sizeof(double) * N * N);
    orc_gll_nodes(N, xi);
    orc_deriv_matrix(N, xi, Dr);
    orc_matmul(N, Dr, Dr, D2);
    for (int jj = 0; jj < Ns; ++jj) {
        double a = jj * L / Ns, b = a + L / Ns;
        for (int j = 0; j < N; ++j) y[jj * (N - 1) + j] = 0.5 * (a + b + (L / Ns) * xi[j]);
    }
    for (int i = 0; i < N * N; ++i) {
        D[i] = Dr[i] * (2.0 * Ns / L);
        D2[i] = D2[i] * (4.0 * Ns * Ns / (L * L));
    }
    free(xi);
    free(Dr);
}

/* ------------------------------------------------------------------- LU -- */

/* In-place LU with scaled partial pivoting, LINPACK storage: multipliers of
 * step k stay in column k and are not swapped by later pivots, and the row
 * scales are not permuted (LU_Decomposition.cpp:7-72).  Returns 0, or 1 when
 * the scaled pivot is <= 1e-12 (the reference's singular check, :49-50). */
int orc_lu_decompose(int n, double* A, int* piv)
{
    double* s = (double*)malloc(sizeof(double) * n);
    for (int p = 0; p < n; ++p) {
        s[p] = fabs(A[p * n]);
        for (int q = 1; q < n; ++q)
            if (fabs(A[p * n + q]) > s[p]) s[p] = fabs(A[p * n + q]);
    }
    for (int k = 0; k < n - 1; ++k) {
        double c = fabs(A[k * n + k]) / s[k];
        int idx = k;
        for (int i = k + 1; i < n; ++i)
            if (fabs(A[i * n + k]) / s[i] > c) { idx = i; c = fabs(A[i * n + k]) / s[i]; }
        piv[k] = idx;
        if (fabs(c) <= 1e-12) { free(s); return 1; }
        if (idx != k)
            for (int j = k; j < n; ++j) { double t = A[k * n + j]; A[k * n + j] = A[idx * n + j]; A[idx * n + j] = t; }
        for (int l = k + 1; l < n; ++l) {
            A[l * n + k] /= A[k * n + k];
            for (int m = k + 1; m < n; ++m) A[l * n + m] -= A[l * n + k] * A[k * n + m];
        }
    }
    if (n > 0) piv[n - 1] = n - 1;
    free(s);
    return 0;
}

/* Forward (interleaved pivot swaps) and back substitution, b overwritten by
 * the solution (LU_Decomposition.cpp:78-108). */
void orc_lu_solve(int n, const double* A, const int* piv, double* b)
{
    for (int k = 0; k < n - 1; ++k) {
        int idx = piv[k];
        if (idx != k) { double t = b[idx]; b[idx] = b[k]; b[k] = t; }
        for (int i = k + 1; i < n; ++i) b[i] -= A[i * n + k] * b[k];
    }
    b[n - 1] /= A[(n - 1) * n + n - 1];
    for (int p = n - 2; p >= 0; --p) {
        double t = 0.0;
        for (int q = p + 1; q < n; ++q) t += A[p * n + q] * b[q];
        b[p] = (b[p] - t) / A[p * n + p];
    }
}

/* ------------------------------------------------------------------ FFT -- */

/* In-place complex radix-2 DFT of length n (power of 2) on (re, im) with
 * element stride `st`.  sign = -1: X_m = sum_j x_j exp(-2 pi i j m / n), no
 * scaling (the reference's isign = +1, Fourier_Quadrature.cpp:543-598);
 * sign = +1: the unscaled inverse. */
static void orc_fft(int n, double* re, double* im, long st, int sign)
{
    for (int i = 1, j = 0; i < n; ++i) {
        int bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) {
            double t = re[i * st]; re[i * st] = re[j * st]; re[j * st] = t;
            t = im[i * st]; im[i * st] = im[j * st]; im[j * st] = t;
        }
    }
    for (int len = 2; len <= n; len <<= 1) {
        int h = len >> 1;
        for (int k = 0; k < h; ++k) {
            double ang = sign * 2.0 * ORC_PI * k / len;
            double wr = cos(ang), wi = sin(ang);
            for (int s = 0; s < n; s += len) {
                long a = (long)(s + k) * st, b = (long)(s + k + h) * st;
                double tr = wr * re[b] - wi * im[b];
                double ti = wr * im[b] + wi * re[b];
                re[b] = re[a] - tr; im[b] = im[a] - ti;
                re[a] += tr; im[a] += ti;
            }
        }
    }
}

static int orc_is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

/* --------------------------------------------- per-wavenumber GLL solve -- */

/* Solve one complex spectral row set sharing one operator: the particular
 * solutions of every element, the homogeneous solutions ul/ur, the
 * element-interface tridiagonal sweep with Robin ends, and the combination
 * (NonPeriodic2D_MPI.cpp:176-223 and the size==1 paths :265-295, :414-424,
 * :466-470).  F, U: [Ns][N] (re or im part, stride `es` between elements).
 * Op: LU of Dyy_int - sigma I; ul, ur: homogeneous solutions [N]. */
static double orc_dot(int N, const double* r, const double* v)
{
    double s = 0.0;
    for (int k = 0; k < N; ++k) s += r[k] * v[k];
    return s;
}

static void orc_row_solve(int N, int Ns, const double* Op, const int* piv, const double* D,
                          const double* ul, const double* ur, double al, double bl, double ar, double br,
                          const double* F, long es, double gl, double gr, double* U, double* work)
{
    int n = N - 2;
    double* phi = work;                    /* [Ns][N] */
    double* b = phi + (size_t)Ns * N;      /* [Ns] */
    double* c = b + Ns;
    double* rhs = c + Ns;
    double* zl = rhs + Ns;
    double* zr = zl + Ns;
    const double* D0 = D;                  /* row 0 of Dy */
    const double* DN = D + (size_t)(N - 1) * N;
    for (int jj = 0; jj < Ns; ++jj) {
        double* p = phi + (size_t)jj * N;
        p[0] = 0.0;
        p[N - 1] = 0.0;
        for (int j = 0; j < n; ++j) p[j + 1] = F[jj * es + j + 1];
        orc_lu_solve(n, Op, piv, p + 1);
    }
    double d0ul = orc_dot(N, D0, ul), d0ur = orc_dot(N, D0, ur), dNul = orc_dot(N, DN, ul), dNur = orc_dot(N, DN, ur);
    b[0] = -al * d0ul + bl;
    c[0] = -al * d0ur;
    rhs[0] = gl + al * orc_dot(N, D0, phi);
    for (int jj = 1; jj < Ns; ++jj) {
        double lb = dNul;
        b[jj] = dNur - d0ul - (c[jj - 1] / b[jj - 1]) * lb;
        c[jj] = -d0ur;
        rhs[jj] = orc_dot(N, D0, phi + (size_t)jj * N) - orc_dot(N, DN, phi + (size_t)(jj - 1) * N) - (rhs[jj - 1] / b[jj - 1]) * lb;
    }
    double lb = ar * dNul;
    double bR = ar * dNur + br - (c[Ns - 1] / b[Ns - 1]) * lb;
    double rR = gr - ar * orc_dot(N, DN, phi + (size_t)(Ns - 1) * N) - (rhs[Ns - 1] / b[Ns - 1]) * lb;
    for (int jj = Ns - 1; jj >= 0; --jj) {
        zr[jj] = (jj == Ns - 1) ? rR / bR : zl[jj + 1];
        zl[jj] = (rhs[jj] - c[jj] * zr[jj]) / b[jj];
    }
    for (int jj = 0; jj < Ns; ++jj)
        for (int j = 0; j < N; ++j)
            U[jj * es + j] = phi[(size_t)jj * N + j] + zl[jj] * ul[j] + zr[jj] * ur[j];
}

/* The same row set for the solver that is periodic in the GLL direction: the
 * particular solutions, then the cyclic interface sweep with its rank-one
 * correction, then the combination (Periodic2D_MPI.cpp:176-223; the size == 1
 * paths of Step 3 :257-295, Step 4 :521-565 and Step 5 :682-686).  One element:
 * u(0) = u(L) = zeta with matching slopes.  Several: a tridiagonal sweep whose
 * first diagonal is shifted, a second right-hand side rhs1 for the shift, and
 * alpha = -(zl + zr) / (1 + el + er) at the last element. */
static void orc_row_solve_periodic(int N, int Ns, const double* Op, const int* piv, const double* D,
                                   const double* ul, const double* ur, const double* F, long es,
                                   double* U, double* work)
{
    int n = N - 2;
    double* phi = work;                    /* [Ns][N] */
    double* b = phi + (size_t)Ns * N;      /* [Ns] each */
    double* c = b + Ns;
    double* r0 = c + Ns;
    double* r1 = r0 + Ns;
    double* zl = r1 + Ns;
    double* zr = zl + Ns;
    double* el = zr + Ns;
    double* er = el + Ns;
    const double* D0 = D;
    const double* DN = D + (size_t)(N - 1) * N;
    for (int jj = 0; jj < Ns; ++jj) {
        double* p = phi + (size_t)jj * N;
        p[0] = 0.0;
        p[N - 1] = 0.0;
        for (int j = 0; j < n; ++j) p[j + 1] = F[jj * es + j + 1];
        orc_lu_solve(n, Op, piv, p + 1);
    }
    double d0ul = orc_dot(N, D0, ul), d0ur = orc_dot(N, D0, ur), dNul = orc_dot(N, DN, ul), dNur = orc_dot(N, DN, ur);
    if (Ns == 1) {
        double bb = (d0ul + d0ur) - (dNul + dNur);
        double z = (orc_dot(N, DN, phi) - orc_dot(N, D0, phi)) / bb;
        zl[0] = z;
        zr[0] = z;
    } else {
        const double* plast = phi + (size_t)(Ns - 1) * N;
        b[0] = dNur - dNul - d0ul;
        c[0] = -d0ur;
        r0[0] = orc_dot(N, D0, phi) - orc_dot(N, DN, plast);
        r1[0] = dNul;
        for (int jj = 1; jj < Ns; ++jj) {
            const double* pj = phi + (size_t)jj * N;
            const double* pp = phi + (size_t)(jj - 1) * N;
            r0[jj] = orc_dot(N, D0, pj) - orc_dot(N, DN, pp) - (r0[jj - 1] / b[jj - 1]) * dNul;
            if (jj < Ns - 1) {
                b[jj] = dNur - d0ul - (c[jj - 1] / b[jj - 1]) * dNul;
                c[jj] = -d0ur;
                r1[jj] = -(r1[jj - 1] / b[jj - 1]) * dNul;
            } else {
                b[jj] = dNur - d0ul + d0ur - (c[jj - 1] / b[jj - 1]) * dNul;
                c[jj] = 0.0;
                r1[jj] = -d0ur - (r1[jj - 1] / b[jj - 1]) * dNul;
            }
        }
        zl[Ns - 1] = r0[Ns - 1] / b[Ns - 1];
        el[Ns - 1] = r1[Ns - 1] / b[Ns - 1];
        for (int jj = Ns - 2; jj >= 0; --jj) {
            zr[jj] = zl[jj + 1];
            er[jj] = el[jj + 1];
            zl[jj] = (r0[jj] - c[jj] * zr[jj]) / b[jj];
            el[jj] = (r1[jj] - c[jj] * er[jj]) / b[jj];
        }
        zr[Ns - 1] = zl[0];
        er[Ns - 1] = el[0];
        double alpha = -(zl[Ns - 1] + zr[Ns - 1]) / (1.0 + el[Ns - 1] + er[Ns - 1]);
        for (int jj = 0; jj < Ns; ++jj) {
            zl[jj] += alpha * el[jj];
            zr[jj] += alpha * er[jj];
        }
    }
    for (int jj = 0; jj < Ns; ++jj)
        for (int j = 0; j < N; ++j)
            U[jj * es + j] = phi[(size_t)jj * N + j] + zl[jj] * ul[j] + zr[jj] * ur[j];
}

/* Build Dyy_int - sigma I, factor it, and form the homogeneous solutions
 * (the ConstructOperator callback of TestNonPeriodic2D_MPI.cpp:67-74 plus
 * NonPeriodic2D_MPI.cpp:194-213).  Returns the LU status. */
static int orc_operator(int N, const double* D2, double sigma, double* Op, int* piv, double* ul, double* ur)
{
    int n = N - 2;
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
            Op[i * n + j] = D2[(i + 1) * N + (j + 1)] - (i == j ? sigma : 0.0);
    if (orc_lu_decompose(n, Op, piv)) return 1;
    ul[0] = 1.0; ul[N - 1] = 0.0;
    ur[0] = 0.0; ur[N - 1] = 1.0;
    for (int j = 0; j < n; ++j) { ul[j + 1] = -D2[(j + 1) * N]; ur[j + 1] = -D2[(j + 1) * N + N - 1]; }
    orc_lu_solve(n, Op, piv, ul + 1);
    orc_lu_solve(n, Op, piv, ur + 1);
    return 0;
}

/* 2D solve (SolvePDE, NonPeriodic2D_MPI.cpp:228-474; periodic in y:
 * Periodic2D_MPI.cpp:228-469).  Returns 0 on success, 2 for a non-power-of-2
 * Nx, 3 for a singular operator. */
static int orc_solve2d_impl(int Nx, int N, int Ns, double Lx, double Ly,
                            double al, double bl, double ar, double br, double lam,
                            const double* f, const double* gl, const double* gr, double* u, int periodic)
{
    if (!orc_is_pow2(Nx)) return 2;
    size_t es = (size_t)Nx * N; /* element stride */
    double* y = malloc(sizeof(double) * (Ns * (N - 1) + 1));
    double* D = malloc(sizeof(double) * N * N);
    double* D2 = malloc(sizeof(double) * N * N);
    double* Fr = malloc(sizeof(double) * Ns * es);
    double* Fi = calloc(Ns * es, sizeof(double));
    double* Ur = malloc(sizeof(double) * Ns * es);
    double* Ui = malloc(sizeof(double) * Ns * es);
    double* Glr = malloc(sizeof(double) * Nx), *Gli = calloc(Nx, sizeof(double));
    double* Grr = malloc(sizeof(double) * Nx), *Gri = calloc(Nx, sizeof(double));
    double* Op = malloc(sizeof(double) * N * N);
    int* piv = malloc(sizeof(int) * N);
    double* ul = malloc(sizeof(double) * N), *ur = malloc(sizeof(double) * N);
    double* work = malloc(sizeof(double) * (Ns * (N + 9) + 8));
    double* Fa = malloc(sizeof(double) * Ns * N), *Ua = malloc(sizeof(double) * Ns * N);
    int status = 0;
    orc_gll_setup(N, Ns, Ly, y, D, D2);
    memcpy(Fr, f, sizeof(double) * Ns * es);
    memcpy(Glr, gl, sizeof(double) * Nx);
    memcpy(Grr, gr, sizeof(double) * Nx);
    for (int jj = 0; jj < Ns; ++jj)
        for (int j = 0; j < N; ++j) orc_fft(Nx, Fr + jj * es + j, Fi + jj * es + j, N, -1);
    orc_fft(Nx, Glr, Gli, 1, -1);
    orc_fft(Nx, Grr, Gri, 1, -1);
    for (int m = 0; m < Nx; ++m) {
        int iw = (m <= Nx / 2) ? m : Nx - m;
        double sigma = lam + 4.0 * ORC_PI * ORC_PI * iw * iw / (Lx * Lx);
        if (orc_operator(N, D2, sigma, Op, piv, ul, ur)) { status = 3; goto done; }
        for (int part = 0; part < 2; ++part) {
            const double* F = part ? Fi : Fr;
            double* U = part ? Ui : Ur;
            for (int jj = 0; jj < Ns; ++jj) memcpy(Fa + jj * N, F + jj * es + (size_t)m * N, sizeof(double) * N);
            if (periodic)
                orc_row_solve_periodic(N, Ns, Op, piv, D, ul, ur, Fa, N, Ua, work);
            else
                orc_row_solve(N, Ns, Op, piv, D, ul, ur, al, bl, ar, br, Fa, N,
                              part ? Gli[m] : Glr[m], part ? Gri[m] : Grr[m], Ua, work);
            for (int jj = 0; jj < Ns; ++jj) memcpy(U + jj * es + (size_t)m * N, Ua + jj * N, sizeof(double) * N);
        }
    }
    for (int jj = 0; jj < Ns; ++jj)
        for (int j = 0; j < N; ++j) orc_fft(Nx, Ur + jj * es + j, Ui + jj * es + j, N, +1);
    for (size_t i = 0; i < Ns * es; ++i) u[i] = Ur[i] / Nx;
done:
    free(y); free(D); free(D2); free(Fr); free(Fi); free(Ur); free(Ui);
    free(Glr); free(Gli); free(Grr); free(Gri); free(Op); free(piv); free(ul); free(ur);
    free(work); free(Fa); free(Ua);
    return status;
}

int orc_solve2d(int Nx, int N, int Ns, double Lx, double Ly,
                double al, double bl, double ar, double br, double lam,
                const double* f, const double* gl, const double* gr, double* u)
{
    return orc_solve2d_impl(Nx, N, Ns, Lx, Ly, al, bl, ar, br, lam, f, gl, gr, u, 0);
}

/* Periodic in y (Periodic2D_MPI.cpp SolvePDE): no boundary data. */
int orc_psolve2d(int Nx, int N, int Ns, double Lx, double Ly, double lam, const double* f, double* u)
{
    double* z = calloc(Nx, sizeof(double));
    int st = orc_solve2d_impl(Nx, N, Ns, Lx, Ly, 0.0, 1.0, 0.0, 1.0, lam, f, z, z, u, 1);
    free(z);
    return st;
}

/* 3D solve (SolvePDE, NonPeriodic3D_MPI.cpp:237-591; periodic in z:
 * Periodic3D_MPI.cpp:233-866): 2D DFT over (x, y), one operator per
 * (|kx|, |ky|), inverse DFT. */
static int orc_solve3d_impl(int Nx, int Ny, int N, int Ns, double Lx, double Ly, double Lz,
                            double al, double bl, double ar, double br, double lam,
                            const double* f, const double* gl, const double* gr, double* u, int periodic)
{
    if (!orc_is_pow2(Nx) || !orc_is_pow2(Ny)) return 2;
    size_t plane = (size_t)Ny * N, es = (size_t)Nx * plane;
    double* z = malloc(sizeof(double) * (Ns * (N - 1) + 1));
    double* D = malloc(sizeof(double) * N * N);
    double* D2 = malloc(sizeof(double) * N * N);
    double* Fr = malloc(sizeof(double) * Ns * es);
    double* Fi = calloc(Ns * es, sizeof(double));
    double* Ur = malloc(sizeof(double) * Ns * es);
    double* Ui = malloc(sizeof(double) * Ns * es);
    size_t nb = (size_t)Nx * Ny;
    double* Glr = malloc(sizeof(double) * nb), *Gli = calloc(nb, sizeof(double));
    double* Grr = malloc(sizeof(double) * nb), *Gri = calloc(nb, sizeof(double));
    double* Op = malloc(sizeof(double) * N * N);
    int* piv = malloc(sizeof(int) * N);
    double* ul = malloc(sizeof(double) * N), *ur = malloc(sizeof(double) * N);
    double* work = malloc(sizeof(double) * (Ns * (N + 9) + 8));
    double* Fa = malloc(sizeof(double) * Ns * N), *Ua = malloc(sizeof(double) * Ns * N);
    int status = 0;
    orc_gll_setup(N, Ns, Lz, z, D, D2);
    memcpy(Fr, f, sizeof(double) * Ns * es);
    memcpy(Glr, gl, sizeof(double) * nb);
    memcpy(Grr, gr, sizeof(double) * nb);
    for (int kk = 0; kk < Ns; ++kk) {
        for (int j = 0; j < Ny; ++j)
            for (int k = 0; k < N; ++k) orc_fft(Nx, Fr + kk * es + (size_t)j * N + k, Fi + kk * es + (size_t)j * N + k, plane, -1);
        for (int i = 0; i < Nx; ++i)
            for (int k = 0; k < N; ++k) orc_fft(Ny, Fr + kk * es + i * plane + k, Fi + kk * es + i * plane + k, N, -1);
    }
    for (int j = 0; j < Ny; ++j) { orc_fft(Nx, Glr + j, Gli + j, Ny, -1); orc_fft(Nx, Grr + j, Gri + j, Ny, -1); }
    for (int i = 0; i < Nx; ++i) { orc_fft(Ny, Glr + (size_t)i * Ny, Gli + (size_t)i * Ny, 1, -1); orc_fft(Ny, Grr + (size_t)i * Ny, Gri + (size_t)i * Ny, 1, -1); }
    for (int iw = 0; iw <= Nx / 2; ++iw)
        for (int jw = 0; jw <= Ny / 2; ++jw) {
            double sigma = lam + 4.0 * ORC_PI * ORC_PI * iw * iw / (Lx * Lx) + 4.0 * ORC_PI * ORC_PI * jw * jw / (Ly * Ly);
            if (orc_operator(N, D2, sigma, Op, piv, ul, ur)) { status = 3; goto done; }
            int ms[2] = {iw, (Nx - iw) % Nx}, ns[2] = {jw, (Ny - jw) % Ny};
            for (int a = 0; a < 2; ++a) {
                if (a == 1 && ms[1] == ms[0]) continue;
                for (int bb = 0; bb < 2; ++bb) {
                    if (bb == 1 && ns[1] == ns[0]) continue;
                    size_t off = (size_t)ms[a] * plane + (size_t)ns[bb] * N, boff = (size_t)ms[a] * Ny + ns[bb];
                    for (int part = 0; part < 2; ++part) {
                        const double* F = part ? Fi : Fr;
                        double* U = part ? Ui : Ur;
                        for (int kk = 0; kk < Ns; ++kk) memcpy(Fa + kk * N, F + kk * es + off, sizeof(double) * N);
                        if (periodic)
                            orc_row_solve_periodic(N, Ns, Op, piv, D, ul, ur, Fa, N, Ua, work);
                        else
                            orc_row_solve(N, Ns, Op, piv, D, ul, ur, al, bl, ar, br, Fa, N,
                                          part ? Gli[boff] : Glr[boff], part ? Gri[boff] : Grr[boff], Ua, work);
                        for (int kk = 0; kk < Ns; ++kk) memcpy(U + kk * es + off, Ua + kk * N, sizeof(double) * N);
                    }
                }
            }
        }
    for (int kk = 0; kk < Ns; ++kk) {
        for (int i = 0; i < Nx; ++i)
            for (int k = 0; k < N; ++k) orc_fft(Ny, Ur + kk * es + i * plane + k, Ui + kk * es + i * plane + k, N, +1);
        for (int j = 0; j < Ny; ++j)
            for (int k = 0; k < N; ++k) orc_fft(Nx, Ur + kk * es + (size_t)j * N + k, Ui + kk * es + (size_t)j * N + k, plane, +1);
    }
    for (size_t i = 0; i < Ns * es; ++i) u[i] = Ur[i] / ((double)Nx * Ny);
done:
    free(z); free(D); free(D2); free(Fr); free(Fi); free(Ur); free(Ui);
    free(Glr); free(Gli); free(Grr); free(Gri); free(Op); free(piv); free(ul); free(ur);
    free(work); free(Fa); free(Ua);
    return status;
}

int orc_solve3d(int Nx, int Ny, int N, int Ns, double Lx, double Ly, double Lz,
                double al, double bl, double ar, double br, double lam,
                const double* f, const double* gl, const double* gr, double* u)
{
    return orc_solve3d_impl(Nx, Ny, N, Ns, Lx, Ly, Lz, al, bl, ar, br, lam, f, gl, gr, u, 0);
}

/* Periodic in z (Periodic3D_MPI.cpp SolvePDE): no boundary data. */
int orc_psolve3d(int Nx, int Ny, int N, int Ns, double Lx, double Ly, double Lz, double lam,
                 const double* f, double* u)
{
    double* z = calloc((size_t)Nx * Ny, sizeof(double));
    int st = orc_solve3d_impl(Nx, Ny, N, Ns, Lx, Ly, Lz, 0.0, 1.0, 0.0, 1.0, lam, f, z, z, u, 1);
    free(z);
    return st;
}

/* ------------------------------------------------ derivative helpers -- */

/* du = M u for `nrows` rows of N values, M the scaled first (order 1) or
 * second (order 2) GLL derivative matrix of one element of length L/Ns
 * (FirstDerivativeY / SecondDerivativeY, NonPeriodic2D_MPI.cpp:497-542;
 * FirstDerivativeZ / SecondDerivativeZ, NonPeriodic3D_MPI.cpp:632-683). */
void orc_gll_deriv(int N, int Ns, double L, int order, long nrows, const double* u, double* du)
{
    double* y = malloc(sizeof(double) * (Ns * (N - 1) + 1));
    double* D = malloc(sizeof(double) * N * N);
    double* D2 = malloc(sizeof(double) * N * N);
    orc_gll_setup(N, Ns, L, y, D, D2);
    const double* M = order == 1 ? D : D2;
    for (long r = 0; r < nrows; ++r)
        for (int j = 0; j < N; ++j) {
            double a = 0.0;
            for (int k = 0; k < N; ++k) a += M[j * N + k] * u[r * N + k];
            du[r * N + j] = a;
        }
    free(y); free(D); free(D2);
}

/* Spectral derivative of the real array u[n0][n1][n2] along axis 0 or 1:
 * forward DFT, multiply by 2 pi K (order 1, times i) or -4 pi^2 K^2 (order 2)
 * with K = k for k < n/2 and k - n otherwise, inverse DFT (/n), real part,
 * divided by L^order (FirstDerivativeFourierX..Y / SecondDerivativeFourierX..Y,
 * Fourier_Quadrature.cpp:1387-1834). */
void orc_fourier_deriv(int n0, int n1, int n2, int axis, int order, double L, const double* u, double* du)
{
    int n = axis == 0 ? n0 : n1;
    long st = axis == 0 ? (long)n1 * n2 : n2;
    double* re = malloc(sizeof(double) * n);
    double* im = malloc(sizeof(double) * n);
    int outer = axis == 0 ? 1 : n0, inner = axis == 0 ? n1 * n2 : n2;
    for (int o = 0; o < outer; ++o)
        for (int c = 0; c < inner; ++c) {
            long base = (axis == 0 ? 0 : (long)o * n1 * n2) + c;
            for (int i = 0; i < n; ++i) { re[i] = u[base + i * st]; im[i] = 0.0; }
            orc_fft(n, re, im, 1, -1);
            for (int i = 0; i < n; ++i) {
                double K = (i < n / 2) ? (double)i : (double)(i - n);
                if (order == 1) {
                    double t = re[i];
                    re[i] = -2.0 * ORC_PI * K * im[i];
                    im[i] = 2.0 * ORC_PI * K * t;
                } else {
                    re[i] *= -4.0 * ORC_PI * ORC_PI * K * K;
                    im[i] *= -4.0 * ORC_PI * ORC_PI * K * K;
                }
            }
            orc_fft(n, re, im, 1, +1);
            double sc = (order == 1 ? L : L * L) * n;
            for (int i = 0; i < n; ++i) du[base + i * st] = re[i] / sc;
        }
    free(re); free(im);
}

/* The collocation residual of a 3D solution, computed directly in FP64:
 * interior GLL rows  r = f - (u_xx + u_yy + D2 u - lambda u)  (spectral x/y
 * derivatives), boundary rows r = g - (Robin operator) u, for Ns = 1.
 * Returns max |r| over all rows and writes the per-point residual to r. */
double orc_residual3d(int Nx, int Ny, int N, double Lx, double Ly, double Lz,
                      double al, double bl, double ar, double br, double lam,
                      const double* f, const double* gl, const double* gr, const double* u, double* r)
{
    size_t plane = (size_t)Ny * N, tot = (size_t)Nx * plane;
    double* z = malloc(sizeof(double) * N);
    double* D = malloc(sizeof(double) * N * N);
    double* D2 = malloc(sizeof(double) * N * N);
    double* Lr = malloc(sizeof(double) * tot), *Li = calloc(tot, sizeof(double));
    orc_gll_setup(N, 1, Lz, z, D, D2);
    memcpy(Lr, u, sizeof(double) * tot);
    for (int j = 0; j < Ny; ++j)
        for (int k = 0; k < N; ++k) orc_fft(Nx, Lr + (size_t)j * N + k, Li + (size_t)j * N + k, plane, -1);
    for (int i = 0; i < Nx; ++i)
        for (int k = 0; k < N; ++k) orc_fft(Ny, Lr + i * plane + k, Li + i * plane + k, N, -1);
    for (int m1 = 0; m1 < Nx; ++m1)
        for (int m2 = 0; m2 < Ny; ++m2) {
            int iw = m1 <= Nx / 2 ? m1 : Nx - m1, jw = m2 <= Ny / 2 ? m2 : Ny - m2;
            double k2 = 4.0 * ORC_PI * ORC_PI * ((double)iw * iw / (Lx * Lx) + (double)jw * jw / (Ly * Ly));
            for (int k = 0; k < N; ++k) {
                size_t o = (size_t)m1 * plane + (size_t)m2 * N + k;
                Lr[o] *= -k2;
                Li[o] *= -k2;
            }
        }
    for (int i = 0; i < Nx; ++i)
        for (int k = 0; k < N; ++k) orc_fft(Ny, Lr + i * plane + k, Li + i * plane + k, N, +1);
    for (int j = 0; j < Ny; ++j)
        for (int k = 0; k < N; ++k) orc_fft(Nx, Lr + (size_t)j * N + k, Li + (size_t)j * N + k, plane, +1);
    double mx = 0.0;
    for (int i = 0; i < Nx; ++i)
        for (int j = 0; j < Ny; ++j) {
            const double* uc = u + i * plane + (size_t)j * N;
            double* rc = r + i * plane + (size_t)j * N;
            for (int k = 1; k < N - 1; ++k) {
                double s = 0.0;
                for (int q = 0; q < N; ++q) s += D2[k * N + q] * uc[q];
                double lap = Lr[i * plane + (size_t)j * N + k] / ((double)Nx * Ny) + s - lam * uc[k];
                rc[k] = f[i * plane + (size_t)j * N + k] - lap;
            }
            double d0 = 0.0, dN = 0.0;
            for (int q = 0; q < N; ++q) { d0 += D[q] * uc[q]; dN += D[(N - 1) * N + q] * uc[q]; }
            rc[0] = gl[(size_t)i * Ny + j] - (-al * d0 + bl * uc[0]);
            rc[N - 1] = gr[(size_t)i * Ny + j] - (ar * dN + br * uc[N - 1]);
            for (int k = 0; k < N; ++k) if (fabs(rc[k]) > mx) mx = fabs(rc[k]);
        }
    free(z); free(D); free(D2); free(Lr); free(Li);
    return mx;
}

/* -------------------------------------------- finite-difference variant -- */

/* FFT/Thomas solve of the second-order finite-difference Helmholtz problem:
 * periodic x and y (dx = Lx/Nx, dy = Ly/Ny), Nz interior points in z with
 * dz = Lz/(Nz+1), and one-sided second-order Robin rows at both z ends,
 * alpha du/dn + beta u = g with the outward normal.  Stencil and boundary rows
 * restate HypreFDM/src/Helmholtz3D_MPI.cpp:297-410 (interior 387-403, back
 * row 310-321, front row 322-333); the periodic directions become modified
 * wavenumbers -(4/dx^2) sin^2(pi m / Nx).  Returns 0 or 2 (non-power-of-2). */
int orc_fd3d_solve(int Nx, int Ny, int Nz, double Lx, double Ly, double Lz,
                   double ab, double bb, double af, double bf, double lam,
                   const double* f, const double* gb, const double* gf, double* u)
{
    if (!orc_is_pow2(Nx) || !orc_is_pow2(Ny)) return 2;
    double dx = Lx / Nx, dy = Ly / Ny, dz = Lz / (Nz + 1);
    double cx1 = 1.0 / (dx * dx), cy1 = 1.0 / (dy * dy), cz0 = 1.0 / dz, cz1 = 1.0 / (dz * dz);
    size_t plane = (size_t)Ny * Nz, tot = (size_t)Nx * plane, nb = (size_t)Nx * Ny;
    double* Fr = malloc(sizeof(double) * tot), *Fi = calloc(tot, sizeof(double));
    double* Br = malloc(sizeof(double) * nb), *Bi = calloc(nb, sizeof(double));
    double* Gr = malloc(sizeof(double) * nb), *Gi = calloc(nb, sizeof(double));
    int M = Nz + 2;
    double* lo = malloc(sizeof(double) * M), *di = malloc(sizeof(double) * M), *up = malloc(sizeof(double) * M);
    double* rr = malloc(sizeof(double) * M), *ri = malloc(sizeof(double) * M);
    memcpy(Fr, f, sizeof(double) * tot);
    memcpy(Br, gb, sizeof(double) * nb);
    memcpy(Gr, gf, sizeof(double) * nb);
    for (int j = 0; j < Ny; ++j)
        for (int k = 0; k < Nz; ++k) orc_fft(Nx, Fr + (size_t)j * Nz + k, Fi + (size_t)j * Nz + k, plane, -1);
    for (int i = 0; i < Nx; ++i)
        for (int k = 0; k < Nz; ++k) orc_fft(Ny, Fr + i * plane + k, Fi + i * plane + k, Nz, -1);
    for (int j = 0; j < Ny; ++j) { orc_fft(Nx, Br + j, Bi + j, Ny, -1); orc_fft(Nx, Gr + j, Gi + j, Ny, -1); }
    for (int i = 0; i < Nx; ++i) { orc_fft(Ny, Br + (size_t)i * Ny, Bi + (size_t)i * Ny, 1, -1); orc_fft(Ny, Gr + (size_t)i * Ny, Gi + (size_t)i * Ny, 1, -1); }
    for (int m1 = 0; m1 < Nx; ++m1)
        for (int m2 = 0; m2 < Ny; ++m2) {
            double sx = sin(ORC_PI * m1 / Nx), sy = sin(ORC_PI * m2 / Ny);
            double dd = -2.0 * cz1 - lam - 4.0 * cx1 * sx * sx - 4.0 * cy1 * sy * sy;
            size_t off = (size_t)m1 * plane + (size_t)m2 * Nz, bo = (size_t)m1 * Ny + m2;
            /* rows 0..M-1: boundary, Nz interior, boundary */
            for (int k = 1; k <= Nz; ++k) {
                lo[k] = cz1; di[k] = dd; up[k] = cz1;
                rr[k] = Fr[off + k - 1]; ri[k] = Fi[off + k - 1];
            }
            /* back row a0 u0 + a1 u1 + a2 u2 = g; remove a2 with interior row 1 */
            double a0 = 1.5 * ab * cz0 + bb, a1 = -2.0 * ab * cz0, a2 = 0.5 * ab * cz0;
            double q = a2 / cz1;
            lo[0] = 0.0; di[0] = a0 - q * cz1; up[0] = a1 - q * dd;
            rr[0] = Br[bo] - q * rr[1]; ri[0] = Bi[bo] - q * ri[1];
            double e0 = 1.5 * af * cz0 + bf, e1 = -2.0 * af * cz0, e2 = 0.5 * af * cz0;
            q = e2 / cz1;
            up[M - 1] = 0.0; di[M - 1] = e0 - q * cz1; lo[M - 1] = e1 - q * dd;
            rr[M - 1] = Gr[bo] - q * rr[M - 2]; ri[M - 1] = Gi[bo] - q * ri[M - 2];
            /* Thomas algorithm */
            for (int k = 1; k < M; ++k) {
                double w = lo[k] / di[k - 1];
                di[k] -= w * up[k - 1];
                rr[k] -= w * rr[k - 1];
                ri[k] -= w * ri[k - 1];
            }
            rr[M - 1] /= di[M - 1]; ri[M - 1] /= di[M - 1];
            for (int k = M - 2; k >= 0; --k) {
                rr[k] = (rr[k] - up[k] * rr[k + 1]) / di[k];
                ri[k] = (ri[k] - up[k] * ri[k + 1]) / di[k];
            }
            for (int k = 1; k <= Nz; ++k) { Fr[off + k - 1] = rr[k]; Fi[off + k - 1] = ri[k]; }
        }
    for (int i = 0; i < Nx; ++i)
        for (int k = 0; k < Nz; ++k) orc_fft(Ny, Fr + i * plane + k, Fi + i * plane + k, Nz, +1);
    for (int j = 0; j < Ny; ++j)
        for (int k = 0; k < Nz; ++k) orc_fft(Nx, Fr + (size_t)j * Nz + k, Fi + (size_t)j * Nz + k, plane, +1);
    for (size_t i = 0; i < tot; ++i) u[i] = Fr[i] / ((double)Nx * Ny);
    free(Fr); free(Fi); free(Br); free(Bi); free(Gr); free(Gi);
    free(lo); free(di); free(up); free(rr); free(ri);
    return 0;
}

/* Stencil residual of the finite-difference system in physical space, FP64,
 * evaluated directly from the HypreFDM stencil (no FFT): returns
 * max |f - A_h u| over the interior rows, with the Dirichlet/Robin end values
 * recovered from the boundary rows.  Used to pin orc_fd3d_solve. */
double orc_fd3d_residual(int Nx, int Ny, int Nz, double Lx, double Ly, double Lz,
                         double ab, double bb, double af, double bf, double lam,
                         const double* f, const double* gb, const double* gf, const double* u)
{
    double dx = Lx / Nx, dy = Ly / Ny, dz = Lz / (Nz + 1);
    double cx1 = 1.0 / (dx * dx), cy1 = 1.0 / (dy * dy), cz0 = 1.0 / dz, cz1 = 1.0 / (dz * dz);
    size_t plane = (size_t)Ny * Nz;
    double mx = 0.0;
    for (int i = 0; i < Nx; ++i)
        for (int j = 0; j < Ny; ++j) {
            const double* uc = u + i * plane + (size_t)j * Nz;
            size_t bo = (size_t)i * Ny + j;
            /* end values from the boundary rows: a0 u0 + a1 u1 + a2 u2 = g */
            double a0 = 1.5 * ab * cz0 + bb, a1 = -2.0 * ab * cz0, a2 = 0.5 * ab * cz0;
            double u0 = (gb[bo] - a1 * uc[0] - a2 * uc[1]) / a0;
            double e0 = 1.5 * af * cz0 + bf, e1 = -2.0 * af * cz0, e2 = 0.5 * af * cz0;
            double uM = (gf[bo] - e1 * uc[Nz - 1] - e2 * uc[Nz - 2]) / e0;
            for (int k = 0; k < Nz; ++k) {
                double um = (k == 0) ? u0 : uc[k - 1];
                double up = (k == Nz - 1) ? uM : uc[k + 1];
                double ux = u[(size_t)((i + Nx - 1) % Nx) * plane + (size_t)j * Nz + k] + u[(size_t)((i + 1) % Nx) * plane + (size_t)j * Nz + k];
                double uy = u[i * plane + (size_t)((j + Ny - 1) % Ny) * Nz + k] + u[i * plane + (size_t)((j + 1) % Ny) * Nz + k];
                double au = cx1 * ux + cy1 * uy + cz1 * (um + up) + (-2.0 * (cx1 + cy1 + cz1) - lam) * uc[k];
                double rr = fabs(f[i * plane + (size_t)j * Nz + k] - au);
                if (rr > mx) mx = rr;
            }
        }
    return mx;
}
