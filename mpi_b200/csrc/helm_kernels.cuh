// Kernel argument blocks shared by the launchers (helm_kernels.cu) and the plan
// (helm_plan.cu).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace helm {

// FFT_C2R_ADJ: the C2R pass of an adjoint solve (FftArgs adj_* fields), a
// separate instantiation so the forward C2R carries none of its code.
// FFT_DERIV: real in, real out -- the forward transform of each pair of real
// columns packed as one complex column, the multiplication by (i deriv_w K)^
// deriv_order, the inverse transform and the scaling, in one kernel.
enum FftMode { FFT_C2C = 0, FFT_R2C = 1, FFT_C2R = 2, FFT_C2R_ADJ = 3, FFT_DERIV = 4 };

// One batched FFT along a strided axis.  The transform index is the row; the
// data of one row are `ncols` contiguous columns; batches are `*_batch` apart.
// Units: elements of the in/out array type (real for the R2C input and the C2R
// output, complex otherwise).
struct FftArgs {
    const void* in;
    void* out;
    long long in_row, out_row;
    long long in_batch, out_batch;
    int ncols;      // complex columns per batch (C2C) or real columns (R2C/C2R)
    int nbatch;
    double scale;   // applied to every output value
    const void* tw; // exp(DIR * 2 pi i e / L), e in [0, L), compute precision
    // R2C only: GLL boundary slots k == 0 / k == P-1 of batch gl_batch /
    // gr_batch read the boundary data gl / gr [row][col / P] instead of the
    // input; the boundary slots of the other batches read 0.  P = 0 disables.
    const double* gl;
    const double* gr;
    long long bc_row;
    int P, gl_batch, gr_batch;
    // bc_add = 1: the boundary slots keep the input and add bc_scale_l * gl /
    // bc_scale_r * gr (finite-difference variant: the Robin rows eliminated
    // into the first and last interior equations).
    int bc_add;
    double bc_scale_l, bc_scale_r;
    // optional per-batch element offsets of the input / output (batched plans of
    // independent problems in a packed buffer); NULL: batch * *_batch
    const long long* in_boff;
    const long long* out_boff;
    // C2R of the adjoint solve (adj_mode != 0): the output is fbar; its GLL
    // boundary slots k = 0 / adj_P - 1 also go to gbar_l / gbar_r (times
    // adj_scale_l / adj_scale_r, index row * bc_row + col / adj_P); mode 1 (GLL)
    // stores 0 in those slots of fbar, mode 2 (finite differences) keeps them;
    // lam_out += sum of fbar * lam_u over the slots fbar keeps (lam_u NULL: no sum)
    int adj_mode, adj_P;
    double adj_scale_l, adj_scale_r;
    double* gbar_l;
    double* gbar_r;
    const double* lam_u;
    double* lam_out;
    // when set, the pass writes 0 to *zero_out first (the lambda sum of the same
    // solve's last pass starts from it; no separate memset)
    double* zero_out;
    // C2R only: spectral derivative, the half-spectrum row k is multiplied by
    // (i deriv_w K)^deriv_order on load, K = k below L/2 and -L/2 at L/2
    // (0: no derivative)
    int deriv_order;
    double deriv_w;
    // R2C only (non-pipelined kernel): when set, the transformed input is
    // in - in_sub, same layout and type as in (the data misfit u - u_obs of the
    // adjoint of a least-squares loss, formed as it is loaded)
    const void* in_sub;
    // C2R only (forward): add the result to out instead of storing it (the
    // correction of a refinement sweep accumulated into the solution)
    int accumulate;
};

// Finite-difference variant: one tridiagonal solve along z per spectrum row.
// Interior rows: cz1 u_{k-1} + (-2 cz1 - lambda - mx[kx] - my[ky]) u_k + cz1 u_{k+1};
// the first row adds d_first to its diagonal and has super-diagonal s_first,
// the last row adds d_last and has sub-diagonal s_last.
struct ThomasArgs {
    void* spec;           // complex [nrows][Nz], overwritten by the solution
    void* cprime;         // scratch [nrows][Nz] real: forward-elimination coefficients
    long long nrows;
    int Ny, Nz;
    const double* mx;     // [Nx/2+1] modified x wavenumbers 4 cx1 sin^2(pi kx / Nx)
    const double* my;     // [Ny]
    double cz1, lambda, d_first, s_first, d_last, s_last;
    int transpose;        // solve with the transposed matrix (adjoint)
    int half;             // Nz <= 256: one row per half-warp instead of per warp
};

// Per-wavenumber solve of the spectrum rows, grouped by shift sigma.
struct RowArgs {
    void* spec;                // complex [Ns][nrows][P]
    long long elem_stride;     // complex elements between GLL elements
    int P, n, Ns;
    int ngroups;
    const int* grp_start;      // [ngroups + 1]
    const int* grp_rows;       // complex row index (spec offset row * P)
    // LU method: per group, column-major combined L\U factor, 1/U_ii, row permutation
    const void* fac;
    const void* dinv;
    const uint8_t* perm;
    int ldf;                   // leading dimension of a factor column
    long long fac_stride;      // elements between two groups' factors
    // FDM method: shared interior eigen-decomposition D2int = V diag(lam) V^-1
    const void* vinvT;         // column-major V^-1: vinvT[k*ldf + j] = Vinv[j][k]
    const void* vT;            // column-major V:    vT[k*ldf + i]    = V[i][k]
    const double* lam;         // eigenvalues [n]
    // homogeneous solutions and scalars (FP64), per group
    const double* hom;         // [ngroups][2][P]: ul, ur
    const double* homs;        // [ngroups][4]: D0.ul, D0.ur, DN.ul, DN.ur
    const double* d0;          // [P] first row of the scaled first-derivative matrix
    const double* dN;          // [P] last row
    const double* sigma;       // [ngroups]
    const double* d2t;         // refinement: column-major interior D2 [n][n]
    int sweeps;
    double al, bl, ar, br;
    // Adjoint (transposed) solve, Ns = 1, FDM: vinvT / vT then hold the
    // transposed transforms, d2t the transposed D2, d0 / dN the boundary
    // columns D2[int][0] / D2[int][N-1], hom the per-group interior vectors
    // pl = -A^-T r0 and pr = -A^-T rN, homs the 2x2 boundary matrix
    // [[m00, m01], [m10, m11]] of the transposed system (row-major).
    int adjoint;
    // periodic in the GLL direction: the interface system is cyclic (u and its
    // slope continuous across the last element's right end into the first
    // element's left end); hom / homs are the forward ul, ur / D0.ul, D0.ur,
    // DN.ul, DN.ur in both directions, and the adjoint (one element) reads
    // pl = A^-T (DN - D0), pr = 0
    int periodic;
    // adjoint with several elements (Ns > 1, not periodic): the forward
    // homogeneous solutions ul, ur [ngroups][2][P], their end slopes
    // [ngroups][4] and the first / last rows of D (the forward data; vinvT / vT
    // then hold the transposed transforms for the interior solves)
    const double* fhom;
    const double* fhoms;
    const double* fd0;
    const double* fdN;
};

// Derivative along the GLL direction of every row of P values: du = M u with
// M the plan's scaled first (order 1, anti-centrosymmetric) or second (order 2,
// centrosymmetric) derivative matrix, applied through its even/odd fold.
struct GllDerivArgs {
    const void* in;
    void* out;
    const double* M;        // [P][P] row-major, FP64
    int P, order;
    long long nrows;        // rows of P values
    int rows_per_x;         // rows in one x row (Ny in 3D, 1 in 2D)
    int nx;                 // x rows per element
    long long x_stride, elem_stride;  // in elements of the io type
    int* err;               // device status word: set when a copy wait ran out, or NULL
};
int launch_gll_deriv(int io_double, const GllDerivArgs& a, cudaStream_t s);

// Launchers (helm_kernels.cu).  Return a cudaError_t.
// T: compute precision (0 = float, 1 = double); io: real element bytes for
// R2C input / C2R output (4 or 8).
// variant: launch shape chosen by the plan's autotuner (0: 256-thread CTAs, 1: 128).
int launch_fft(int L, int mode, int dir, int t_double, int io_bytes, const FftArgs& a, long long total_cols,
               cudaStream_t s, int variant = 0);
// method: 1 = LU, 2 = FDM; prec: 0 = FP64, 1 = FP32, 2 = FP32 with FP64 refinement
int launch_rows(int method, int prec, const RowArgs& a, cudaStream_t s);
int launch_thomas(int prec, const ThomasArgs& a, cudaStream_t s);
// Dynamic shared memory rows_kernel needs for this method / precision / size.
size_t rows_smem_bytes(int method, int prec, int n, int ld);
constexpr size_t kMaxSmemPerBlock = 232448;  // 227 KB opt-in limit of sm_100

}  // namespace helm
