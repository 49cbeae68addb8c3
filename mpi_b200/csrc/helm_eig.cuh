// Eigen-basis pipeline of the one-element Dirichlet solve (helm_eig.cu).
#pragma once
#include <cstddef>
#include <cuda_runtime.h>

namespace helm {

// The folded transforms have 32 slots per fold (GLL up to 66 points); a row of
// the coefficient spectrum holds both folds, 64 complex values.
constexpr int EIG_LD = 32;
constexpr int EIG_SLOTS = 2 * EIG_LD;

struct EigArgs {
    const double* f;        // input [x][y][P] (x stride x_stride, y stride P)
    double* u;              // output, same layout
    double* S;              // coefficient spectrum [Nx/2+1][Ny][64] complex
    const double* gl;       // boundary data [x * bc_x_stride + y], or NULL (zero)
    const double* gr;
    double ibl, ibr;        // 1 / beta_l, 1 / beta_r
    long long x_stride, bc_x_stride;
    int Ny, P, n, m, ms;
    const double* mats;     // the four folded transforms in m8n8k4 fragment order [4][4][8][32]
    const double* hbc;      // [4][32]: first transform of the folded boundary columns (s|l, s|r, a|l, a|r)
    const double* recip;    // [groups][64]: 1 / (eigenvalue - sigma), symmetric then antisymmetric fold
    const int* grp_of_row;  // shift group of spectrum row kx * Ny + ky
    const void* tw_x;       // exp(-2 pi i e / Nx), FP64 complex
    const void* tw_y;       // exp(-2 pi i e / Ny)
    double scale;           // 1 / (Nx Ny)
    // batched 2D problems of one size class (helm2d_batch_*): element offset of
    // each problem's f / u block (NULL: one problem); problem b's spectrum rows
    // are b (Nx/2+1) + kx in grp_of_row
    const long long* boff;
    // adjoint solves (the transposed map): first pass reads ubar - sub (sub may
    // be NULL); last pass writes fbar (boundary slots 0), the boundary
    // cotangents (NULL: not wanted) and adds sum(fbar u) into *lam_out (NULL:
    // not wanted; zeroed by the first pass)
    int adjoint;
    const double* sub;
    double* gbar_l;
    double* gbar_r;
    const double* lam_u;
    double* lam_out;
    // 3D pass 1: load each plane of f (and u_obs) with tensor-memory-accelerator
    // copies (16-byte aligned arrays with an even x stride), and
    // the device status word that a copy wait which ran out sets (NULL: none)
    int tma;
    int* err;
    // 3D pass 2 CTA shape: 0 = 16 columns x 256 threads, 1 = 8 columns x 128
    // threads (Ny = 512: 8 or 4 columns, 256 threads)
    int conv_var;
    // 3D passes 1 and 3 (Nx >= 64): each plane on a cluster of two CTAs, half
    // the rows each (the x FFT split by wavenumber parity across the pair)
    int split;
};

// Whether pass 1 can load these arrays with TMA copies (Nx: plane rows).
bool eig_tma_ok(const EigArgs& a, int Nx);

// Whether the pipeline covers a plan of this shape (FP64 arithmetic).
bool eig_shape_ok(int dim, int Nx, int Ny, int P);
// One launch of the pipeline.  3D: pass 0 = GLL transform + x FFT, pass 1 = y
// convolution, pass 2 = inverse x FFT + inverse GLL transform.  2D: pass 0 is
// the whole solve of `nprob` problems (one CTA each); passes 1 and 2 do nothing.
int launch_eig_pass(int pass, int dim, int Nx, const EigArgs& a, int nprob, cudaStream_t s);

}  // namespace helm
