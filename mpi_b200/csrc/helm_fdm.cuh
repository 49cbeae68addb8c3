// Arguments of the folded fast-diagonalisation row solve (helm_fdm.cu).
#pragma once
#include <cstddef>
#include <cuda_runtime.h>

namespace helm {

struct FdmArgs {
    void* spec;          // complex spectrum rows [nrows_total][P]
    int P, n, m, ms, ma; // GLL points, interior n = P-2, m = n/2, ms = m + n%2, ma = m
    int ld;              // padded fold length (32 * ceil(ms/32))
    int nrows;           // rows to solve
    const int* rows;     // spectrum row of each work item (grouped by shift)
    const int* row_grp;  // shift group of each work item
    const void* mats;    // 4 column-major ld x ld blocks: first/second transform of the
                         // symmetric block, then of the antisymmetric block
    const double* d2f;   // refinement: the folded blocks of D2int (column-major), 2 x ld*ld
    const void* recip;   // [groups][2][ld]: 1/(lambda_s - sigma), 1/(lambda_a - sigma)
    const double* sigma; // [groups]
    int sweeps;
    const double* e0f;   // [2][ld] folded weights of the first boundary functional
    const double* eNf;   // [2][ld] folded weights of the second
    const double* hvec;  // [groups][2][P] vectors combined with the boundary values (NULL: none)
    const double* hscal; // [groups][4] scalars of the boundary system
    int hzero;           // hvec is zero: skip its reads (boundary values still computed)
    double al, bl, ar, br;
    int adjoint;
    // periodic in the GLL direction (one element): u(0) = u(L) = zeta with
    // matching slopes; hscal then holds D0.ul, D0.ur, DN.ul, DN.ur in both
    // directions, and the adjoint's hvec the interior vectors A^-T (DN - D0), 0
    int periodic;
    // FP64 tensor-core variant: the four transforms of `mats` in mma.sync
    // m8n8k4 A-fragment order, [4][ld/8][ld/4][32] (NULL: not prepared)
    const double* mma_mats;
    const double* mma16_mats;  // the same transforms in m16n8k8 fragment order, [4][ld/16][ld/8][32][4]
    // refined plans with ld = 32: the transforms split into TF32 hi + lo, and the
    // folded D2int blocks in f64 fragment order (launch_fdm_tc_refine)
    const void* tc_mats;
    const double* tc_m;
};

int launch_fdm_fast(int prec, const FdmArgs& a, cudaStream_t s, int variant = 0);
size_t fdm_fast_smem_bytes(int prec, int ld);
// FP64 plans: the folded solve with its transforms on the FP64 tensor cores.
int launch_fdm_mma(const FdmArgs& a, cudaStream_t s, int variant = 0);
// The transforms `cm` (4 column-major ld x ld blocks) in the A-fragment order
// launch_fdm_mma reads.
void fdm_mma_swizzle(const double* cm, int ld, double* out);
void fdm_mma16_swizzle(const double* cm, int ld, double* out);
// Refined plans (ld = 32, one sweep): FP32-accurate solves as three TF32
// tensor products, FP64 residual on the FP64 tensor cores.
int launch_fdm_tc_refine(const FdmArgs& a, cudaStream_t s);
// FP64 3D plans with Ns = 1, ld = 32 and Ny in {64, 128, 256}: y-FFT, row solve
// and inverse y-FFT fused per kx slab in a cluster of two CTAs.  H0 = (P + 1) / 2
// GLL columns in the first CTA; HS its shared-memory row stride (odd);
// grp_of_row: the shift group of each spectrum row.
int launch_slab(const FdmArgs& a, int Ny, int H0, int HS, const void* tw, const int* grp_of_row, int nkx,
                cudaStream_t s);
bool slab_fits(int Ny, int P, int ld);
void fdm_tc_swizzle(const double* cm, int ld, float* out);    // [4][2][ld/16][ld/8][32][4]
void fdm_m16_swizzle2(const double* cm, int ld, double* out);  // [2 blocks][2 planes][ld/16][ld/8][32][2]

}  // namespace helm
