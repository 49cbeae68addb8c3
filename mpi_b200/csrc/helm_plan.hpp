// The plan object behind helm_plan_t (include/helm_b200.h).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/helm_b200.h"
#include "helm_setup.hpp"

namespace helm {

struct Plan {
    int dim = 2;                 // 2: Fourier x GLL, 3: Fourier x Fourier x GLL
    int Nx = 0, Ny = 1, N = 0, Ns = 1, n = 0;
    int nslot = 1, ld = 32;      // 32-lane slots per interior vector, padded length
    double xl = 0, xr = 1, yl = 0, yr = 1, zl = 0, zr = 1;
    double Lx = 1, Ly = 1, Lgll = 1;
    helm_robin_t bc{0.0, 1.0, 0.0, 1.0};
    bool periodic = false;       // periodic in the GLL direction (no boundary data)
    // user operators (helm_plan_set_operator_callback): per wavenumber pair, in
    // place of D2int - sigma I; the plan then runs the LU method
    helm_operator_fn op_cb = nullptr;
    void* op_user = nullptr;
    double lambda = 0;
    int precision = HELM_FP64, method = HELM_METHOD_AUTO;
    int io_bytes = 8, sweeps = 1;
    long long x_stride = 0, elem_stride = 0, bc_x_stride = 0;
    int device = 0;
    GllSetup gll;

    // rows grouped by shift
    int ngroups = 0;
    long long nrows = 0, elem_spec = 0;
    std::vector<int> grp_start, grp_rows, grp_iw, grp_jw;
    std::vector<double> sigma;
    std::vector<double> h_lam, h_V, h_Vi;

    // device memory
    void* d_spec = nullptr;
    size_t spec_bytes = 0, cprime_bytes = 0;
    void* d_tw_x = nullptr;
    void* d_tw_y = nullptr;
    int* d_grp_start = nullptr;
    int* d_grp_rows = nullptr;
    double* d_sigma = nullptr;
    void* d_fac = nullptr;
    void* d_dinv = nullptr;
    uint8_t* d_perm = nullptr;
    void* d_vinvT = nullptr;
    void* d_vT = nullptr;
    double* d_lam = nullptr;
    double* d_hom = nullptr;
    double* d_homs = nullptr;
    double* d_d0 = nullptr;
    double* d_dN = nullptr;
    double* d_d2t = nullptr;
    double* d_Dfull = nullptr;   // [N][N] scaled first-derivative matrix (derivative helpers)
    double* d_D2full = nullptr;  // [N][N] second-derivative matrix
    // adjoint (transposed) solve data, FDM plans with one element
    bool adj_ready = false;
    void* d_vtT = nullptr;        // column-major V^T
    void* d_vinvtT = nullptr;     // column-major V^-T
    double* d_d2row = nullptr;    // column-major D2int^T (= row-major D2int)
    double* d_c0 = nullptr;       // [P] D2[int][0] in the interior slots
    double* d_cN = nullptr;       // [P] D2[int][N-1]
    double* d_hom_adj = nullptr;  // [G][2][P] pl, pr
    double* d_homs_adj = nullptr; // [G][4] 2x2 boundary matrix
    // folded fast-diagonalisation path (FDM plans with one element)
    bool fast = false;
    int fm = 0, fms = 0, fma = 0, fld = 32;
    void* d_fmats = nullptr;       // forward transforms [4][fld][fld]
    void* d_fmats_adj = nullptr;   // transposed transforms
    double* d_fmma = nullptr;      // FP64 plans: the transforms in tensor-core fragment order
    double* d_fmma_adj = nullptr;
    double* d_fmma16 = nullptr;    // the same in m16n8k8 fragment order
    double* d_fmma16_adj = nullptr;
    float* d_ftc = nullptr;        // refined plans: TF32 hi/lo transforms (tensor-core refine)
    float* d_ftc_adj = nullptr;
    double* d_ftcm = nullptr;      // folded D2int blocks, f64 fragment order
    double* d_ftcm_adj = nullptr;
    double* d_fd2 = nullptr;       // folded D2int blocks (refinement)
    double* d_fd2_adj = nullptr;   // their transposes
    void* d_frecip = nullptr;      // [G][2][fld] reciprocal shifts
    int* d_row_grp = nullptr;      // group of each grouped row
    double* d_fe0 = nullptr;       // folded D[0][int], D[N-1][int]
    double* d_feN = nullptr;
    double* d_fc0 = nullptr;       // folded D2[int][0], D2[int][N-1]
    double* d_fcN = nullptr;
    // batched independent 2D problems of one size class (helm_batch_*): their
    // lambdas, and the element offsets of each problem in the caller's packed
    // f / u buffers
    int batch = 1;
    std::vector<double> lambdas;
    long long* d_boff = nullptr;
    long long packed_elems = 0;  // length of the caller's packed buffers
    // finite-difference variant (FFT in x and y, Thomas along z)
    bool fd = false;
    double fd_cz1 = 0, fd_dfirst = 0, fd_sfirst = 0, fd_dlast = 0, fd_slast = 0;
    double fd_scale_l = 0, fd_scale_r = 0;  // weights of gl / gr in the first / last equation
    double* d_mx = nullptr;
    double* d_my = nullptr;
    void* d_cprime = nullptr;
    // HELM_FP32_REFINE finite-difference plans: FP32 internals with FP64
    // residual sweeps, and their FP32 residual / correction array
    bool fd_refine = false;
    void* d_refine = nullptr;
    size_t refine_bytes = 0;
    // autotuned launch shapes of the four FFT stages (x, y, inverse y, inverse x)
    int fft_var[4] = {0, 0, 0, 0};
    // launch variant of the spectral derivative passes (-1: chosen by length)
    int deriv_var = -1;
    // row-solve variant: 0, 1 launch shapes of the plan precision's folded kernel;
    // 2 fused y-FFT / rows / inverse y (slab, FP64 arithmetic); 3 refined plans:
    // the FP64 tensor-core row kernel; 4 the eigen-basis pipeline (whole solve)
    int row_var = 0;
    bool slab_ok = false;          // FP64 3D plans whose kx slab fits a two-CTA cluster
    // eigen-basis pipeline (helm_eig.cu; row variant 4): one element, Dirichlet
    // ends, FP64 arithmetic (FP64 and refined plans)
    bool eig_cand = false;         // shape and boundary conditions allow it
    bool eig_ok = false;           // its data are on the device
    double* d_hbc = nullptr;       // [4][32] first transform of the folded boundary columns
    double* d_frecip64 = nullptr;  // FP64 reciprocal shifts (refined plans; FP64 plans use d_frecip)
    int* d_grp_of_row = nullptr;   // shift group of each spectrum row (slab kernel)
    // device status word of the eigen-basis pipeline's TMA loads: a bounded wait
    // that ran out sets it to a nonzero code (helm_plan_device_status)
    int* d_status = nullptr;
    bool stage_timing = false;
    cudaEvent_t ev[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    std::string kernel_names;       // helm_plan_kernels
    std::vector<void*> allocations;
    long long device_bytes = 0;

    int alloc(void** p, size_t bytes);
    int upload(void** p, const void* host, size_t bytes);
    void release();
};

// Scratch that one solve writes: the spectrum workspace and, for
// finite-difference plans whose Nz exceeds the one-warp tridiagonal kernel, the
// forward-elimination coefficients.  A solve given no workspace uses the plan's
// own buffers; the plan itself is never modified by a solve.
struct Workspace {
    void* spec = nullptr;
    void* cprime = nullptr;
    void* refine = nullptr;
};

// Bytes of spectrum and elimination scratch a solve of this plan writes.
size_t spec_bytes(const Plan& p);
size_t cprime_bytes(const Plan& p);
size_t refine_bytes(const Plan& p);

// Argument checks shared by every solve entry point (status, last error set).
int check_solve_args(const Plan& p, const void* f, const double* gl, const double* gr, const void* u);

int solve(Plan& p, const void* f, const double* gl, const double* gr, void* u, cudaStream_t s,
          const Workspace* ws = nullptr);

// One size class of a batch: `lams.size()` independent 2D problems with Nx
// Fourier modes and N GLL points on one domain, homogeneous Dirichlet in y,
// stored in the caller's packed buffers at element offsets `offs`.
int create_batch_class(int Nx, int N, double xl, double xr, double yl, double yr, const std::vector<double>& lams,
                       const std::vector<long long>& offs, long long packed_elems, int precision, Plan** out);
void set_last_error(const char* msg);
// The host-side allocation fault hook (helm_debug_fail_alloc): true when the
// caller's next device allocation is to fail (the last error then says so).
bool alloc_fault_fires();

}  // namespace helm
