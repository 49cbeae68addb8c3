/*
 * helm_b200.h -- C ABI of the B200 (sm_100a) pseudo-spectral Helmholtz solver.
 *
 * Solves (d2/dx2 + d2/dy2 [+ d2/dz2] - lambda) u = f with Fourier collocation
 * in the periodic directions and Gauss-Lobatto-Legendre (GLL) collocation in the
 * last direction, with Robin conditions alpha du/dn + beta u = g (outward
 * normal) at both ends of the GLL direction:
 *     bottom:  betal u - alphal du/dy = gl        top:  betar u + alphar du/dy = gr
 * exactly as the reference's DirectPseudoSpectral solvers do.  The solve is an
 * FFT along the periodic directions, one collocation system per wavenumber, an
 * element-interface tridiagonal sweep, and the inverse FFT.
 *
 * Every entry point returns an int status (HELM_OK = 0); none aborts.  All
 * array arguments of the solve calls are DEVICE pointers on the plan's device;
 * `stream` is a cudaStream_t passed as void* (NULL = legacy default stream).
 *
 * Array layouts (row-major, GLL index fastest, as the reference stores them):
 *   2D   f, u : [Ns][Nx][N]        gl, gr : [Nx]
 *   3D   f, u : [Ns][Nx][Ny][N]    gl, gr : [Nx][Ny]
 * with the strides of helm_plan_set_layout (default: compact).  The reference's
 * own arrays (rhsPDE[Ns][2Nx][N], U.phi[2Nx][N]; 3D [Ns][2Nx][2Ny][N],
 * leftBC[2Nx][2Ny]) are addressed by passing their strides.  f is read only at
 * the interior GLL nodes of each element, like the reference (its boundary
 * slots carry no equation).
 *
 * Grid convention kept from the reference: the GLL nodes of element jj lie on
 * [jj*L/Ns, (jj+1)*L/Ns] measured from 0 (not from the user's lower bound), and
 * x_i = xl + i*Lx/Nx.  helm_plan_get_grid returns the nodes.
 */
#ifndef HELM_B200_H
#define HELM_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (the reference calls ErrorMessage -> exit(1) instead) ---- */
enum {
    HELM_OK = 0,
    HELM_ERR_INVALID = 1,     /* bad size / argument / NULL pointer                      */
    HELM_ERR_NOT_POW2 = 2,    /* Fourier size not a power of 2 (Fourier_Quadrature.cpp:429-432) */
    HELM_ERR_SINGULAR = 3,    /* a shifted GLL operator is singular (LU_Decomposition.cpp:49-50) */
    HELM_ERR_OOM = 4,         /* device or host allocation failed (General.h:311-312)     */
    HELM_ERR_CUDA = 5,        /* a CUDA call or kernel launch failed                       */
    HELM_ERR_UNSUPPORTED = 6, /* combination not built (e.g. size beyond the kernels' range) */
    HELM_ERR_NO_DEVICE = 7    /* no usable CUDA device                                     */
};

/* ---- arithmetic of the solve ---- */
enum {
    HELM_FP64 = 0,        /* FFTs, back-solves and epilogue in FP64                       */
    HELM_FP32 = 1,        /* everything in FP32 (FP32 factors, FP32 spectrum)             */
    HELM_FP32_REFINE = 2  /* FP64 FFTs; FP32 back-solves with FP64-residual refinement   */
};

/* ---- per-wavenumber solve method ---- */
enum {
    HELM_METHOD_AUTO = 0, /* the autotuner's choice for this shape                        */
    HELM_METHOD_LU = 1,   /* per-wavenumber LU with scaled partial pivoting (the reference's) */
    HELM_METHOD_FDM = 2   /* fast diagonalisation of the interior GLL operator            */
};

typedef struct helm_plan_s* helm_plan_t;

/* Robin coefficients of the two ends of the GLL direction (the reference's
 * globals alphal, betal, alphar, betar; NonPeriodic2D_MPI.h:27). */
typedef struct {
    double alphal, betal, alphar, betar;
} helm_robin_t;

/* Replaces CreatePDEPlan(Nx,Ny,N,xl,xr,yl,yr) + CreateFFTPlan(Nx)
 * (NonPeriodic2D_MPI.h:33, Fourier_Quadrature.h:43) together with the
 * reference's globals Lambda/alphal..betar and its ConstructOperator callback
 * (TestNonPeriodic2D_MPI.cpp:67-74): every shifted operator is built and
 * factored here, once, in FP64.  Ny/N elements: Ns = ceil(Ny/N)
 * (NonPeriodic2D_MPI.cpp:62, one rank).  bc == NULL means Dirichlet (0,1,0,1). */
int helm2d_plan_create(int Nx, int Ny, int N, double xl, double xr, double yl, double yr,
                       const helm_robin_t* bc, double lambda, int precision, int method,
                       helm_plan_t* plan);

/* Replaces CreatePDEPlan(Nx,Ny,Nz,N,xl,xr,yl,yr,zl,zr) + CreateFFTPlan(max(Nx,Ny))
 * (NonPeriodic3D_MPI.h:33) with the operator of TestNonPeriodic3D_MPI.cpp:71-79. */
int helm3d_plan_create(int Nx, int Ny, int Nz, int N, double xl, double xr, double yl, double yr,
                       double zl, double zr, const helm_robin_t* bc, double lambda, int precision,
                       int method, helm_plan_t* plan);

/* Solvers periodic in the GLL direction as well: replaces the CreatePDEPlan of
 * Periodic2D_MPI.h:31 (and Periodic3D_MPI.h:31 for helm3d_periodic_plan_create)
 * with the ConstructOperator of TestPeriodic2D_MPI.cpp:44-51
 * (TestPeriodic3D_MPI.cpp:46-54).  The GLL elements close on themselves: u and
 * its slope are continuous from the last element's right end into the first
 * element's left end (one element: u(0) = u(L), u'(0) = u'(L)), solved by the
 * reference's cyclic interface sweep with its rank-one correction
 * (Periodic2D_MPI.cpp:257-565).  helm_solve takes gl = gr = NULL; the GLL
 * boundary slots of f are not read.  helm_solve_adjoint (Ns = 1) takes
 * glbar = grbar = NULL.  Same size limits as helm2d_plan_create /
 * helm3d_plan_create; lambda > 0 (lambda = 0 leaves the constant mode singular,
 * HELM_ERR_SINGULAR). */
int helm2d_periodic_plan_create(int Nx, int Ny, int N, double xl, double xr, double yl, double yr, double lambda,
                                int precision, int method, helm_plan_t* plan);
int helm3d_periodic_plan_create(int Nx, int Ny, int Nz, int N, double xl, double xr, double yl, double yr,
                                double zl, double zr, double lambda, int precision, int method, helm_plan_t* plan);

/* User operator of a wavenumber pair, the replacement of the reference's
 * ConstructOperator callback (SolvePDE(FieldVariable U[], void
 * (*ConstructOperator)(const int)), NonPeriodic2D_MPI.h:37; (const int, const
 * int) in NonPeriodic3D_MPI.h:37; the periodic twins Periodic2D_MPI.h:35,
 * Periodic3D_MPI.h:35).  The reference calls it once per |iw| (2D) or per
 * (|iw|, |jw|) pair (3D) inside every SolvePDE (NonPeriodic2D_MPI.cpp:239-241,
 * NonPeriodic3D_MPI.cpp:248-253), and the callback fills the interior operator
 * Operator[N-2][N-2] (TestNonPeriodic2D_MPI.cpp:67-74).  Here the callback
 * writes that n x n operator (n = N - 2 interior GLL points) row-major into
 * `op` with leading dimension `ld`, for iw = 0 .. Nx/2 and (3D) jw = 0 .. Ny/2
 * (2D: jw = 0); `user` is passed through.  The operator of -iw (and -jw) is
 * taken to be the same, as the reference's loop over |iw| assumes. */
typedef void (*helm_operator_fn)(int iw, int jw, double* op, int ld, void* user);

/* Replaces the plan's shifted operators D2int - sigma I by the callback's, one
 * per wavenumber pair: the callback runs now, once per pair, on the calling
 * thread (serially), each operator is LU-factored in FP64 with the
 * reference's scaled partial pivoting, and later solves use those factors
 * (the LU method; the boundary columns, interface sweep and Robin rows stay
 * the GLL ones).  Rebuilds the plan in place: its handle, layout, I/O width
 * and refinement count are kept, the launch variants are re-tuned.  FP64 and
 * FP32 plans (refined plans have no residual for a foreign operator:
 * HELM_ERR_UNSUPPORTED), non-periodic or periodic, not finite-difference
 * plans.  A singular operator gives HELM_ERR_SINGULAR and leaves the plan as
 * it was.  Adjoint solves of such a plan are HELM_ERR_UNSUPPORTED. */
int helm_plan_set_operator_callback(helm_plan_t plan, helm_operator_fn op, void* user);

/* The GLL grid of one direction as the reference's CreatePDEPlan builds it
 * (NonPeriodic2D_MPI.cpp:88-123): nodes[Ns*(N-1)+1] of Ns elements of length
 * L/Ns placed from 0, the first-derivative matrix D[N][N] scaled by 2Ns/L
 * (FirstDerivativeMatrix, GLLQuadrature.cpp:198-213) and D2 = D D scaled by
 * 4Ns^2/L^2 (SecondDerivativeMatrix, GLLQuadrature.cpp:250-262).  Host only:
 * no device, no plan.  Any pointer may be NULL. */
int helm_gll_grid(int N, int Ns, double L, double* nodes, double* D, double* D2);

/* FP64 LU with scaled partial pivoting of a dense row-major n x n matrix in
 * place -- the pivot rule of the reference's LUDecomposition
 * (LU_Decomposition.cpp:7-72) -- stored as P A = L U (unit L below the
 * diagonal, U on and above it; perm[i] = the original row of position i) with
 * the determinant (may be NULL); HELM_ERR_SINGULAR below a scaled pivot of
 * 1e-12.  helm_lu_solve solves A x = b with those factors, b overwritten
 * (LUSolve, LU_Decomposition.cpp:78-108).  Host only. */
int helm_lu_factor(int n, double* A, int* perm, double* determinant);
int helm_lu_solve(int n, const double* LU, const int* perm, double* b);

/* max |a - b| over the solution points of a (single-problem) plan's arrays --
 * every element, x row and GLL node of the plan's layout, the 3D y index
 * included -- reduced on the device into *result (a DEVICE double, written on
 * `stream`; a NaN anywhere gives NaN).  The device form of the reference's
 * ComputeError (NonPeriodic2D_MPI.cpp:547-566, NonPeriodic3D_MPI.cpp:688-708),
 * which takes a = the solution and b = the exact values. */
int helm_max_abs_diff(helm_plan_t plan, const double* a, const double* b, double* result, void* stream);

/* Second-order finite-difference variant: the 7-point stencil of the
 * reference's HypreFDM solver (HelmholtzSolvers/HypreFDM/src/Helmholtz3D_MPI.cpp:
 * CreatePDEPlan 117-269, SetA 297-410, Setb 424-466) with x and y periodic
 * (dx = Lx/Nx, dy = Ly/Ny) and Nz interior points in z (dz = Lz/(Nz+1)), solved
 * directly: FFT in x and y, one Thomas solve along z per wavenumber, inverse
 * FFT (the reference solves the same system iteratively with HYPRE).  bc gives
 * the Robin coefficients of the back (z = zl: alphal, betal) and front (z = zr:
 * alphar, betar) rows, with the reference's one-sided second-order rows.
 * Arrays: f, u [Nx][Ny][Nz] interior points; gl = back data, gr = front data,
 * [Nx][Ny].  helm_solve / helm_solve_adjoint / helm_plan_destroy apply.
 * HELM_FP32_REFINE plans solve in FP32 (FP32 spectrum and tridiagonal solves,
 * FP64 arrays in and out) and refine: per sweep (2 by default,
 * helm_plan_set_refine_sweeps) the residual f - A_h u of the stencil in FP64
 * and an FP32 solve of its correction, added to u; the adjoint refines the same
 * way with the transposed stencil (fbar, the boundary cotangents and
 * lambda_bar).  Each sweep multiplies the error by about the FP32 solve's
 * relative error. */
int helm_fd3d_plan_create(int Nx, int Ny, int Nz, double xl, double xr, double yl, double yr, double zl, double zr,
                          const helm_robin_t* bc, double lambda, int precision, helm_plan_t* plan);

/* Strides (in elements) of f/u and of gl/gr; 0 keeps the compact value.
 *   x_stride    : between consecutive x rows of f and u   (compact: N in 2D, Ny*N in 3D)
 *   elem_stride : between consecutive GLL elements         (compact: Nx*x_stride)
 *   bc_x_stride : 3D only, between x rows of gl and gr     (compact: Ny)
 * The reference's own arrays: 2D x_stride=N, elem_stride=2*Nx*N;
 * 3D x_stride=2*Ny*N, elem_stride=2*Nx*2*Ny*N, bc_x_stride=2*Ny. */
int helm_plan_set_layout(helm_plan_t plan, long long x_stride, long long elem_stride, long long bc_x_stride);

/* Element type of f and u for HELM_FP32 plans: 8 (double, default) or 4 (float).
 * FP64 and FP32_REFINE plans always read and write double. */
int helm_plan_set_io_bytes(helm_plan_t plan, int bytes);

/* Number of refinement sweeps of a HELM_FP32_REFINE plan (default 1, 0..8). */
int helm_plan_set_refine_sweeps(helm_plan_t plan, int sweeps);

/* SolvePDE(U, ConstructOperator) (NonPeriodic2D_MPI.cpp:228-474,
 * NonPeriodic3D_MPI.cpp:237-591): u = solution, device pointers.  Unlike the
 * reference, f is not overwritten by its spectrum.  gl/gr may be NULL (zero
 * boundary data).  Asynchronous on `stream`. */
int helm_solve(helm_plan_t plan, const void* f, const double* gl, const double* gr, void* u, void* stream);

/* Adjoint of helm_solve as a linear map (f, gl, gr) -> u.  Given ubar = dL/du
 * (same layout as u), writes fbar = dL/df (zero on the GLL boundary slots, which
 * the solve never reads), glbar = dL/dgl, grbar = dL/dgr (any may be NULL), and,
 * when lambda_bar != NULL, the scalar
 *     dL/dlambda = sum over the interior collocation nodes of fbar * u
 * (d(A u)/d lambda = -u on the interior rows, so du/dlambda = A^-1 u), where u
 * must be the forward solution of the same plan; the sum is written to the
 * DEVICE double *lambda_bar.  Plans with the FDM method (one GLL element, or
 * several elements not periodic in the GLL direction) and finite-difference
 * plans; LU plans (operator callbacks) return HELM_ERR_UNSUPPORTED.  No
 * counterpart in the reference, which has no gradients. */
int helm_solve_adjoint(helm_plan_t plan, const double* ubar, double* fbar, double* glbar, double* grbar,
                       const double* u, double* lambda_bar, void* stream);

/* The adjoint of the least-squares loss L = 1/2 ||u - u_obs||^2 in one call:
 * helm_solve_adjoint with ubar = u - u_obs, formed as the first pass loads its
 * input (no ubar array, no separate kernel); u must be the forward solution of
 * the same plan (it is also the u of dL/dlambda).  Outputs as helm_solve_adjoint.
 * No counterpart in the reference, which has no gradients. */
int helm_solve_adjoint_misfit(helm_plan_t plan, const double* u, const double* u_obs, double* fbar, double* glbar,
                              double* grbar, double* lambda_bar, void* stream);

/* Derivative along the GLL direction, element by element: du = Dy u (order 1)
 * or Dyy u (order 2) with the plan's scaled matrices (helm_plan_get_grid), at
 * every node of every Fourier row.  Replaces FirstDerivativeY /
 * SecondDerivativeY of the 2D solvers (NonPeriodic2D_MPI.cpp:497-542,
 * Periodic2D_MPI.cpp:714-763) and FirstDerivativeZ / SecondDerivativeZ of the 3D
 * ones (NonPeriodic3D_MPI.cpp:632-683, Periodic3D_MPI.cpp:905-957).  u, du: the
 * plan's layout and io type (helm_plan_set_layout / helm_plan_set_io_bytes),
 * device pointers; du may equal u.  Not for finite-difference plans. */
int helm_gll_derivative(helm_plan_t plan, int order, const void* u, void* du, void* stream);

/* Spectral derivative along a Fourier direction: axis 0 = x, axis 1 = y (3D
 * plans) of a real field in the plan's layout: forward FFT along the axis,
 * multiplication by (2 pi i K / L)^order with K = k below L/2 and K = -L/2 at
 * the Nyquist index, inverse FFT, real part.  Replaces FirstDerivativeFourierX
 * / FirstDerivativeFourierY and SecondDerivativeFourierX / ...Y
 * (Fourier_Quadrature.cpp:1387-1834) on the solver's arrays (the reference's
 * solver-level FirstDerivativeX of NonPeriodic2D_MPI.cpp:479-483 is an empty
 * stub).  Every GLL node is differentiated, boundary slots included; du must
 * not overlap u.  Uses the plan's spectrum scratch: do not run it concurrently
 * with a solve of the same plan on another stream. */
int helm_fourier_derivative(helm_plan_t plan, int axis, int order, const void* u, void* du, void* stream);

/* Output writers (host code; u is a HOST array in the plan's compact layout):
 * the reference's WriteFile (NonPeriodic2D_MPI.cpp:571-650,
 * NonPeriodic3D_MPI.cpp:713-795, and the Periodic twins) in the same text
 * format -- fixed notation, 8 decimals, tab-separated, x fastest, then y, then
 * the GLL node of each element (element boundaries twice).  helm_write_tecplot
 * writes the TECPLOT branch (columns X, Y, [Z,] U, Exact; `exact` may be NULL
 * for zeros, 2D plans get z = 0); helm_write_vtk the VISIT branch (legacy VTK
 * structured grid, scalar Phi).  The reference picks the file name from its
 * rank ("Output/Solution-%04d.tec"); here the caller passes `path`. */
int helm_write_tecplot(helm_plan_t plan, const double* u, double (*exact)(double x, double y, double z),
                       const char* path);
int helm_write_vtk(helm_plan_t plan, const double* u, const char* path);

/* Node coordinates: 2D y[Ns*(N-1)+1] / 3D z[...], and the scaled first and
 * second GLL derivative matrices D[N*N], D2[N*N] (row-major), host pointers,
 * any may be NULL.  The reference's globals y/z, Dy/Dz, Dyy/Dzz. */
int helm_plan_get_grid(helm_plan_t plan, double* nodes, double* D, double* D2);

/* Plan facts: Ns, the number of distinct shifted operators, the method the
 * plan runs, and the device bytes it holds. */
int helm_plan_info(helm_plan_t plan, int* Ns, int* n_operators, int* method, long long* device_bytes);

/* Stage timing: when enabled, helm_solve and helm_solve_adjoint record CUDA events on their stream
 * around each of its kernels; helm_plan_stage_times then waits for the last
 * solve and returns the five stage durations in ms: x-FFT, y-FFT, row solves,
 * inverse y-FFT, inverse x-FFT (y stages are 0 in 2D).  The reference times
 * only the whole SolvePDE with a host clock (TestNonPeriodic2D_MPI.cpp:103-131). */
int helm_plan_set_stage_timing(helm_plan_t plan, int enable);
int helm_plan_stage_times(helm_plan_t plan, float* ms5);

/* Device status of the plan's tensor-memory-accelerator and bulk copies (the
 * first pass of the 3D eigen-basis pipeline: code 1; the GLL derivative of
 * FP64 arrays in the packed layout: code 8): 0, or the code of a wait on a
 * copy that ran out of its iteration limit (the kernel then skipped that work,
 * so that call's output is not valid).  Waits for the device; reset != 0
 * clears the word afterwards.  Plans without such copies report 0.  No
 * counterpart in the reference. */
int helm_plan_device_status(helm_plan_t plan, int* code, int reset);

/* Kernel launch variants of the plan: fft4[i] (0..15) for the x, y, inverse y
 * and inverse x FFT passes -- bit 0: 128-thread CTAs, bit 1: radix-8 schedule
 * (lengths 128, 256), bit 2: persistent pipelined pass, bit 3: 512-thread CTAs
 * for passes of length 512 or 1024 (ignored for shorter ones; with bit 2 the
 * tile exceeds shared memory and the solve fails with HELM_ERR_CUDA) -- and rows (0..4) for
 * the row solve: 0, 1 the two kernel shapes of the plan's precision (finite-
 * difference plans: a tridiagonal row per warp, or per half-warp when Nz <= 256); 2 (FP64 and
 * refined 3D plans with one element, at most 65 GLL points and Ny in {64, 128,
 * 256}) the y pass, the row solve and the inverse y pass fused into one kernel
 * per kx slab, the two y entries of fft4 then unused; 3 (refined plans with one
 * element) the FP64 tensor-core row kernel on the refined plan's FP64 spectrum;
 * 4 (FP64 and refined plans with one element, Dirichlet ends, at most 66 GLL
 * points, Nx in {8, ..., 256}, Ny in {4, ..., 512}, powers of 2) the eigen-basis
 * pipeline of the whole forward solve -- GLL eigen-transform fused with the x
 * FFT, the y FFT, diagonal scaling and inverse y FFT in one pass, and the
 * inverse of the first pass: three kernels in 3D, one in 2D; in 3D bit 0 of
 * fft4[1] picks the CTA shape of the middle pass and bit 1 (Nx >= 64) runs the
 * first and last passes on pairs of CTAs, each holding half of a plane (the
 * other fft4 entries are unused); adjoint solves run the transposed pipeline.  Plan creation times every
 * variant on the plan's own shape and keeps the fastest (environment
 * HELM_AUTOTUNE=0: all 0, rows 4 where it applies).  Setting them
 * pins the choice, e.g. to reproduce a run bit for bit.  Every variant
 * computes the same solve; the last bits of the results may differ between
 * variants.  No counterpart in the reference, which has one code path. */
int helm_plan_get_launch_variants(helm_plan_t plan, int* fft4, int* rows);
int helm_plan_set_launch_variants(helm_plan_t plan, const int* fft4, int rows);

/* Launch variant of the spectral derivative passes (helm_fourier_derivative),
 * with the bits of the FFT variants above (bit 2: the persistent pipelined
 * kernel).  -1, the default, picks by transform length and precision:
 * 512-thread CTAs from length 512; below, the radix-8 schedule, pipelined for
 * FP32 plans.  Pipelined shapes whose tile buffers exceed shared memory are
 * refused with HELM_ERR_CUDA and launch nothing.  Every
 * variant computes the same derivative up to the last bits.  No counterpart in
 * the reference, which has one code path. */
int helm_plan_set_derivative_variant(helm_plan_t plan, int variant);
int helm_plan_get_derivative_variant(helm_plan_t plan, int* variant);

/* The kernels a forward helm_solve of the plan launches, as a short
 * space-separated list of kernel names in launch order (for reports: which
 * row kernel ran, e.g. whether a refined plan ran its FP32 tensor-core kernel or
 * the FP64 one).  The string stays valid until the plan is destroyed or its
 * variants change.  No counterpart in the reference. */
const char* helm_plan_kernels(helm_plan_t plan);

/* Test hook for the out-of-memory paths (host-side fault injection): with
 * n >= 0 the n-th device allocation made by plan creation from now on (0: the
 * next) fails as a failed cudaMalloc would -- the call returns HELM_ERR_OOM
 * after freeing what it had allocated -- and the hook disarms itself; n < 0
 * disarms it.  The reference exits on allocation failure (General.h:320-392,
 * no status); this hook has no counterpart there. */
int helm_debug_fail_alloc(long long n);

/* helm_solve with the spectrum workspace taken from a fixed 16 MiB device
 * array inside this library instead of the plan's buffer; the call allocates
 * no device memory.  For callers whose memory manager owns the device memory
 * or whose device footprint must stay fixed after start-up.  Plans whose
 * spectrum needs more than 16 MiB get HELM_ERR_UNSUPPORTED.  The first call on
 * a device looks up the array's address and should come before any stream
 * capture; calls that overlap on the GPU share the array and race.  No
 * counterpart in the reference. */
int helm_solve_static_scratch(helm_plan_t plan, const void* f, const double* gl, const double* gr, void* u,
                              void* stream);

/* ---- batches of independent 2D problems of uneven sizes ----
 * No counterpart in the reference, which solves one problem per plan
 * (NonPeriodic2D_MPI.h:33-37).  Problem p is the 2D problem of
 * helm2d_plan_create with Nx[p] Fourier modes, one GLL element of N[p] points,
 * lambda[p], homogeneous Dirichlet rows in y, on the common domain
 * [xl, xr) x [yl, yr].  f and u are packed: problem p is the compact
 * [Nx[p]][N[p]] block at element offset sum_{q<p} Nx[q] N[q].
 * FP64 and refined batches whose problems all have Nx in 8 .. 512 and 4 .. 129
 * GLL points run as ONE persistent kernel launch (after one memset of its work
 * queue): every problem is solved in the eigen basis of its GLL operator, cut
 * into row, column and row items that persistent CTAs take from one ordered
 * queue (FP64 arithmetic; a refined batch computes in FP64 throughout).
 * Other batches (FP32, or sizes outside that range) group their problems into
 * size classes (Nx, N), three kernels per class covering all its problems.
 * helm_batch_solve runs the solve as one CUDA graph with a single
 * cudaGraphLaunch on `stream` (the size classes on concurrent streams inside
 * it).  The graph is captured at the first call and again whenever f or u
 * differ from the last call's.  Calls on one batch whose kernels overlap on the
 * GPU race on its workspace: serialise them. */
typedef struct helm_batch_s* helm_batch_t;

int helm2d_batch_create(int nprob, const int* Nx, const int* N, const double* lambda, double xl, double xr,
                        double yl, double yr, int precision, helm_batch_t* batch);

/* Element offsets of the problems in the packed buffers (host array of nprob,
 * may be NULL) and the packed length. */
int helm_batch_offsets(helm_batch_t batch, long long* offsets, long long* total_elems);

/* Distinct problem sizes (Nx, N), kernel launches inside one solve (1 for the
 * persistent launch), device bytes held. */
int helm_batch_info(helm_batch_t batch, int* n_classes, int* kernels_per_solve, long long* device_bytes);

/* Status word of the persistent batch kernel: 0, or 7 when a wait of an item
 * for the items it depends on ran out of its iteration limit (that solve's
 * output is not valid).  Waits for the device; reset != 0 clears it. */
int helm_batch_device_status(helm_batch_t batch, int* code, int reset);

/* enable = 0: helm_batch_solve launches its kernels directly on `stream`
 * (the classes one after another) instead of through the graph (default 1). */
int helm_batch_set_graph(helm_batch_t batch, int enable);

/* u = solution of every problem; f, u DEVICE double arrays of the packed length. */
int helm_batch_solve(helm_batch_t batch, const double* f, double* u, void* stream);

int helm_batch_destroy(helm_batch_t batch);

/* Replaces DestroyPDEPlan() + DestroyFFTPlan(). NULL is accepted. */
int helm_plan_destroy(helm_plan_t plan);

/* Human-readable status text (static storage). */
const char* helm_status_string(int status);

/* Last CUDA error text recorded by this library on the calling thread. */
const char* helm_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* HELM_B200_H */
