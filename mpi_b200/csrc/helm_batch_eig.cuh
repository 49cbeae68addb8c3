// Batches of independent 2D problems in one persistent launch (helm_batch_eig.cu).
#pragma once
#include <cuda_runtime.h>

namespace helm {

struct BatchEig;

// Tables of the one-launch batch solve, or HELM_ERR_UNSUPPORTED (*out = NULL,
// last error set) when a problem lies outside its range (Nx of 8 .. 512, at
// most 129 GLL points) or its shifted operator is singular.  offs: element
// offsets of the problems in the packed f / u buffers.
int batch_eig_create(int nprob, const int* Nx, const int* N, const double* lambda, double xl, double xr, double yl,
                     double yr, const long long* offs, int device, BatchEig** out);
// One solve: a reset of the work queue (one memset) and one kernel launch.
int batch_eig_solve(BatchEig* be, const double* f, double* u, cudaStream_t s);
long long batch_eig_device_bytes(const BatchEig* be);
// Device status word: nonzero when a dependency wait of the kernel ran out.
int* batch_eig_status(BatchEig* be);
void batch_eig_destroy(BatchEig* be);

}  // namespace helm
