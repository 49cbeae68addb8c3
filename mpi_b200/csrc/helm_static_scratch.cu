// helm_solve_static_scratch: the solve of helm_solve with its spectrum
// workspace taken from a fixed, file-scope device array instead of the plan's
// own buffer, for callers that must not allocate device memory at call time.
//
// Who needs it: applications whose own memory manager has taken the device
// memory (a cudaMalloc on the solve path would fail or fragment its pool), and
// services that must keep their device footprint fixed after start-up.  Such a
// caller creates its plan once at start-up and afterwards only solves; the
// plan's setup still allocates, the solve call does not.
//
// Limits and behaviour:
//   * The workspace is kHelmStaticScratchBytes = 16 MiB per device; a plan whose
//     spectrum (plus, for finite-difference plans with more than 512 points in
//     z, its elimination coefficients, and for refined finite-difference plans
//     their residual array) needs more is rejected with
//     HELM_ERR_UNSUPPORTED.  Every GPU that
//     loads this library holds the 16 MiB until the process exits.
//   * The first call on a device looks up the array's device address
//     (cudaGetSymbolAddress) with that device current; make that first call
//     before any stream capture.
//   * All calls share the one array and it keeps the last call's contents.
//     Nothing in it has to start at zero: a solve writes every element it later
//     reads.  Two calls of this entry point whose kernels overlap on the GPU
//     (different streams, or different host threads) race on the array;
//     serialise them.  The plan object is only read, so helm_solve and the
//     other entry points may use the same plan concurrently with this call.
//   * Argument checks are those of helm_solve (plans periodic in the GLL
//     direction take no boundary data).
//   * The call itself allocates nothing: no cudaMalloc, cudaFree or allocating
//     library routine.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/helm_b200.h"
#include "helm_plan.hpp"

namespace helm {

constexpr size_t kHelmStaticScratchBytes = 16u << 20;  // 16 MiB
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_helm_static_scratch[kHelmStaticScratchBytes];

static std::mutex g_scratch_mutex;
static void* g_scratch_addr[kMaxDevices] = {nullptr};

// Device address of the array on `device` (current), looked up once per device.
static int static_scratch_address(int device, void** out)
{
    if (device < 0 || device >= kMaxDevices) {
        set_last_error("device ordinal out of range for the static scratch table");
        return HELM_ERR_INVALID;
    }
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_addr[device]) {
        void* ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_helm_static_scratch);
        if (e != cudaSuccess || !ptr) {
            cudaGetLastError();
            set_last_error((std::string("cudaGetSymbolAddress of the static scratch: ") +
                            (e != cudaSuccess ? cudaGetErrorString(e) : "null address"))
                               .c_str());
            return HELM_ERR_CUDA;
        }
        g_scratch_addr[device] = ptr;
    }
    *out = g_scratch_addr[device];
    return HELM_OK;
}

}  // namespace helm

extern "C" int helm_solve_static_scratch(helm_plan_t plan, const void* f, const double* gl, const double* gr, void* u,
                                         void* stream)
{
    if (!plan) return HELM_ERR_INVALID;
    helm::Plan& p = *reinterpret_cast<helm::Plan*>(plan);
    if (int st = helm::check_solve_args(p, f, gl, gr, u)) return st;
    // the spectrum, then (finite-difference plans with long z lines) the
    // elimination coefficients, each at a 256-byte boundary
    const size_t spec = (helm::spec_bytes(p) + 255) & ~(size_t)255;
    const size_t cpr = (helm::cprime_bytes(p) + 255) & ~(size_t)255;
    const size_t need = spec + cpr + helm::refine_bytes(p);
    if (need > helm::kHelmStaticScratchBytes) {
        helm::set_last_error("plan needs more than the 16 MiB static scratch");
        return HELM_ERR_UNSUPPORTED;
    }
    int cur = 0;
    if (cudaGetDevice(&cur) != cudaSuccess) {
        cudaGetLastError();
        helm::set_last_error("cudaGetDevice failed");
        return HELM_ERR_CUDA;
    }
    if (cur != p.device && cudaSetDevice(p.device) != cudaSuccess) {
        cudaGetLastError();
        helm::set_last_error("cudaSetDevice to the plan's device failed");
        return HELM_ERR_CUDA;
    }
    void* scratch = nullptr;
    int st = helm::static_scratch_address(p.device, &scratch);
    if (st == HELM_OK) {
        // the plan is only read: its own workspace stays in place for other calls
        helm::Workspace ws;
        ws.spec = scratch;
        ws.cprime = helm::cprime_bytes(p) ? static_cast<unsigned char*>(scratch) + spec : nullptr;
        ws.refine = helm::refine_bytes(p) ? static_cast<unsigned char*>(scratch) + spec + cpr : nullptr;
        st = helm::solve(p, f, gl, gr, u, static_cast<cudaStream_t>(stream), &ws);
    }
    if (cur != p.device) cudaSetDevice(cur);
    return st;
}
