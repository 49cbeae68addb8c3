// Batched independent 2D solves of uneven sizes (helm2d_batch_* of
// include/helm_b200.h).
//
// The problems are grouped into size classes (Nx, N).  Each class is one plan
// whose three kernels cover all of its problems at once: the x FFT reads every
// problem of the class from the caller's packed f through a per-problem offset
// table, the row solve runs all (problem, kx) rows with each problem's own
// shifts k^2 + lambda_p, and the inverse x FFT writes through the same table
// into the packed u.  A solve is one CUDA graph: the classes' kernel chains
// are captured on one stream per class, forked from and joined back to a
// capture stream, so that the chains run concurrently; the graph is launched
// with one cudaGraphLaunch on the caller's stream.  The graph holds the f and u
// pointers and is captured again when a call passes different ones.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <utility>
#include <vector>

#include "../../include/helm_b200.h"
#include "helm_batch_eig.cuh"
#include "helm_plan.hpp"

namespace helm {

struct Batch {
    int nprob = 0, device = 0, precision = HELM_FP64;
    // FP64 and refined batches within its range: one persistent launch
    // (helm_batch_eig.cu) in place of the size classes
    BatchEig* be = nullptr;
    int n_sizes = 0;  // distinct (Nx, N) of the batch
    std::vector<long long> offs;  // element offset of each problem in the packed buffers
    long long total = 0;          // elements of the packed buffers
    std::vector<Plan*> classes;
    std::vector<cudaStream_t> streams;  // one per class (capture fork)
    std::vector<cudaEvent_t> joins;
    cudaStream_t origin = nullptr;      // capture stream
    cudaEvent_t fork = nullptr;
    bool use_graph = true;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    const void* graph_f = nullptr;
    void* graph_u = nullptr;
    std::mutex mu;

    void release()
    {
        batch_eig_destroy(be);
        be = nullptr;
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
        for (Plan* p : classes) {
            p->release();
            delete p;
        }
        classes.clear();
        for (cudaStream_t s : streams) cudaStreamDestroy(s);
        streams.clear();
        for (cudaEvent_t e : joins) cudaEventDestroy(e);
        joins.clear();
        if (origin) cudaStreamDestroy(origin);
        if (fork) cudaEventDestroy(fork);
        origin = nullptr;
        fork = nullptr;
    }
};

static int cuda_status(cudaError_t e, const char* what)
{
    std::string msg = std::string(what) + ": " + cudaGetErrorString(e);
    set_last_error(msg.c_str());
    return HELM_ERR_CUDA;
}

// The class chains, each on its own stream, ordered after `fork` on `origin`
// and joined back into `origin`.
static int launch_classes(Batch& b, const void* f, void* u)
{
    if (b.be) return batch_eig_solve(b.be, static_cast<const double*>(f), static_cast<double*>(u), b.origin);
    cudaError_t e = cudaEventRecord(b.fork, b.origin);
    if (e != cudaSuccess) return cuda_status(e, "cudaEventRecord");
    for (size_t c = 0; c < b.classes.size(); ++c) {
        if ((e = cudaStreamWaitEvent(b.streams[c], b.fork, 0)) != cudaSuccess) return cuda_status(e, "cudaStreamWaitEvent");
        int st = solve(*b.classes[c], f, nullptr, nullptr, u, b.streams[c]);
        if (st) return st;
        if ((e = cudaEventRecord(b.joins[c], b.streams[c])) != cudaSuccess) return cuda_status(e, "cudaEventRecord");
        if ((e = cudaStreamWaitEvent(b.origin, b.joins[c], 0)) != cudaSuccess) return cuda_status(e, "cudaStreamWaitEvent");
    }
    return HELM_OK;
}

static int capture(Batch& b, const void* f, void* u)
{
    if (b.exec) cudaGraphExecDestroy(b.exec);
    if (b.graph) cudaGraphDestroy(b.graph);
    b.exec = nullptr;
    b.graph = nullptr;
    b.graph_f = nullptr;
    b.graph_u = nullptr;
    cudaError_t e = cudaStreamBeginCapture(b.origin, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return cuda_status(e, "cudaStreamBeginCapture");
    const int st = launch_classes(b, f, u);
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(b.origin, &g);
    if (st) {
        if (g) cudaGraphDestroy(g);
        return st;
    }
    if (e != cudaSuccess) return cuda_status(e, "cudaStreamEndCapture");
    if ((e = cudaGraphInstantiate(&b.exec, g, 0)) != cudaSuccess) {
        cudaGraphDestroy(g);
        b.exec = nullptr;
        return cuda_status(e, "cudaGraphInstantiate");
    }
    b.graph = g;
    b.graph_f = f;
    b.graph_u = u;
    return HELM_OK;
}

}  // namespace helm

using helm::Batch;

extern "C" {

int helm2d_batch_create(int nprob, const int* Nx, const int* N, const double* lambda, double xl, double xr,
                        double yl, double yr, int precision, helm_batch_t* batch)
{
    if (!batch) return HELM_ERR_INVALID;
    *batch = nullptr;
    if (nprob < 1 || !Nx || !N || !lambda) {
        helm::set_last_error("empty batch or NULL size arrays");
        return HELM_ERR_INVALID;
    }
    if (precision < HELM_FP64 || precision > HELM_FP32_REFINE) return HELM_ERR_INVALID;
    if (!(xr > xl) || !(yr > yl)) {
        helm::set_last_error("empty domain");
        return HELM_ERR_INVALID;
    }
    for (int i = 0; i < nprob; ++i) {
        if (N[i] < 3 || N[i] > 129 || Nx[i] < 4 || !std::isfinite(lambda[i])) {
            helm::set_last_error("problem size or lambda out of range");
            return HELM_ERR_INVALID;
        }
        if (Nx[i] & (Nx[i] - 1)) {
            helm::set_last_error("N has to be 2^n");
            return HELM_ERR_NOT_POW2;
        }
        if (Nx[i] > 1024) {
            helm::set_last_error("Fourier size beyond 4..1024");
            return HELM_ERR_UNSUPPORTED;
        }
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
        cudaGetLastError();
        helm::set_last_error("no CUDA device");
        return HELM_ERR_NO_DEVICE;
    }
    Batch* b = new (std::nothrow) Batch();
    if (!b) return HELM_ERR_OOM;
    cudaGetDevice(&b->device);
    b->nprob = nprob;
    b->precision = precision;
    b->offs.resize(nprob);
    long long off = 0;
    for (int i = 0; i < nprob; ++i) {
        b->offs[i] = off;
        off += (long long)Nx[i] * N[i];
    }
    b->total = off;
    // size classes in order of first appearance of (Nx, N)
    std::map<std::pair<int, int>, int> cls_of;
    std::vector<std::pair<int, int>> cls_key;
    std::vector<std::vector<int>> members;
    for (int i = 0; i < nprob; ++i) {
        auto key = std::make_pair(Nx[i], N[i]);
        auto it = cls_of.find(key);
        if (it == cls_of.end()) {
            it = cls_of.emplace(key, (int)cls_key.size()).first;
            cls_key.push_back(key);
            members.emplace_back();
        }
        members[it->second].push_back(i);
    }
    b->n_sizes = (int)cls_key.size();
    int st = HELM_OK;
    if (precision != HELM_FP32) {
        st = helm::batch_eig_create(nprob, Nx, N, lambda, xl, xr, yl, yr, b->offs.data(), b->device, &b->be);
        if (st == HELM_ERR_UNSUPPORTED) st = HELM_OK;  // outside its range: the size classes below
    }
    for (size_t c = 0; c < cls_key.size() && !st && !b->be; ++c) {
        std::vector<double> lams;
        std::vector<long long> offs;
        for (int i : members[c]) {
            lams.push_back(lambda[i]);
            offs.push_back(b->offs[i]);
        }
        helm::Plan* p = nullptr;
        st = helm::create_batch_class(cls_key[c].first, cls_key[c].second, xl, xr, yl, yr, lams, offs, b->total,
                                      precision, &p);
        if (!st) b->classes.push_back(p);
    }
    cudaError_t e = cudaSuccess;
    if (!st && (e = cudaStreamCreateWithFlags(&b->origin, cudaStreamNonBlocking)) != cudaSuccess)
        st = helm::cuda_status(e, "cudaStreamCreate");
    if (!st && (e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming)) != cudaSuccess)
        st = helm::cuda_status(e, "cudaEventCreate");
    for (size_t c = 0; c < b->classes.size() && !st; ++c) {
        cudaStream_t s = nullptr;
        cudaEvent_t ev = nullptr;
        if ((e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)) != cudaSuccess) {
            st = helm::cuda_status(e, "cudaStreamCreate");
            break;
        }
        b->streams.push_back(s);
        if ((e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess) {
            st = helm::cuda_status(e, "cudaEventCreate");
            break;
        }
        b->joins.push_back(ev);
    }
    if (st) {
        b->release();
        delete b;
        return st;
    }
    *batch = reinterpret_cast<helm_batch_t>(b);
    return HELM_OK;
}

int helm_batch_offsets(helm_batch_t batch, long long* offsets, long long* total_elems)
{
    if (!batch) return HELM_ERR_INVALID;
    Batch* b = reinterpret_cast<Batch*>(batch);
    if (offsets) std::copy(b->offs.begin(), b->offs.end(), offsets);
    if (total_elems) *total_elems = b->total;
    return HELM_OK;
}

int helm_batch_info(helm_batch_t batch, int* n_classes, int* kernels_per_solve, long long* device_bytes)
{
    if (!batch) return HELM_ERR_INVALID;
    Batch* b = reinterpret_cast<Batch*>(batch);
    if (n_classes) *n_classes = b->n_sizes;
    if (kernels_per_solve) *kernels_per_solve = b->be ? 1 : 3 * (int)b->classes.size();
    if (device_bytes) {
        long long s = b->be ? helm::batch_eig_device_bytes(b->be) : 0;
        for (const helm::Plan* p : b->classes) s += p->device_bytes;
        *device_bytes = s;
    }
    return HELM_OK;
}

int helm_batch_set_graph(helm_batch_t batch, int enable)
{
    if (!batch) return HELM_ERR_INVALID;
    Batch* b = reinterpret_cast<Batch*>(batch);
    std::lock_guard<std::mutex> lock(b->mu);
    b->use_graph = enable != 0;
    return HELM_OK;
}

int helm_batch_solve(helm_batch_t batch, const double* f, double* u, void* stream)
{
    if (!batch || !f || !u) return HELM_ERR_INVALID;
    Batch* b = reinterpret_cast<Batch*>(batch);
    std::lock_guard<std::mutex> lock(b->mu);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != b->device) cudaSetDevice(b->device);
    int st = HELM_OK;
    if (!b->use_graph) {
        if (b->be) st = helm::batch_eig_solve(b->be, f, u, s);
        for (helm::Plan* p : b->classes)
            if ((st = helm::solve(*p, f, nullptr, nullptr, u, s))) break;
    } else {
        if (!b->exec || b->graph_f != f || b->graph_u != u) st = helm::capture(*b, f, u);
        if (!st) {
            cudaError_t e = cudaGraphLaunch(b->exec, s);
            if (e != cudaSuccess) st = helm::cuda_status(e, "cudaGraphLaunch");
        }
    }
    if (cur != b->device) cudaSetDevice(cur);
    return st;
}

int helm_batch_device_status(helm_batch_t batch, int* code, int reset)
{
    if (!batch || !code) return HELM_ERR_INVALID;
    Batch* b = reinterpret_cast<Batch*>(batch);
    *code = 0;
    if (!b->be) return HELM_OK;
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != b->device) cudaSetDevice(b->device);
    int* d = helm::batch_eig_status(b->be);
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(code, d, sizeof(int), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && reset) e = cudaMemset(d, 0, sizeof(int));
    if (cur != b->device) cudaSetDevice(cur);
    return e == cudaSuccess ? HELM_OK : helm::cuda_status(e, "device status");
}

int helm_batch_destroy(helm_batch_t batch)
{
    if (!batch) return HELM_OK;
    Batch* b = reinterpret_cast<Batch*>(batch);
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != b->device) cudaSetDevice(b->device);
    b->release();
    if (cur != b->device) cudaSetDevice(cur);
    delete b;
    return HELM_OK;
}

}  // extern "C"
