// Batches of independent 2D problems (helm2d_batch_*) in one persistent
// launch, FP64, sm_100a.
//
// Each problem (Nx Fourier modes, P GLL points, its own lambda, homogeneous
// Dirichlet ends) is solved in the eigen basis of its interior GLL operator,
// as the reference solves each one with per-wavenumber LU
// (DPS/src/NonPeriodic2D_MPI.cpp:228-474, one CreatePDEPlan / SolvePDE per
// problem): u_int = V (x-FFT^-1 diag(1/(mu_j - sigma(kx))) x-FFT) V^-1 f_int,
// with V, V^-1 the folded transforms of helm_fdm.cu.  The work is cut into
// three kinds of items that persistent CTAs take from one ordered queue:
//   1. (problem, 4096 / ld x rows): fold and first transform of f's rows on the
//      FP64 tensor cores -> the problem's coefficient rows C[x][2 ld] (scratch);
//   2. (problem, up to 16 coefficient column pairs): x FFT, scaling by
//      1 / ((mu_j - sigma) Nx), inverse x FFT, in place in C;
//   3. (problem, 4096 / ld x rows): second transform, unfold -> u rows.
// A kind-2 item waits until every kind-1 item of its problem is done, a kind-3
// item until every kind-2 item is (per-problem counters, bounded waits).  The
// queue holds every kind-1 item before any kind-2 item before any kind-3 item,
// so a CTA only waits for items that running CTAs have already taken: the
// launch needs no co-residency guarantee.  Big problems spread over many CTAs
// (a 512 x 129 problem is 8 + 8 + 8 items), small ones cost one item each.
// The coefficient scratch (sum of Nx * 2 ld doubles) mostly stays in L2.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <new>
#include <numeric>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/helm_b200.h"
#include "helm_batch_eig.cuh"
#include "helm_device.cuh"
#include "helm_plan.hpp"
#include "helm_setup.hpp"

namespace helm {

namespace {

constexpr int BE_THREADS = 256;   // 8 warps; two or three CTAs share an SM
constexpr int BE_MINB = 2;        // resident CTAs per SM the kernel is built for
// x rows of a kind-1 / kind-3 item of a class with ld slots: 4096 / ld (512 for
// ld = 8 down to 64 for ld = 64), so that each warp runs eight 8-row m-tiles of
// one n-tile in every class (the same work and registers as ld = 64)
__host__ __device__ constexpr int be_item_rows(int ld) { return 4096 / ld; }
constexpr int BE_MTW = 8;         // m-tiles per warp in a row item

// Complex columns of a kind-2 item: as many as the CTA's FFT transforms in
// one round (256 threads over nx / r0 threads per column, r0 the first radix
// of a length-nx transform), at most ld.  The tile (nx rows of CT + 1
// double2) stays at or below 74 KB, so two CTAs fit an SM.
__host__ __device__ constexpr int be_cols(int nx, int ld)
{
    const int r0 = (nx >= 128) ? 16 : nx <= 16 ? nx : 8;  // 512: the radix-16-first schedule
    const int cap = 256 * r0 / nx;
    return ld < cap ? ld : cap;
}
constexpr long long BE_WAIT_LIMIT = 1ll << 24;
constexpr double kBePi = 3.1415926535897932;  // the reference's PI (General.h:14)

struct BeProblem {
    long long off;   // element offset of f / u in the packed buffers
    long long coff;  // offset (doubles) of the coefficient rows in the scratch
    double lam;
    int nx, cls, nchunk, ngroup;
};

struct BeClass {
    int P, n, m, ms, ma, ld, pitch;  // pitch: doubles per staged f row
    const double* first;             // m8n8k4 B fragments [2][ld/8][ld/4][32] of Vs^-1 | Va^-1
    const double* second;            // of Vs | Va
    const double* mu;                // [2 ld]: ms symmetric then ma antisymmetric eigenvalues
};

struct BeArgs {
    const double* f;
    double* u;
    double* C;
    const BeProblem* prob;
    const BeClass* cls;
    const int* items;
    int nitems;
    int* head;                // queue position
    int* done1;               // kind-1 items finished, per problem
    int* done2;               // kind-2 items finished, per problem
    int* err;                 // status word: 7 when a dependency wait ran out
    const double2* tw[10];    // exp(-2 pi i e / 2^k), k = 3 .. 9
    double w2;                // (2 pi / Lx)^2: the shift of wavenumber kx is lam + w2 kx^2
};

__device__ __forceinline__ void red_release_add(int* p)
{
    asm volatile("red.release.gpu.global.add.s32 [%0], 1;\n" ::"l"(p) : "memory");
}

__device__ __forceinline__ int ld_acquire(const int* p)
{
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Kind 1: rows x0 .. x0+R-1 of problem pr -> coefficient rows.  The rows
// are staged once for the CTA; warp w then owns n-tile w % NT of both folds
// over eight consecutive 8-row m-tiles, so each B fragment it loads feeds
// eight products of each fold.
template <int LD>
__device__ void be_rows_in(const BeArgs& a, const BeProblem& pr, const BeClass& c, int idx, double* sm)
{
    constexpr int NT = LD / 8, KK = LD / 4, IR = be_item_rows(LD);
    const int R = pr.nx < IR ? pr.nx : IR, x0 = idx * IR, P = c.P, pitch = c.pitch;
    double* st = sm;  // [R][pitch]; the boundary slots stay zero (homogeneous Dirichlet)
    const double* f = a.f + pr.off + (long long)x0 * P;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, q = lane & 3;
    // a warp per row, lanes along the row: asynchronous copies, all in flight
    // before the one wait
    for (int r = warp; r < R; r += BE_THREADS / 32)
        for (int k = lane; k < P; k += 32) {
            if (k > 0 && k < P - 1) cp_async_bytes8(st + r * pitch + k, f + r * P + k, true);
            else st[r * pitch + k] = 0.0;
        }
    cp_async_commit();
    cp_async_wait_all();
    __syncthreads();
    // fold each row in place, once: slots [0, LD) the symmetric fold, [LD, 2 LD)
    // the antisymmetric one, zero past ms / m (a warp per row: all reads, then
    // all writes)
    const int n = c.n, m = c.m, ms = c.ms;
    for (int r = warp; r < R; r += BE_THREADS / 32) {
        double* row = st + r * pitch;
        double fs[(LD + 31) / 32], fa[(LD + 31) / 32];
#pragma unroll
        for (int i = 0; i < (LD + 31) / 32; ++i) {
            const int k = lane + 32 * i;
            double vs = 0.0, va = 0.0;
            if (k < m) {
                const double lo = row[1 + k], hi = row[n - k];
                vs = kR2 * (lo + hi);
                va = kR2 * (lo - hi);
            } else if (k < ms) {
                vs = row[1 + k];
            }
            fs[i] = vs;
            fa[i] = va;
        }
        __syncwarp();
#pragma unroll
        for (int i = 0; i < (LD + 31) / 32; ++i) {
            const int k = lane + 32 * i;
            if (k < LD) {
                row[k] = fs[i];
                row[LD + k] = fa[i];
            }
        }
    }
    __syncthreads();
    const int nt = warp % NT, mt0 = (warp / NT) * BE_MTW;
    if (mt0 * 8 >= R) return;
    const int nmt = min(BE_MTW, R / 8 - mt0);  // live m-tiles of this warp
    double cs[BE_MTW][2], ca[BE_MTW][2];
#pragma unroll
    for (int t = 0; t < BE_MTW; ++t) cs[t][0] = cs[t][1] = ca[t][0] = ca[t][1] = 0.0;
    const double* Bs = c.first + (size_t)nt * KK * 32 + lane;
    const double* Ba = c.first + (size_t)(NT + nt) * KK * 32 + lane;
#pragma unroll 4
    for (int kk = 0; kk < KK; ++kk) {
        const double bs = __ldg(Bs + kk * 32), ba = __ldg(Ba + kk * 32);
#pragma unroll
        for (int t = 0; t < BE_MTW; ++t) {
            if (t < nmt) {
                const double* row = st + ((mt0 + t) * 8 + g) * pitch;
                dmma_8x8x4(cs[t][0], cs[t][1], row[4 * kk + q], bs);
                dmma_8x8x4(ca[t][0], ca[t][1], row[LD + 4 * kk + q], ba);
            }
        }
    }
#pragma unroll
    for (int t = 0; t < BE_MTW; ++t) {
        if (t < nmt) {
            double* crow = a.C + pr.coff + (long long)(x0 + (mt0 + t) * 8 + g) * 2 * LD;
            *reinterpret_cast<double2*>(crow + nt * 8 + 2 * q) = make_double2(cs[t][0], cs[t][1]);
            *reinterpret_cast<double2*>(crow + LD + nt * 8 + 2 * q) = make_double2(ca[t][0], ca[t][1]);
        }
    }
}

// Eigenvalue of real coefficient column j; live = false on padding slots.
__device__ __forceinline__ double be_mu(const BeClass& c, int j, bool& live)
{
    const int ld = c.ld;
    live = j < ld ? j < c.ms : (j - ld) < c.ma;
    return live ? c.mu[j < ld ? j : c.ms + (j - ld)] : 0.0;
}

// Kind 2: column pairs [16 idx, 16 idx + CT) of problem pr, along x.
template <int L>
__device__ void be_columns(const BeArgs& a, const BeProblem& pr, const BeClass& c, int idx, double* sm)
{
    constexpr int LOG2 = L == 8 ? 3 : L == 16 ? 4 : L == 32 ? 5 : L == 64 ? 6 : L == 128 ? 7 : L == 256 ? 8 : 9;
    const int ld2 = 2 * c.ld, CT = be_cols(L, c.ld), col0 = idx * 2 * CT, HS = CT + 1;
    double2* z = reinterpret_cast<double2*>(sm);  // [L][HS]
    double* Cb = a.C + pr.coff;
    for (int e = threadIdx.x; e < L * CT; e += BE_THREADS) {
        const int x = e / CT, cc = e - x * CT;
        cp_async_bytes16(&z[x * HS + cc], Cb + (long long)x * ld2 + col0 + 2 * cc, true);
    }
    cp_async_commit();
    cp_async_wait_all();
    __syncthreads();
    const double2* tw = a.tw[LOG2];
    using RS = typename std::conditional<L == 512, Radix512Wide, Radix<L>>::type;
    slab_fft<L, -1, BE_THREADS, 0, 1, RS>(z, HS, CT, tw);
    // real-to-complex split of each column pair, scaling, and the assembly of
    // the full-length spectrum for the inverse (imaginary parts dropped at
    // kx = 0 and L / 2)
    // a thread keeps one column pair (BE_THREADS is a multiple of CT): its two
    // eigenvalues are loaded once, the shift of each kx is lam + w2 kx^2
    const double scale = 1.0 / L;
    const int cc = threadIdx.x % CT;
    bool live0, live1;
    const double mu0 = be_mu(c, col0 + 2 * cc, live0), mu1 = be_mu(c, col0 + 2 * cc + 1, live1);
    for (int e = threadIdx.x; e < (L / 2 + 1) * CT; e += BE_THREADS) {
        const int kx = e / CT, km = (L - kx) & (L - 1);
        const double2 zk = z[kx * HS + cc], zm = z[km * HS + cc];
        double2 X = make_double2(0.5 * (zk.x + zm.x), 0.5 * (zk.y - zm.y));
        double2 Y = make_double2(0.5 * (zk.y + zm.y), 0.5 * (zm.x - zk.x));
        const double sig = pr.lam + a.w2 * (double)(kx * kx);
        const double r0 = live0 ? scale / (mu0 - sig) : 0.0, r1 = live1 ? scale / (mu1 - sig) : 0.0;
        X = make_double2(X.x * r0, X.y * r0);
        Y = make_double2(Y.x * r1, Y.y * r1);
        if (kx == 0 || kx == L / 2) { X.y = 0.0; Y.y = 0.0; }
        z[kx * HS + cc] = make_double2(X.x - Y.y, X.y + Y.x);
        if (kx > 0 && kx < L / 2) z[km * HS + cc] = make_double2(X.x + Y.y, Y.x - X.y);
    }
    __syncthreads();
    slab_fft<L, 1, BE_THREADS, 0, 1, RS>(z, HS, CT, tw);
    for (int e = threadIdx.x; e < L * CT; e += BE_THREADS) {
        const int x = e / CT, cc = e - x * CT;
        __stcg(reinterpret_cast<double2*>(Cb + (long long)x * ld2 + col0 + 2 * cc), z[x * HS + cc]);
    }
}

// Kind 3: coefficient rows x0 .. x0+R-1 -> second transform, unfold -> u rows.
// The coefficient rows are staged once for the CTA; warp w owns n-tile w % NT
// of both folds over eight m-tiles (as kind 1), and after every warp has read the
// rows its results overwrite them, ready for the unfold.
template <int LD>
__device__ void be_rows_out(const BeArgs& a, const BeProblem& pr, const BeClass& c, int idx, double* sm)
{
    constexpr int NT = LD / 8, KK = LD / 4, PITCH = 2 * LD + 4, IR = be_item_rows(LD);
    const int R = pr.nx < IR ? pr.nx : IR, x0 = idx * IR, P = c.P;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, q = lane & 3;
    double* rows = sm;  // [R][PITCH]: coefficients (s | d), then the transformed values
    const double* Cb = a.C + pr.coff + (long long)x0 * 2 * LD;
    for (int e = threadIdx.x; e < R * LD; e += BE_THREADS) {
        const int r = e / LD, j2 = 2 * (e - r * LD);
        cp_async_bytes16(rows + r * PITCH + j2, Cb + (long long)r * 2 * LD + j2, true);
    }
    cp_async_commit();
    cp_async_wait_all();
    __syncthreads();
    const int nt = warp % NT, mt0 = (warp / NT) * BE_MTW;
    const int nmt = mt0 * 8 >= R ? 0 : min(BE_MTW, R / 8 - mt0);
    double vs[BE_MTW][2], vd[BE_MTW][2];
#pragma unroll
    for (int t = 0; t < BE_MTW; ++t) vs[t][0] = vs[t][1] = vd[t][0] = vd[t][1] = 0.0;
    const double* Bs = c.second + (size_t)nt * KK * 32 + lane;
    const double* Bd = c.second + (size_t)(NT + nt) * KK * 32 + lane;
#pragma unroll 4
    for (int kk = 0; kk < KK; ++kk) {
        const double bs = __ldg(Bs + kk * 32), bd = __ldg(Bd + kk * 32);
#pragma unroll
        for (int t = 0; t < BE_MTW; ++t) {
            if (t < nmt) {
                const double* row = rows + ((mt0 + t) * 8 + g) * PITCH;
                dmma_8x8x4(vs[t][0], vs[t][1], row[4 * kk + q], bs);
                dmma_8x8x4(vd[t][0], vd[t][1], row[LD + 4 * kk + q], bd);
            }
        }
    }
    __syncthreads();  // every warp has read the coefficients
#pragma unroll
    for (int t = 0; t < BE_MTW; ++t) {
        if (t < nmt) {
            double* row = rows + ((mt0 + t) * 8 + g) * PITCH;
            *reinterpret_cast<double2*>(row + nt * 8 + 2 * q) = make_double2(vs[t][0], vs[t][1]);
            *reinterpret_cast<double2*>(row + LD + nt * 8 + 2 * q) = make_double2(vd[t][0], vd[t][1]);
        }
    }
    __syncthreads();
    const int n = c.n, m = c.m, ms = c.ms;
    double* u = a.u + pr.off + (long long)x0 * P;
    for (int r = warp; r < R; r += BE_THREADS / 32) {
        const double* sr = rows + r * PITCH;
        for (int k = lane; k < P; k += 32) {
            double v = 0.0;
            if (k > 0 && k < P - 1) {
                const int j = k - 1;
                if (j < m) v = kR2 * (sr[j] + sr[LD + j]);
                else if (j < ms) v = sr[j];
                else v = kR2 * (sr[n - 1 - j] - sr[LD + n - 1 - j]);
            }
            u[r * P + k] = v;
        }
    }
}

__global__ void __launch_bounds__(BE_THREADS, BE_MINB) batch_eig_kernel(BeArgs a)
{
    extern __shared__ __align__(16) double bsm[];
    __shared__ int s_item, s_next, s_ok;
    pdl_enter();
    if (threadIdx.x == 0) s_item = atomicAdd(a.head, 1);
    for (;;) {
        __syncthreads();
        const int it = s_item;
        if (it >= a.nitems) break;
        // take the next item now; it is used after this one (items are still
        // taken in queue order, so every wait is on an earlier item)
        if (threadIdx.x == 0) s_next = atomicAdd(a.head, 1);
        const int code = a.items[it];
        const int kind = code >> 28, b = (code >> 12) & 0xffff, idx = code & 0xfff;
        const BeProblem pr = a.prob[b];
        const BeClass c = a.cls[pr.cls];
        if (kind > 1) {
            // wait for the items this one depends on (taken earlier from the queue)
            if (threadIdx.x == 0) {
                const int* cnt = kind == 2 ? &a.done1[b] : &a.done2[b];
                const int need = kind == 2 ? pr.nchunk : pr.ngroup;
                int ok = 1;
                for (long long w = 0; ld_acquire(cnt) < need; ++w) {
                    if (w >= BE_WAIT_LIMIT) {
                        ok = 0;
                        atomicExch(a.err, 7);
                        break;
                    }
                    __nanosleep(64);
                }
                s_ok = ok;
            }
            __syncthreads();
        } else if (threadIdx.x == 0) {
            s_ok = 1;
        }
        __syncthreads();
        if (s_ok) {
            if (kind == 1 || kind == 3) {
                switch (c.ld) {
                    case 8: kind == 1 ? be_rows_in<8>(a, pr, c, idx, bsm) : be_rows_out<8>(a, pr, c, idx, bsm); break;
                    case 16: kind == 1 ? be_rows_in<16>(a, pr, c, idx, bsm) : be_rows_out<16>(a, pr, c, idx, bsm); break;
                    case 32: kind == 1 ? be_rows_in<32>(a, pr, c, idx, bsm) : be_rows_out<32>(a, pr, c, idx, bsm); break;
                    default: kind == 1 ? be_rows_in<64>(a, pr, c, idx, bsm) : be_rows_out<64>(a, pr, c, idx, bsm); break;
                }
            } else {
                switch (pr.nx) {
                    case 8: be_columns<8>(a, pr, c, idx, bsm); break;
                    case 16: be_columns<16>(a, pr, c, idx, bsm); break;
                    case 32: be_columns<32>(a, pr, c, idx, bsm); break;
                    case 64: be_columns<64>(a, pr, c, idx, bsm); break;
                    case 128: be_columns<128>(a, pr, c, idx, bsm); break;
                    case 256: be_columns<256>(a, pr, c, idx, bsm); break;
                    default: be_columns<512>(a, pr, c, idx, bsm); break;
                }
            }
        }
        // publish: the CTA's writes, then one release increment of the counter
        __syncthreads();
        if (threadIdx.x == 0) {
            if (kind < 3) red_release_add(kind == 1 ? &a.done1[b] : &a.done2[b]);
            s_item = s_next;
        }
    }
}

// m8n8k4 B fragments of an ld x ld block M (row-major, out = M in): lane l of
// (nt, kk) holds M[8 nt + l / 4][4 kk + l % 4].
void swizzle_b(const std::vector<double>& M, int dim, int ld, double* out)
{
    const int NT = ld / 8, KK = ld / 4;
    for (int nt = 0; nt < NT; ++nt)
        for (int kk = 0; kk < KK; ++kk)
            for (int l = 0; l < 32; ++l) {
                const int i = nt * 8 + (l >> 2), k = kk * 4 + (l & 3);
                out[((size_t)nt * KK + kk) * 32 + l] = (i < dim && k < dim) ? M[(size_t)i * dim + k] : 0.0;
            }
}

}  // namespace

struct BatchEig {
    int device = 0, nprob = 0, nitems = 0, nsm = 148;
    size_t smem = 0;
    BeArgs args{};
    int* d_counters = nullptr;  // head, done1[nprob], done2[nprob]
    size_t counter_bytes = 0;
    std::vector<void*> allocs;
    long long bytes = 0;

    int alloc(void** p, size_t n)
    {
        if (alloc_fault_fires()) {
            *p = nullptr;
            return HELM_ERR_OOM;
        }
        if (cudaMalloc(p, n) != cudaSuccess) {
            cudaGetLastError();
            *p = nullptr;
            set_last_error("cudaMalloc failed for the batch tables");
            return HELM_ERR_OOM;
        }
        allocs.push_back(*p);
        bytes += (long long)n;
        return HELM_OK;
    }
    int upload(void** p, const void* h, size_t n)
    {
        if (int st = alloc(p, n)) return st;
        if (cudaMemcpy(*p, h, n, cudaMemcpyHostToDevice) != cudaSuccess) {
            cudaGetLastError();
            set_last_error("cudaMemcpy failed for the batch tables");
            return HELM_ERR_CUDA;
        }
        return HELM_OK;
    }
    void release()
    {
        for (void* p : allocs) cudaFree(p);
        allocs.clear();
    }
};

int batch_eig_create(int nprob, const int* Nx, const int* N, const double* lambda, double xl, double xr, double yl,
                     double yr, const long long* offs, int device, BatchEig** out)
{
    *out = nullptr;
    if (nprob > 0xffff) {
        set_last_error("more problems than the one-launch batch takes");
        return HELM_ERR_UNSUPPORTED;
    }
    for (int i = 0; i < nprob; ++i)
        if (Nx[i] < 8 || Nx[i] > 512 || N[i] < 4 || N[i] > 129) {
            set_last_error("problem outside the one-launch batch range (Nx 8..512, 4..129 GLL points)");
            return HELM_ERR_UNSUPPORTED;
        }
    const double Lx = xr - xl, Ly = yr - yl;
    BatchEig* be = new (std::nothrow) BatchEig();
    if (!be) return HELM_ERR_OOM;
    be->device = device;
    be->nprob = nprob;
    int st = HELM_OK;
    // one class per GLL size: folded eigen-decomposition and its fragments
    std::map<int, int> cls_of;
    std::vector<BeClass> cls;
    std::vector<FoldedEigen> eig;
    for (int i = 0; i < nprob && !st; ++i) {
        if (cls_of.count(N[i])) continue;
        const int P = N[i], n = P - 2;
        const GllSetup gll = build_gll_setup(P, 1, Ly);
        std::vector<double> A0((size_t)n * n);
        for (int r = 0; r < n; ++r)
            for (int q = 0; q < n; ++q) A0[(size_t)r * n + q] = gll.D2[(size_t)(r + 1) * P + q + 1];
        FoldedEigen fe;
        if (!fold_eigen(n, A0, fe)) {
            set_last_error("no eigen-decomposition of the GLL operator for the one-launch batch");
            st = HELM_ERR_UNSUPPORTED;
            break;
        }
        BeClass c{};
        c.P = P;
        c.n = n;
        c.m = fe.m;
        c.ms = fe.ms;
        c.ma = fe.ma;
        c.ld = fe.ms <= 8 ? 8 : fe.ms <= 16 ? 16 : fe.ms <= 32 ? 32 : 64;
        const int ld = c.ld;
        // staged row: the P values, then in place their two folds (2 ld slots);
        // = 4 mod 16 doubles: conflict-free fragment loads
        c.pitch = 4;
        while (c.pitch < std::max(P, 2 * ld)) c.pitch += 16;
        const size_t frag = (size_t)ld * ld;
        std::vector<double> first(2 * frag), second(2 * frag), mu(2 * (size_t)ld, 0.0);
        swizzle_b(fe.Vsi, fe.ms, ld, first.data());
        swizzle_b(fe.Vai, fe.ma, ld, first.data() + frag);
        swizzle_b(fe.Vs, fe.ms, ld, second.data());
        swizzle_b(fe.Va, fe.ma, ld, second.data() + frag);
        for (int j = 0; j < fe.ms; ++j) mu[j] = fe.ls[j];
        for (int j = 0; j < fe.ma; ++j) mu[fe.ms + j] = fe.la[j];
        void *d1 = nullptr, *d2 = nullptr, *d3 = nullptr;
        if ((st = be->upload(&d1, first.data(), first.size() * sizeof(double)))) break;
        if ((st = be->upload(&d2, second.data(), second.size() * sizeof(double)))) break;
        if ((st = be->upload(&d3, mu.data(), mu.size() * sizeof(double)))) break;
        c.first = static_cast<const double*>(d1);
        c.second = static_cast<const double*>(d2);
        c.mu = static_cast<const double*>(d3);
        cls_of[P] = (int)cls.size();
        cls.push_back(c);
        eig.push_back(std::move(fe));
    }
    // problems: scratch offsets, item counts, and the singularity check of the
    // class path (a shift too close to an eigenvalue)
    std::vector<BeProblem> prob(nprob);
    long long coff = 0;
    size_t smem = 0;
    for (int i = 0; i < nprob && !st; ++i) {
        const int ci = cls_of[N[i]];
        const BeClass& c = cls[ci];
        const FoldedEigen& fe = eig[ci];
        const double w2 = 4.0 * kBePi * kBePi / (Lx * Lx);  // as the kernel forms the shift
        for (int kx = 0; kx <= Nx[i] / 2 && !st; ++kx) {
            const double sig = lambda[i] + w2 * (double)(kx * kx);
            for (double l : fe.ls)
                if (!(std::fabs(l - sig) > 1e-12 * std::max(std::fabs(l), std::fabs(sig)))) st = HELM_ERR_SINGULAR;
            for (double l : fe.la)
                if (!(std::fabs(l - sig) > 1e-12 * std::max(std::fabs(l), std::fabs(sig)))) st = HELM_ERR_SINGULAR;
        }
        if (st) {
            set_last_error("shifted GLL operator is singular");
            break;
        }
        BeProblem& p = prob[i];
        p.off = offs[i];
        p.coff = coff;
        p.lam = lambda[i];
        p.nx = Nx[i];
        p.cls = ci;
        p.nchunk = (Nx[i] + be_item_rows(c.ld) - 1) / be_item_rows(c.ld);
        p.ngroup = c.ld / be_cols(Nx[i], c.ld);
        coff += (long long)Nx[i] * 2 * c.ld;
        const int R = std::min(Nx[i], be_item_rows(c.ld));
        smem = std::max(smem, (size_t)R * c.pitch * sizeof(double));
        smem = std::max(smem, (size_t)R * (2 * c.ld + 4) * sizeof(double));
        smem = std::max(smem, (size_t)Nx[i] * (be_cols(Nx[i], c.ld) + 1) * sizeof(double2));
    }
    if (st) {
        be->release();
        delete be;
        return st;
    }
    // the ordered queue: every kind-1 item, then every kind-2, then every
    // kind-3, problems in order of decreasing work so the big ones start first
    std::vector<int> order(nprob);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
        const long long cx = (long long)prob[x].nx * cls[prob[x].cls].ld * cls[prob[x].cls].ld;
        const long long cy = (long long)prob[y].nx * cls[prob[y].cls].ld * cls[prob[y].cls].ld;
        return cx > cy;
    });
    std::vector<int> items;
    for (int kind = 1; kind <= 3; ++kind)
        for (int b : order) {
            const int cnt = kind == 2 ? prob[b].ngroup : prob[b].nchunk;
            for (int k = 0; k < cnt; ++k) items.push_back((kind << 28) | (b << 12) | k);
        }
    BeArgs& a = be->args;
    void *dp = nullptr, *dc = nullptr, *di = nullptr, *dC = nullptr, *dcnt = nullptr, *derr = nullptr;
    if (!st) st = be->upload(&dp, prob.data(), prob.size() * sizeof(BeProblem));
    if (!st) st = be->upload(&dc, cls.data(), cls.size() * sizeof(BeClass));
    if (!st) st = be->upload(&di, items.data(), items.size() * sizeof(int));
    if (!st) st = be->alloc(&dC, (size_t)coff * sizeof(double));
    be->counter_bytes = (1 + 2 * (size_t)nprob) * sizeof(int);
    if (!st) st = be->alloc(&dcnt, be->counter_bytes);
    const int zero = 0;
    if (!st) st = be->upload(&derr, &zero, sizeof(int));
    for (int k = 3; k <= 9 && !st; ++k) {
        const int L = 1 << k;
        std::vector<double> tw(2 * (size_t)L);
        for (int e = 0; e < L; ++e) {
            const long double ang = -2.0L * 3.14159265358979323846264338327950288L * e / L;
            tw[2 * e] = (double)std::cos(ang);
            tw[2 * e + 1] = (double)std::sin(ang);
        }
        void* d = nullptr;
        if (!(st = be->upload(&d, tw.data(), tw.size() * sizeof(double)))) a.tw[k] = static_cast<const double2*>(d);
    }
    if (st) {
        be->release();
        delete be;
        return st;
    }
    a.prob = static_cast<const BeProblem*>(dp);
    a.cls = static_cast<const BeClass*>(dc);
    a.items = static_cast<const int*>(di);
    a.nitems = (int)items.size();
    a.C = static_cast<double*>(dC);
    be->d_counters = static_cast<int*>(dcnt);
    a.head = be->d_counters;
    a.done1 = be->d_counters + 1;
    a.done2 = be->d_counters + 1 + nprob;
    a.err = static_cast<int*>(derr);
    a.w2 = 4.0 * kBePi * kBePi / (Lx * Lx);
    be->nitems = a.nitems;
    be->smem = smem;
    int nsm = 0;
    if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device) == cudaSuccess && nsm > 0) be->nsm = nsm;
    cudaGetLastError();
    if (cudaFuncSetAttribute(batch_eig_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
        cudaGetLastError();
        be->release();
        delete be;
        set_last_error("the one-launch batch kernel does not get its shared memory");
        return HELM_ERR_UNSUPPORTED;
    }
    *out = be;
    return HELM_OK;
}

int batch_eig_solve(BatchEig* be, const double* f, double* u, cudaStream_t s)
{
    BeArgs a = be->args;
    a.f = f;
    a.u = u;
    cudaError_t e = cudaMemsetAsync(be->d_counters, 0, be->counter_bytes, s);
    if (e == cudaSuccess) {
        const int grid = std::min(BE_MINB * be->nsm, be->nitems);
        e = launch_k(batch_eig_kernel, dim3(grid), dim3(BE_THREADS), be->smem, s, a);
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        set_last_error(cudaGetErrorString(e));
        return HELM_ERR_CUDA;
    }
    return HELM_OK;
}

long long batch_eig_device_bytes(const BatchEig* be) { return be->bytes; }
int* batch_eig_status(BatchEig* be) { return be->args.err; }

void batch_eig_destroy(BatchEig* be)
{
    if (!be) return;
    be->release();
    delete be;
}

}  // namespace helm
