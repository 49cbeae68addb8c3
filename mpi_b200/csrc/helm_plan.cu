// Plan objects and the C ABI of include/helm_b200.h.
//
// A plan holds everything of the reference's CreatePDEPlan/CreateFFTPlan and of
// the ConstructOperator callbacks it would call inside SolvePDE, precomputed
// once in FP64 on the host and uploaded: the GLL grid and derivative rows,
// one shifted operator per distinct shift sigma = lambda + kx^2 + ky^2 (LU
// factors for the LU method, or the shared eigen-decomposition for the
// fast-diagonalisation method), the homogeneous solutions ul/ur of every
// shift, FFT twiddles, and the spectrum workspace.  helm_solve then runs five
// kernels on the caller's stream: x-FFT (R2C) -> y-FFT -> row solves -> inverse
// y-FFT -> x-FFT (C2R); 2D plans skip the y passes.
#include "../../include/helm_b200.h"
#include "helm_kernels.cuh"
#include "helm_plan.hpp"
#include "helm_setup.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <string>
#include <thread>
#include <vector>

namespace helm {

static thread_local std::string g_last_error;

static int set_cuda_error(cudaError_t e, const char* what)
{
    g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
    return HELM_ERR_CUDA;
}

static bool is_pow2(int v) { return v > 0 && (v & (v - 1)) == 0; }

// The reference's constant (General.h:15), so sigma is computed with the same
// double arithmetic as its ConstructOperator callbacks.
static const double kRefPi = 3.1415926535897932;

void Plan::release()
{
    for (void* p : allocations) cudaFree(p);
    allocations.clear();
    device_bytes = 0;
}

int Plan::alloc(void** p, size_t bytes)
{
    *p = nullptr;
    if (bytes == 0) return HELM_OK;
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
        g_last_error = "cudaMalloc failed";
        return HELM_ERR_OOM;
    }
    allocations.push_back(*p);
    device_bytes += (long long)bytes;
    return HELM_OK;
}

int Plan::upload(void** p, const void* host, size_t bytes)
{
    int st = alloc(p, bytes);
    if (st) return st;
    if (bytes) {
        cudaError_t e = cudaMemcpy(*p, host, bytes, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return set_cuda_error(e, "upload");
    }
    return HELM_OK;
}

template <typename T>
static std::vector<T> twiddles(int L)
{
    std::vector<T> t(2 * L);
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int e = 0; e < L; ++e) {
        long double a = -2.0L * pi * e / L;
        t[2 * e] = (T)std::cos(a);
        t[2 * e + 1] = (T)std::sin(a);
    }
    return t;
}

// Groups of spectrum rows that share one shifted operator.
static void build_groups(Plan& p)
{
    const int nkx = p.Nx / 2 + 1;
    const int Nyf = p.dim == 3 ? p.Ny : 1;
    const bool merge = (p.dim == 3) && (p.Lx == p.Ly);  // sigma depends on kx^2+ky^2 only
    std::map<long long, std::vector<int>> by_key;
    std::map<long long, std::pair<int, int>> key_pair;
    for (int kx = 0; kx < nkx; ++kx)
        for (int ky = 0; ky < Nyf; ++ky) {
            const int jw = p.dim == 3 ? std::min(ky, p.Ny - ky) : 0;
            const long long key = merge ? (long long)kx * kx + (long long)jw * jw : (long long)kx * 4096 + jw;
            by_key[key].push_back(kx * Nyf + ky);
            if (!key_pair.count(key)) key_pair[key] = {kx, jw};
        }
    p.grp_start.assign(1, 0);
    p.grp_rows.clear();
    p.grp_iw.clear();
    p.grp_jw.clear();
    p.sigma.clear();
    for (auto& kv : by_key) {
        const int iw = key_pair[kv.first].first, jw = key_pair[kv.first].second;
        double s = p.lambda + 4.0 * kRefPi * kRefPi * iw * iw / (p.Lx * p.Lx);
        if (p.dim == 3) s = s + 4.0 * kRefPi * kRefPi * jw * jw / (p.Ly * p.Ly);
        p.sigma.push_back(s);
        p.grp_iw.push_back(iw);
        p.grp_jw.push_back(jw);
        for (int r : kv.second) p.grp_rows.push_back(r);
        p.grp_start.push_back((int)p.grp_rows.size());
    }
    p.ngroups = (int)p.sigma.size();
}

static int setup_plan(Plan& p)
{
    const int N = p.N, n = N - 2;
    p.n = n;
    p.nslot = (n + 31) / 32;
    p.ld = 32 * p.nslot;
    p.gll = build_gll_setup(N, p.Ns, p.Lgll);
    const std::vector<double>& D = p.gll.D;
    const std::vector<double>& D2 = p.gll.D2;
    build_groups(p);
    const int G = p.ngroups, ld = p.ld;

    // interior operator and the boundary columns of D2
    std::vector<double> A0(n * n), bl(n), br(n);
    for (int i = 0; i < n; ++i) {
        for (int j = 0; j < n; ++j) A0[i * n + j] = D2[(i + 1) * N + (j + 1)];
        bl[i] = -D2[(i + 1) * N + 0];
        br[i] = -D2[(i + 1) * N + (N - 1)];
    }
    const int prec_code = p.precision == HELM_FP64 ? 0 : (p.precision == HELM_FP32 ? 1 : 2);
    if (p.method == HELM_METHOD_AUTO) p.method = HELM_METHOD_FDM;
    // the FDM transforms live in shared memory; beyond its capacity use the LU method
    if (p.method == HELM_METHOD_FDM && rows_smem_bytes(2, prec_code, n, p.ld) > kMaxSmemPerBlock)
        p.method = HELM_METHOD_LU;
    if (rows_smem_bytes(p.method, prec_code, n, p.ld) > kMaxSmemPerBlock) {
        g_last_error = "GLL size too large for the row-solve kernel at this precision";
        return HELM_ERR_UNSUPPORTED;
    }
    std::vector<double> lam(n), V(n * n), Vi(n * n);
    bool have_eig = false;
    if (p.method == HELM_METHOD_FDM) {
        have_eig = real_eigen(n, A0.data(), lam.data(), V.data(), Vi.data());
        if (!have_eig) p.method = HELM_METHOD_LU;  // fall back to the per-shift factorisation
    }

    // per-group homogeneous solutions (and LU factors for the LU method)
    const bool lu = p.method == HELM_METHOD_LU;
    std::vector<double> fac(lu ? (size_t)G * n * ld : 0), dinv(lu ? (size_t)G * ld : 0);
    std::vector<uint8_t> perm(lu ? (size_t)G * ld : 0);
    std::vector<double> hom((size_t)G * 2 * N), homs((size_t)G * 4);
    std::vector<int> bad(G, 0);
    std::vector<double> h0(n), hN(n);
    if (!lu) {
        for (int j = 0; j < n; ++j) {
            double s0 = 0, s1 = 0;
            for (int k = 0; k < n; ++k) { s0 += Vi[j * n + k] * bl[k]; s1 += Vi[j * n + k] * br[k]; }
            h0[j] = s0;
            hN[j] = s1;
        }
    }
    auto work = [&](int g0, int g1) {
        std::vector<double> A(n * n), x(n), y(n);
        std::vector<int> pv(n);
        for (int g = g0; g < g1; ++g) {
            const double sig = p.sigma[g];
            double* ul = &hom[(size_t)g * 2 * N];
            double* ur = ul + N;
            if (lu) {
                A = A0;
                for (int i = 0; i < n; ++i) A[i * n + i] -= sig;
                if (!lu_factor(n, A.data(), pv.data())) { bad[g] = 1; continue; }
                // column k: U above the diagonal, L below it (the kernel masks by
                // position), the diagonal as 1/U_kk in dinv
                for (int k = 0; k < n; ++k) {
                    for (int i = 0; i < n; ++i) fac[(size_t)g * n * ld + (size_t)k * ld + i] = (i == k) ? 0.0 : A[i * n + k];
                    dinv[(size_t)g * ld + k] = 1.0 / A[k * n + k];
                    perm[(size_t)g * ld + k] = (uint8_t)pv[k];
                }
                x = bl;
                lu_solve(n, A.data(), pv.data(), x.data());
                y = br;
                lu_solve(n, A.data(), pv.data(), y.data());
            } else {
                double mind = 1e300;
                for (int j = 0; j < n; ++j) mind = std::min(mind, std::fabs(lam[j] - sig));
                double scale = std::max(std::fabs(lam[0]), std::fabs(sig));
                if (!(mind > 1e-12 * scale)) { bad[g] = 1; continue; }
                for (int i = 0; i < n; ++i) {
                    double s0 = 0, s1 = 0;
                    for (int j = 0; j < n; ++j) {
                        const double r = 1.0 / (lam[j] - sig);
                        s0 += V[i * n + j] * h0[j] * r;
                        s1 += V[i * n + j] * hN[j] * r;
                    }
                    x[i] = s0;
                    y[i] = s1;
                }
            }
            ul[0] = 1.0; ul[N - 1] = 0.0;
            ur[0] = 0.0; ur[N - 1] = 1.0;
            for (int i = 0; i < n; ++i) { ul[i + 1] = x[i]; ur[i + 1] = y[i]; }
            double s[4] = {0, 0, 0, 0};
            for (int k = 0; k < N; ++k) {
                s[0] += D[k] * ul[k];
                s[1] += D[k] * ur[k];
                s[2] += D[(N - 1) * N + k] * ul[k];
                s[3] += D[(N - 1) * N + k] * ur[k];
            }
            for (int q = 0; q < 4; ++q) homs[(size_t)g * 4 + q] = s[q];
        }
    };
    int nth = (int)std::min<unsigned>(std::max(1u, std::thread::hardware_concurrency()), 16u);
    if (G < 64) nth = 1;
    std::vector<std::thread> th;
    for (int t = 0; t < nth; ++t) th.emplace_back(work, (int)((long long)G * t / nth), (int)((long long)G * (t + 1) / nth));
    for (auto& t : th) t.join();
    for (int g = 0; g < G; ++g)
        if (bad[g]) { g_last_error = "shifted GLL operator is singular"; return HELM_ERR_SINGULAR; }

    // ---- device uploads ----
    const bool td = p.precision != HELM_FP32;           // spectrum / FFT precision is double
    const bool fd = p.precision == HELM_FP64;           // factor / transform precision is double
    const size_t nkx = p.Nx / 2 + 1, Nyf = p.dim == 3 ? p.Ny : 1;
    p.nrows = (long long)nkx * Nyf;
    p.elem_spec = p.nrows * N;
    int st;
    if ((st = p.alloc(&p.d_spec, (size_t)p.Ns * p.elem_spec * (td ? 16 : 8)))) return st;
    auto up_tw = [&](int L, void** d) -> int {
        if (td) { auto t = twiddles<double>(L); return p.upload(d, t.data(), t.size() * sizeof(double)); }
        auto t = twiddles<float>(L);
        return p.upload(d, t.data(), t.size() * sizeof(float));
    };
    if ((st = up_tw(p.Nx, &p.d_tw_x))) return st;
    if (p.dim == 3 && (st = up_tw(p.Ny, &p.d_tw_y))) return st;
    if ((st = p.upload((void**)&p.d_grp_start, p.grp_start.data(), p.grp_start.size() * sizeof(int)))) return st;
    if ((st = p.upload((void**)&p.d_grp_rows, p.grp_rows.data(), p.grp_rows.size() * sizeof(int)))) return st;
    if ((st = p.upload((void**)&p.d_sigma, p.sigma.data(), p.sigma.size() * sizeof(double)))) return st;
    if ((st = p.upload((void**)&p.d_hom, hom.data(), hom.size() * sizeof(double)))) return st;
    if ((st = p.upload((void**)&p.d_homs, homs.data(), homs.size() * sizeof(double)))) return st;
    if ((st = p.upload((void**)&p.d_d0, D.data(), N * sizeof(double)))) return st;
    if ((st = p.upload((void**)&p.d_dN, D.data() + (size_t)(N - 1) * N, N * sizeof(double)))) return st;
    // refinement: interior D2 column-major with leading dimension ld
    std::vector<double> d2t((size_t)n * ld, 0.0);
    for (int k = 0; k < n; ++k)
        for (int i = 0; i < n; ++i) d2t[(size_t)k * ld + i] = A0[i * n + k];
    if ((st = p.upload((void**)&p.d_d2t, d2t.data(), d2t.size() * sizeof(double)))) return st;
    auto up_mat = [&](const std::vector<double>& h, void** d) -> int {
        if (fd) return p.upload(d, h.data(), h.size() * sizeof(double));
        std::vector<float> f(h.begin(), h.end());
        return p.upload(d, f.data(), f.size() * sizeof(float));
    };
    if (lu) {
        if ((st = up_mat(fac, &p.d_fac))) return st;
        if ((st = up_mat(dinv, &p.d_dinv))) return st;
        if ((st = p.upload((void**)&p.d_perm, perm.data(), perm.size()))) return st;
    } else {
        std::vector<double> vinvT((size_t)n * ld, 0.0), vT((size_t)n * ld, 0.0);
        for (int k = 0; k < n; ++k)
            for (int i = 0; i < n; ++i) {
                vinvT[(size_t)k * ld + i] = Vi[i * n + k];
                vT[(size_t)k * ld + i] = V[i * n + k];
            }
        if ((st = up_mat(vinvT, &p.d_vinvT))) return st;
        if ((st = up_mat(vT, &p.d_vT))) return st;
        if ((st = p.upload((void**)&p.d_lam, lam.data(), lam.size() * sizeof(double)))) return st;
    }
    p.h_lam = lam;
    p.h_V = V;
    p.h_Vi = Vi;
    return HELM_OK;
}

static int fft_pass(Plan& p, int L, int mode, int dir, const void* in, void* out, long long in_row, long long out_row,
                    long long in_batch, long long out_batch, int ncols, int nbatch, double scale, const void* tw,
                    const double* gl, const double* gr, cudaStream_t s)
{
    FftArgs a{};
    a.in = in;
    a.out = out;
    a.in_row = in_row;
    a.out_row = out_row;
    a.in_batch = in_batch;
    a.out_batch = out_batch;
    a.ncols = ncols;
    a.nbatch = nbatch;
    a.scale = scale;
    a.tw = tw;
    a.gl = gl;
    a.gr = gr;
    a.bc_row = p.dim == 3 ? p.bc_x_stride : 1;
    a.P = (mode == FFT_R2C) ? p.N : 0;
    a.gl_batch = 0;
    a.gr_batch = p.Ns - 1;
    const long long ccols = (mode == FFT_C2C) ? ncols : (ncols + 1) / 2;
    const int td = p.precision != HELM_FP32;
    const int io = td ? 8 : p.io_bytes;
    int e = launch_fft(L, mode, dir, td, io, a, ccols * nbatch, s);
    if (e) return set_cuda_error((cudaError_t)e, "fft launch");
    return HELM_OK;
}

int solve(Plan& p, const void* f, const double* gl, const double* gr, void* u, cudaStream_t s)
{
    const int N = p.N;
    const long long cols = (long long)(p.dim == 3 ? p.Ny : 1) * N;  // real columns per x row
    const int nkx = p.Nx / 2 + 1;
    int st;
    // 1. x: real-to-complex, GLL boundary slots take the boundary data
    if ((st = fft_pass(p, p.Nx, FFT_R2C, -1, f, p.d_spec, p.x_stride, cols, p.elem_stride, p.elem_spec, (int)cols, p.Ns,
                       1.0, p.d_tw_x, gl, gr, s)))
        return st;
    // 2. y: complex-to-complex along the middle axis
    if (p.dim == 3 &&
        (st = fft_pass(p, p.Ny, FFT_C2C, -1, p.d_spec, p.d_spec, N, N, (long long)p.Ny * N, (long long)p.Ny * N, N,
                       p.Ns * nkx, 1.0, p.d_tw_y, nullptr, nullptr, s)))
        return st;
    // 3. per-wavenumber collocation solves + interface sweep + combination
    RowArgs r{};
    r.spec = p.d_spec;
    r.elem_stride = p.elem_spec;
    r.P = N;
    r.n = p.n;
    r.Ns = p.Ns;
    r.ngroups = p.ngroups;
    r.grp_start = p.d_grp_start;
    r.grp_rows = p.d_grp_rows;
    r.fac = p.d_fac;
    r.dinv = p.d_dinv;
    r.perm = p.d_perm;
    r.ldf = p.ld;
    r.fac_stride = (long long)p.n * p.ld;
    r.vinvT = p.d_vinvT;
    r.vT = p.d_vT;
    r.lam = p.d_lam;
    const bool hom = p.Ns > 1 || p.bc.alphal != 0.0 || p.bc.alphar != 0.0 || gl != nullptr || gr != nullptr;
    r.hom = hom ? p.d_hom : nullptr;
    r.homs = p.d_homs;
    r.d0 = p.d_d0;
    r.dN = p.d_dN;
    r.sigma = p.d_sigma;
    r.d2t = p.d_d2t;
    r.sweeps = p.sweeps;
    r.al = p.bc.alphal;
    r.bl = p.bc.betal;
    r.ar = p.bc.alphar;
    r.br = p.bc.betar;
    const int prec = p.precision == HELM_FP64 ? 0 : (p.precision == HELM_FP32 ? 1 : 2);
    int e = launch_rows(p.method, prec, r, s);
    if (e) return set_cuda_error((cudaError_t)e, "row-solve launch");
    // 4. inverse y
    if (p.dim == 3 &&
        (st = fft_pass(p, p.Ny, FFT_C2C, 1, p.d_spec, p.d_spec, N, N, (long long)p.Ny * N, (long long)p.Ny * N, N,
                       p.Ns * nkx, 1.0, p.d_tw_y, nullptr, nullptr, s)))
        return st;
    // 5. x: complex-to-real, scaled by 1/(Nx Ny) (the reference's /Nx, /Ny)
    const double scale = 1.0 / ((double)p.Nx * (p.dim == 3 ? p.Ny : 1));
    if ((st = fft_pass(p, p.Nx, FFT_C2R, 1, p.d_spec, u, cols, p.x_stride, p.elem_spec, p.elem_stride, (int)cols, p.Ns,
                       scale, p.d_tw_x, nullptr, nullptr, s)))
        return st;
    return HELM_OK;
}

static int create_plan(int dim, int Nx, int Ny, int Ngll_total, int N, double xl, double xr, double yl, double yr,
                       double zl, double zr, const helm_robin_t* bc, double lambda, int precision, int method,
                       helm_plan_t* out)
{
    if (!out) return HELM_ERR_INVALID;
    *out = nullptr;
    if (N < 3 || N > 129 || Nx < 4 || Ngll_total < 1) { g_last_error = "size out of range"; return HELM_ERR_INVALID; }
    if (!is_pow2(Nx) || (dim == 3 && !is_pow2(Ny))) { g_last_error = "N has to be 2^n"; return HELM_ERR_NOT_POW2; }
    if (Nx > 1024 || (dim == 3 && (Ny < 4 || Ny > 1024))) { g_last_error = "Fourier size beyond 4..1024"; return HELM_ERR_UNSUPPORTED; }
    if (precision < HELM_FP64 || precision > HELM_FP32_REFINE) return HELM_ERR_INVALID;
    if (method < HELM_METHOD_AUTO || method > HELM_METHOD_FDM) return HELM_ERR_INVALID;
    if (!(xr > xl) || !(yr > yl) || (dim == 3 && !(zr > zl))) { g_last_error = "empty domain"; return HELM_ERR_INVALID; }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        g_last_error = "no CUDA device";
        return HELM_ERR_NO_DEVICE;
    }
    Plan* p = new (std::nothrow) Plan();
    if (!p) return HELM_ERR_OOM;
    cudaGetDevice(&p->device);
    p->dim = dim;
    p->Nx = Nx;
    p->Ny = dim == 3 ? Ny : 1;
    p->N = N;
    p->Ns = (int)std::ceil((double)Ngll_total / N);  // NonPeriodic2D_MPI.cpp:62, one rank
    if (p->Ns > 64) { delete p; g_last_error = "more than 64 GLL elements"; return HELM_ERR_UNSUPPORTED; }
    p->xl = xl; p->xr = xr; p->yl = yl; p->yr = yr; p->zl = zl; p->zr = zr;
    p->Lx = xr - xl;
    p->Ly = yr - yl;
    p->Lgll = dim == 3 ? zr - zl : yr - yl;
    p->bc = bc ? *bc : helm_robin_t{0.0, 1.0, 0.0, 1.0};
    p->lambda = lambda;
    p->precision = precision;
    p->method = method;
    const long long cols = (long long)p->Ny * N;
    p->x_stride = cols;
    p->elem_stride = (long long)Nx * cols;
    p->bc_x_stride = p->Ny;
    int st = setup_plan(*p);
    if (st) { p->release(); delete p; return st; }
    *out = reinterpret_cast<helm_plan_t>(p);
    return HELM_OK;
}

}  // namespace helm

using helm::Plan;

extern "C" {

int helm2d_plan_create(int Nx, int Ny, int N, double xl, double xr, double yl, double yr, const helm_robin_t* bc,
                       double lambda, int precision, int method, helm_plan_t* plan)
{
    try {
        return helm::create_plan(2, Nx, 1, Ny, N, xl, xr, yl, yr, 0.0, 1.0, bc, lambda, precision, method, plan);
    } catch (...) {
        return HELM_ERR_OOM;
    }
}

int helm3d_plan_create(int Nx, int Ny, int Nz, int N, double xl, double xr, double yl, double yr, double zl, double zr,
                       const helm_robin_t* bc, double lambda, int precision, int method, helm_plan_t* plan)
{
    try {
        return helm::create_plan(3, Nx, Ny, Nz, N, xl, xr, yl, yr, zl, zr, bc, lambda, precision, method, plan);
    } catch (...) {
        return HELM_ERR_OOM;
    }
}

int helm_plan_set_layout(helm_plan_t plan, long long x_stride, long long elem_stride, long long bc_x_stride)
{
    if (!plan) return HELM_ERR_INVALID;
    Plan& p = *reinterpret_cast<Plan*>(plan);
    const long long cols = (long long)p.Ny * p.N;
    const long long xs = x_stride ? x_stride : cols;
    const long long es = elem_stride ? elem_stride : (long long)p.Nx * xs;
    const long long bs = bc_x_stride ? bc_x_stride : p.Ny;
    if (xs < cols || es < (long long)p.Nx * xs || bs < p.Ny) return HELM_ERR_INVALID;
    p.x_stride = xs;
    p.elem_stride = es;
    p.bc_x_stride = bs;
    return HELM_OK;
}

int helm_plan_set_io_bytes(helm_plan_t plan, int bytes)
{
    if (!plan || (bytes != 4 && bytes != 8)) return HELM_ERR_INVALID;
    Plan& p = *reinterpret_cast<Plan*>(plan);
    if (bytes == 4 && p.precision != HELM_FP32) return HELM_ERR_UNSUPPORTED;
    p.io_bytes = bytes;
    return HELM_OK;
}

int helm_plan_set_refine_sweeps(helm_plan_t plan, int sweeps)
{
    if (!plan || sweeps < 0 || sweeps > 8) return HELM_ERR_INVALID;
    reinterpret_cast<Plan*>(plan)->sweeps = sweeps;
    return HELM_OK;
}

int helm_solve(helm_plan_t plan, const void* f, const double* gl, const double* gr, void* u, void* stream)
{
    if (!plan || !f || !u) return HELM_ERR_INVALID;
    Plan& p = *reinterpret_cast<Plan*>(plan);
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != p.device) cudaSetDevice(p.device);
    int st = helm::solve(p, f, gl, gr, u, static_cast<cudaStream_t>(stream));
    if (cur != p.device) cudaSetDevice(cur);
    return st;
}

int helm_solve_adjoint(helm_plan_t plan, const double* ubar, double* fbar, double* glbar, double* grbar,
                       const double* u, double* lambda_bar, void* stream)
{
    (void)plan; (void)ubar; (void)fbar; (void)glbar; (void)grbar; (void)u; (void)lambda_bar; (void)stream;
    return HELM_ERR_UNSUPPORTED;
}

int helm_plan_get_grid(helm_plan_t plan, double* nodes, double* D, double* D2)
{
    if (!plan) return HELM_ERR_INVALID;
    const Plan& p = *reinterpret_cast<const Plan*>(plan);
    if (nodes) std::memcpy(nodes, p.gll.nodes.data(), p.gll.nodes.size() * sizeof(double));
    if (D) std::memcpy(D, p.gll.D.data(), p.gll.D.size() * sizeof(double));
    if (D2) std::memcpy(D2, p.gll.D2.data(), p.gll.D2.size() * sizeof(double));
    return HELM_OK;
}

int helm_plan_info(helm_plan_t plan, int* Ns, int* n_operators, int* method, long long* device_bytes)
{
    if (!plan) return HELM_ERR_INVALID;
    const Plan& p = *reinterpret_cast<const Plan*>(plan);
    if (Ns) *Ns = p.Ns;
    if (n_operators) *n_operators = p.ngroups;
    if (method) *method = p.method;
    if (device_bytes) *device_bytes = p.device_bytes;
    return HELM_OK;
}

int helm_plan_destroy(helm_plan_t plan)
{
    if (!plan) return HELM_OK;
    Plan* p = reinterpret_cast<Plan*>(plan);
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != p->device) cudaSetDevice(p->device);
    p->release();
    if (cur != p->device) cudaSetDevice(cur);
    delete p;
    return HELM_OK;
}

const char* helm_status_string(int status)
{
    switch (status) {
        case HELM_OK: return "ok";
        case HELM_ERR_INVALID: return "invalid argument";
        case HELM_ERR_NOT_POW2: return "Fourier size has to be a power of 2";
        case HELM_ERR_SINGULAR: return "shifted GLL operator is singular";
        case HELM_ERR_OOM: return "allocation failed";
        case HELM_ERR_CUDA: return "CUDA error";
        case HELM_ERR_UNSUPPORTED: return "unsupported size or option";
        case HELM_ERR_NO_DEVICE: return "no CUDA device";
        default: return "unknown status";
    }
}

const char* helm_last_error(void) { return helm::g_last_error.c_str(); }

}  // extern "C"
