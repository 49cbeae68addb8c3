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
#include "helm_fdm.cuh"
#include "helm_kernels.cuh"
#include "helm_plan.hpp"
#include "helm_eig.cuh"
#include "helm_fd_refine.cuh"
#include "helm_setup.hpp"

#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
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
    for (cudaEvent_t& e : ev)
        if (e) { cudaEventDestroy(e); e = nullptr; }
    for (void* p : allocations) cudaFree(p);
    allocations.clear();
    device_bytes = 0;
}

// Host-side fault injection for tests of the out-of-memory paths: while armed
// with n >= 0, the n-th device allocation of a plan from then on (0: the next)
// fails as a cudaMalloc failure would, and the hook disarms itself.
static std::atomic<long long> g_alloc_fault{-1};

bool alloc_fault_fires()
{
    if (g_alloc_fault.load() >= 0 && g_alloc_fault.fetch_sub(1) == 0) {
        g_last_error = "device allocation failure injected by helm_debug_fail_alloc";
        return true;
    }
    return false;
}

int Plan::alloc(void** p, size_t bytes)
{
    *p = nullptr;
    if (bytes == 0) return HELM_OK;
    if (alloc_fault_fires()) return HELM_ERR_OOM;
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

// Groups of spectrum rows that share one shifted operator (per problem of a
// batched plan: problem b's rows follow problem b-1's in the spectrum).
static void build_groups(Plan& p)
{
    const int nkx = p.Nx / 2 + 1;
    const int Nyf = p.dim == 3 ? p.Ny : 1;
    // sigma depends on kx^2+ky^2 only; a user operator may tell (kx, ky) pairs apart
    const bool merge = (p.dim == 3) && (p.Lx == p.Ly) && !p.op_cb;
    p.grp_start.assign(1, 0);
    p.grp_rows.clear();
    p.grp_iw.clear();
    p.grp_jw.clear();
    p.sigma.clear();
    for (int b = 0; b < p.batch; ++b) {
        const double lam = p.batch > 1 ? p.lambdas[b] : p.lambda;
        const int row0 = b * nkx * Nyf;
        std::map<long long, std::vector<int>> by_key;
        std::map<long long, std::pair<int, int>> key_pair;
        for (int kx = 0; kx < nkx; ++kx)
            for (int ky = 0; ky < Nyf; ++ky) {
                const int jw = p.dim == 3 ? std::min(ky, p.Ny - ky) : 0;
                const long long key = merge ? (long long)kx * kx + (long long)jw * jw : (long long)kx * 4096 + jw;
                by_key[key].push_back(row0 + kx * Nyf + ky);
                if (!key_pair.count(key)) key_pair[key] = {kx, jw};
            }
        for (auto& kv : by_key) {
            const int iw = key_pair[kv.first].first, jw = key_pair[kv.first].second;
            double s = lam + 4.0 * kRefPi * kRefPi * iw * iw / (p.Lx * p.Lx);
            if (p.dim == 3) s = s + 4.0 * kRefPi * kRefPi * jw * jw / (p.Ly * p.Ly);
            p.sigma.push_back(s);
            p.grp_iw.push_back(iw);
            p.grp_jw.push_back(jw);
            for (int r : kv.second) p.grp_rows.push_back(r);
            p.grp_start.push_back((int)p.grp_rows.size());
        }
    }
    p.ngroups = (int)p.sigma.size();
}

// Data of the transposed per-wavenumber system M_sigma^T v = w (one element,
// FDM): M_sigma has the interior rows D2[k][:] - sigma e_k and the Robin rows
// (betal - alphal D[0][0], -alphal D[0][int], -alphal D[0][N-1]) and
// (alphar D[N-1][0], alphar D[N-1][int], betar + alphar D[N-1][N-1]).
// Eliminating the interior, v_int = psi + v0 pl + vN pr with psi = A^-T w_int,
// pl = -A^-T r0, pr = -A^-T rN, and (v0, vN) solve a 2x2 system.
//
// Periodic plans: the forward map is u_int = A^-1 f_int + zeta h_int, u_0 =
// u_{N-1} = zeta with zeta = (DN - D0).phi / b and b = (D0 - DN).(ul + ur), so
// the transpose is fbar_int = psi + mu A^-T (DN - D0), mu = (w_0 + w_{N-1} -
// c0.psi - cN.psi) / b: pl = A^-T (DN - D0) (r0 = D0 - DN), pr = 0, and the
// boundary scalars stay the forward D0.ul, D0.ur, DN.ul, DN.ur (`fwd_homs`).
static int setup_adjoint(Plan& p, const std::vector<double>& A0, const std::vector<double>& lam,
                         const std::vector<double>& V, const std::vector<double>& Vi, int prec_code,
                         const std::vector<double>& fwd_homs)
{
    const int N = p.N, n = p.n, ld = p.ld, G = p.ngroups;
    const std::vector<double>& D = p.gll.D;
    const std::vector<double>& D2 = p.gll.D2;
    const double al = p.bc.alphal, bl = p.bc.betal, ar = p.bc.alphar, br = p.bc.betar;
    std::vector<double> r0(n), rN(n), c0(N, 0.0), cN(N, 0.0);
    for (int i = 0; i < n; ++i) {
        r0[i] = p.periodic ? D[i + 1] - D[(N - 1) * N + i + 1] : -al * D[i + 1];
        rN[i] = p.periodic ? 0.0 : ar * D[(N - 1) * N + i + 1];
        c0[i + 1] = D2[(i + 1) * N];
        cN[i + 1] = D2[(i + 1) * N + N - 1];
    }
    const double a00 = bl - al * D[0], a0N = -al * D[N - 1];
    const double aN0 = ar * D[(N - 1) * N], aNN = br + ar * D[(N - 1) * N + N - 1];
    std::vector<double> vr0(n), vrN(n);  // V^T r0, V^T rN
    for (int j = 0; j < n; ++j) {
        double s0 = 0, s1 = 0;
        for (int k = 0; k < n; ++k) { s0 += V[k * n + j] * r0[k]; s1 += V[k * n + j] * rN[k]; }
        vr0[j] = s0;
        vrN[j] = s1;
    }
    std::vector<double> hom((size_t)G * 2 * N, 0.0), homs((size_t)G * 4);
    for (int g = 0; g < G; ++g) {
        double* pl = &hom[(size_t)g * 2 * N];
        double* pr = pl + N;
        const double sig = p.sigma[g];
        for (int i = 0; i < n; ++i) {
            double s0 = 0, s1 = 0;
            for (int j = 0; j < n; ++j) {
                const double rr = 1.0 / (lam[j] - sig);
                s0 += Vi[j * n + i] * vr0[j] * rr;
                s1 += Vi[j * n + i] * vrN[j] * rr;
            }
            pl[i + 1] = -s0;
            pr[i + 1] = -s1;
        }
        double c0pl = 0, c0pr = 0, cNpl = 0, cNpr = 0;
        for (int i = 1; i <= n; ++i) {
            c0pl += c0[i] * pl[i]; c0pr += c0[i] * pr[i];
            cNpl += cN[i] * pl[i]; cNpr += cN[i] * pr[i];
        }
        if (p.periodic) {
            for (int q = 0; q < 4; ++q) homs[(size_t)g * 4 + q] = fwd_homs[(size_t)g * 4 + q];
            continue;
        }
        homs[(size_t)g * 4 + 0] = a00 + c0pl;
        homs[(size_t)g * 4 + 1] = aN0 + c0pr;
        homs[(size_t)g * 4 + 2] = a0N + cNpl;
        homs[(size_t)g * 4 + 3] = aNN + cNpr;
        const double det = homs[g * 4] * homs[g * 4 + 3] - homs[g * 4 + 1] * homs[g * 4 + 2];
        if (!(std::fabs(det) > 0.0)) { g_last_error = "singular boundary system of the adjoint"; return HELM_ERR_SINGULAR; }
    }
    std::vector<double> vtT((size_t)n * ld, 0.0), vinvtT((size_t)n * ld, 0.0), d2row((size_t)n * ld, 0.0);
    for (int k = 0; k < n; ++k)
        for (int i = 0; i < n; ++i) {
            vtT[(size_t)k * ld + i] = V[k * n + i];
            vinvtT[(size_t)k * ld + i] = Vi[k * n + i];
            d2row[(size_t)k * ld + i] = A0[k * n + i];
        }
    int st;
    auto up_mat = [&](const std::vector<double>& h, void** d) -> int {
        if (prec_code == 0) return p.upload(d, h.data(), h.size() * sizeof(double));
        std::vector<float> f(h.begin(), h.end());
        return p.upload(d, f.data(), f.size() * sizeof(float));
    };
    if ((st = up_mat(vtT, &p.d_vtT))) return st;
    if ((st = up_mat(vinvtT, &p.d_vinvtT))) return st;
    if ((st = p.upload((void**)&p.d_d2row, d2row.data(), d2row.size() * sizeof(double)))) return st;
    if ((st = p.upload((void**)&p.d_c0, c0.data(), c0.size() * sizeof(double)))) return st;
    if ((st = p.upload((void**)&p.d_cN, cN.data(), cN.size() * sizeof(double)))) return st;
    if ((st = p.upload((void**)&p.d_hom_adj, hom.data(), hom.size() * sizeof(double)))) return st;
    if ((st = p.upload((void**)&p.d_homs_adj, homs.data(), homs.size() * sizeof(double)))) return st;
    p.adj_ready = true;
    return HELM_OK;
}

// Transposed interior solves of a plan with several GLL elements (not
// periodic): A^T = V^-T diag(lam) V^T and D2int^T for the refinement residual.
// The interface system is transposed inside the row kernel from the forward
// homogeneous solutions and end slopes, which such a plan already holds.
static int setup_adjoint_multi(Plan& p, const std::vector<double>& A0, const std::vector<double>& V,
                               const std::vector<double>& Vi, int prec_code)
{
    const int n = p.n, ld = p.ld;
    std::vector<double> vtT((size_t)n * ld, 0.0), vinvtT((size_t)n * ld, 0.0), d2row((size_t)n * ld, 0.0);
    for (int k = 0; k < n; ++k)
        for (int i = 0; i < n; ++i) {
            vtT[(size_t)k * ld + i] = V[k * n + i];
            vinvtT[(size_t)k * ld + i] = Vi[k * n + i];
            d2row[(size_t)k * ld + i] = A0[k * n + i];
        }
    auto up_mat = [&](const std::vector<double>& h, void** d) -> int {
        if (prec_code == 0) return p.upload(d, h.data(), h.size() * sizeof(double));
        std::vector<float> f(h.begin(), h.end());
        return p.upload(d, f.data(), f.size() * sizeof(float));
    };
    int st;
    if ((st = up_mat(vtT, &p.d_vtT))) return st;
    if ((st = up_mat(vinvtT, &p.d_vinvtT))) return st;
    if ((st = p.upload((void**)&p.d_d2row, d2row.data(), d2row.size() * sizeof(double)))) return st;
    p.adj_ready = true;
    return HELM_OK;
}

// Folded fast-diagonalisation data (helm_fdm.cu): the orthogonal even/odd
// fold Q of the interior nodes block-diagonalises the centrosymmetric D2int,
// Q D2int Q^T = diag(Ms, Ma); each block gets its own eigen-decomposition.
static int setup_fast(Plan& p, const std::vector<double>& A0, int prec_code)
{
    const int n = p.n, m = n / 2, odd = n % 2, ms = m + odd, ma = m, N = p.N, G = p.ngroups;
    const int ld = 32 * ((ms + 31) / 32);
    if (fdm_fast_smem_bytes(prec_code, ld) > kMaxSmemPerBlock || ld > 64) return HELM_OK;  // stay on rows_kernel
    FoldedEigen fe;
    if (!fold_eigen(n, A0, fe)) return HELM_OK;  // not centrosymmetric to rounding, or no decomposition: rows_kernel
    const std::vector<double>&Q = fe.Q, &Ms = fe.Ms, &Ma = fe.Ma, &ls = fe.ls, &Vs = fe.Vs, &Vsi = fe.Vsi,
                               &la = fe.la, &Va = fe.Va, &Vai = fe.Vai;

    const size_t L2 = (size_t)ld * ld;
    std::vector<double> fw(4 * L2, 0.0), fa(4 * L2, 0.0), d2f(2 * L2, 0.0), d2a(2 * L2, 0.0);
    for (int i = 0; i < ms; ++i)
        for (int j = 0; j < ms; ++j) {
            fw[0 * L2 + (size_t)j * ld + i] = Vsi[(size_t)i * ms + j];  // first: Vs^-1, column-major
            fw[1 * L2 + (size_t)j * ld + i] = Vs[(size_t)i * ms + j];   // second: Vs
            fa[0 * L2 + (size_t)j * ld + i] = Vs[(size_t)j * ms + i];   // adjoint first: Vs^T
            fa[1 * L2 + (size_t)j * ld + i] = Vsi[(size_t)j * ms + i];  // adjoint second: Vs^-T
            d2f[0 * L2 + (size_t)j * ld + i] = Ms[(size_t)i * ms + j];
            d2a[0 * L2 + (size_t)j * ld + i] = Ms[(size_t)j * ms + i];
        }
    for (int i = 0; i < ma; ++i)
        for (int j = 0; j < ma; ++j) {
            fw[2 * L2 + (size_t)j * ld + i] = Vai[(size_t)i * ma + j];
            fw[3 * L2 + (size_t)j * ld + i] = Va[(size_t)i * ma + j];
            fa[2 * L2 + (size_t)j * ld + i] = Va[(size_t)j * ma + i];
            fa[3 * L2 + (size_t)j * ld + i] = Vai[(size_t)j * ma + i];
            d2f[1 * L2 + (size_t)j * ld + i] = Ma[(size_t)i * ma + j];
            d2a[1 * L2 + (size_t)j * ld + i] = Ma[(size_t)j * ma + i];
        }
    std::vector<double> recip((size_t)G * 2 * ld, 0.0);
    for (int g = 0; g < G; ++g) {
        const double sg = p.sigma[g];
        for (int j = 0; j < ms; ++j) {
            const double d = ls[j] - sg;
            if (!(std::fabs(d) > 1e-12 * std::max(std::fabs(ls[j]), std::fabs(sg)))) {
                g_last_error = "shifted GLL operator is singular";
                return HELM_ERR_SINGULAR;
            }
            recip[(size_t)g * 2 * ld + j] = 1.0 / d;
        }
        for (int j = 0; j < ma; ++j) {
            const double d = la[j] - sg;
            if (!(std::fabs(d) > 1e-12 * std::max(std::fabs(la[j]), std::fabs(sg)))) {
                g_last_error = "shifted GLL operator is singular";
                return HELM_ERR_SINGULAR;
            }
            recip[(size_t)g * 2 * ld + ld + j] = 1.0 / d;
        }
    }
    // folded boundary functionals: e_f = Q e restricted to the two blocks
    auto fold = [&](const std::vector<double>& e) {
        std::vector<double> out(2 * ld, 0.0);
        for (int i = 0; i < n; ++i) {
            double s = 0;
            for (int k = 0; k < n; ++k) s += Q[(size_t)i * n + k] * e[k];
            if (i < ms) out[i] = s; else out[ld + (i - ms)] = s;
        }
        return out;
    };
    const std::vector<double>& D = p.gll.D;
    const std::vector<double>& D2 = p.gll.D2;
    std::vector<double> e0(n), eN(n), c0(n), cN(n);
    for (int i = 0; i < n; ++i) {
        e0[i] = D[i + 1];
        eN[i] = D[(size_t)(N - 1) * N + i + 1];
        c0[i] = D2[(size_t)(i + 1) * N];
        cN[i] = D2[(size_t)(i + 1) * N + N - 1];
    }
    std::vector<double> fe0 = fold(e0), feN = fold(eN), fc0 = fold(c0), fcN = fold(cN);
    std::vector<int> row_grp(p.grp_rows.size());
    for (int g = 0; g < G; ++g)
        for (int rr = p.grp_start[g]; rr < p.grp_start[g + 1]; ++rr) row_grp[rr] = g;
    int st;
    auto up_t = [&](const std::vector<double>& h, void** d) -> int {
        if (prec_code == 0) return p.upload(d, h.data(), h.size() * sizeof(double));
        std::vector<float> f(h.begin(), h.end());
        return p.upload(d, f.data(), f.size() * sizeof(float));
    };
    if ((st = up_t(fw, &p.d_fmats))) return st;
    if ((st = up_t(fa, &p.d_fmats_adj))) return st;
    if (prec_code == 2 && ld == 32) {
        std::vector<float> tf(8 * L2);
        fdm_tc_swizzle(fw.data(), ld, tf.data());
        if ((st = p.upload((void**)&p.d_ftc, tf.data(), tf.size() * sizeof(float)))) return st;
        fdm_tc_swizzle(fa.data(), ld, tf.data());
        if ((st = p.upload((void**)&p.d_ftc_adj, tf.data(), tf.size() * sizeof(float)))) return st;
        std::vector<double> mm(2 * L2);
        fdm_m16_swizzle2(d2f.data(), ld, mm.data());
        if ((st = p.upload((void**)&p.d_ftcm, mm.data(), mm.size() * sizeof(double)))) return st;
        fdm_m16_swizzle2(d2a.data(), ld, mm.data());
        if ((st = p.upload((void**)&p.d_ftcm_adj, mm.data(), mm.size() * sizeof(double)))) return st;
    }
    // FP64 tensor-core transforms: FP64 plans, and refined plans (whose FP64
    // spectrum the FP64 row kernel and the eigen-basis pipeline can also solve)
    if (prec_code == 0 || prec_code == 2) {
        std::vector<double> sw(4 * L2);
        fdm_mma_swizzle(fw.data(), ld, sw.data());
        if ((st = p.upload((void**)&p.d_fmma, sw.data(), sw.size() * sizeof(double)))) return st;
        fdm_mma_swizzle(fa.data(), ld, sw.data());
        if ((st = p.upload((void**)&p.d_fmma_adj, sw.data(), sw.size() * sizeof(double)))) return st;
        fdm_mma16_swizzle(fw.data(), ld, sw.data());
        if ((st = p.upload((void**)&p.d_fmma16, sw.data(), sw.size() * sizeof(double)))) return st;
        fdm_mma16_swizzle(fa.data(), ld, sw.data());
        if ((st = p.upload((void**)&p.d_fmma16_adj, sw.data(), sw.size() * sizeof(double)))) return st;
    }
    if ((st = up_t(recip, &p.d_frecip))) return st;
    if (prec_code == 2 && (st = p.upload((void**)&p.d_frecip64, recip.data(), recip.size() * sizeof(double)))) return st;
    if (prec_code == 0) p.d_frecip64 = static_cast<double*>(p.d_frecip);
    if ((st = p.upload((void**)&p.d_fd2, d2f.data(), d2f.size() * sizeof(double)))) return st;
    if ((st = p.upload((void**)&p.d_fd2_adj, d2a.data(), d2a.size() * sizeof(double)))) return st;
    if ((st = p.upload((void**)&p.d_row_grp, row_grp.data(), row_grp.size() * sizeof(int)))) return st;
    const bool slab = prec_code != 1 && p.dim == 3 && p.batch == 1 && slab_fits(p.Ny, N, ld);
    const bool eig = p.eig_cand && ld == EIG_LD && prec_code != 1;
    if (slab || eig) {
        std::vector<int> gor((size_t)p.nrows * p.batch, 0);
        for (int g = 0; g < G; ++g)
            for (int rr = p.grp_start[g]; rr < p.grp_start[g + 1]; ++rr) gor[p.grp_rows[rr]] = g;
        if ((st = p.upload((void**)&p.d_grp_of_row, gor.data(), gor.size() * sizeof(int)))) return st;
        p.slab_ok = slab;
    }
    if (eig) {
        // first transform of the folded boundary columns bl = -D2[int][0],
        // br = -D2[int][N-1]: the coefficients that zl = gl / beta_l and
        // zr = gr / beta_r add to each row's
        std::vector<double> bl(n), br(n);
        for (int i = 0; i < n; ++i) {
            bl[i] = -D2[(size_t)(i + 1) * N];
            br[i] = -D2[(size_t)(i + 1) * N + N - 1];
        }
        const std::vector<double> fbl = fold(bl), fbr = fold(br);
        std::vector<double> hbc(4 * EIG_LD, 0.0);
        for (int i = 0; i < ms; ++i)
            for (int j = 0; j < ms; ++j) {
                hbc[i] += Vsi[(size_t)i * ms + j] * fbl[j];
                hbc[EIG_LD + i] += Vsi[(size_t)i * ms + j] * fbr[j];
            }
        for (int i = 0; i < ma; ++i)
            for (int j = 0; j < ma; ++j) {
                hbc[2 * EIG_LD + i] += Vai[(size_t)i * ma + j] * fbl[ld + j];
                hbc[3 * EIG_LD + i] += Vai[(size_t)i * ma + j] * fbr[ld + j];
            }
        if ((st = p.upload((void**)&p.d_hbc, hbc.data(), hbc.size() * sizeof(double)))) return st;
        p.eig_ok = true;
    }
    if ((st = p.upload((void**)&p.d_fe0, fe0.data(), fe0.size() * sizeof(double)))) return st;
    if ((st = p.upload((void**)&p.d_feN, feN.data(), feN.size() * sizeof(double)))) return st;
    if ((st = p.upload((void**)&p.d_fc0, fc0.data(), fc0.size() * sizeof(double)))) return st;
    if ((st = p.upload((void**)&p.d_fcN, fcN.data(), fcN.size() * sizeof(double)))) return st;
    p.fm = m;
    p.fms = ms;
    p.fma = ma;
    p.fld = ld;
    p.fast = true;
    return HELM_OK;
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
    // user operators: one LU factor per wavenumber pair, harvested here serially
    // (the callback may use global state, as the reference's does)
    std::vector<double> user_ops;
    if (p.op_cb) {
        p.method = HELM_METHOD_LU;
        user_ops.assign((size_t)G * n * n, 0.0);
        for (int g = 0; g < G; ++g) p.op_cb(p.grp_iw[g], p.grp_jw[g], &user_ops[(size_t)g * n * n], n, p.op_user);
    }
    // one-element plans run the folded FDM kernel, whose half-size transforms fit
    // shared memory up to 129 points at every precision
    const int fold_ld = 32 * (((n / 2 + n % 2) + 31) / 32);
    const bool fold_fits = p.Ns == 1 && fold_ld <= 64 && fdm_fast_smem_bytes(prec_code, fold_ld) <= kMaxSmemPerBlock;
    // the unfolded FDM transforms live in shared memory; beyond its capacity use the LU method
    if (p.method == HELM_METHOD_FDM && !fold_fits && rows_smem_bytes(2, prec_code, n, p.ld) > kMaxSmemPerBlock)
        p.method = HELM_METHOD_LU;
    if (!(p.method == HELM_METHOD_FDM && fold_fits) && rows_smem_bytes(p.method, prec_code, n, p.ld) > kMaxSmemPerBlock) {
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
                if (p.op_cb) {
                    A.assign(user_ops.begin() + (size_t)g * n * n, user_ops.begin() + (size_t)(g + 1) * n * n);
                } else {
                    A = A0;
                    for (int i = 0; i < n; ++i) A[i * n + i] -= sig;
                }
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
    if (p.periodic) {
        // the real coefficients of the cyclic interface sweep (the kernels' divisors)
        // must not vanish: lambda = 0 leaves the constant mode without an equation
        for (int g = 0; g < G; ++g) {
            const double* h = &homs[(size_t)g * 4];
            const double d0ul = h[0], d0ur = h[1], dNul = h[2], dNur = h[3];
            const double tol = 1e-12 * (std::fabs(d0ul) + std::fabs(d0ur) + std::fabs(dNul) + std::fabs(dNur));
            bool ok = true;
            if (p.Ns == 1) {
                ok = std::fabs((d0ul + d0ur) - (dNul + dNur)) > tol;
            } else {
                std::vector<double> b(p.Ns), c(p.Ns), r1(p.Ns);
                for (int jj = 0; jj < p.Ns && ok; ++jj) {
                    if (jj == 0) { b[0] = dNur - dNul - d0ul; c[0] = -d0ur; r1[0] = dNul; }
                    else if (jj < p.Ns - 1) {
                        b[jj] = dNur - d0ul - (c[jj - 1] / b[jj - 1]) * dNul;
                        c[jj] = -d0ur;
                        r1[jj] = -(r1[jj - 1] / b[jj - 1]) * dNul;
                    } else {
                        b[jj] = dNur - d0ul + d0ur - (c[jj - 1] / b[jj - 1]) * dNul;
                        c[jj] = 0.0;
                        r1[jj] = -d0ur - (r1[jj - 1] / b[jj - 1]) * dNul;
                    }
                    ok = std::fabs(b[jj]) > tol;
                }
                if (ok) {
                    double el = r1[p.Ns - 1] / b[p.Ns - 1];
                    const double elast = el;
                    for (int jj = p.Ns - 2; jj >= 0; --jj) el = (r1[jj] - c[jj] * el) / b[jj];
                    ok = std::fabs(1.0 + elast + el) > 1e-12 * (1.0 + std::fabs(elast) + std::fabs(el));
                }
            }
            if (!ok) {
                g_last_error = "periodic interface system is singular (lambda = 0 leaves the constant mode free)";
                return HELM_ERR_SINGULAR;
            }
        }
    }

    // ---- device uploads ----
    const bool td = p.precision != HELM_FP32;           // spectrum / FFT precision is double
    const bool fd = p.precision == HELM_FP64;           // factor / transform precision is double
    const size_t nkx = p.Nx / 2 + 1, Nyf = p.dim == 3 ? p.Ny : 1;
    p.nrows = (long long)nkx * Nyf;
    p.elem_spec = p.nrows * N;
    int st;
    // the spectrum scratch also holds the half spectra of a derivative along y
    // (Nx x (Ny/2+1) rows per element), larger than the solve's when Nx > Ny,
    // and the coefficient spectrum of the eigen-basis pipeline (64 per row)
    p.eig_cand = p.Ns == 1 && !p.periodic && !p.fd && p.bc.alphal == 0.0 && p.bc.alphar == 0.0 &&
                 p.precision != HELM_FP32 && p.method == HELM_METHOD_FDM && (p.batch == 1 || p.dim == 2) &&
                 eig_shape_ok(p.dim, p.Nx, p.Ny, N);
    long long spec_elems = std::max(p.elem_spec, p.dim == 3 ? (long long)p.Nx * (p.Ny / 2 + 1) * N : 0LL);
    if (p.eig_cand && p.dim == 3) spec_elems = std::max(spec_elems, p.nrows * (long long)EIG_SLOTS);
    p.spec_bytes = (size_t)p.Ns * p.batch * spec_elems * (td ? 16 : 8);
    if ((st = p.alloc(&p.d_spec, p.spec_bytes))) return st;
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
    if ((st = p.upload((void**)&p.d_Dfull, D.data(), (size_t)N * N * sizeof(double)))) return st;
    {
        const int zero = 0;  // device status word of the kernels with bounded copy waits
        if ((st = p.upload((void**)&p.d_status, &zero, sizeof(int)))) return st;
    }
    if ((st = p.upload((void**)&p.d_D2full, D2.data(), (size_t)N * N * sizeof(double)))) return st;
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
    if (!lu && p.Ns == 1) {
        if (p.packed_elems == 0 && (st = setup_adjoint(p, A0, lam, V, Vi, prec_code, homs))) return st;
        if ((st = setup_fast(p, A0, prec_code))) return st;
    } else if (!lu && !p.periodic && p.packed_elems == 0 && p.batch == 1) {
        if ((st = setup_adjoint_multi(p, A0, V, Vi, prec_code))) return st;
    }
    if (!p.fast && rows_smem_bytes(p.method, prec_code, n, p.ld) > kMaxSmemPerBlock) {
        g_last_error = "GLL size too large for the row-solve kernel at this precision";
        return HELM_ERR_UNSUPPORTED;
    }
    return HELM_OK;
}

// Per-call options of a pipeline run (refinement sweeps of finite-difference
// plans): element size of the input read by the first pass and of the output
// written by the last (0: the plan's), and whether the last pass adds its
// result to the output (and, in an adjoint run, to the boundary cotangents and
// the lambda sum, which it then does not zero first).
struct PipeOpts {
    int io_in = 0, io_out = 0;
    bool accumulate = false;
};

// Outputs of the adjoint solve that its last (C2R) pass writes besides fbar.
struct AdjOut {
    double* glbar;
    double* grbar;
    const double* u;       // forward solution (lambda sum), or NULL
    double* lambda_bar;    // device scalar, zeroed before the pass, or NULL
    const double* sub;     // the first pass reads ubar - sub (data misfit), or NULL
};

static int fft_pass(Plan& p, int L, int mode, int dir, const void* in, void* out, long long in_row, long long out_row,
                    long long in_batch, long long out_batch, int ncols, int nbatch, double scale, const void* tw,
                    const double* gl, const double* gr, bool inject, bool io_double, int stage, cudaStream_t s,
                    const AdjOut* adj = nullptr, int deriv_order = 0, double deriv_w = 0.0,
                    const PipeOpts* po = nullptr)
{
    FftArgs a{};
    a.deriv_order = deriv_order;
    a.deriv_w = deriv_w;
    // the misfit subtrahend is read by the non-pipelined R2C kernel only
    const bool sub = adj && adj->sub && mode == FFT_R2C && stage == 0;
    a.in_sub = sub ? adj->sub : nullptr;
    if (adj && mode == FFT_C2R) {
        a.adj_mode = p.fd ? 2 : 1;
        a.adj_P = p.N;
        a.adj_scale_l = p.fd ? p.fd_scale_l : 1.0;
        a.adj_scale_r = p.fd ? p.fd_scale_r : 1.0;
        a.gbar_l = adj->glbar;
        a.gbar_r = adj->grbar;
        a.lam_u = adj->lambda_bar ? adj->u : nullptr;
        a.lam_out = adj->lambda_bar;
    }
    const bool acc = po && po->accumulate;
    if (adj && stage == 0 && !acc) a.zero_out = adj->lambda_bar;
    a.accumulate = (acc && stage == 3) ? 1 : 0;
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
    a.P = (mode == FFT_R2C && inject) ? p.N : 0;
    a.gl_batch = 0;
    a.gr_batch = p.Ns - 1;
    a.bc_add = p.fd ? 1 : 0;
    a.bc_scale_l = p.fd_scale_l;
    a.bc_scale_r = p.fd_scale_r;
    // batched plans: the caller's packed f (x pass) and u (inverse x pass)
    a.in_boff = stage == 0 ? p.d_boff : nullptr;
    a.out_boff = stage == 3 ? p.d_boff : nullptr;
    const long long ccols = (mode == FFT_C2C) ? ncols : (ncols + 1) / 2;
    const int td = p.precision != HELM_FP32;
    int io = (td || io_double) ? 8 : p.io_bytes;
    if (po && stage == 0 && po->io_in) io = po->io_in;
    if (po && stage == 3 && po->io_out) io = po->io_out;
    const int kmode = a.adj_mode ? (int)FFT_C2R_ADJ : mode;
    // Spectral derivatives take their own launch shape: the solve's variant of
    // the same stage is tuned for another kernel (on eigen-basis plans the
    // stage-1 bits select the y-convolution pass).  Unless pinned: 512-thread
    // CTAs from length 512; below, the radix-8 schedule, in the persistent
    // pipelined kernel for FP32 transforms.  Measured at 256^2 x 65 (FP64 I/O):
    // FP64 d/dx 33.8 us (radix-16 shapes 44.0, pipelined 37.9), FP32 31.7 us
    // (plain 33.8); at 512^2 x 33 FP64 d/dx 62.4 us (256 threads 76.7).
    const int dvar = p.deriv_var >= 0 ? p.deriv_var : (L >= 512 ? 8 : td ? 2 : 6);
    const int var = mode == FFT_DERIV ? dvar : sub ? (p.fft_var[stage] & ~4) : p.fft_var[stage];
    int e = launch_fft(L, kmode, dir, td, io, a, ccols * nbatch, s, var);
    if (e) return set_cuda_error((cudaError_t)e, "fft launch");
    return HELM_OK;
}

// The five kernels of a solve.  Forward: in = f with gl/gr injected into the
// GLL boundary slots of the spectrum, out = u.  Adjoint: in = ubar read in
// every slot, the transposed row solve, out = A^-T ubar in every slot.
static int run_pipeline(Plan& p, const void* in, const double* gl, const double* gr, void* out, bool adjoint,
                        cudaStream_t s, const AdjOut* adj = nullptr, const Workspace* ws = nullptr,
                        const PipeOpts* po = nullptr)
{
    const int N = p.N;
    void* const spec = ws ? ws->spec : p.d_spec;
    void* const cprime = ws ? ws->cprime : p.d_cprime;
    const long long cols = (long long)(p.dim == 3 ? p.Ny : 1) * N;  // real columns per x row
    const int nkx = p.Nx / 2 + 1;
    int st;
    auto mark = [&](int i) {
        if (p.stage_timing) cudaEventRecord(p.ev[i], s);
    };
    mark(0);
    // row variant in effect: the eigen-basis pipeline covers forward solves
    int rv = p.row_var;
    if (rv == 4 && (!p.eig_ok || (adjoint && !p.d_fmma_adj))) rv = p.precision == HELM_FP64 ? 0 : 3;
    if (rv == 3 && (p.precision != HELM_FP32_REFINE || !p.d_fmma)) rv = 0;
    if (rv == 4) {
        // three launches (3D) or one (2D): GLL transform + x FFT, y convolution,
        // inverse; stage events 1 and 4 bracket the middle pass
        EigArgs ea{};
        ea.f = static_cast<const double*>(in);
        ea.u = static_cast<double*>(out);
        ea.S = static_cast<double*>(spec);
        ea.gl = gl;
        ea.gr = gr;
        ea.ibl = 1.0 / p.bc.betal;
        ea.ibr = 1.0 / p.bc.betar;
        ea.x_stride = p.x_stride;
        ea.bc_x_stride = p.dim == 3 ? p.bc_x_stride : 1;
        ea.Ny = p.dim == 3 ? p.Ny : 1;
        ea.P = N;
        ea.n = p.n;
        ea.m = p.fm;
        ea.ms = p.fms;
        ea.mats = adjoint ? p.d_fmma_adj : p.d_fmma;
        if (adjoint) {
            ea.adjoint = 1;
            ea.sub = adj ? adj->sub : nullptr;
            ea.gbar_l = adj ? adj->glbar : nullptr;
            ea.gbar_r = adj ? adj->grbar : nullptr;
            ea.lam_out = adj ? adj->lambda_bar : nullptr;
            ea.lam_u = ea.lam_out ? adj->u : nullptr;
        }
        ea.hbc = p.d_hbc;
        ea.recip = p.d_frecip64;
        ea.grp_of_row = p.d_grp_of_row;
        ea.tw_x = p.d_tw_x;
        ea.tw_y = p.d_tw_y;
        ea.scale = 1.0 / ((double)p.Nx * (p.dim == 3 ? p.Ny : 1));
        ea.boff = p.d_boff;  // size-class plans of a batch: the packed offsets (one problem or more)
        ea.err = p.d_status;
        ea.tma = (p.dim == 3 && eig_tma_ok(ea, p.Nx)) ? 1 : 0;
        ea.conv_var = p.fft_var[1] & 1;
        ea.split = (p.dim == 3 && p.Nx >= 64 && (p.fft_var[1] & 2)) ? 1 : 0;
        int e = launch_eig_pass(0, p.dim, p.Nx, ea, p.batch, s);
        if (e) return set_cuda_error((cudaError_t)e, "eigen-basis pass 1");
        mark(1);
        if (p.dim == 3 && (e = launch_eig_pass(1, p.dim, p.Nx, ea, 1, s)))
            return set_cuda_error((cudaError_t)e, "eigen-basis pass 2");
        mark(2);
        mark(3);
        mark(4);
        if (p.dim == 3 && (e = launch_eig_pass(2, p.dim, p.Nx, ea, 1, s)))
            return set_cuda_error((cudaError_t)e, "eigen-basis pass 3");
        mark(5);
        return HELM_OK;
    }
    // 1. x: real-to-complex (forward: GLL boundary slots take the boundary data)
    if ((st = fft_pass(p, p.Nx, FFT_R2C, -1, in, spec, p.x_stride, cols, p.elem_stride, p.elem_spec, (int)cols,
                       p.Ns * p.batch, 1.0, p.d_tw_x, gl, gr, !adjoint, adjoint, 0, s, adj, 0, 0.0, po)))
        return st;
    mark(1);
    // FP64 and refined 3D plans may run stages 2-4 as one fused kernel per kx slab
    const bool slab = rv == 2 && p.slab_ok && p.fast && p.precision != HELM_FP32;
    // the FP64 tensor-core row kernels (FP64 plans; refined plans with variant 2, 3)
    const bool rows64 = p.precision == HELM_FP64 || slab || rv == 3;
    // 2. y: complex-to-complex along the middle axis
    if (p.dim == 3 && !slab &&
        (st = fft_pass(p, p.Ny, FFT_C2C, -1, spec, spec, N, N, (long long)p.Ny * N, (long long)p.Ny * N, N,
                       p.Ns * nkx, 1.0, p.d_tw_y, nullptr, nullptr, false, false, 1, s)))
        return st;
    mark(2);
    // 3. per-wavenumber collocation solves + interface sweep + combination
    RowArgs r{};
    r.spec = spec;
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
    r.lam = p.d_lam;
    r.sigma = p.d_sigma;
    r.sweeps = p.sweeps;
    r.al = p.bc.alphal;
    r.bl = p.bc.betal;
    r.ar = p.bc.alphar;
    r.br = p.bc.betar;
    if (!adjoint) {
        r.vinvT = p.d_vinvT;
        r.vT = p.d_vT;
        const bool hom = p.Ns > 1 || p.periodic || p.bc.alphal != 0.0 || p.bc.alphar != 0.0 || gl != nullptr ||
                         gr != nullptr;
        r.hom = hom ? p.d_hom : nullptr;
        r.homs = p.d_homs;
        r.d0 = p.d_d0;
        r.dN = p.d_dN;
        r.d2t = p.d_d2t;
    } else {
        r.adjoint = 1;
        r.vinvT = p.d_vtT;
        r.vT = p.d_vinvtT;
        r.hom = p.d_hom_adj;
        r.homs = p.d_homs_adj;
        r.d0 = p.d_c0;
        r.dN = p.d_cN;
        r.d2t = p.d_d2row;
        r.fhom = p.d_hom;
        r.fhoms = p.d_homs;
        r.fd0 = p.d_d0;
        r.fdN = p.d_dN;
    }
    r.periodic = p.periodic ? 1 : 0;
    const int prec = p.precision == HELM_FP64 ? 0 : (p.precision == HELM_FP32 ? 1 : 2);
    int e;
    if (p.fd) {
        ThomasArgs ta{};
        ta.spec = spec;
        ta.cprime = cprime;
        ta.nrows = p.nrows;
        ta.Ny = p.Ny;
        ta.Nz = N;
        ta.mx = p.d_mx;
        ta.my = p.d_my;
        ta.cz1 = p.fd_cz1;
        ta.lambda = p.lambda;
        ta.d_first = p.fd_dfirst;
        ta.s_first = p.fd_sfirst;
        ta.d_last = p.fd_dlast;
        ta.s_last = p.fd_slast;
        ta.transpose = adjoint ? 1 : 0;
        ta.half = rv & 1;
        e = launch_thomas(prec, ta, s);
    } else if (p.fast) {
        FdmArgs fa{};
        fa.spec = spec;
        fa.P = N;
        fa.n = p.n;
        fa.m = p.fm;
        fa.ms = p.fms;
        fa.ma = p.fma;
        fa.ld = p.fld;
        fa.nrows = (int)p.grp_rows.size();
        fa.rows = p.d_grp_rows;
        fa.row_grp = p.d_row_grp;
        fa.mats = adjoint ? p.d_fmats_adj : p.d_fmats;
        fa.d2f = adjoint ? p.d_fd2_adj : p.d_fd2;
        fa.recip = rows64 ? (const void*)p.d_frecip64 : p.d_frecip;
        fa.sigma = p.d_sigma;
        fa.sweeps = p.sweeps;
        fa.e0f = adjoint ? p.d_fc0 : p.d_fe0;
        fa.eNf = adjoint ? p.d_fcN : p.d_feN;
        fa.hvec = adjoint ? p.d_hom_adj : r.hom;
        fa.hscal = adjoint ? p.d_homs_adj : p.d_homs;
        // the transposed system's pl, pr are -A^-T of the Robin rows' interior
        // entries, which vanish for Dirichlet ends
        fa.hzero = (adjoint && !p.periodic && p.bc.alphal == 0.0 && p.bc.alphar == 0.0) ? 1 : 0;
        fa.periodic = p.periodic ? 1 : 0;
        fa.al = p.bc.alphal;
        fa.bl = p.bc.betal;
        fa.ar = p.bc.alphar;
        fa.br = p.bc.betar;
        fa.adjoint = adjoint ? 1 : 0;
        fa.mma_mats = adjoint ? p.d_fmma_adj : p.d_fmma;
        fa.mma16_mats = adjoint ? p.d_fmma16_adj : p.d_fmma16;
        fa.tc_mats = adjoint ? (const void*)p.d_ftc_adj : (const void*)p.d_ftc;
        fa.tc_m = adjoint ? p.d_ftcm_adj : p.d_ftcm;
        if (slab)
            e = launch_slab(fa, p.Ny, (N + 1) / 2, ((N + 1) / 2) | 1, p.d_tw_y, p.d_grp_of_row, nkx, s);
        else if (rows64 && fa.mma_mats)
            e = launch_fdm_mma(fa, s, rv == 3 ? 0 : rv & 1);
        else if (prec == 2 && fa.tc_mats && p.sweeps == 1 && rv == 0)
            e = launch_fdm_tc_refine(fa, s);
        else
            e = launch_fdm_fast(prec, fa, s, rv & 1);
    } else {
        e = launch_rows(p.method, prec, r, s);
    }
    if (e) return set_cuda_error((cudaError_t)e, "row-solve launch");
    mark(3);
    // 4. inverse y
    if (p.dim == 3 && !slab &&
        (st = fft_pass(p, p.Ny, FFT_C2C, 1, spec, spec, N, N, (long long)p.Ny * N, (long long)p.Ny * N, N,
                       p.Ns * nkx, 1.0, p.d_tw_y, nullptr, nullptr, false, false, 2, s)))
        return st;
    mark(4);
    // 5. x: complex-to-real, scaled by 1/(Nx Ny) (the reference's /Nx, /Ny)
    const double scale = 1.0 / ((double)p.Nx * (p.dim == 3 ? p.Ny : 1));
    if ((st = fft_pass(p, p.Nx, FFT_C2R, 1, spec, out, cols, p.x_stride, p.elem_spec, p.elem_stride, (int)cols,
                       p.Ns * p.batch, scale, p.d_tw_x, nullptr, nullptr, false, adjoint, 3, s, adj, 0, 0.0, po)))
        return st;
    mark(5);
    return HELM_OK;
}

// Autotuner, at plan creation, on the plan's own shape (zero input, CUDA
// events around each stage of whole solves):
//   1. the FFT launch variants 0..7 (and 8..15, the 512-thread CTAs, when a pass
//      is 512 or 1024 long), with the row variant held at its default, the
//      fastest kept per FFT stage;
//   2. with those FFT variants, each row variant of the plan's precision
//      (refined plans: the FP32 tensor-core kernels and the FP64 tensor-core
//      kernel), the fastest row stage kept;
//   3. whole solves of the fused alternatives (the slab kernel, the eigen-basis
//      pipeline) against the result of 1 and 2, the fastest kept.
// Results are cached per shape for the process; HELM_AUTOTUNE=0 in the
// environment keeps the default variants.
static std::mutex g_tune_mutex;
static std::map<std::string, std::array<int, 5>> g_tune_cache;  // 4 FFT variants, row variant

// Mean event times of the five stages over `reps` solves after one warm-up.
static bool time_stages(Plan& p, const void* f, void* u, int reps, float (&ms)[5])
{
    for (float& t : ms) t = 0.f;
    for (int rep = 0; rep <= reps; ++rep) {
        if (solve(p, f, nullptr, nullptr, u, 0)) return false;
        if (cudaEventSynchronize(p.ev[5]) != cudaSuccess) return false;
        if (rep == 0) continue;
        for (int i = 0; i < 5; ++i) {
            float t = 0;
            cudaEventElapsedTime(&t, p.ev[i], p.ev[i + 1]);
            ms[i] += t / reps;
        }
    }
    return true;
}

static int autotune(Plan& p)
{
    const char* env = std::getenv("HELM_AUTOTUNE");
    if (env && env[0] == '0') {
        if (p.eig_ok) p.row_var = 4;
        return HELM_OK;
    }
    const std::string key = std::string(p.fd ? "fd:" : "gll:") + std::to_string(p.dim) + ":" + std::to_string(p.Nx) +
                            ":" + std::to_string(p.Ny) + ":" +
                            std::to_string(p.N) + ":" + std::to_string(p.Ns) + ":" + std::to_string(p.precision) +
                            ":" + std::to_string(p.io_bytes) + ":" + std::to_string(p.x_stride) + ":" +
                            std::to_string(p.batch) + ":" + std::to_string(p.periodic) + ":" +
                            std::to_string(p.eig_ok) + ":" + std::to_string(p.sweeps) + ":" +
                            std::to_string(p.method);
    {
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) {
            for (int i = 0; i < 4; ++i) p.fft_var[i] = it->second[i];
            p.row_var = it->second[4];
            return HELM_OK;
        }
    }
    const long long elems = std::max((long long)p.Ns * p.elem_stride, p.packed_elems);
    const size_t bytes = (size_t)elems * (p.precision == HELM_FP32 ? p.io_bytes : 8);
    void *f = nullptr, *u = nullptr;
    if (cudaMalloc(&f, bytes) != cudaSuccess || cudaMalloc(&u, bytes) != cudaSuccess) {
        cudaGetLastError();
        if (f) cudaFree(f);
        if (p.eig_ok) p.row_var = 4;
        return HELM_OK;  // keep the defaults
    }
    cudaMemset(f, 0, bytes);
    const bool had = p.stage_timing;
    if (!p.ev[0])
        for (cudaEvent_t& e : p.ev) cudaEventCreate(&e);
    p.stage_timing = true;
    // 1. FFT variants, row variant 0
    float best[5] = {1e30f, 1e30f, 1e30f, 1e30f, 1e30f};
    int pick[5] = {0, 0, 0, 0, 0};
    const int nvar = (p.Nx >= 512 || (p.dim == 3 && p.Ny >= 512)) ? 16 : 8;
    p.row_var = 0;
    float ms[5];
    for (int v = 0; v < nvar; ++v) {
        for (int i = 0; i < 4; ++i) p.fft_var[i] = v;
        if (!time_stages(p, f, u, 3, ms)) { cudaGetLastError(); continue; }
        for (int i = 0; i < 5; ++i)
            if (i != 2 && ms[i] < best[i]) { best[i] = ms[i]; pick[i] = v; }
    }
    cudaGetLastError();
    const int stage_of_fft[4] = {0, 1, 3, 4};
    for (int i = 0; i < 4; ++i) p.fft_var[i] = pick[stage_of_fft[i]];
    // 2. row variants with the chosen FFT variants
    std::vector<int> rows_cand;
    if (p.fast) {
        rows_cand = {0, 1};
        if (p.precision == HELM_FP32_REFINE && p.d_fmma) rows_cand.push_back(3);
    } else if (p.fd && p.N <= 256) {
        rows_cand = {0, 1};  // the tridiagonal solves: a row per warp or per half-warp
    } else {
        rows_cand = {0};
    }
    float best_rows = 1e30f;
    int best_rv = 0;
    for (int rv : rows_cand) {
        p.row_var = rv;
        if (!time_stages(p, f, u, 3, ms)) { cudaGetLastError(); continue; }
        if (ms[2] < best_rows) { best_rows = ms[2]; best_rv = rv; }
    }
    cudaGetLastError();
    p.row_var = best_rv;
    // 3. fused alternatives, whole solves
    // (row variant, y-pass variant): the eigen-basis pipeline takes bit 0 of the
    // y-pass variant as the CTA shape of its second pass and bit 1 as the
    // pair-split form of its first and third passes
    const int yv = p.fft_var[1];
    std::vector<std::pair<int, int>> whole = {{p.row_var, yv}};
    if (p.slab_ok) whole.push_back({2, yv});
    if (p.eig_ok) whole.push_back({4, 0});
    if (p.eig_ok && p.dim == 3) whole.push_back({4, 1});
    if (p.eig_ok && p.dim == 3 && p.Nx >= 64) {
        whole.push_back({4, 2});
        whole.push_back({4, 3});
    }
    if (whole.size() > 1) {
        std::vector<float> tot(whole.size(), 0.f);
        bool ok = true;
        for (int rep = 0; rep < 6 && ok; ++rep)
            for (size_t k = 0; k < whole.size() && ok; ++k) {
                p.row_var = whole[k].first;
                p.fft_var[1] = whole[k].second;
                if (solve(p, f, nullptr, nullptr, u, 0) || cudaEventSynchronize(p.ev[5]) != cudaSuccess) {
                    ok = false;
                    break;
                }
                float t = 0;
                cudaEventElapsedTime(&t, p.ev[0], p.ev[5]);
                if (rep > 0) tot[k] += t;
            }
        cudaGetLastError();
        size_t bk = 0;
        if (ok)
            for (size_t k = 1; k < whole.size(); ++k)
                if (tot[k] < tot[bk]) bk = k;
        p.row_var = whole[bk].first;
        p.fft_var[1] = whole[bk].second;
    }
    p.stage_timing = had;
    cudaFree(f);
    cudaFree(u);
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    g_tune_cache[key] = {p.fft_var[0], p.fft_var[1], p.fft_var[2], p.fft_var[3], p.row_var};
    return HELM_OK;
}

// The stencil coefficients of a finite-difference plan's residual.
static FdResidualArgs fd_residual_args(const Plan& p)
{
    FdResidualArgs r{};
    const double dx = p.Lx / p.Nx, dy = p.Ly / p.Ny;
    r.Nx = p.Nx;
    r.Ny = p.Ny;
    r.Nz = p.N;
    r.cx1 = 1.0 / (dx * dx);
    r.cy1 = 1.0 / (dy * dy);
    r.cz1 = p.fd_cz1;
    r.lam = p.lambda;
    r.dfirst = p.fd_dfirst;
    r.sfirst = p.fd_sfirst;
    r.dlast = p.fd_dlast;
    r.slast = p.fd_slast;
    r.scale_l = p.fd_scale_l;
    r.scale_r = p.fd_scale_r;
    return r;
}

// Refined finite-difference solve (HELM_FP32_REFINE): the FP32 solve of the
// FP64 data, then p.sweeps times the FP64 residual r = f - A_h u and an FP32
// solve of A_h d = r whose last pass adds d into u.  The adjoint runs the same
// with the transposed stencil; its last passes also add into the boundary
// cotangents and the lambda sum.
static int refine_fd(Plan& p, const void* in, const double* gl, const double* gr, void* out, bool adjoint,
                     cudaStream_t s, const AdjOut* adj, const Workspace* ws)
{
    float* r = static_cast<float*>(ws && ws->refine ? ws->refine : p.d_refine);
    int st = run_pipeline(p, in, gl, gr, out, adjoint, s, adj, ws);
    FdResidualArgs ra = fd_residual_args(p);
    ra.rhs = static_cast<const double*>(in);
    ra.sub = adjoint && adj ? adj->sub : nullptr;
    ra.gl = adjoint ? nullptr : gl;
    ra.gr = adjoint ? nullptr : gr;
    ra.v = static_cast<const double*>(out);
    ra.r = r;
    ra.transpose = adjoint ? 1 : 0;
    PipeOpts po;
    po.io_in = 4;
    po.io_out = 8;
    po.accumulate = true;
    AdjOut cadj{};
    if (adj) {
        cadj = *adj;
        cadj.sub = nullptr;  // the residual already holds ubar - u_obs
    }
    for (int k = 0; k < p.sweeps && !st; ++k) {
        if (int e = launch_fd_residual(ra, s)) return set_cuda_error((cudaError_t)e, "refinement residual");
        st = run_pipeline(p, r, nullptr, nullptr, out, adjoint, s, adj ? &cadj : nullptr, ws, &po);
    }
    return st;
}

int solve(Plan& p, const void* f, const double* gl, const double* gr, void* u, cudaStream_t s, const Workspace* ws)
{
    if (p.fd_refine) return refine_fd(p, f, gl, gr, u, false, s, nullptr, ws);
    return run_pipeline(p, f, gl, gr, u, false, s, nullptr, ws);
}

size_t spec_bytes(const Plan& p) { return p.spec_bytes; }
size_t cprime_bytes(const Plan& p) { return p.d_cprime ? p.cprime_bytes : 0; }
size_t refine_bytes(const Plan& p) { return p.d_refine ? p.refine_bytes : 0; }

int check_solve_args(const Plan& p, const void* f, const double* gl, const double* gr, const void* u)
{
    if (!f || !u) {
        g_last_error = "f and u must be device pointers";
        return HELM_ERR_INVALID;
    }
    if (p.periodic && (gl || gr)) {
        g_last_error = "a plan periodic in the GLL direction takes no boundary data";
        return HELM_ERR_INVALID;
    }
    return HELM_OK;
}

int solve_adjoint(Plan& p, const double* ubar, double* fbar, double* glbar, double* grbar, const double* u,
                  double* lambda_bar, cudaStream_t s, const double* sub = nullptr)
{
    if (!p.adj_ready) {
        g_last_error = "adjoint needs a fast-diagonalisation plan (one GLL element, or several not periodic)";
        return HELM_ERR_UNSUPPORTED;
    }
    if (lambda_bar && !u) {
        g_last_error = "lambda_bar needs the forward solution u";
        return HELM_ERR_INVALID;
    }
    // the first pass zeroes lambda_bar; the last writes fbar, splits off glbar /
    // grbar and sums fbar * u into lambda_bar
    const AdjOut adj{glbar, grbar, u, lambda_bar, sub};
    if (p.fd_refine) return refine_fd(p, ubar, nullptr, nullptr, fbar, true, s, &adj, nullptr);
    return run_pipeline(p, ubar, nullptr, nullptr, fbar, true, s, &adj);
}

// du = M u along the GLL index of every row (helm_deriv.cu).
int gll_derivative(Plan& p, int order, const void* u, void* du, cudaStream_t s)
{
    if (p.fd || p.batch > 1 || !p.d_Dfull) {
        g_last_error = "GLL derivative needs a Fourier x GLL plan";
        return HELM_ERR_UNSUPPORTED;
    }
    GllDerivArgs a{};
    a.in = u;
    a.out = du;
    a.M = order == 1 ? p.d_Dfull : p.d_D2full;
    a.P = p.N;
    a.order = order;
    a.nx = p.Nx;
    a.rows_per_x = p.dim == 3 ? p.Ny : 1;
    a.nrows = (long long)p.Ns * p.Nx * a.rows_per_x;
    a.x_stride = p.x_stride;
    a.elem_stride = p.elem_stride;
    a.err = p.d_status;
    const int io_double = (p.precision != HELM_FP32 || p.io_bytes == 8) ? 1 : 0;
    const int e = launch_gll_deriv(io_double, a, s);
    if (e) return set_cuda_error((cudaError_t)e, "GLL derivative launch");
    return HELM_OK;
}

// Spectral derivative along x (axis 0) or y (axis 1, 3D): a real-to-complex
// pass along the axis into the spectrum scratch, then the complex-to-real pass
// back with the multiplier (i 2 pi K / L)^order applied on its load.
int fourier_derivative(Plan& p, int axis, int order, const void* u, void* du, cudaStream_t s)
{
    if (p.batch > 1) { g_last_error = "derivative of a batched plan"; return HELM_ERR_UNSUPPORTED; }
    // one launch per call (per element when elements are not packed back to
    // back along y): forward transform, multiplication, inverse transform
    const int N = p.N;
    const bool tdbl = p.precision != HELM_FP32;
    int st;
    if (axis == 0) {
        const long long cols = (long long)(p.dim == 3 ? p.Ny : 1) * N;
        const double w = 2.0 * kRefPi / p.Lx;
        return fft_pass(p, p.Nx, FFT_DERIV, -1, u, du, p.x_stride, p.x_stride, p.elem_stride, p.elem_stride,
                        (int)cols, p.Ns, 1.0 / p.Nx, p.d_tw_x, nullptr, nullptr, false, false, 0, s, nullptr, order, w);
    }
    if (axis != 1 || p.dim != 3) {
        g_last_error = "axis must be 0 (x) or, for 3D plans, 1 (y)";
        return HELM_ERR_INVALID;
    }
    const double w = 2.0 * kRefPi / p.Ly;
    const bool uniform = p.elem_stride == (long long)p.Nx * p.x_stride;
    const int nb = uniform ? p.Ns * p.Nx : p.Nx;
    const size_t esz = (tdbl || p.io_bytes == 8) ? 8 : 4;
    for (int e = 0; e < (uniform ? 1 : p.Ns); ++e) {
        const char* ue = static_cast<const char*>(u) + (size_t)e * p.elem_stride * esz;
        char* de = static_cast<char*>(du) + (size_t)e * p.elem_stride * esz;
        if ((st = fft_pass(p, p.Ny, FFT_DERIV, -1, ue, de, N, N, p.x_stride, p.x_stride, N, nb, 1.0 / p.Ny, p.d_tw_y,
                           nullptr, nullptr, false, false, 1, s, nullptr, order, w)))
            return st;
    }
    return HELM_OK;
}

// Finite-difference variant: the second-order stencil of HypreFDM
// (HelmholtzSolvers/HypreFDM/src/Helmholtz3D_MPI.cpp:297-410) with periodic x
// and y (dx = Lx/Nx, dy = Ly/Ny) and Nz interior points in z (dz = Lz/(Nz+1)),
// one-sided second-order Robin rows at z = zl (back) and z = zr (front).  The
// Robin rows are eliminated into the first and last interior equations, whose
// right-hand sides then carry -cz1/a0 * g_back and -cz1/e0 * g_front.
static int create_fd_plan(int Nx, int Ny, int Nz, double xl, double xr, double yl, double yr, double zl, double zr,
                          const helm_robin_t* bc, double lambda, int precision, helm_plan_t* out)
{
    if (!out) return HELM_ERR_INVALID;
    *out = nullptr;
    if (Nz < 2 || Nz > 4096 || Nx < 4 || Ny < 4) { g_last_error = "size out of range"; return HELM_ERR_INVALID; }
    if (!is_pow2(Nx) || !is_pow2(Ny)) { g_last_error = "N has to be 2^n"; return HELM_ERR_NOT_POW2; }
    if (Nx > 1024 || Ny > 1024) { g_last_error = "Fourier size beyond 4..1024"; return HELM_ERR_UNSUPPORTED; }
    if (precision < HELM_FP64 || precision > HELM_FP32_REFINE) return HELM_ERR_INVALID;
    if (!(xr > xl) || !(yr > yl) || !(zr > zl)) { g_last_error = "empty domain"; return HELM_ERR_INVALID; }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        g_last_error = "no CUDA device";
        return HELM_ERR_NO_DEVICE;
    }
    Plan* p = new (std::nothrow) Plan();
    if (!p) return HELM_ERR_OOM;
    cudaGetDevice(&p->device);
    p->fd = true;
    p->dim = 3;
    p->Nx = Nx;
    p->Ny = Ny;
    p->N = Nz;
    p->n = Nz;
    p->Ns = 1;
    p->xl = xl; p->xr = xr; p->yl = yl; p->yr = yr; p->zl = zl; p->zr = zr;
    p->Lx = xr - xl;
    p->Ly = yr - yl;
    p->Lgll = zr - zl;
    p->bc = bc ? *bc : helm_robin_t{0.0, 1.0, 0.0, 1.0};
    p->lambda = lambda;
    // HELM_FP32_REFINE: FP32 spectrum and tridiagonal solves, FP64 input and
    // output, two FP64-residual refinement sweeps per solve (refine_fd)
    p->fd_refine = precision == HELM_FP32_REFINE;
    p->precision = precision == HELM_FP64 ? HELM_FP64 : HELM_FP32;
    if (p->fd_refine) p->sweeps = 2;
    p->method = HELM_METHOD_LU;
    p->x_stride = (long long)Ny * Nz;
    p->elem_stride = (long long)Nx * Ny * Nz;
    p->bc_x_stride = Ny;
    const double dx = p->Lx / Nx, dy = p->Ly / Ny, dz = p->Lgll / (Nz + 1);
    const double cx1 = 1.0 / (dx * dx), cy1 = 1.0 / (dy * dy), cz0 = 1.0 / dz, cz1 = 1.0 / (dz * dz);
    const double a0 = 1.5 * p->bc.alphal * cz0 + p->bc.betal, a1 = -2.0 * p->bc.alphal * cz0,
                 a2 = 0.5 * p->bc.alphal * cz0;
    const double e0 = 1.5 * p->bc.alphar * cz0 + p->bc.betar, e1 = -2.0 * p->bc.alphar * cz0,
                 e2 = 0.5 * p->bc.alphar * cz0;
    if (a0 == 0.0 || e0 == 0.0) {
        delete p;
        g_last_error = "degenerate Robin row";
        return HELM_ERR_SINGULAR;
    }
    p->fd_cz1 = cz1;
    p->fd_dfirst = -cz1 * a1 / a0;
    p->fd_sfirst = cz1 - cz1 * a2 / a0;
    p->fd_dlast = -cz1 * e1 / e0;
    p->fd_slast = cz1 - cz1 * e2 / e0;
    p->fd_scale_l = -cz1 / a0;
    p->fd_scale_r = -cz1 / e0;
    const int nkx = Nx / 2 + 1;
    std::vector<double> mx(nkx), my(Ny);
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int k = 0; k < nkx; ++k) { const long double s = std::sin(pi * k / Nx); mx[k] = (double)(4.0L * cx1 * s * s); }
    for (int k = 0; k < Ny; ++k) { const long double s = std::sin(pi * k / Ny); my[k] = (double)(4.0L * cy1 * s * s); }
    p->nrows = (long long)nkx * Ny;
    p->elem_spec = p->nrows * Nz;
    const bool td = p->precision != HELM_FP32;
    p->spec_bytes = (size_t)p->elem_spec * (td ? 16 : 8);
    int st = p->alloc(&p->d_spec, p->spec_bytes);
    // elimination scratch of the thread-per-row tridiagonal kernel (Nz > 512 only)
    p->cprime_bytes = (size_t)p->elem_spec * (td ? 8 : 4);
    if (!st && Nz > 512) st = p->alloc(&p->d_cprime, p->cprime_bytes);
    // the residual of a refinement sweep, then its correction (FP32)
    p->refine_bytes = (size_t)Nx * Ny * Nz * sizeof(float);
    if (!st && p->fd_refine) st = p->alloc(&p->d_refine, p->refine_bytes);
    if (!st) st = p->upload((void**)&p->d_mx, mx.data(), mx.size() * sizeof(double));
    if (!st) st = p->upload((void**)&p->d_my, my.data(), my.size() * sizeof(double));
    auto up_tw = [&](int L, void** d) -> int {
        if (td) { auto t = twiddles<double>(L); return p->upload(d, t.data(), t.size() * sizeof(double)); }
        auto t = twiddles<float>(L);
        return p->upload(d, t.data(), t.size() * sizeof(float));
    };
    if (!st) st = up_tw(Nx, &p->d_tw_x);
    if (!st) st = up_tw(Ny, &p->d_tw_y);
    p->adj_ready = true;
    if (!st) st = autotune(*p);
    if (st) { p->release(); delete p; return st; }
    *out = reinterpret_cast<helm_plan_t>(p);
    return HELM_OK;
}

static int create_plan(int dim, int Nx, int Ny, int Ngll_total, int N, double xl, double xr, double yl, double yr,
                       double zl, double zr, const helm_robin_t* bc, double lambda, int precision, int method,
                       helm_plan_t* out, bool periodic = false, helm_operator_fn op = nullptr,
                       void* op_user = nullptr)
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
    p->periodic = periodic;
    if (periodic) p->bc = helm_robin_t{0.0, 1.0, 0.0, 1.0};  // unused: no boundary rows
    p->lambda = lambda;
    p->precision = precision;
    p->method = method;
    p->op_cb = op;
    p->op_user = op_user;
    const long long cols = (long long)p->Ny * N;
    p->x_stride = cols;
    p->elem_stride = (long long)Nx * cols;
    p->bc_x_stride = p->Ny;
    int st = setup_plan(*p);
    if (!st) st = autotune(*p);
    if (st) { p->release(); delete p; return st; }
    *out = reinterpret_cast<helm_plan_t>(p);
    return HELM_OK;
}

void set_last_error(const char* msg) { g_last_error = msg; }

int create_batch_class(int Nx, int N, double xl, double xr, double yl, double yr, const std::vector<double>& lams,
                       const std::vector<long long>& offs, long long packed_elems, int precision, Plan** out)
{
    *out = nullptr;
    if (lams.empty() || lams.size() != offs.size()) return HELM_ERR_INVALID;
    if (N < 3 || N > 129 || Nx < 4) { g_last_error = "size out of range"; return HELM_ERR_INVALID; }
    if (!is_pow2(Nx)) { g_last_error = "N has to be 2^n"; return HELM_ERR_NOT_POW2; }
    if (Nx > 1024) { g_last_error = "Fourier size beyond 4..1024"; return HELM_ERR_UNSUPPORTED; }
    Plan* p = new (std::nothrow) Plan();
    if (!p) return HELM_ERR_OOM;
    cudaGetDevice(&p->device);
    p->dim = 2;
    p->Nx = Nx;
    p->Ny = 1;
    p->N = N;
    p->Ns = 1;
    p->xl = xl; p->xr = xr; p->yl = yl; p->yr = yr;
    p->Lx = xr - xl;
    p->Ly = yr - yl;
    p->Lgll = yr - yl;
    p->bc = helm_robin_t{0.0, 1.0, 0.0, 1.0};
    p->batch = (int)lams.size();
    p->lambdas = lams;
    p->lambda = lams[0];
    p->precision = precision;
    p->method = HELM_METHOD_AUTO;
    p->x_stride = N;
    p->elem_stride = (long long)Nx * N;
    p->bc_x_stride = 1;
    p->packed_elems = packed_elems;
    int st = setup_plan(*p);
    if (!st && !p->fast) { g_last_error = "batched plans need the folded fast-diagonalisation path"; st = HELM_ERR_UNSUPPORTED; }
    if (!st) st = p->upload((void**)&p->d_boff, offs.data(), offs.size() * sizeof(long long));
    if (!st) st = autotune(*p);
    if (st) { p->release(); delete p; return st; }
    *out = p;
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

int helm_fd3d_plan_create(int Nx, int Ny, int Nz, double xl, double xr, double yl, double yr, double zl, double zr,
                          const helm_robin_t* bc, double lambda, int precision, helm_plan_t* plan)
{
    try {
        return helm::create_fd_plan(Nx, Ny, Nz, xl, xr, yl, yr, zl, zr, bc, lambda, precision, plan);
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

int helm2d_periodic_plan_create(int Nx, int Ny, int N, double xl, double xr, double yl, double yr, double lambda,
                                int precision, int method, helm_plan_t* plan)
{
    try {
        return helm::create_plan(2, Nx, 1, Ny, N, xl, xr, yl, yr, 0.0, 1.0, nullptr, lambda, precision, method, plan,
                                 true);
    } catch (...) {
        return HELM_ERR_OOM;
    }
}

int helm3d_periodic_plan_create(int Nx, int Ny, int Nz, int N, double xl, double xr, double yl, double yr, double zl,
                                double zr, double lambda, int precision, int method, helm_plan_t* plan)
{
    try {
        return helm::create_plan(3, Nx, Ny, Nz, N, xl, xr, yl, yr, zl, zr, nullptr, lambda, precision, method, plan,
                                 true);
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
    if (bytes == 4 && (p.precision != HELM_FP32 || p.fd_refine)) return HELM_ERR_UNSUPPORTED;
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
    if (!plan) return HELM_ERR_INVALID;
    Plan& p = *reinterpret_cast<Plan*>(plan);
    if (int st = helm::check_solve_args(p, f, gl, gr, u)) return st;
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
    if (!plan || !ubar || !fbar || (lambda_bar && !u)) return HELM_ERR_INVALID;
    Plan& p = *reinterpret_cast<Plan*>(plan);
    if (p.periodic && (glbar || grbar)) {
        helm::set_last_error("a plan periodic in the GLL direction has no boundary data to differentiate");
        return HELM_ERR_INVALID;
    }
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != p.device) cudaSetDevice(p.device);
    int st = helm::solve_adjoint(p, ubar, fbar, glbar, grbar, u, lambda_bar, static_cast<cudaStream_t>(stream));
    if (cur != p.device) cudaSetDevice(cur);
    return st;
}

int helm_gll_derivative(helm_plan_t plan, int order, const void* u, void* du, void* stream)
{
    if (!plan || !u || !du || (order != 1 && order != 2)) return HELM_ERR_INVALID;
    Plan& p = *reinterpret_cast<Plan*>(plan);
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != p.device) cudaSetDevice(p.device);
    int st = helm::gll_derivative(p, order, u, du, static_cast<cudaStream_t>(stream));
    if (cur != p.device) cudaSetDevice(cur);
    return st;
}

int helm_fourier_derivative(helm_plan_t plan, int axis, int order, const void* u, void* du, void* stream)
{
    if (!plan || !u || !du || (order != 1 && order != 2)) return HELM_ERR_INVALID;
    Plan& p = *reinterpret_cast<Plan*>(plan);
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != p.device) cudaSetDevice(p.device);
    int st = helm::fourier_derivative(p, axis, order, u, du, static_cast<cudaStream_t>(stream));
    if (cur != p.device) cudaSetDevice(cur);
    return st;
}

int helm_solve_adjoint_misfit(helm_plan_t plan, const double* u, const double* u_obs, double* fbar, double* glbar,
                              double* grbar, double* lambda_bar, void* stream)
{
    if (!plan || !u || !u_obs || !fbar) return HELM_ERR_INVALID;
    Plan& p = *reinterpret_cast<Plan*>(plan);
    if (p.periodic && (glbar || grbar)) {
        helm::set_last_error("a plan periodic in the GLL direction has no boundary data to differentiate");
        return HELM_ERR_INVALID;
    }
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != p.device) cudaSetDevice(p.device);
    int st = helm::solve_adjoint(p, u, fbar, glbar, grbar, u, lambda_bar, static_cast<cudaStream_t>(stream), u_obs);
    if (cur != p.device) cudaSetDevice(cur);
    return st;
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

int helm_plan_device_status(helm_plan_t plan, int* code, int reset)
{
    if (!plan || !code) return HELM_ERR_INVALID;
    Plan& p = *reinterpret_cast<Plan*>(plan);
    *code = 0;
    if (!p.d_status) return HELM_OK;
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != p.device) cudaSetDevice(p.device);
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(code, p.d_status, sizeof(int), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && reset) e = cudaMemset(p.d_status, 0, sizeof(int));
    if (cur != p.device) cudaSetDevice(cur);
    if (e != cudaSuccess) return helm::set_cuda_error(e, "device status");
    return HELM_OK;
}

int helm_plan_set_stage_timing(helm_plan_t plan, int enable)
{
    if (!plan) return HELM_ERR_INVALID;
    Plan& p = *reinterpret_cast<Plan*>(plan);
    if (enable && !p.ev[0])
        for (cudaEvent_t& e : p.ev) {
            cudaError_t err = cudaEventCreate(&e);
            if (err != cudaSuccess) return helm::set_cuda_error(err, "cudaEventCreate");
        }
    p.stage_timing = enable != 0;
    return HELM_OK;
}

int helm_plan_stage_times(helm_plan_t plan, float* ms5)
{
    if (!plan || !ms5) return HELM_ERR_INVALID;
    Plan& p = *reinterpret_cast<Plan*>(plan);
    if (!p.stage_timing) return HELM_ERR_INVALID;
    cudaError_t err = cudaEventSynchronize(p.ev[5]);
    if (err != cudaSuccess) return helm::set_cuda_error(err, "cudaEventSynchronize");
    for (int i = 0; i < 5; ++i) {
        float t = 0.0f;
        err = cudaEventElapsedTime(&t, p.ev[i], p.ev[i + 1]);
        if (err != cudaSuccess) return helm::set_cuda_error(err, "cudaEventElapsedTime");
        ms5[i] = t;
    }
    return HELM_OK;
}

int helm_plan_get_launch_variants(helm_plan_t plan, int* fft4, int* rows)
{
    if (!plan) return HELM_ERR_INVALID;
    const Plan& p = *reinterpret_cast<const Plan*>(plan);
    if (fft4)
        for (int i = 0; i < 4; ++i) fft4[i] = p.fft_var[i];
    if (rows) *rows = p.row_var;
    return HELM_OK;
}

int helm_plan_set_launch_variants(helm_plan_t plan, const int* fft4, int rows)
{
    if (!plan || !fft4 || rows < 0 || rows > 4) return HELM_ERR_INVALID;
    for (int i = 0; i < 4; ++i)
        if (fft4[i] < 0 || fft4[i] > 15) return HELM_ERR_INVALID;
    Plan& p = *reinterpret_cast<Plan*>(plan);
    if (rows == 2 && !p.slab_ok) {
        helm::set_last_error("the fused slab kernel needs an FP64 or refined 3D plan with one element, at most 65 points, Ny in {64, 128, 256}");
        return HELM_ERR_UNSUPPORTED;
    }
    if (rows == 3 && (p.precision != HELM_FP32_REFINE || !p.d_fmma)) {
        helm::set_last_error("row variant 3 (FP64 tensor-core rows) is for refined plans with one element");
        return HELM_ERR_UNSUPPORTED;
    }
    if (rows == 4 && !p.eig_ok) {
        helm::set_last_error("the eigen-basis pipeline needs an FP64 or refined plan with one element, Dirichlet ends, "
                             "at most 66 points, Nx in {8..256} and Ny in {4..512}");
        return HELM_ERR_UNSUPPORTED;
    }
    for (int i = 0; i < 4; ++i) p.fft_var[i] = fft4[i];
    p.row_var = rows;
    return HELM_OK;
}

int helm_plan_set_derivative_variant(helm_plan_t plan, int variant)
{
    if (!plan || variant < -1 || variant > 15) return HELM_ERR_INVALID;
    reinterpret_cast<Plan*>(plan)->deriv_var = variant;
    return HELM_OK;
}

int helm_plan_get_derivative_variant(helm_plan_t plan, int* variant)
{
    if (!plan || !variant) return HELM_ERR_INVALID;
    *variant = reinterpret_cast<Plan*>(plan)->deriv_var;
    return HELM_OK;
}

int helm_plan_set_operator_callback(helm_plan_t plan, helm_operator_fn op, void* user)
{
    if (!plan || !op) return HELM_ERR_INVALID;
    Plan& p = *reinterpret_cast<Plan*>(plan);
    if (p.fd || p.batch > 1) {
        helm::set_last_error("operator callbacks apply to the GLL plans (not finite-difference or batch plans)");
        return HELM_ERR_UNSUPPORTED;
    }
    if (p.precision == HELM_FP32_REFINE) {
        helm::set_last_error("a refined plan has no FP64 residual for a user operator: use an FP64 or FP32 plan");
        return HELM_ERR_UNSUPPORTED;
    }
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != p.device) cudaSetDevice(p.device);
    helm_plan_t fresh = nullptr;
    const int st = helm::create_plan(p.dim, p.Nx, p.Ny, p.Ns * p.N, p.N, p.xl, p.xr, p.yl, p.yr, p.zl, p.zr, &p.bc,
                                     p.lambda, p.precision, HELM_METHOD_LU, &fresh, p.periodic, op, user);
    if (cur != p.device) cudaSetDevice(cur);
    if (st) return st;
    Plan& q = *reinterpret_cast<Plan*>(fresh);
    q.x_stride = p.x_stride;
    q.elem_stride = p.elem_stride;
    q.bc_x_stride = p.bc_x_stride;
    q.io_bytes = p.io_bytes;
    q.sweeps = p.sweeps;
    std::swap(p, q);
    return helm_plan_destroy(fresh);  // frees the old plan's contents
}

int helm_debug_fail_alloc(long long n)
{
    helm::g_alloc_fault.store(n < 0 ? -1 : n);
    return HELM_OK;
}

const char* helm_plan_kernels(helm_plan_t plan)
{
    if (!plan) return "";
    Plan& p = *reinterpret_cast<Plan*>(plan);
    int rv = p.row_var;
    if (rv == 4 && !p.eig_ok) rv = p.precision == HELM_FP64 ? 0 : 3;
    if (rv == 3 && (p.precision != HELM_FP32_REFINE || !p.d_fmma)) rv = 0;
    std::string k;
    if (rv == 4) {
        if (p.dim != 3) k = "eig_solve2d_kernel";
        else if (p.Nx >= 64 && (p.fft_var[1] & 2)) k = "eig_fwd_split_kernel eig_conv_kernel eig_inv_split_kernel";
        else k = "eig_fwd_kernel eig_conv_kernel eig_inv_kernel";
    } else {
        const bool slab = rv == 2 && p.slab_ok && p.fast && p.precision != HELM_FP32;
        std::string rows;
        if (p.fd) rows = p.N <= 512 ? "thomas_warp_kernel" : "thomas_kernel";
        else if (!p.fast) rows = "rows_kernel";
        else if (slab) rows = "slab_kernel";
        else if ((p.precision == HELM_FP64 || rv == 3) && p.d_fmma) rows = (rv == 3 || rv == 0) ? "fdm_mma16_kernel" : "fdm_mma_kernel";
        else if (p.precision == HELM_FP32_REFINE && p.d_ftc && p.sweeps == 1 && rv == 0) rows = "fdm_tc_refine_kernel";
        else rows = "fdm_fast_kernel";
        const std::string fft = p.fft_var[0] & 4 ? "fft_pipe_kernel" : "fft_kernel";
        k = fft + "(x)";
        if (p.dim == 3 && !slab) k += " fft_kernel(y)";
        k += " " + rows;
        if (p.dim == 3 && !slab) k += " fft_kernel(y-inv)";
        k += std::string(" ") + (p.fft_var[3] & 4 ? "fft_pipe_kernel" : "fft_kernel") + "(x-inv)";
        if (p.fd_refine) {  // per sweep: the residual, then a correction solve
            const std::string one = k;
            for (int i = 0; i < p.sweeps; ++i) k += " fd_residual_kernel " + one;
        }
    }
    p.kernel_names = k;
    return p.kernel_names.c_str();
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
