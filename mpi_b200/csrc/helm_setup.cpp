// Host-side FP64 setup of a Helmholtz plan (see helm_setup.hpp).
#include "helm_setup.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace helm {

using ld = long double;

static const ld kPiL = 3.141592653589793238462643383279502884L;

// P_n(x) and P_n'(x) by the three-term recurrence, long double.
static void legendre(int n, ld x, ld& p, ld& dp)
{
    ld pm1 = 1.0L, pc = x;
    if (n == 0) { p = 1.0L; dp = 0.0L; return; }
    for (int k = 2; k <= n; ++k) {
        ld pn = ((2.0L * k - 1.0L) * x * pc - (k - 1.0L) * pm1) / k;
        pm1 = pc;
        pc = pn;
    }
    p = pc;
    dp = (n == 1) ? 1.0L : n * (x * pc - pm1) / (x * x - 1.0L);
}

void gll_nodes(int N, double* x)
{
    const int n = N - 1;
    std::vector<ld> t(N);
    t[0] = -1.0L;
    t[N - 1] = 1.0L;
    for (int i = 1; i < N - 1; ++i) {
        ld s = -std::cos(kPiL * i / n);  // Chebyshev-Gauss-Lobatto start
        for (int it = 0; it < 200; ++it) {
            ld p, dp;
            legendre(n, s, p, dp);
            // Legendre ODE: (1-s^2) P'' = 2 s P' - n(n+1) P
            ld d2p = (2.0L * s * dp - n * (n + 1.0L) * p) / (1.0L - s * s);
            ld ds = dp / d2p;
            s -= ds;
            if (std::fabs(ds) < 1e-21L) break;
        }
        t[i] = s;
    }
    for (int i = 0; i < N / 2; ++i) {  // exact symmetry about 0
        ld h = 0.5L * (t[N - 1 - i] - t[i]);
        t[i] = -h;
        t[N - 1 - i] = h;
    }
    if (N % 2) t[N / 2] = 0.0L;
    for (int i = 0; i < N; ++i) x[i] = (double)t[i];
}

void gll_derivative(int N, const double* x, double* D)
{
    std::vector<ld> P(N);
    for (int i = 0; i < N; ++i) { ld dp; legendre(N - 1, (ld)x[i], P[i], dp); }
    for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j)
            D[i * N + j] = (i == j) ? 0.0 : (double)(P[i] / (P[j] * ((ld)x[i] - (ld)x[j])));
    D[0] = -0.25 * N * (N - 1);
    D[N * N - 1] = 0.25 * N * (N - 1);
}

void matmul(int N, const double* A, const double* B, double* C)
{
    for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j) {
            double s = 0.0;
            for (int k = 0; k < N; ++k) s += A[i * N + k] * B[k * N + j];
            C[i * N + j] = s;
        }
}

bool lu_factor(int n, double* A, int* perm)
{
    std::vector<double> scale(n);
    for (int r = 0; r < n; ++r) {
        double m = 0.0;
        for (int c = 0; c < n; ++c) m = std::max(m, std::fabs(A[r * n + c]));
        scale[r] = m;
        perm[r] = r;
    }
    for (int k = 0; k < n - 1; ++k) {
        int best = k;
        double bestv = std::fabs(A[k * n + k]) / scale[k];
        for (int r = k + 1; r < n; ++r) {
            double v = std::fabs(A[r * n + k]) / scale[r];
            if (v > bestv) { bestv = v; best = r; }
        }
        if (!(bestv > 1e-12)) return false;
        if (best != k) {
            for (int c = 0; c < n; ++c) std::swap(A[k * n + c], A[best * n + c]);
            std::swap(perm[k], perm[best]);
        }
        const double inv = A[k * n + k];
        for (int r = k + 1; r < n; ++r) {
            double m = A[r * n + k] / inv;
            A[r * n + k] = m;
            for (int c = k + 1; c < n; ++c) A[r * n + c] -= m * A[k * n + c];
        }
    }
    return std::fabs(A[(n - 1) * n + n - 1]) > 0.0;
}

void lu_solve(int n, const double* LU, const int* perm, double* b)
{
    std::vector<double> y(n);
    for (int i = 0; i < n; ++i) y[i] = b[perm[i]];
    for (int i = 1; i < n; ++i) {
        double s = y[i];
        for (int k = 0; k < i; ++k) s -= LU[i * n + k] * y[k];
        y[i] = s;
    }
    for (int i = n - 1; i >= 0; --i) {
        double s = y[i];
        for (int k = i + 1; k < n; ++k) s -= LU[i * n + k] * y[k];
        y[i] = s / LU[i * n + i];
    }
    for (int i = 0; i < n; ++i) b[i] = y[i];
}

// ----------------------------------------------------------- eigen solver --

// Long-double LU with partial pivoting (for inverse iteration and V^-1).
static bool lu_ld(int n, std::vector<ld>& A, std::vector<int>& p)
{
    p.resize(n);
    for (int i = 0; i < n; ++i) p[i] = i;
    for (int k = 0; k < n; ++k) {
        int best = k;
        for (int r = k + 1; r < n; ++r)
            if (std::fabs(A[r * n + k]) > std::fabs(A[best * n + k])) best = r;
        if (A[best * n + k] == 0.0L) A[best * n + k] = 1e-30L;  // exactly singular shift
        if (best != k) {
            for (int c = 0; c < n; ++c) std::swap(A[k * n + c], A[best * n + c]);
            std::swap(p[k], p[best]);
        }
        for (int r = k + 1; r < n; ++r) {
            ld m = A[r * n + k] / A[k * n + k];
            A[r * n + k] = m;
            for (int c = k + 1; c < n; ++c) A[r * n + c] -= m * A[k * n + c];
        }
    }
    return true;
}

static void lu_ld_solve(int n, const std::vector<ld>& LU, const std::vector<int>& p, std::vector<ld>& b)
{
    std::vector<ld> y(n);
    for (int i = 0; i < n; ++i) y[i] = b[p[i]];
    for (int i = 1; i < n; ++i)
        for (int k = 0; k < i; ++k) y[i] -= LU[i * n + k] * y[k];
    for (int i = n - 1; i >= 0; --i) {
        for (int k = i + 1; k < n; ++k) y[i] -= LU[i * n + k] * y[k];
        y[i] /= LU[i * n + i];
    }
    b = y;
}

// Eigenvalues of a real upper-Hessenberg matrix with real spectrum by
// explicitly shifted QR (Givens rotations) with Wilkinson shifts and
// deflation at the bottom of the active block.
static bool hessenberg_qr_eigenvalues(int n, std::vector<ld>& H, std::vector<ld>& ev)
{
    ev.assign(n, 0.0L);
    int hi = n - 1;
    int iter = 0;
    std::vector<ld> cs(n), sn(n);
    while (hi >= 0) {
        if (hi == 0) { ev[0] = H[0]; break; }
        // find the start of the unreduced block ending at hi
        int lo = hi;
        while (lo > 0) {
            ld s = std::fabs(H[(lo - 1) * n + lo - 1]) + std::fabs(H[lo * n + lo]);
            if (std::fabs(H[lo * n + lo - 1]) <= 1e-21L * s) { H[lo * n + lo - 1] = 0.0L; break; }
            --lo;
        }
        if (lo == hi) { ev[hi] = H[hi * n + hi]; --hi; iter = 0; continue; }
        if (++iter > 500) return false;
        // Wilkinson shift from the trailing 2x2 block
        ld a = H[(hi - 1) * n + hi - 1], b = H[(hi - 1) * n + hi];
        ld c = H[hi * n + hi - 1], d = H[hi * n + hi];
        ld tr = a + d, det = a * d - b * c, disc = 0.25L * tr * tr - det;
        ld mu;
        if (disc >= 0.0L) {
            ld r = std::sqrt(disc);
            ld l1 = 0.5L * tr + r, l2 = 0.5L * tr - r;
            mu = (std::fabs(l1 - d) < std::fabs(l2 - d)) ? l1 : l2;
        } else {
            mu = d;
        }
        if (iter % 11 == 10) mu += std::fabs(c);  // exceptional shift
        // QR step on block [lo, hi]: H - mu I = Q R, H <- R Q + mu I
        for (int i = lo; i <= hi; ++i) H[i * n + i] -= mu;
        for (int k = lo; k < hi; ++k) {
            ld x = H[k * n + k], y = H[(k + 1) * n + k];
            ld r = std::hypot(x, y);
            ld cc = (r == 0.0L) ? 1.0L : x / r, ss = (r == 0.0L) ? 0.0L : y / r;
            cs[k] = cc;
            sn[k] = ss;
            for (int j = k; j < n; ++j) {
                ld t1 = H[k * n + j], t2 = H[(k + 1) * n + j];
                H[k * n + j] = cc * t1 + ss * t2;
                H[(k + 1) * n + j] = -ss * t1 + cc * t2;
            }
        }
        for (int k = lo; k < hi; ++k) {
            ld cc = cs[k], ss = sn[k];
            int rmax = std::min(hi, k + 2);
            for (int i = 0; i <= rmax; ++i) {
                ld t1 = H[i * n + k], t2 = H[i * n + k + 1];
                H[i * n + k] = cc * t1 + ss * t2;
                H[i * n + k + 1] = -ss * t1 + cc * t2;
            }
        }
        for (int i = lo; i <= hi; ++i) H[i * n + i] += mu;
    }
    return true;
}

bool real_eigen(int n, const double* Ain, double* lam, double* V, double* Vinv)
{
    std::vector<ld> A(n * n), H(n * n);
    for (int i = 0; i < n * n; ++i) A[i] = Ain[i];
    H = A;
    // Householder reduction to upper Hessenberg form
    std::vector<ld> v(n);
    for (int k = 0; k < n - 2; ++k) {
        ld alpha = 0.0L;
        for (int i = k + 1; i < n; ++i) alpha += H[i * n + k] * H[i * n + k];
        alpha = std::sqrt(alpha);
        if (alpha == 0.0L) continue;
        if (H[(k + 1) * n + k] > 0) alpha = -alpha;
        for (int i = 0; i < n; ++i) v[i] = 0.0L;
        v[k + 1] = H[(k + 1) * n + k] - alpha;
        for (int i = k + 2; i < n; ++i) v[i] = H[i * n + k];
        ld vv = 0.0L;
        for (int i = k + 1; i < n; ++i) vv += v[i] * v[i];
        if (vv == 0.0L) continue;
        for (int j = 0; j < n; ++j) {  // H <- (I - 2vv^T/vv) H
            ld s = 0.0L;
            for (int i = k + 1; i < n; ++i) s += v[i] * H[i * n + j];
            s = 2.0L * s / vv;
            for (int i = k + 1; i < n; ++i) H[i * n + j] -= s * v[i];
        }
        for (int i = 0; i < n; ++i) {  // H <- H (I - 2vv^T/vv)
            ld s = 0.0L;
            for (int j = k + 1; j < n; ++j) s += H[i * n + j] * v[j];
            s = 2.0L * s / vv;
            for (int j = k + 1; j < n; ++j) H[i * n + j] -= s * v[j];
        }
    }
    std::vector<ld> ev;
    if (!hessenberg_qr_eigenvalues(n, H, ev)) return false;
    std::sort(ev.begin(), ev.end());
    // inverse iteration for each eigenvector, eigenvalue refined by the
    // Rayleigh quotient along the way
    std::vector<ld> Vl(n * n), M(n * n), x(n);
    std::vector<int> piv;
    for (int j = 0; j < n; ++j) {
        ld mu = ev[j];
        for (int i = 0; i < n; ++i) x[i] = 1.0L + 0.01L * ((i * 7919 + j * 104729) % 97) / 97.0L;
        for (int it = 0; it < 4; ++it) {
            M = A;
            for (int i = 0; i < n; ++i) M[i * n + i] -= mu;
            lu_ld(n, M, piv);
            lu_ld_solve(n, M, piv, x);
            ld nrm = 0.0L;
            for (int i = 0; i < n; ++i) nrm += x[i] * x[i];
            nrm = std::sqrt(nrm);
            for (int i = 0; i < n; ++i) x[i] /= nrm;
        }
        // sign convention: largest component positive
        int im = 0;
        for (int i = 1; i < n; ++i) if (std::fabs(x[i]) > std::fabs(x[im])) im = i;
        ld sg = x[im] < 0 ? -1.0L : 1.0L;
        // Rayleigh quotient x^T A x (x normalised)
        ld rq = 0.0L;
        for (int i = 0; i < n; ++i) {
            ld s = 0.0L;
            for (int k = 0; k < n; ++k) s += A[i * n + k] * x[k];
            rq += x[i] * s;
        }
        (void)rq;
        ev[j] = mu;
        for (int i = 0; i < n; ++i) Vl[i * n + j] = sg * x[i];
    }
    // V^-1 by LU of V
    std::vector<ld> LV = Vl, Wi(n * n), e(n);
    lu_ld(n, LV, piv);
    for (int j = 0; j < n; ++j) {
        for (int i = 0; i < n; ++i) e[i] = (i == j) ? 1.0L : 0.0L;
        lu_ld_solve(n, LV, piv, e);
        for (int i = 0; i < n; ++i) Wi[i * n + j] = e[i];
    }
    // residual checks: |A V - V diag(ev)| and |V V^-1 - I|
    ld anorm = 0.0L;
    for (int i = 0; i < n * n; ++i) anorm = std::max(anorm, std::fabs(A[i]));
    ld r1 = 0.0L, r2 = 0.0L;
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            ld s = 0.0L, t = 0.0L;
            for (int k = 0; k < n; ++k) {
                s += A[i * n + k] * Vl[k * n + j];
                t += Vl[i * n + k] * Wi[k * n + j];
            }
            r1 = std::max(r1, std::fabs(s - Vl[i * n + j] * ev[j]));
            r2 = std::max(r2, std::fabs(t - (i == j ? 1.0L : 0.0L)));
        }
    if (!(r1 <= 1e-14L * anorm) || !(r2 <= 1e-13L)) return false;
    for (int i = 0; i < n; ++i) lam[i] = (double)ev[i];
    for (int i = 0; i < n * n; ++i) { V[i] = (double)Vl[i]; Vinv[i] = (double)Wi[i]; }
    return true;
}

GllSetup build_gll_setup(int N, int Ns, double L)
{
    GllSetup s;
    s.N = N;
    s.Ns = Ns;
    s.L = L;
    std::vector<double> xi(N), Dr(N * N), D2r(N * N);
    gll_nodes(N, xi.data());
    gll_derivative(N, xi.data(), Dr.data());
    matmul(N, Dr.data(), Dr.data(), D2r.data());
    s.nodes.resize(Ns * (N - 1) + 1);
    for (int jj = 0; jj < Ns; ++jj) {
        double a = jj * L / Ns, b = a + L / Ns;
        for (int j = 0; j < N; ++j) s.nodes[jj * (N - 1) + j] = 0.5 * (a + b + (L / Ns) * xi[j]);
    }
    s.D.resize(N * N);
    s.D2.resize(N * N);
    for (int i = 0; i < N * N; ++i) {
        s.D[i] = Dr[i] * (2.0 * Ns / L);
        s.D2[i] = D2r[i] * (4.0 * Ns * Ns / (L * L));
    }
    return s;
}

}  // namespace helm

namespace helm {

bool fold_eigen(int n, const std::vector<double>& A0, FoldedEigen& fe)
{
    const int m = n / 2, odd = n % 2, ms = m + odd, ma = m;
    const double r2 = 0.70710678118654752440;
    fe.n = n;
    fe.m = m;
    fe.ms = ms;
    fe.ma = ma;
    fe.Q.assign((size_t)n * n, 0.0);
    std::vector<double>& Q = fe.Q;
    for (int k = 0; k < m; ++k) {
        Q[(size_t)k * n + k] = r2;
        Q[(size_t)k * n + n - 1 - k] = r2;
        Q[(size_t)(ms + k) * n + k] = r2;
        Q[(size_t)(ms + k) * n + n - 1 - k] = -r2;
    }
    if (odd) Q[(size_t)m * n + m] = 1.0;
    std::vector<double> T((size_t)n * n, 0.0), Mf((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i)  // T = Q A0
        for (int j = 0; j < n; ++j) {
            double s = 0;
            for (int k = 0; k < n; ++k) s += Q[(size_t)i * n + k] * A0[(size_t)k * n + j];
            T[(size_t)i * n + j] = s;
        }
    double amax = 0, off = 0;
    for (int i = 0; i < n; ++i)  // Mf = T Q^T
        for (int j = 0; j < n; ++j) {
            double s = 0;
            for (int k = 0; k < n; ++k) s += T[(size_t)i * n + k] * Q[(size_t)j * n + k];
            Mf[(size_t)i * n + j] = s;
            amax = std::max(amax, std::fabs(s));
            if ((i < ms) != (j < ms)) off = std::max(off, std::fabs(s));
        }
    if (off > 1e-11 * amax) return false;
    fe.Ms.assign((size_t)ms * ms, 0.0);
    fe.Ma.assign((size_t)ma * ma, 0.0);
    for (int i = 0; i < ms; ++i)
        for (int j = 0; j < ms; ++j) fe.Ms[(size_t)i * ms + j] = Mf[(size_t)i * n + j];
    for (int i = 0; i < ma; ++i)
        for (int j = 0; j < ma; ++j) fe.Ma[(size_t)i * ma + j] = Mf[(size_t)(ms + i) * n + ms + j];
    fe.ls.assign(ms, 0.0);
    fe.Vs.assign((size_t)ms * ms, 0.0);
    fe.Vsi.assign((size_t)ms * ms, 0.0);
    fe.la.assign(ma, 0.0);
    fe.Va.assign((size_t)ma * ma, 0.0);
    fe.Vai.assign((size_t)ma * ma, 0.0);
    if (!real_eigen(ms, fe.Ms.data(), fe.ls.data(), fe.Vs.data(), fe.Vsi.data())) return false;
    if (ma > 0 && !real_eigen(ma, fe.Ma.data(), fe.la.data(), fe.Va.data(), fe.Vai.data())) return false;
    return true;
}

}  // namespace helm
