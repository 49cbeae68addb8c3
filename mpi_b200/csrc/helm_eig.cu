// Eigen-basis pipeline of the one-element solve with Dirichlet ends, FP64,
// sm_100a.
//
// The per-wavenumber solve of the reference (ConstructFundamentalSolutions +
// LUSolve, DPS/src/NonPeriodic3D_MPI.cpp:184-232, with the Dirichlet ends of
// the interface step :328-369 and the combination :582-587) is, for every
// spectrum row (kx, ky),
//     u_int = (D2int - sigma(kx, ky) I)^-1 (f_int + zl bl + zr br),
//     u(0) = zl = gl / beta_l,  u(N-1) = zr = gr / beta_r,
// with bl, br minus the boundary columns of D2.  D2int = V diag(mu) V^-1 (the
// folded blocks of helm_fdm.cu), so the solve is V^-1 along the GLL index, a
// diagonal scaling by 1 / (mu_j - sigma), and V along the GLL index.  V and
// V^-1 act on the GLL index only and commute with the Fourier transforms along
// x and y, which act on the other two.  The solve therefore runs as
//   pass 1 (one CTA per y plane): load f[x][y][:] for all x, fold, apply V^-1
//          (plus the boundary columns times zl, zr) on the FP64 tensor cores,
//          real-to-complex FFT along x, store the coefficient spectrum
//          S[kx][y][64];
//   pass 2 (one CTA per kx and 16 coefficients): FFT along y, scale by
//          1 / (mu_j - sigma) / (Nx Ny), inverse FFT along y, in place;
//   pass 3 (one CTA per y plane): complex-to-real FFT along x, apply V on the
//          tensor cores, unfold, write u[x][y][:] with the boundary values.
// f is read once, u written once, and S crosses the memory system four times
// (34 MB each at 256 x 256 x 65): three launches instead of five.  A 2D problem
// is one plane: its whole solve is one CTA, one launch.
#include "helm_device.cuh"
#include "helm_eig.cuh"
#include "helm_kernels.cuh"
#include "helm_tma.cuh"

#include <cstring>

namespace helm {

namespace {

constexpr int EP_PITCH = 68;     // doubles per row of a plane in shared memory (P <= 66, 64 slots, 4 of pad)
constexpr int EP_HS = EP_PITCH / 2;
constexpr int EP_FRAG = 4 * 8 * 32;  // doubles of one fold's transform in fragment order

template <int L>
struct EpShape {
    static constexpr int WARPS = (L / 8 < 16) ? L / 8 : 16;
    static constexpr int THREADS = 32 * WARPS;
    static constexpr int RW = L / WARPS;  // rows of the plane per warp
    static constexpr int MTW = RW / 8;    // 8-row tiles per warp
    static_assert(MTW >= 1 && RW % 8 == 0, "plane rows per warp");
    // plane, then the transforms it applies (2 folds, or all 4 for the fused 2D solve)
    static constexpr size_t smem(int nmats) { return ((size_t)L * EP_PITCH + (size_t)nmats * EP_FRAG) * sizeof(double); }
};

__device__ __forceinline__ void copy_mats(double* dst, const double* src, int blk0, int blk1)
{
    const double2* s0 = reinterpret_cast<const double2*>(src + (size_t)blk0 * EP_FRAG);
    const double2* s1 = reinterpret_cast<const double2*>(src + (size_t)blk1 * EP_FRAG);
    double2* d = reinterpret_cast<double2*>(dst);
    for (int e = threadIdx.x; e < EP_FRAG; e += blockDim.x) d[e] = (e < EP_FRAG / 2) ? s0[e] : s1[e - EP_FRAG / 2];
}

// Loads plane y of f (rows x = 0..L-1, GLL slots 1..P-2) into buf and the
// scaled boundary values zl, zr into slots 0 and P-1.
template <int L>
__device__ __forceinline__ void load_plane(const EigArgs& a, const double* f, const double* gl, const double* gr,
                                           long long yoff, long long bc_off, double* buf)
{
    const int P = a.P;
    for (int e = threadIdx.x; e < L * P; e += blockDim.x) {
        const int x = e / P, k = e - x * P;
        double* d = buf + x * EP_PITCH + k;
        const double* s = f + (long long)x * a.x_stride + yoff + k;
        if (k == 0) *d = gl ? gl[(long long)x * a.bc_x_stride + bc_off] * a.ibl : 0.0;
        else if (k == P - 1) *d = gr ? gr[(long long)x * a.bc_x_stride + bc_off] * a.ibr : 0.0;
        else cp_async_bytes8(d, s, true);
    }
    cp_async_commit();
    cp_async_wait_all();
    if (a.sub) {  // adjoint of a least-squares misfit: ubar = u - u_obs at the interior slots
        __syncthreads();
        for (int e = threadIdx.x; e < L * P; e += blockDim.x) {
            const int x = e / P, k = e - x * P;
            if (k > 0 && k < P - 1) buf[x * EP_PITCH + k] -= a.sub[(long long)x * a.x_stride + yoff + k];
        }
    }
}

// First transform of the warp's rows (8 MTW rows at `rows`): coefficients of
// the folded interior plus the boundary columns, written back over the rows as
// slots 0..31 (symmetric fold) and 32..63 (antisymmetric fold).
template <int MTW>
__device__ __forceinline__ void first_transform(const EigArgs& a, double* rows, const double* Ms, const double* Ma,
                                                const double* hbc, int lane)
{
    const int g = lane >> 2, q = lane & 3;
    const int n = a.n, m = a.m, ms = a.ms, P = a.P;
    double cs[MTW][4][2], ca[MTW][4][2];
#pragma unroll
    for (int mt = 0; mt < MTW; ++mt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) cs[mt][nt][0] = cs[mt][nt][1] = ca[mt][nt][0] = ca[mt][nt][1] = 0.0;
#pragma unroll 2
    for (int kk = 0; kk < 8; ++kk) {
        const int k = 4 * kk + q;
        double as[MTW], aa[MTW];
#pragma unroll
        for (int mt = 0; mt < MTW; ++mt) {
            const double* row = rows + (mt * 8 + g) * EP_PITCH;
            double vs = 0.0, va = 0.0;
            if (k < m) {
                const double lo = row[1 + k], hi = row[n - k];
                vs = kR2 * (lo + hi);
                va = kR2 * (lo - hi);
            } else if (k < ms) {
                vs = row[1 + k];
            }
            as[mt] = vs;
            aa[mt] = va;
        }
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) {
            const double bs = Ms[(nt * 8 + kk) * 32 + lane], ba = Ma[(nt * 8 + kk) * 32 + lane];
#pragma unroll
            for (int mt = 0; mt < MTW; ++mt) {
                dmma_8x8x4(cs[mt][nt][0], cs[mt][nt][1], as[mt], bs);
                dmma_8x8x4(ca[mt][nt][0], ca[mt][nt][1], aa[mt], ba);
            }
        }
    }
    double zl[MTW], zr[MTW];
#pragma unroll
    for (int mt = 0; mt < MTW; ++mt) {
        const double* row = rows + (mt * 8 + g) * EP_PITCH;
        zl[mt] = row[0];
        zr[mt] = row[P - 1];
    }
    __syncwarp();
#pragma unroll
    for (int nt = 0; nt < 4; ++nt)
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const int i = nt * 8 + 2 * q + j;
            const double hsl = hbc[i], hsr = hbc[32 + i], hal = hbc[64 + i], har = hbc[96 + i];
#pragma unroll
            for (int mt = 0; mt < MTW; ++mt) {
                cs[mt][nt][j] += zl[mt] * hsl + zr[mt] * hsr;
                ca[mt][nt][j] += zl[mt] * hal + zr[mt] * har;
            }
        }
#pragma unroll
    for (int mt = 0; mt < MTW; ++mt) {
        double* row = rows + (mt * 8 + g) * EP_PITCH;
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) {
            *reinterpret_cast<double2*>(row + nt * 8 + 2 * q) = make_double2(cs[mt][nt][0], cs[mt][nt][1]);
            *reinterpret_cast<double2*>(row + 32 + nt * 8 + 2 * q) = make_double2(ca[mt][nt][0], ca[mt][nt][1]);
        }
    }
    __syncwarp();
}

// Second transform of the warp's rows (coefficients in slots 0..63), unfolded
// into GLL slots 1..P-2 of the same rows; slots 0 and P-1 keep the boundary
// values the caller puts there.
template <int MTW>
__device__ __forceinline__ void second_transform(const EigArgs& a, double* rows, const double* Ms, const double* Ma,
                                                 int lane)
{
    const int g = lane >> 2, q = lane & 3;
    const int n = a.n, m = a.m, ms = a.ms;
    double cs[MTW][4][2], ca[MTW][4][2];
#pragma unroll
    for (int mt = 0; mt < MTW; ++mt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) cs[mt][nt][0] = cs[mt][nt][1] = ca[mt][nt][0] = ca[mt][nt][1] = 0.0;
#pragma unroll 2
    for (int kk = 0; kk < 8; ++kk) {
        const int k = 4 * kk + q;
        double as[MTW], aa[MTW];
#pragma unroll
        for (int mt = 0; mt < MTW; ++mt) {
            const double* row = rows + (mt * 8 + g) * EP_PITCH;
            as[mt] = row[k];
            aa[mt] = row[32 + k];
        }
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) {
            const double bs = Ms[(nt * 8 + kk) * 32 + lane], ba = Ma[(nt * 8 + kk) * 32 + lane];
#pragma unroll
            for (int mt = 0; mt < MTW; ++mt) {
                dmma_8x8x4(cs[mt][nt][0], cs[mt][nt][1], as[mt], bs);
                dmma_8x8x4(ca[mt][nt][0], ca[mt][nt][1], aa[mt], ba);
            }
        }
    }
    __syncwarp();
#pragma unroll
    for (int mt = 0; mt < MTW; ++mt) {
        double* row = rows + (mt * 8 + g) * EP_PITCH;
#pragma unroll
        for (int nt = 0; nt < 4; ++nt)
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                const int i = nt * 8 + 2 * q + j;
                const double s = cs[mt][nt][j], d = ca[mt][nt][j];
                if (i < m) {
                    row[1 + i] = kR2 * (s + d);
                    row[n - i] = kR2 * (s - d);
                } else if (i < ms) {
                    row[1 + i] = s;
                }
            }
    }
    __syncwarp();
}

// Real-to-complex split of the 32 column pairs of the transformed plane into
// the half spectrum X (slot 2c) and Y (slot 2c+1) of row kx; emit(kx, c, X, Y).
template <int L, typename Emit>
__device__ __forceinline__ void r2c_split(const double2* z, int warp, int lane, Emit emit)
{
    for (int kx = warp; kx <= L / 2; kx += EpShape<L>::WARPS) {
        const double2 zk = z[kx * EP_HS + lane], zm = z[((L - kx) & (L - 1)) * EP_HS + lane];
        const double2 X = make_double2(0.5 * (zk.x + zm.x), 0.5 * (zk.y - zm.y));
        const double2 Y = make_double2(0.5 * (zk.y + zm.y), 0.5 * (zm.x - zk.x));
        emit(kx, lane, X, Y);
    }
}

// Complex-to-real assembly: full-length Z[k] = X_k + i Y_k from the half
// spectra of the 32 column pairs (imaginary parts dropped at k = 0 and L/2, as
// the real part of the reference's inverse transform does); fetch(kx, c, X, Y).
template <int L, typename Fetch>
__device__ __forceinline__ void c2r_assemble(double2* z, int warp, int lane, Fetch fetch)
{
    for (int kx = warp; kx <= L / 2; kx += EpShape<L>::WARPS) {
        double2 X, Y;
        fetch(kx, lane, X, Y);
        if (kx == 0 || kx == L / 2) { X.y = 0.0; Y.y = 0.0; }
        z[kx * EP_HS + lane] = make_double2(X.x - Y.y, X.y + Y.x);
        if (kx > 0 && kx < L / 2) z[(L - kx) * EP_HS + lane] = make_double2(X.x + Y.y, Y.x - X.y);
    }
}

// ------------------------------------------------------------------ pass 1 --
template <int L>
__global__ void __launch_bounds__(EpShape<L>::THREADS, 1) eig_fwd_kernel(EigArgs a)
{
    using S = EpShape<L>;
    extern __shared__ __align__(16) double esm[];
    double* buf = esm;
    double* Mt = esm + (size_t)L * EP_PITCH;
    copy_mats(Mt, a.mats, 0, 2);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int y = blockIdx.x;
    pdl_enter();
    if (a.lam_out && blockIdx.x == 0 && threadIdx.x == 0) *a.lam_out = 0.0;
    load_plane<L>(a, a.f, a.adjoint ? nullptr : a.gl, a.adjoint ? nullptr : a.gr, (long long)y * a.P, y, buf);
    __syncthreads();
    first_transform<S::MTW>(a, buf + warp * S::RW * EP_PITCH, Mt, Mt + EP_FRAG, a.hbc, lane);
    __syncthreads();
    double2* z = reinterpret_cast<double2*>(buf);
    slab_fft<L, -1, S::THREADS>(z, EP_HS, 32, static_cast<const double2*>(a.tw_x));
    double2* Sg = reinterpret_cast<double2*>(a.S);
    const long long Ny = a.Ny;
    r2c_split<L>(z, warp, lane, [&](int kx, int c, double2 X, double2 Y) {
        double2* row = Sg + ((long long)kx * Ny + y) * EIG_SLOTS;
        row[2 * c] = X;
        row[2 * c + 1] = Y;
    });
}

// ------------------------------------------------------------------ pass 2 --
template <int NY, int CT>
__global__ void __launch_bounds__(256) eig_conv_kernel(EigArgs a)
{
    extern __shared__ __align__(16) double esm[];
    double2* sm = reinterpret_cast<double2*>(esm);
    constexpr int TILES = EIG_SLOTS / CT;
    const int kx = blockIdx.x / TILES, j0 = (blockIdx.x - kx * TILES) * CT;
    double2* Sg = reinterpret_cast<double2*>(a.S) + (long long)kx * NY * EIG_SLOTS + j0;
    pdl_enter();
    for (int e = threadIdx.x; e < NY * CT; e += blockDim.x) {
        const int ky = e / CT, c = e - ky * CT;
        cp_async_bytes16(&sm[ky * CT + c], &Sg[(long long)ky * EIG_SLOTS + c], true);
    }
    cp_async_commit();
    cp_async_wait_all();
    __syncthreads();
    const double2* tw = static_cast<const double2*>(a.tw_y);
    slab_fft<NY, -1, 256>(sm, CT, CT, tw);
    const double* rc = a.recip;
    for (int e = threadIdx.x; e < NY * CT; e += blockDim.x) {
        const int ky = e / CT, c = e - ky * CT;
        const double r = rc[(long long)a.grp_of_row[kx * NY + ky] * EIG_SLOTS + j0 + c] * a.scale;
        const double2 v = sm[ky * CT + c];
        sm[ky * CT + c] = make_double2(v.x * r, v.y * r);
    }
    __syncthreads();
    slab_fft<NY, 1, 256>(sm, CT, CT, tw);
    for (int e = threadIdx.x; e < NY * CT; e += blockDim.x) {
        const int ky = e / CT, c = e - ky * CT;
        Sg[(long long)ky * EIG_SLOTS + c] = sm[ky * CT + c];
    }
}

// Adjoint: the boundary terms of the transposed map for the warp's rows,
// b_l . fbar_int = hsl . cs + hal . ca (and the same with the right-hand
// vectors), from the coefficients in slots 0..63 before the second transform.
template <int L>
__device__ __forceinline__ void adjoint_boundary_dots(const EigArgs& a, const double* rows, int lane, double* dl,
                                                      double* dr)
{
    using S = EpShape<L>;
    const double hs0 = a.hbc[lane], hs1 = a.hbc[EIG_LD + lane], ha0 = a.hbc[2 * EIG_LD + lane],
                 ha1 = a.hbc[3 * EIG_LD + lane];
    for (int r = 0; r < S::RW; ++r) {
        const double cs = rows[r * EP_PITCH + lane], ca = rows[r * EP_PITCH + 32 + lane];
        double vl = hs0 * cs + ha0 * ca, vr = hs1 * cs + ha1 * ca;
        for (int o = 16; o > 0; o >>= 1) {
            vl += __shfl_xor_sync(0xffffffffu, vl, o);
            vr += __shfl_xor_sync(0xffffffffu, vr, o);
        }
        if (lane == r) { *dl = vl; *dr = vr; }
    }
}

// Adjoint: writes the warp's rows of fbar (boundary slots 0), the boundary
// cotangents gbar = (ubar_boundary + dot) / beta, and returns this lane's share
// of sum(fbar u).
template <int L>
__device__ __forceinline__ double store_adjoint_rows(const EigArgs& a, double* fbar, const double* ubar,
                                                     long long yoff, long long bc_off, double* rows, int x0, int lane,
                                                     double dl, double dr)
{
    using S = EpShape<L>;
    const int P = a.P;
    if (lane < S::RW) {
        const long long x = x0 + lane;
        const long long o = x * a.x_stride + yoff;
        if (a.gbar_l) {
            const double u0 = ubar[o] - (a.sub ? a.sub[o] : 0.0);
            a.gbar_l[x * a.bc_x_stride + bc_off] = (u0 + dl) * a.ibl;
        }
        if (a.gbar_r) {
            const double uN = ubar[o + P - 1] - (a.sub ? a.sub[o + P - 1] : 0.0);
            a.gbar_r[x * a.bc_x_stride + bc_off] = (uN + dr) * a.ibr;
        }
        rows[lane * EP_PITCH] = 0.0;
        rows[lane * EP_PITCH + P - 1] = 0.0;
    }
    __syncwarp();
    double acc = 0.0;
    for (int r = 0; r < S::RW; ++r) {
        const long long o = (long long)(x0 + r) * a.x_stride + yoff;
        for (int k = lane; k < P; k += 32) {
            const double v = rows[r * EP_PITCH + k];
            fbar[o + k] = v;
            if (a.lam_u) acc += v * a.lam_u[o + k];
        }
    }
    return acc;
}

// Adds every thread's acc into *a.lam_out, one atomic per CTA (all threads call).
__device__ __forceinline__ void eig_lambda_sum(const EigArgs& a, double acc)
{
    __shared__ double red[32];
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double sum = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) sum += red[w];
        atomicAdd(a.lam_out, sum);
    }
}

// ------------------------------------------------------------------ pass 3 --
// Writes the warp's rows of plane y: boundary slots from gl, gr, then the rows.
template <int L>
__device__ __forceinline__ void store_plane_rows(const EigArgs& a, double* u, const double* gl, const double* gr,
                                                 long long yoff, long long bc_off, double* rows, int x0, int lane)
{
    using S = EpShape<L>;
    const int P = a.P;
    if (lane < S::RW) {
        const long long x = x0 + lane;
        rows[lane * EP_PITCH] = gl ? gl[x * a.bc_x_stride + bc_off] * a.ibl : 0.0;
        rows[lane * EP_PITCH + P - 1] = gr ? gr[x * a.bc_x_stride + bc_off] * a.ibr : 0.0;
    }
    __syncwarp();
    for (int r = 0; r < S::RW; ++r) {
        double* dst = u + (long long)(x0 + r) * a.x_stride + yoff;
        for (int k = lane; k < P; k += 32) dst[k] = rows[r * EP_PITCH + k];
    }
}

template <int L>
__global__ void __launch_bounds__(EpShape<L>::THREADS, 1) eig_inv_kernel(EigArgs a)
{
    using S = EpShape<L>;
    extern __shared__ __align__(16) double esm[];
    double* buf = esm;
    double* Mt = esm + (size_t)L * EP_PITCH;
    copy_mats(Mt, a.mats, 1, 3);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int y = blockIdx.x;
    double2* z = reinterpret_cast<double2*>(buf);
    const double2* Sg = reinterpret_cast<const double2*>(a.S);
    const long long Ny = a.Ny;
    pdl_enter();
    c2r_assemble<L>(z, warp, lane, [&](int kx, int c, double2& X, double2& Y) {
        const double2* row = Sg + ((long long)kx * Ny + y) * EIG_SLOTS;
        X = row[2 * c];
        Y = row[2 * c + 1];
    });
    __syncthreads();
    slab_fft<L, 1, S::THREADS>(z, EP_HS, 32, static_cast<const double2*>(a.tw_x));
    double* rows = buf + warp * S::RW * EP_PITCH;
    if (!a.adjoint) {
        second_transform<S::MTW>(a, rows, Mt, Mt + EP_FRAG, lane);
        store_plane_rows<L>(a, a.u, a.gl, a.gr, (long long)y * a.P, y, rows, warp * S::RW, lane);
        return;
    }
    double dl = 0.0, dr = 0.0;
    adjoint_boundary_dots<L>(a, rows, lane, &dl, &dr);
    __syncwarp();
    second_transform<S::MTW>(a, rows, Mt, Mt + EP_FRAG, lane);
    const double acc =
        store_adjoint_rows<L>(a, a.u, a.f, (long long)y * a.P, y, rows, warp * S::RW, lane, dl, dr);
    if (a.lam_out) eig_lambda_sum(a, acc);
}

// --------------------------------------------------------- fused 2D solve --
// One CTA per problem: the whole pipeline on one plane, the diagonal scaling
// applied to the half spectrum in shared memory between the two FFTs.
template <int L>
__global__ void __launch_bounds__(EpShape<L>::THREADS, 1) eig_solve2d_kernel(EigArgs a)
{
    using S = EpShape<L>;
    extern __shared__ __align__(16) double esm[];
    double* buf = esm;
    double* M1 = esm + (size_t)L * EP_PITCH;
    double* M2 = M1 + 2 * EP_FRAG;
    copy_mats(M1, a.mats, 0, 2);
    copy_mats(M2, a.mats, 1, 3);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int b = blockIdx.x;
    const long long off = a.boff ? a.boff[b] : 0;
    // batched problems have no boundary data (homogeneous Dirichlet rows);
    // adjoint solves read none
    const double* gl = (a.boff || a.adjoint) ? nullptr : a.gl;
    const double* gr = (a.boff || a.adjoint) ? nullptr : a.gr;
    pdl_enter();
    if (a.lam_out && threadIdx.x == 0) *a.lam_out = 0.0;
    load_plane<L>(a, a.f + off, gl, gr, 0, 0, buf);
    __syncthreads();
    double* rows = buf + warp * S::RW * EP_PITCH;
    first_transform<S::MTW>(a, rows, M1, M1 + EP_FRAG, a.hbc, lane);
    __syncthreads();
    double2* z = reinterpret_cast<double2*>(buf);
    const double2* tw = static_cast<const double2*>(a.tw_x);
    slab_fft<L, -1, S::THREADS>(z, EP_HS, 32, tw);
    // split, scale and reassemble each pair of rows (kx, L - kx) in place
    for (int kx = warp; kx <= L / 2; kx += S::WARPS) {
        const int km = (L - kx) & (L - 1);
        const double2 zk = z[kx * EP_HS + lane], zm = z[km * EP_HS + lane];
        double2 X = make_double2(0.5 * (zk.x + zm.x), 0.5 * (zk.y - zm.y));
        double2 Y = make_double2(0.5 * (zk.y + zm.y), 0.5 * (zm.x - zk.x));
        const double* rc = a.recip + (long long)a.grp_of_row[(long long)b * (L / 2 + 1) + kx] * EIG_SLOTS;
        const double r0 = rc[2 * lane] * a.scale, r1 = rc[2 * lane + 1] * a.scale;
        X = make_double2(X.x * r0, X.y * r0);
        Y = make_double2(Y.x * r1, Y.y * r1);
        if (kx == 0 || kx == L / 2) { X.y = 0.0; Y.y = 0.0; }
        z[kx * EP_HS + lane] = make_double2(X.x - Y.y, X.y + Y.x);
        if (kx > 0 && kx < L / 2) z[km * EP_HS + lane] = make_double2(X.x + Y.y, Y.x - X.y);
    }
    __syncthreads();
    slab_fft<L, 1, S::THREADS>(z, EP_HS, 32, tw);
    if (!a.adjoint) {
        second_transform<S::MTW>(a, rows, M2, M2 + EP_FRAG, lane);
        store_plane_rows<L>(a, a.u + off, gl, gr, 0, 0, rows, warp * S::RW, lane);
        return;
    }
    double dl = 0.0, dr = 0.0;
    adjoint_boundary_dots<L>(a, rows, lane, &dl, &dr);
    __syncwarp();
    second_transform<S::MTW>(a, rows, M2, M2 + EP_FRAG, lane);
    const double acc = store_adjoint_rows<L>(a, a.u, a.f, 0, 0, rows, warp * S::RW, lane, dl, dr);
    if (a.lam_out) eig_lambda_sum(a, acc);
}

// Tensor maps of one solve (kernel parameter, built on the host per call).
struct EigMaps {
    CUtensorMap f;    // pass 1: f as [Nx][x_stride] doubles, box 68 x 16
    CUtensorMap sub;  // pass 1, misfit adjoint: u_obs, the same
    CUtensorMap S;    // pass 3: S as [nkx][Ny][128] doubles, box 128 x 1 x 16
    CUtensorMap T;    // pass 2: the same array, box 2 CT x min(Ny, 256) x 1
};

// ------------------------------------------------ persistent TMA passes --
// Row variant 5: the three 3D passes as persistent kernels, one CTA per SM,
// each with one producer warp that moves tiles by TMA (cp.async.bulk.tensor)
// through a ring of shared-memory slots guarded by mbarriers, and consumer
// warps that transform them.  A CTA works through its share of planes (passes
// 1 and 3) or tiles (pass 2) while the producer already fetches the next ones,
// so HBM latency hides behind the FP64 tensor-core and FFT work.
//   pass 1: f rows in 16-row chunks (tensor map over f, box 68 x 16; the
//           chunk's first element rounded down to a 16-byte boundary, the
//           shift taken out in shared memory) -> fold, first transform on the
//           FP64 tensor cores -> the plane's coefficient rows; then the x FFT
//           and plain stores of the coefficient spectrum S[kx][y][64];
//   pass 2: (kx, 16 coefficient slots) tiles of S (box 32 x Ny x 1) ->
//           y FFT, scaling, inverse y FFT in place -> TMA store of the tile;
//   pass 3: S rows of plane y in 16-kx chunks (box 128 x 1 x 16) -> full
//           spectra of the 32 column pairs -> inverse x FFT, second transform,
//           unfold, stores of u.
// Every wait is bounded (kTmaWaitLimit); a wait that runs out records an
// error in *a.err, and later waits of the CTA return at once, so the kernel
// ends with every named barrier still met.
constexpr int TP_PITCH = EP_PITCH;   // doubles per staged f row = box inner extent (68)
constexpr int TP_F_SLOTS = 8;        // pass 1 ring: f chunks (pairs of slots: f and u_obs, misfit adjoint)
constexpr int TP_S_SLOTS = 4;        // pass 3 ring: S chunks
constexpr int TP_C_SLOTS = 3;        // pass 2 ring: S tiles

template <int L>
struct TmaShape {
    using E = EpShape<L>;
    static constexpr int CW = E::WARPS;            // consumer warps
    static constexpr int CT = E::THREADS;          // consumer threads
    static constexpr int THREADS = CT + 32;        // + the producer warp
    static constexpr int RC = L < 16 ? L : 16;     // f rows per chunk (pass 1)
    static constexpr int NCH1 = L / RC;
    static constexpr int KC = 16;                  // kx rows per S chunk (pass 3)
    static constexpr int NCH3 = (L / 2) / KC + 1;  // chunks covering kx = 0 .. L/2
    static constexpr size_t plane = (size_t)L * TP_PITCH * sizeof(double);
    static constexpr size_t fslot = (size_t)RC * TP_PITCH * sizeof(double);
    static constexpr size_t sslot = (size_t)KC * 2 * EIG_SLOTS * sizeof(double);
    static constexpr size_t mats = 2 * EP_FRAG * sizeof(double);
    static constexpr size_t smem1 = plane + TP_F_SLOTS * fslot + mats + 2 * TP_F_SLOTS * sizeof(uint64_t);
    static constexpr size_t smem3 = plane + TP_S_SLOTS * sslot + mats + 2 * TP_S_SLOTS * sizeof(uint64_t);
};

// Bounded wait of a consumer or producer; false (and the error recorded) once
// any wait of the CTA has run out.
__device__ __forceinline__ bool tp_wait(uint64_t* bar, uint32_t parity, volatile int* s_err, int* err, int code)
{
    if (*s_err) return false;
    if (mbar_wait(bar, parity)) return true;
    *s_err = 1;
    if (err) atomicExch(err, code);
    return false;
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}

template <int THREADS>
__device__ __forceinline__ void consumers_sync()
{
    asm volatile("bar.sync 1, %0;\n" ::"n"(THREADS) : "memory");
}

template <int L>
__global__ void __launch_bounds__(TmaShape<L>::THREADS, 1)
    eig_fwd_tma_kernel(EigArgs a, const __grid_constant__ EigMaps tm)
{
    using T = TmaShape<L>;
    extern __shared__ __align__(1024) unsigned char tsm[];
    double* coef = reinterpret_cast<double*>(tsm);                                   // [L][68]
    double* ring = reinterpret_cast<double*>(tsm + T::plane);                         // [8][RC][68]
    double* Mt = reinterpret_cast<double*>(tsm + T::plane + TP_F_SLOTS * T::fslot);   // first transforms, sym | anti
    uint64_t* full = reinterpret_cast<uint64_t*>(tsm + T::plane + TP_F_SLOTS * T::fslot + T::mats);
    uint64_t* empty = full + TP_F_SLOTS;
    __shared__ int s_err;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int P = a.P, n = a.n, m = a.m, ms = a.ms, Ny = a.Ny;
    const bool sub = a.sub != nullptr;
    const int nslot = sub ? TP_F_SLOTS / 2 : TP_F_SLOTS;   // chunk slots (doubled in the misfit adjoint)
    if (tid == 0) {
        s_err = 0;
        for (int i = 0; i < TP_F_SLOTS; ++i) {
            mbar_init(&full[i], 1);
            mbar_init(&empty[i], T::CW);
        }
        fence_mbar_init();
    }
    copy_mats(Mt, a.mats, 0, 2);
    __syncthreads();
    pdl_enter();
    if (a.lam_out && blockIdx.x == 0 && tid == 0) *a.lam_out = 0.0;
    if (warp == T::CW) {
        // producer: every chunk of every plane of this CTA, in order
        int i = 0;
        for (int y = blockIdx.x; y < Ny; y += gridDim.x) {
            const int c0 = y * P - ((y * P) & 1);
            for (int c = 0; c < T::NCH1; ++c, ++i) {
                const int s = i % nslot;
                const uint32_t par = ((i / nslot) & 1) ^ 1;
                if (lane == 0 && tp_wait(&empty[s], par, &s_err, a.err, 1)) {
                    double* dst = ring + (size_t)s * (sub ? 2 : 1) * T::RC * TP_PITCH;
                    mbar_arrive_expect_tx(&full[s], (uint32_t)((sub ? 2 : 1) * T::fslot));
                    tma_load_2d(dst, &tm.f, c0, c * T::RC, &full[s]);
                    if (sub) tma_load_2d(dst + T::RC * TP_PITCH, &tm.sub, c0, c * T::RC, &full[s]);
                }
                __syncwarp();
            }
        }
        // every load issued has landed before the CTA may end (consumers wait
        // for each; after an error, wait here for the last ones in flight)
        if (lane == 0 && s_err) {
            const int last = i;
            for (int j = (last > nslot ? last - nslot : 0); j < last; ++j) mbar_wait(&full[j % nslot], (j / nslot) & 1);
        }
    } else {
        const int g = lane >> 2, q = lane & 3;
        const double* gl = a.adjoint ? nullptr : a.gl;
        const double* gr = a.adjoint ? nullptr : a.gr;
        int i = 0;
        for (int y = blockIdx.x; y < Ny; y += gridDim.x) {
            const int sh = (y * P) & 1;
            for (int c = 0; c < T::NCH1; ++c, ++i) {
                const int s = i % nslot;
                const bool ok = tp_wait(&full[s], (i / nslot) & 1, &s_err, a.err, 2);
                const double* st = ring + (size_t)s * (sub ? 2 : 1) * T::RC * TP_PITCH;
                for (int t = warp; ok && t < (T::RC / 8) * 8; t += T::CW) {
                    const int mt = t >> 3, ntg = t & 7, fold = ntg >> 2, nt = ntg & 3;
                    const double* Mb = Mt + fold * EP_FRAG;
                    const int r = mt * 8 + g;
                    const double* rowp = st + r * TP_PITCH + sh;
                    const double* rows = sub ? rowp + T::RC * TP_PITCH : nullptr;
                    double c0 = 0.0, c1 = 0.0, d0 = 0.0, d1 = 0.0;
#pragma unroll
                    for (int kk = 0; kk < 8; kk += 2) {
                        const double v0 = fold_value(rowp, rows, 4 * kk + q, fold, n, m, ms);
                        const double v1 = fold_value(rowp, rows, 4 * kk + 4 + q, fold, n, m, ms);
                        dmma_8x8x4(c0, c1, v0, Mb[(nt * 8 + kk) * 32 + lane]);
                        dmma_8x8x4(d0, d1, v1, Mb[(nt * 8 + kk + 1) * 32 + lane]);
                    }
                    const long long x = (long long)c * T::RC + r;
                    const int i0 = nt * 8 + 2 * q;
                    double o0 = c0 + d0, o1 = c1 + d1;
                    if (gl) {
                        const double zl = gl[x * a.bc_x_stride + y] * a.ibl;
                        o0 += zl * a.hbc[fold * 2 * EIG_LD + i0];
                        o1 += zl * a.hbc[fold * 2 * EIG_LD + i0 + 1];
                    }
                    if (gr) {
                        const double zr = gr[x * a.bc_x_stride + y] * a.ibr;
                        o0 += zr * a.hbc[fold * 2 * EIG_LD + EIG_LD + i0];
                        o1 += zr * a.hbc[fold * 2 * EIG_LD + EIG_LD + i0 + 1];
                    }
                    *reinterpret_cast<double2*>(coef + x * TP_PITCH + ntg * 8 + 2 * q) = make_double2(o0, o1);
                }
                __syncwarp();
                if (lane == 0) mbar_arrive(&empty[s]);
            }
            consumers_sync<T::CT>();
            double2* z = reinterpret_cast<double2*>(coef);
            slab_fft<L, -1, T::CT, 1>(z, EP_HS, 32, static_cast<const double2*>(a.tw_x));
            double2* Sg = reinterpret_cast<double2*>(a.S);
            r2c_split<L>(z, warp, lane, [&](int kx, int cc, double2 X, double2 Y) {
                double2* row = Sg + ((long long)kx * Ny + y) * EIG_SLOTS;
                row[2 * cc] = X;
                row[2 * cc + 1] = Y;
            });
            consumers_sync<T::CT>();  // the coefficient rows are rewritten by the next plane
        }
    }
}

template <int L>
__global__ void __launch_bounds__(TmaShape<L>::THREADS, 1)
    eig_inv_tma_kernel(EigArgs a, const __grid_constant__ EigMaps tm)
{
    using T = TmaShape<L>;
    using S = EpShape<L>;
    extern __shared__ __align__(1024) unsigned char tsm[];
    double* buf = reinterpret_cast<double*>(tsm);                                   // [L][68]
    double* ring = reinterpret_cast<double*>(tsm + T::plane);                        // [4][16][128]
    double* Mt = reinterpret_cast<double*>(tsm + T::plane + TP_S_SLOTS * T::sslot);  // second transforms
    uint64_t* full = reinterpret_cast<uint64_t*>(tsm + T::plane + TP_S_SLOTS * T::sslot + T::mats);
    uint64_t* empty = full + TP_S_SLOTS;
    __shared__ int s_err;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int Ny = a.Ny;
    if (tid == 0) {
        s_err = 0;
        for (int i = 0; i < TP_S_SLOTS; ++i) {
            mbar_init(&full[i], 1);
            mbar_init(&empty[i], T::CW);
        }
        fence_mbar_init();
    }
    copy_mats(Mt, a.mats, 1, 3);
    __syncthreads();
    pdl_enter();
    double lam_acc = 0.0;
    if (warp == T::CW) {
        int i = 0;
        for (int y = blockIdx.x; y < Ny; y += gridDim.x)
            for (int c = 0; c < T::NCH3; ++c, ++i) {
                const int s = i % TP_S_SLOTS;
                if (lane == 0 && tp_wait(&empty[s], ((i / TP_S_SLOTS) & 1) ^ 1, &s_err, a.err, 3)) {
                    mbar_arrive_expect_tx(&full[s], (uint32_t)T::sslot);
                    tma_load_3d(ring + (size_t)s * T::KC * 2 * EIG_SLOTS, &tm.S, 0, y, c * T::KC, &full[s]);
                }
                __syncwarp();
            }
        if (lane == 0 && s_err) {
            const int last = i;
            for (int j = (last > TP_S_SLOTS ? last - TP_S_SLOTS : 0); j < last; ++j)
                mbar_wait(&full[j % TP_S_SLOTS], (j / TP_S_SLOTS) & 1);
        }
    } else {
        double2* z = reinterpret_cast<double2*>(buf);
        double* rows = buf + warp * S::RW * EP_PITCH;
        int i = 0;
        for (int y = blockIdx.x; y < Ny; y += gridDim.x) {
            for (int c = 0; c < T::NCH3; ++c, ++i) {
                const int s = i % TP_S_SLOTS;
                const bool ok = tp_wait(&full[s], (i / TP_S_SLOTS) & 1, &s_err, a.err, 4);
                const double2* st = reinterpret_cast<const double2*>(ring + (size_t)s * T::KC * 2 * EIG_SLOTS);
                // full-length spectra Z = X + i Y of the column pairs (imaginary
                // parts dropped at kx = 0 and L / 2, as the real part of the
                // reference's inverse transform does)
                for (int e = tid; ok && e < T::KC * 32; e += T::CT) {
                    const int r = e >> 5, cc = e & 31, kx = c * T::KC + r;
                    if (kx > L / 2) continue;
                    double2 X = st[r * EIG_SLOTS + 2 * cc], Y = st[r * EIG_SLOTS + 2 * cc + 1];
                    if (kx == 0 || kx == L / 2) { X.y = 0.0; Y.y = 0.0; }
                    z[kx * EP_HS + cc] = make_double2(X.x - Y.y, X.y + Y.x);
                    if (kx > 0 && kx < L / 2) z[(L - kx) * EP_HS + cc] = make_double2(X.x + Y.y, Y.x - X.y);
                }
                __syncwarp();
                if (lane == 0) mbar_arrive(&empty[s]);
            }
            consumers_sync<T::CT>();
            slab_fft<L, 1, T::CT, 1>(z, EP_HS, 32, static_cast<const double2*>(a.tw_x));
            if (!a.adjoint) {
                second_transform<S::MTW>(a, rows, Mt, Mt + EP_FRAG, lane);
                store_plane_rows<L>(a, a.u, a.gl, a.gr, (long long)y * a.P, y, rows, warp * S::RW, lane);
            } else {
                double dl = 0.0, dr = 0.0;
                adjoint_boundary_dots<L>(a, rows, lane, &dl, &dr);
                __syncwarp();
                second_transform<S::MTW>(a, rows, Mt, Mt + EP_FRAG, lane);
                lam_acc += store_adjoint_rows<L>(a, a.u, a.f, (long long)y * a.P, y, rows, warp * S::RW, lane, dl, dr);
            }
            consumers_sync<T::CT>();  // the plane buffer is rewritten by the next plane
        }
    }
    if (a.lam_out) eig_lambda_sum(a, lam_acc);
}

template <int NY, int CT>
struct ConvShape {
    static constexpr int CONS = 256;                       // consumer threads
    static constexpr int THREADS = CONS + 32;
    static constexpr int TILES_PER_KX = EIG_SLOTS / CT;
    static constexpr int BOX_Y = NY < 256 ? NY : 256;
    static constexpr size_t tile = (size_t)NY * CT * sizeof(double2);
    static constexpr size_t smem = TP_C_SLOTS * tile + 2 * TP_C_SLOTS * sizeof(uint64_t);
    static constexpr int PER = (NY * CT + CONS - 1) / CONS;  // elements scaled per consumer thread
};

template <int NY, int CT>
__global__ void __launch_bounds__(ConvShape<NY, CT>::THREADS, 1)
    eig_conv_tma_kernel(EigArgs a, const __grid_constant__ EigMaps tm)
{
    using C = ConvShape<NY, CT>;
    extern __shared__ __align__(1024) unsigned char tsm[];
    double2* ring = reinterpret_cast<double2*>(tsm);
    uint64_t* full = reinterpret_cast<uint64_t*>(tsm + TP_C_SLOTS * C::tile);
    uint64_t* done = full + TP_C_SLOTS;
    __shared__ int s_err;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int ntiles = a.nkx * C::TILES_PER_KX;
    int mine = 0;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) ++mine;
    if (tid == 0) {
        s_err = 0;
        for (int i = 0; i < TP_C_SLOTS; ++i) {
            mbar_init(&full[i], 1);
            mbar_init(&done[i], 1);
        }
        fence_mbar_init();
    }
    __syncthreads();
    pdl_enter();
    auto coords = [&](int i, int& kx, int& j0) {
        const int t = blockIdx.x + i * gridDim.x;
        kx = t / C::TILES_PER_KX;
        j0 = (t - kx * C::TILES_PER_KX) * CT;
    };
    if (warp == C::CONS / 32) {
        if (lane == 0) {
            for (int i = 0; i < mine + TP_C_SLOTS; ++i) {
                if (i >= TP_C_SLOTS) {  // tile i - SLOTS solved: store it back
                    const int j = i - TP_C_SLOTS, s = j % TP_C_SLOTS;
                    if (tp_wait(&done[s], (j / TP_C_SLOTS) & 1, &s_err, a.err, 5)) {
                        int kx, j0;
                        coords(j, kx, j0);
                        for (int yb = 0; yb < NY; yb += C::BOX_Y)
                            tma_store_3d(&tm.T, 2 * j0, yb, kx, ring + (size_t)s * NY * CT + (size_t)yb * CT);
                        tma_store_commit();
                    }
                }
                if (i < mine) {
                    const int s = i % TP_C_SLOTS;
                    tma_store_wait_read<0>();  // the store of this slot's previous tile has read it
                    if (!s_err) {
                        int kx, j0;
                        coords(i, kx, j0);
                        mbar_arrive_expect_tx(&full[s], (uint32_t)C::tile);
                        for (int yb = 0; yb < NY; yb += C::BOX_Y)
                            tma_load_3d(ring + (size_t)s * NY * CT + (size_t)yb * CT, &tm.T, 2 * j0, yb, kx, &full[s]);
                    }
                }
            }
            tma_store_wait_all();
            if (s_err)
                for (int j = (mine > TP_C_SLOTS ? mine - TP_C_SLOTS : 0); j < mine; ++j)
                    mbar_wait(&full[j % TP_C_SLOTS], (j / TP_C_SLOTS) & 1);
        }
        __syncwarp();
    } else {
        const double2* tw = static_cast<const double2*>(a.tw_y);
        for (int i = 0; i < mine; ++i) {
            const int s = i % TP_C_SLOTS;
            int kx, j0;
            coords(i, kx, j0);
            // this thread's scale factors, fetched while the tile is in flight
            double r[C::PER];
#pragma unroll
            for (int k = 0; k < C::PER; ++k) {
                const int e = tid + k * C::CONS, ky = e / CT, cc = e - ky * CT;
                r[k] = e < NY * CT ? a.recip[(long long)a.grp_of_row[kx * NY + ky] * EIG_SLOTS + j0 + cc] * a.scale
                                   : 0.0;
            }
            const bool ok = tp_wait(&full[s], (i / TP_C_SLOTS) & 1, &s_err, a.err, 6);
            double2* sm = ring + (size_t)s * NY * CT;
            if (ok) slab_fft<NY, -1, C::CONS, 1>(sm, CT, CT, tw);
#pragma unroll
            for (int k = 0; k < C::PER; ++k) {
                const int e = tid + k * C::CONS;
                if (ok && e < NY * CT) sm[e] = make_double2(sm[e].x * r[k], sm[e].y * r[k]);
            }
            consumers_sync<C::CONS>();
            if (ok) slab_fft<NY, 1, C::CONS, 1>(sm, CT, CT, tw);
            fence_proxy_async_smem();
            consumers_sync<C::CONS>();
            if (tid == 0) mbar_arrive(&done[s]);
        }
    }
}

template <typename K>
cudaError_t prep(K k, size_t smem)
{
    return cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

template <int NY>
int run_conv_tma(const EigArgs& a, EigMaps& tm, cudaStream_t s)
{
    constexpr int CT = NY <= 256 ? 16 : 8;
    using C = ConvShape<NY, CT>;
    const uint64_t dims[3] = {2 * EIG_SLOTS, (uint64_t)NY, (uint64_t)a.nkx};
    const uint64_t str[2] = {2 * EIG_SLOTS * sizeof(double), (uint64_t)NY * 2 * EIG_SLOTS * sizeof(double)};
    const uint32_t box[3] = {2 * CT, (uint32_t)C::BOX_Y, 1};
    if (!encode_tmap_f64_3d(&tm.T, a.S, dims, str, box)) return (int)cudaErrorInvalidValue;
    cudaError_t e = prep(eig_conv_tma_kernel<NY, CT>, C::smem);
    if (e != cudaSuccess) return (int)e;
    const int ntiles = a.nkx * C::TILES_PER_KX;
    const int grid = ntiles < a.nsm ? ntiles : a.nsm;
    return (int)launch_k(eig_conv_tma_kernel<NY, CT>, dim3(grid), dim3(C::THREADS), C::smem, s, a, tm);
}

template <int L>
int run_3d_tma(int pass, const EigArgs& a, cudaStream_t s)
{
    using T = TmaShape<L>;
    EigMaps tm;
    std::memset(&tm, 0, sizeof(tm));
    const int grid = a.Ny < a.nsm ? a.Ny : a.nsm;
    cudaError_t e;
    if (pass == 0) {
        const uint64_t dims[2] = {(uint64_t)a.x_stride, (uint64_t)L};
        const uint64_t str[1] = {(uint64_t)a.x_stride * sizeof(double)};
        const uint32_t box[2] = {TP_PITCH, T::RC};
        if (!encode_tmap_f64_2d(&tm.f, a.f, dims, str, box)) return (int)cudaErrorInvalidValue;
        if (a.sub && !encode_tmap_f64_2d(&tm.sub, a.sub, dims, str, box)) return (int)cudaErrorInvalidValue;
        if ((e = prep(eig_fwd_tma_kernel<L>, T::smem1)) != cudaSuccess) return (int)e;
        return (int)launch_k(eig_fwd_tma_kernel<L>, dim3(grid), dim3(T::THREADS), T::smem1, s, a, tm);
    }
    if (pass == 2) {
        const uint64_t dims[3] = {2 * EIG_SLOTS, (uint64_t)a.Ny, (uint64_t)a.nkx};
        const uint64_t str[2] = {2 * EIG_SLOTS * sizeof(double), (uint64_t)a.Ny * 2 * EIG_SLOTS * sizeof(double)};
        const uint32_t box[3] = {2 * EIG_SLOTS, 1, (uint32_t)T::KC};
        if (!encode_tmap_f64_3d(&tm.S, a.S, dims, str, box)) return (int)cudaErrorInvalidValue;
        if ((e = prep(eig_inv_tma_kernel<L>, T::smem3)) != cudaSuccess) return (int)e;
        return (int)launch_k(eig_inv_tma_kernel<L>, dim3(grid), dim3(T::THREADS), T::smem3, s, a, tm);
    }
    switch (a.Ny) {
        case 4: return run_conv_tma<4>(a, tm, s);
        case 8: return run_conv_tma<8>(a, tm, s);
        case 16: return run_conv_tma<16>(a, tm, s);
        case 32: return run_conv_tma<32>(a, tm, s);
        case 64: return run_conv_tma<64>(a, tm, s);
        case 128: return run_conv_tma<128>(a, tm, s);
        case 256: return run_conv_tma<256>(a, tm, s);
        case 512: return run_conv_tma<512>(a, tm, s);
        default: return (int)cudaErrorInvalidValue;
    }
}

template <int L>
int run_3d(int pass, const EigArgs& a, cudaStream_t s)
{
    using S = EpShape<L>;
    cudaError_t e;
    const size_t sm1 = S::smem(2);
    if (a.tma) return run_3d_tma<L>(pass, a, s);
    if (pass == 0) {
        if ((e = prep(eig_fwd_kernel<L>, sm1)) != cudaSuccess) return (int)e;
        return (int)launch_k(eig_fwd_kernel<L>, dim3(a.Ny), dim3(S::THREADS), sm1, s, a);
    }
    if (pass == 2) {
        if ((e = prep(eig_inv_kernel<L>, sm1)) != cudaSuccess) return (int)e;
        return (int)launch_k(eig_inv_kernel<L>, dim3(a.Ny), dim3(S::THREADS), sm1, s, a);
    }
    const int nkx = L / 2 + 1;
    switch (a.Ny) {
#define HELM_EIG_CONV(NY, CT)                                                                                   \
    case NY: {                                                                                                  \
        const size_t sm2 = (size_t)NY * CT * sizeof(double2);                                                   \
        if ((e = prep(eig_conv_kernel<NY, CT>, sm2)) != cudaSuccess) return (int)e;                             \
        return (int)launch_k(eig_conv_kernel<NY, CT>, dim3(nkx * (EIG_SLOTS / CT)), dim3(256), sm2, s, a);      \
    }
        HELM_EIG_CONV(4, 16)
        HELM_EIG_CONV(8, 16)
        HELM_EIG_CONV(16, 16)
        HELM_EIG_CONV(32, 16)
        HELM_EIG_CONV(64, 16)
        HELM_EIG_CONV(128, 16)
        HELM_EIG_CONV(256, 16)
        HELM_EIG_CONV(512, 8)
#undef HELM_EIG_CONV
        default: return (int)cudaErrorInvalidValue;
    }
}

template <int L>
int run_2d(const EigArgs& a, int nprob, cudaStream_t s)
{
    using S = EpShape<L>;
    const size_t sm = S::smem(4);
    cudaError_t e = prep(eig_solve2d_kernel<L>, sm);
    if (e != cudaSuccess) return (int)e;
    return (int)launch_k(eig_solve2d_kernel<L>, dim3(nprob), dim3(S::THREADS), sm, s, a);
}

}  // namespace

bool eig_tma_ok(const EigArgs& a)
{
    auto al = [](const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; };
    return al(a.f) && (!a.sub || al(a.sub)) && al(a.S) && (a.x_stride & 1) == 0;
}

bool eig_shape_ok(int dim, int Nx, int Ny, int P)
{
    if (P < 4 || P > 2 * EIG_LD + 2) return false;
    if (Nx < 8 || Nx > 256 || (Nx & (Nx - 1))) return false;
    if (dim == 2) return true;
    return Ny >= 4 && Ny <= 512 && !(Ny & (Ny - 1));
}

int launch_eig_pass(int pass, int dim, int Nx, const EigArgs& a, int nprob, cudaStream_t s)
{
    if (dim == 3) {
        switch (Nx) {
            case 8: return run_3d<8>(pass, a, s);
            case 16: return run_3d<16>(pass, a, s);
            case 32: return run_3d<32>(pass, a, s);
            case 64: return run_3d<64>(pass, a, s);
            case 128: return run_3d<128>(pass, a, s);
            case 256: return run_3d<256>(pass, a, s);
            default: return (int)cudaErrorInvalidValue;
        }
    }
    if (pass != 0) return 0;
    switch (Nx) {
        case 8: return run_2d<8>(a, nprob, s);
        case 16: return run_2d<16>(a, nprob, s);
        case 32: return run_2d<32>(a, nprob, s);
        case 64: return run_2d<64>(a, nprob, s);
        case 128: return run_2d<128>(a, nprob, s);
        case 256: return run_2d<256>(a, nprob, s);
        default: return (int)cudaErrorInvalidValue;
    }
}

}  // namespace helm
