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

#include <cooperative_groups.h>
#include <cstring>

namespace cg = cooperative_groups;

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

// Loads rows x0 .. x0 + L - 1 of plane y of f (GLL slots 1..P-2) into buf and
// the scaled boundary values zl, zr into slots 0 and P-1.
template <int L>
__device__ __forceinline__ void load_plane(const EigArgs& a, const double* f, const double* gl, const double* gr,
                                           long long yoff, long long bc_off, double* buf, int x0 = 0)
{
    const int P = a.P;
    for (int e = threadIdx.x; e < L * P; e += blockDim.x) {
        const int xl = e / P, k = e - xl * P;
        const long long x = x0 + xl;
        double* d = buf + xl * EP_PITCH + k;
        const double* s = f + x * a.x_stride + yoff + k;
        if (k == 0) *d = gl ? gl[x * a.bc_x_stride + bc_off] * a.ibl : 0.0;
        else if (k == P - 1) *d = gr ? gr[x * a.bc_x_stride + bc_off] * a.ibr : 0.0;
        else cp_async_bytes8(d, s, true);
    }
    cp_async_commit();
    cp_async_wait_all();
    if (a.sub) {  // adjoint of a least-squares misfit: ubar = u - u_obs at the interior slots
        __syncthreads();
        for (int e = threadIdx.x; e < L * P; e += blockDim.x) {
            const int xl = e / P, k = e - xl * P;
            if (k > 0 && k < P - 1) buf[xl * EP_PITCH + k] -= a.sub[(long long)(x0 + xl) * a.x_stride + yoff + k];
        }
    }
}

// First transform of the warp's rows (8 MTW rows at `rows`): coefficients of
// the folded interior plus the boundary columns, written back over the rows as
// slots 0..31 (symmetric fold) and 32..63 (antisymmetric fold).
template <int MTW>
__device__ __forceinline__ void first_transform(const EigArgs& a, double* rows, const double* Ms, const double* Ma,
                                                const double* hbc, int lane, int in_off = 0,
                                                const double* sub_rows = nullptr)
{
    // the staged rows start in_off doubles into each row (a TMA copy whose
    // source began 8 bytes before the row); the coefficients go to slot 0 on.
    // sub_rows: the same rows of u_obs, subtracted (misfit adjoint)
    const double* src = rows + in_off;
    const double* sbs = sub_rows ? sub_rows + in_off : nullptr;
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
            const double* row = src + (mt * 8 + g) * EP_PITCH;
            const double* srow = sbs ? sbs + (mt * 8 + g) * EP_PITCH : nullptr;
            double vs = 0.0, va = 0.0;
            if (k < m) {
                double lo = row[1 + k], hi = row[n - k];
                if (srow) {
                    lo -= srow[1 + k];
                    hi -= srow[n - k];
                }
                vs = kR2 * (lo + hi);
                va = kR2 * (lo - hi);
            } else if (k < ms) {
                vs = srow ? row[1 + k] - srow[1 + k] : row[1 + k];
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
        const double* row = src + (mt * 8 + g) * EP_PITCH;
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
    // three rows per round, fetched before any is used
    constexpr int W = EpShape<L>::WARPS, NB = 3;
    for (int k0 = warp; k0 <= L / 2; k0 += NB * W) {
        double2 X[NB], Y[NB];
#pragma unroll
        for (int b = 0; b < NB; ++b)
            if (k0 + b * W <= L / 2) fetch(k0 + b * W, lane, X[b], Y[b]);
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            const int kx = k0 + b * W;
            if (kx > L / 2) break;
            if (kx == 0 || kx == L / 2) { X[b].y = 0.0; Y[b].y = 0.0; }
            z[kx * EP_HS + lane] = make_double2(X[b].x - Y[b].y, X[b].y + Y[b].x);
            if (kx > 0 && kx < L / 2) z[(L - kx) * EP_HS + lane] = make_double2(X[b].x + Y[b].y, Y[b].x - X[b].y);
        }
    }
}

// ------------------------------------------------------------------ pass 1 --
// Tensor map of pass 1 (kernel parameter, built on the host per solve): f as
// [Nx][x_stride] doubles, box EP_PITCH x (Nx / 4) (x / 4 rows of one plane).
struct EigMaps {
    CUtensorMap f;
    CUtensorMap sub;  // the misfit adjoint's u_obs, the same shape (planes up to 128 rows)
};

template <int L>
struct FwdBoxes {
    static constexpr int NQ = L >= 32 ? 4 : 1;  // TMA boxes per plane (row quarters)
    static constexpr int QR = L / NQ;           // rows per box
};

template <int L>
__global__ void __launch_bounds__(EpShape<L>::THREADS, 1) eig_fwd_kernel(EigArgs a, const __grid_constant__ EigMaps tm)
{
    using S = EpShape<L>;
    using B = FwdBoxes<L>;
    extern __shared__ __align__(128) double esm[];
    __shared__ __align__(8) uint64_t bar[B::NQ];
    double* buf = esm;
    double* Mt = esm + (size_t)L * EP_PITCH;
    // misfit adjoint with TMA loads: u_obs's plane after the transforms
    double* sbuf = (a.tma && a.sub) ? Mt + 2 * EP_FRAG : nullptr;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int y = blockIdx.x;
    const bool tma = a.tma != 0;
    if (tma && threadIdx.x == 0) {
        for (int q = 0; q < B::NQ; ++q) mbar_init(&bar[q], 1);
        fence_mbar_init();
    }
    copy_mats(Mt, a.mats, 0, 2);
    __syncthreads();
    pdl_enter();
    if (a.lam_out && blockIdx.x == 0 && threadIdx.x == 0) *a.lam_out = 0.0;
    double* rows = buf + warp * S::RW * EP_PITCH;
    bool tma_ok = true;
    if (tma) {
        // the plane in four boxes (one bulk copy each); a warp starts on its
        // rows as soon as their box has landed.  The copies start at the
        // 16-byte boundary at or before the plane's first element: element k
        // of a row lands in slot k + sh.
        const int sh = (int)(((long long)y * a.P) & 1);
        if (threadIdx.x == 0) {
            const int c0 = y * a.P - sh;
            const uint32_t box = (uint32_t)(B::QR * EP_PITCH * sizeof(double));
            for (int q = 0; q < B::NQ; ++q) {
                mbar_arrive_expect_tx(&bar[q], sbuf ? 2 * box : box);
                tma_load_2d(buf + (size_t)q * B::QR * EP_PITCH, &tm.f, c0, q * B::QR, &bar[q]);
                if (sbuf) tma_load_2d(sbuf + (size_t)q * B::QR * EP_PITCH, &tm.sub, c0, q * B::QR, &bar[q]);
            }
        }
        tma_ok = mbar_wait(&bar[(warp * S::RW) / B::QR], 0);
        if (!tma_ok && lane == 0 && a.err) atomicExch(a.err, 1);
        const double* gl = a.adjoint ? nullptr : a.gl;
        const double* gr = a.adjoint ? nullptr : a.gr;
        if (lane < S::RW) {  // the GLL boundary slots take zl = gl / beta_l, zr = gr / beta_r
            const long long x = (long long)warp * S::RW + lane;
            rows[lane * EP_PITCH + sh] = gl ? gl[x * a.bc_x_stride + y] * a.ibl : 0.0;
            rows[lane * EP_PITCH + sh + a.P - 1] = gr ? gr[x * a.bc_x_stride + y] * a.ibr : 0.0;
        }
        __syncwarp();
        if (tma_ok)
            first_transform<S::MTW>(a, rows, Mt, Mt + EP_FRAG, a.hbc, lane, sh,
                                    sbuf ? sbuf + warp * S::RW * EP_PITCH : nullptr);
    } else {
        load_plane<L>(a, a.f, a.adjoint ? nullptr : a.gl, a.adjoint ? nullptr : a.gr, (long long)y * a.P, y, buf);
        __syncthreads();
        first_transform<S::MTW>(a, rows, Mt, Mt + EP_FRAG, a.hbc, lane);
    }
    __syncthreads();
    if (tma && threadIdx.x == 0 && !tma_ok)  // copies still in flight land before the CTA ends
        for (int q = 0; q < B::NQ; ++q) mbar_wait(&bar[q], 0);
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
// CTA shapes of pass 2: 16 coefficient columns per tile and 256 threads (two
// CTAs per SM), or 8 columns and 128 threads (four per SM, more tiles in
// flight); launch variant bit 0 of the y pass picks one.
template <int NY, int CT, int THREADS>
__global__ void __launch_bounds__(THREADS, 512 / THREADS) eig_conv_kernel(EigArgs a)
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
    // this thread's scale factors, fetched while the tile is in flight
    constexpr int PER = (NY * CT + THREADS - 1) / THREADS;
    double r[PER];
    const double* rc = a.recip;
#pragma unroll
    for (int k = 0; k < PER; ++k) {
        const int e = threadIdx.x + THREADS * k, ky = e / CT, c = e - ky * CT;
        r[k] = e < NY * CT ? rc[(long long)a.grp_of_row[kx * NY + ky] * EIG_SLOTS + j0 + c] * a.scale : 0.0;
    }
    cp_async_wait_all();
    __syncthreads();
    const double2* tw = static_cast<const double2*>(a.tw_y);
    slab_fft<NY, -1, THREADS>(sm, CT, CT, tw);
#pragma unroll
    for (int k = 0; k < PER; ++k) {
        const int e = threadIdx.x + THREADS * k;
        if (e < NY * CT) sm[e] = make_double2(sm[e].x * r[k], sm[e].y * r[k]);
    }
    __syncthreads();
    slab_fft<NY, 1, THREADS>(sm, CT, CT, tw);
    for (int e = threadIdx.x; e < NY * CT; e += blockDim.x) {
        const int ky = e / CT, c = e - ky * CT;
        Sg[(long long)ky * EIG_SLOTS + c] = sm[ky * CT + c];
    }
}

// Adjoint: the boundary terms of the transposed map for the warp's rows,
// b_l . fbar_int = hsl . cs + hal . ca (and the same with the right-hand
// vectors), from the coefficients in slots 0..63 before the second transform.
template <int RW>
__device__ __forceinline__ void adjoint_boundary_dots(const EigArgs& a, const double* rows, int lane, double* dl,
                                                      double* dr)
{
    const double hs0 = a.hbc[lane], hs1 = a.hbc[EIG_LD + lane], ha0 = a.hbc[2 * EIG_LD + lane],
                 ha1 = a.hbc[3 * EIG_LD + lane];
    for (int r = 0; r < RW; ++r) {
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
template <int RW>
__device__ __forceinline__ double store_adjoint_rows(const EigArgs& a, double* fbar, const double* ubar,
                                                     long long yoff, long long bc_off, double* rows, int x0, int lane,
                                                     double dl, double dr)
{
    const int P = a.P;
    if (lane < RW) {
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
    for (int r = 0; r < RW; ++r) {
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
template <int RW>
__device__ __forceinline__ void store_plane_rows(const EigArgs& a, double* u, const double* gl, const double* gr,
                                                 long long yoff, long long bc_off, double* rows, int x0, int lane)
{
    const int P = a.P;
    if (lane < RW) {
        const long long x = x0 + lane;
        rows[lane * EP_PITCH] = gl ? gl[x * a.bc_x_stride + bc_off] * a.ibl : 0.0;
        rows[lane * EP_PITCH + P - 1] = gr ? gr[x * a.bc_x_stride + bc_off] * a.ibr : 0.0;
    }
    __syncwarp();
    for (int r = 0; r < RW; ++r) {
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
        store_plane_rows<S::RW>(a, a.u, a.gl, a.gr, (long long)y * a.P, y, rows, warp * S::RW, lane);
        return;
    }
    double dl = 0.0, dr = 0.0;
    adjoint_boundary_dots<S::RW>(a, rows, lane, &dl, &dr);
    __syncwarp();
    second_transform<S::MTW>(a, rows, Mt, Mt + EP_FRAG, lane);
    const double acc =
        store_adjoint_rows<S::RW>(a, a.u, a.f, (long long)y * a.P, y, rows, warp * S::RW, lane, dl, dr);
    if (a.lam_out) eig_lambda_sum(a, acc);
}

// ------------------------------------------------- pair-split passes 1, 3 --
// Passes 1 and 3 with each plane shared by a cluster of two CTAs: CTA rank r
// holds rows x = r H .. r H + H - 1 (H = L / 2), so a CTA needs half the
// shared memory and two fit on an SM, overlapping one CTA's copies with the
// other's arithmetic.  The length-L FFT along x is split by the parity of
// the wavenumber: pass 1 takes the first radix-2 step of a decimation in
// frequency across the pair (rank 0 keeps a_m = z_m + z_{m+H}, rank 1 keeps
// b_m = (z_m - z_{m+H}) w^m, w = exp(-2 pi i / L)), reading the partner's rows
// from its shared memory, then a length-H FFT gives the even (rank 0) or odd
// (rank 1) wavenumbers.  Pass 3 runs the mirror image: a length-H inverse FFT
// of its parity's wavenumbers, then the last step of a decimation in time
// across the pair, x_m = E_m + conj(w^m) O_m (rank 0) and x_{m+H} = E_m -
// conj(w^m) O_m (rank 1).
template <int L>
struct SplitShape {
    static constexpr int H = L / 2;
    static constexpr int WARPS = (H / 16 < 8) ? H / 16 : 8;
    static constexpr int THREADS = 32 * WARPS;
    static constexpr int RW = H / WARPS;  // 16 rows per warp
    static constexpr int MTW = RW / 8;
    static constexpr int NQ = 2;          // TMA boxes per CTA
    static constexpr int QR = H / NQ;
    static_assert(RW == 16 && QR == FwdBoxes<L>::QR, "pair-split shape");
    static constexpr size_t smem(int nmats) { return ((size_t)H * EP_PITCH + (size_t)nmats * EP_FRAG) * sizeof(double); }
};

// The cross-pair butterfly on the [H][EP_HS] complex rows z: every thread
// reads its elements of the partner's rows, the pair synchronises (both have
// read), and combine(m, own, partner) replaces each element.  The caller has
// synchronised the pair after its last write of z.
template <int L, typename Combine>
__device__ __forceinline__ void pair_exchange(cg::cluster_group& cluster, double2* z, Combine combine)
{
    using S = SplitShape<L>;
    constexpr int PER = S::H * 32 / S::THREADS;
    const double2* zp = cluster.map_shared_rank(z, (int)cluster.block_rank() ^ 1);
    double2 pv[PER];
#pragma unroll
    for (int k = 0; k < PER; ++k) {
        const int e = threadIdx.x + k * S::THREADS, m = e >> 5, c = e & 31;
        pv[k] = zp[m * EP_HS + c];
    }
    cluster.sync();
#pragma unroll
    for (int k = 0; k < PER; ++k) {
        const int e = threadIdx.x + k * S::THREADS, m = e >> 5, c = e & 31;
        z[m * EP_HS + c] = combine(m, z[m * EP_HS + c], pv[k]);
    }
    __syncthreads();
}

template <int L>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(SplitShape<L>::THREADS, 2)
    eig_fwd_split_kernel(EigArgs a, const __grid_constant__ EigMaps tm)
{
    using S = SplitShape<L>;
    constexpr int H = S::H;
    extern __shared__ __align__(128) double esm[];
    __shared__ __align__(8) uint64_t bar[S::NQ];
    cg::cluster_group cluster = cg::this_cluster();
    const int rank = (int)cluster.block_rank();
    double* buf = esm;
    double* Mt = esm + (size_t)H * EP_PITCH;
    double* sbuf = (a.tma && a.sub) ? Mt + 2 * EP_FRAG : nullptr;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int y = blockIdx.x >> 1, x0 = rank * H;
    const bool tma = a.tma != 0;
    if (tma && threadIdx.x == 0) {
        for (int q = 0; q < S::NQ; ++q) mbar_init(&bar[q], 1);
        fence_mbar_init();
    }
    copy_mats(Mt, a.mats, 0, 2);
    __syncthreads();
    pdl_enter();
    if (a.lam_out && blockIdx.x == 0 && threadIdx.x == 0) *a.lam_out = 0.0;
    double* rows = buf + warp * S::RW * EP_PITCH;
    bool tma_ok = true;
    if (tma) {
        const int sh = (int)(((long long)y * a.P) & 1);
        if (threadIdx.x == 0) {
            const int c0 = y * a.P - sh;
            const uint32_t box = (uint32_t)(S::QR * EP_PITCH * sizeof(double));
            for (int q = 0; q < S::NQ; ++q) {
                mbar_arrive_expect_tx(&bar[q], sbuf ? 2 * box : box);
                tma_load_2d(buf + (size_t)q * S::QR * EP_PITCH, &tm.f, c0, x0 + q * S::QR, &bar[q]);
                if (sbuf) tma_load_2d(sbuf + (size_t)q * S::QR * EP_PITCH, &tm.sub, c0, x0 + q * S::QR, &bar[q]);
            }
        }
        tma_ok = mbar_wait(&bar[(warp * S::RW) / S::QR], 0);
        if (!tma_ok && lane == 0 && a.err) atomicExch(a.err, 1);
        const double* gl = a.adjoint ? nullptr : a.gl;
        const double* gr = a.adjoint ? nullptr : a.gr;
        if (lane < S::RW) {
            const long long x = x0 + (long long)warp * S::RW + lane;
            rows[lane * EP_PITCH + sh] = gl ? gl[x * a.bc_x_stride + y] * a.ibl : 0.0;
            rows[lane * EP_PITCH + sh + a.P - 1] = gr ? gr[x * a.bc_x_stride + y] * a.ibr : 0.0;
        }
        __syncwarp();
        if (tma_ok)
            first_transform<S::MTW>(a, rows, Mt, Mt + EP_FRAG, a.hbc, lane, sh,
                                    sbuf ? sbuf + warp * S::RW * EP_PITCH : nullptr);
    } else {
        load_plane<H>(a, a.f, a.adjoint ? nullptr : a.gl, a.adjoint ? nullptr : a.gr, (long long)y * a.P, y, buf, x0);
        __syncthreads();
        first_transform<S::MTW>(a, rows, Mt, Mt + EP_FRAG, a.hbc, lane);
    }
    __syncthreads();
    if (tma && threadIdx.x == 0 && !tma_ok)  // copies still in flight land before the CTA ends
        for (int q = 0; q < S::NQ; ++q) mbar_wait(&bar[q], 0);
    cluster.sync();  // both halves of the plane are transformed
    double2* z = reinterpret_cast<double2*>(buf);
    const double2* tw = static_cast<const double2*>(a.tw_x);
    pair_exchange<L>(cluster, z, [&](int m, double2 own, double2 other) {
        if (rank == 0) return make_double2(own.x + other.x, own.y + other.y);
        return cmul(make_double2(other.x - own.x, other.y - own.y), tw[m]);
    });
    slab_fft<H, -1, S::THREADS, 0, 2>(z, EP_HS, 32, tw);
    // local row k' holds wavenumber 2 k' + rank; its mirror L - k is local
    // row (H - k') mod H (even) or H - 1 - k' (odd)
    double2* Sg = reinterpret_cast<double2*>(a.S);
    const long long Ny = a.Ny;
    const int kmax = rank == 0 ? H / 2 : H / 2 - 1;
    for (int kp = warp; kp <= kmax; kp += S::WARPS) {
        const int km = rank == 0 ? ((H - kp) & (H - 1)) : (H - 1 - kp);
        const double2 zk = z[kp * EP_HS + lane], zm = z[km * EP_HS + lane];
        double2* row = Sg + ((long long)(2 * kp + rank) * Ny + y) * EIG_SLOTS;
        row[2 * lane] = make_double2(0.5 * (zk.x + zm.x), 0.5 * (zk.y - zm.y));
        row[2 * lane + 1] = make_double2(0.5 * (zk.y + zm.y), 0.5 * (zm.x - zk.x));
    }
}

template <int L>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(SplitShape<L>::THREADS, 2) eig_inv_split_kernel(EigArgs a)
{
    using S = SplitShape<L>;
    constexpr int H = S::H;
    extern __shared__ __align__(16) double esm[];
    cg::cluster_group cluster = cg::this_cluster();
    const int rank = (int)cluster.block_rank();
    double* buf = esm;
    double* Mt = esm + (size_t)H * EP_PITCH;
    copy_mats(Mt, a.mats, 1, 3);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int y = blockIdx.x >> 1, x0 = rank * H;
    double2* z = reinterpret_cast<double2*>(buf);
    const double2* Sg = reinterpret_cast<const double2*>(a.S);
    const long long Ny = a.Ny;
    pdl_enter();
    // wavenumbers of this rank's parity, kx = 2 kp + rank <= L / 2, three
    // rows per round fetched before any is used
    constexpr int W = S::WARPS, NB = 3;
    const int kmax = rank == 0 ? H / 2 : H / 2 - 1;
    for (int k0 = warp; k0 <= kmax; k0 += NB * W) {
        double2 X[NB], Y[NB];
#pragma unroll
        for (int b = 0; b < NB; ++b)
            if (k0 + b * W <= kmax) {
                const double2* row = Sg + ((long long)(2 * (k0 + b * W) + rank) * Ny + y) * EIG_SLOTS;
                X[b] = row[2 * lane];
                Y[b] = row[2 * lane + 1];
            }
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            const int kp = k0 + b * W;
            if (kp > kmax) break;
            const int kx = 2 * kp + rank;
            if (kx == 0 || kx == L / 2) { X[b].y = 0.0; Y[b].y = 0.0; }
            z[kp * EP_HS + lane] = make_double2(X[b].x - Y[b].y, X[b].y + Y[b].x);
            if (kx > 0 && kx < L / 2) z[((L - kx - rank) / 2) * EP_HS + lane] = make_double2(X[b].x + Y[b].y, Y[b].x - X[b].y);
        }
    }
    __syncthreads();
    const double2* tw = static_cast<const double2*>(a.tw_x);
    slab_fft<H, 1, S::THREADS, 0, 2>(z, EP_HS, 32, tw);
    cluster.sync();  // both parities are transformed
    pair_exchange<L>(cluster, z, [&](int m, double2 own, double2 other) {
        if (rank == 0) {
            const double2 t = cmulc(other, tw[m]);
            return make_double2(own.x + t.x, own.y + t.y);
        }
        const double2 t = cmulc(own, tw[m]);
        return make_double2(other.x - t.x, other.y - t.y);
    });
    double* rows = buf + warp * S::RW * EP_PITCH;
    const int xw = x0 + warp * S::RW;
    if (!a.adjoint) {
        second_transform<S::MTW>(a, rows, Mt, Mt + EP_FRAG, lane);
        store_plane_rows<S::RW>(a, a.u, a.gl, a.gr, (long long)y * a.P, y, rows, xw, lane);
        return;
    }
    double dl = 0.0, dr = 0.0;
    adjoint_boundary_dots<S::RW>(a, rows, lane, &dl, &dr);
    __syncwarp();
    second_transform<S::MTW>(a, rows, Mt, Mt + EP_FRAG, lane);
    const double acc = store_adjoint_rows<S::RW>(a, a.u, a.f, (long long)y * a.P, y, rows, xw, lane, dl, dr);
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
        store_plane_rows<S::RW>(a, a.u + off, gl, gr, 0, 0, rows, warp * S::RW, lane);
        return;
    }
    double dl = 0.0, dr = 0.0;
    adjoint_boundary_dots<S::RW>(a, rows, lane, &dl, &dr);
    __syncwarp();
    second_transform<S::MTW>(a, rows, M2, M2 + EP_FRAG, lane);
    const double acc = store_adjoint_rows<S::RW>(a, a.u, a.f, 0, 0, rows, warp * S::RW, lane, dl, dr);
    if (a.lam_out) eig_lambda_sum(a, acc);
}

template <typename K>
cudaError_t prep(K k, size_t smem)
{
    return cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

template <int L>
int run_3d(int pass, const EigArgs& a, cudaStream_t s)
{
    using S = EpShape<L>;
    cudaError_t e;
    const size_t sm1 = S::smem(2);
    if (pass == 0) {
        EigMaps tm;
        std::memset(&tm, 0, sizeof(tm));
        EigArgs a1 = a;
        if (a1.tma) {
            const uint64_t dims[2] = {(uint64_t)a.x_stride, (uint64_t)L};
            const uint64_t str[1] = {(uint64_t)a.x_stride * sizeof(double)};
            const uint32_t box[2] = {EP_PITCH, (uint32_t)FwdBoxes<L>::QR};
            if (!encode_tmap_f64_2d(&tm.f, a.f, dims, str, box) ||
                (a.sub && !encode_tmap_f64_2d(&tm.sub, a.sub, dims, str, box)))
                a1.tma = 0;  // element-wise loads instead
        }
        if constexpr (L >= 64) {
            if (a.split) {
                using SS = SplitShape<L>;
                const size_t sms = SS::smem(2) + ((a1.tma && a1.sub) ? (size_t)SS::H * EP_PITCH * sizeof(double) : 0);
                if ((e = prep(eig_fwd_split_kernel<L>, sms)) != cudaSuccess) return (int)e;
                return (int)launch_k(eig_fwd_split_kernel<L>, dim3(2 * a.Ny), dim3(SS::THREADS), sms, s, a1, tm);
            }
        }
        // the misfit adjoint's TMA path stages u_obs's plane beside f's
        const size_t smf = (a1.tma && a1.sub) ? sm1 + (size_t)L * EP_PITCH * sizeof(double) : sm1;
        if ((e = prep(eig_fwd_kernel<L>, smf)) != cudaSuccess) return (int)e;
        return (int)launch_k(eig_fwd_kernel<L>, dim3(a.Ny), dim3(S::THREADS), smf, s, a1, tm);
    }
    if (pass == 2) {
        if constexpr (L >= 64) {
            if (a.split) {
                using SS = SplitShape<L>;
                if ((e = prep(eig_inv_split_kernel<L>, SS::smem(2))) != cudaSuccess) return (int)e;
                return (int)launch_k(eig_inv_split_kernel<L>, dim3(2 * a.Ny), dim3(SS::THREADS), SS::smem(2), s, a);
            }
        }
        if ((e = prep(eig_inv_kernel<L>, sm1)) != cudaSuccess) return (int)e;
        return (int)launch_k(eig_inv_kernel<L>, dim3(a.Ny), dim3(S::THREADS), sm1, s, a);
    }
    const int nkx = L / 2 + 1;
    const bool narrow = a.conv_var & 1;
    switch (a.Ny) {
#define HELM_EIG_CONV(NY, CT, TH)                                                                               \
    {                                                                                                           \
        const size_t sm2 = (size_t)NY * CT * sizeof(double2);                                                   \
        if ((e = prep(eig_conv_kernel<NY, CT, TH>, sm2)) != cudaSuccess) return (int)e;                         \
        return (int)launch_k(eig_conv_kernel<NY, CT, TH>, dim3(nkx * (EIG_SLOTS / CT)), dim3(TH), sm2, s, a);   \
    }
#define HELM_EIG_CONV2(NY)                                                                                      \
    case NY:                                                                                                    \
        if (narrow) HELM_EIG_CONV(NY, 8, 128) else HELM_EIG_CONV(NY, 16, 256)
        HELM_EIG_CONV2(4)
        HELM_EIG_CONV2(8)
        HELM_EIG_CONV2(16)
        HELM_EIG_CONV2(32)
        HELM_EIG_CONV2(64)
        HELM_EIG_CONV2(128)
        HELM_EIG_CONV2(256)
        case 512:
            if (narrow) HELM_EIG_CONV(512, 4, 256) else HELM_EIG_CONV(512, 8, 256)
#undef HELM_EIG_CONV2
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

bool eig_tma_ok(const EigArgs& a, int Nx)
{
    auto al = [](const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; };
    // with u_obs the two planes share the shared memory: planes of at most 128 rows
    return al(a.f) && (a.x_stride & 1) == 0 && (!a.sub || (al(a.sub) && Nx <= 128));
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
