// Derivative along the GLL direction (sm_100a): du = M u for every row of P
// values, M the plan's scaled first- or second-derivative matrix.  Replaces the
// reference's per-element loops FirstDerivativeY / SecondDerivativeY
// (NonPeriodic2D_MPI.cpp:497-542, Periodic2D_MPI.cpp:714-763) and
// FirstDerivativeZ / SecondDerivativeZ (NonPeriodic3D_MPI.cpp:632-683,
// Periodic3D_MPI.cpp:905-957).
//
// The GLL derivative matrices are anti-centrosymmetric (first) or
// centrosymmetric (second), so with the fold s_k = u_k + u_{P-1-k},
// a_k = u_k - u_{P-1-k} (k < h = P/2; s_h = u_h for odd P) every output pair
// comes from two half-size products:
//     sigma_j = sum_k E[j][k] s_k,   E[j][k] = (M[j][k] + M[j][P-1-k]) / 2  (E[j][h] = M[j][h])
//     alpha_j = sum_k F[j][k] a_k,   F[j][k] = (M[j][k] - M[j][P-1-k]) / 2
//     du_j = sigma_j + alpha_j,      du_{P-1-j} = -/+ (sigma_j - alpha_j)  (first / second)
// which halves the multiply-adds of the dense product.
//
// FP64 arrays run both products on the FP64 tensor cores (gll_deriv_bulk_kernel
// for the packed layout, gll_deriv_mma_kernel for any other);
// FP32 arrays run them on the CUDA cores, one lane per row (gll_deriv_kernel).
// Each warp owns 32 rows of a tile in shared memory (raw rows, then their
// folded halves) and never waits on another warp.  The raw rows of
// the warp's next tile are copied in by cp.async while it folds, multiplies and
// stores the current one; E and F are built once per CTA and read as
// broadcasts.  HBM-bound: 2 P values (read + write) per row.
#include "helm_device.cuh"
#include "helm_kernels.cuh"
#include "helm_tma.cuh"

namespace helm {

constexpr int GD_JB = 8;   // outputs per register block

struct GdLayout {
    int h, odd, hs, hsp, hap, hsr, rs, os;
    size_t ef_bytes, warp_bytes;
};

template <typename T>
static GdLayout gd_layout(int P)
{
    GdLayout L{};
    L.h = P / 2;
    L.odd = P & 1;
    L.hs = L.h + L.odd;
    L.hsp = (L.hs + 1) & ~1;                 // k loops run in pairs (16-byte loads)
    L.hap = (L.h + 1) & ~1;
    L.hsr = (L.hs + GD_JB - 1) / GD_JB * GD_JB;  // E / F rows padded to whole register blocks
    L.rs = L.hsp + L.hap;                    // folded row stride: = 2 mod 4 elements, so the
    while ((L.rs & 3) != 2) ++L.rs;          //   per-lane 16-byte loads of 8 rows hit distinct banks
    L.os = P | 1;                            // raw row stride: odd
    L.ef_bytes = (size_t)L.hsr * (L.hsp + L.hap) * sizeof(T);
    L.warp_bytes = (size_t)32 * (L.rs + 2 * L.os) * sizeof(T);  // folded rows + two raw buffers
    return L;
}

__device__ __forceinline__ long long gd_row_offset(const GllDerivArgs& a, long long R)
{
    const long long per_elem = (long long)a.nx * a.rows_per_x;
    const long long e = R / per_elem;
    const long long rem = R - e * per_elem;
    const long long i = rem / a.rows_per_x;
    const long long j = rem - i * a.rows_per_x;
    return e * a.elem_stride + i * a.x_stride + j * a.P;
}

template <typename T>
__global__ void gll_deriv_kernel(GllDerivArgs a, GdLayout L)
{
    pdl_enter();
    using V2 = typename std::conditional<sizeof(T) == 8, double2, float2>::type;
    extern __shared__ __align__(16) unsigned char gd_smem[];
    const int P = a.P, h = L.h, hs = L.hs, hsp = L.hsp, hap = L.hap;
    T* E = reinterpret_cast<T*>(gd_smem);                 // [hsr][hsp]
    T* F = E + (size_t)L.hsr * hsp;                       // [hsr][hap]
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    T* fin = reinterpret_cast<T*>(gd_smem + L.ef_bytes + (size_t)warp * L.warp_bytes);  // [32][rs]
    T* raw = fin + (size_t)32 * L.rs;                                                    // [2][32][os]

    for (int e = threadIdx.x; e < L.hsr * hsp; e += blockDim.x) {
        const int j = e / hsp, k = e - j * hsp;
        double v = 0.0;
        if (j < hs) {
            if (k < h) v = 0.5 * (a.M[j * P + k] + a.M[j * P + P - 1 - k]);
            else if (k == h && L.odd) v = a.M[j * P + h];
        }
        E[e] = (T)v;
    }
    for (int e = threadIdx.x; e < L.hsr * hap; e += blockDim.x) {
        const int j = e / hap, k = e - j * hap;
        double v = 0.0;
        if (j < hs && k < h) v = 0.5 * (a.M[j * P + k] - a.M[j * P + P - 1 - k]);
        F[e] = (T)v;
    }
    __syncthreads();

    const T* in = static_cast<const T*>(a.in);
    T* out = static_cast<T*>(a.out);
    const T sgn = a.order == 1 ? (T)-1 : (T)1;
    const long long tiles = (a.nrows + 31) / 32;
    const long long wstride = (long long)gridDim.x * (blockDim.x >> 5);
    // raw rows of tile t land in raw[buf] by cp.async, issued one tile ahead
    auto issue = [&](long long t, T* dst) {
        const long long R0 = t * 32;
        const int nr = (int)min(32LL, a.nrows - R0);
        const long long my = lane < nr ? gd_row_offset(a, R0 + lane) : 0;
        for (int r = 0; r < nr; ++r) {
            const long long off = __shfl_sync(0xffffffffu, my, r);
            for (int k = lane; k < P; k += 32) cp_async_elem<sizeof(T)>(dst + r * L.os + k, in + off + k, true);
        }
        cp_async_commit();
    };
    long long t = (long long)warp * gridDim.x + blockIdx.x;  // warp-major: small jobs still reach every SM
    int buf = 0;
    if (t < tiles) issue(t, raw);
    for (; t < tiles; t += wstride, buf ^= 1) {
        T* cur = raw + (size_t)buf * 32 * L.os;
        const long long R0 = t * 32;
        const int nr = (int)min(32LL, a.nrows - R0);
        if (t + wstride < tiles) {
            issue(t + wstride, raw + (size_t)(buf ^ 1) * 32 * L.os);
            cp_async_wait_prev();
        } else {
            cp_async_wait_all();
        }
        __syncwarp();
        // fold
        for (int r = 0; r < nr; ++r) {
            const T* u = cur + r * L.os;
            T* f = fin + r * L.rs;
            for (int k = lane; k < hsp; k += 32) {
                T s = 0;
                if (k < h) s = u[k] + u[P - 1 - k];
                else if (k == h && L.odd) s = u[h];
                f[k] = s;
            }
            for (int k = lane; k < hap; k += 32) f[hsp + k] = (k < h) ? u[k] - u[P - 1 - k] : (T)0;
        }
        __syncwarp();
        // lane = row: half-size products in register blocks of GD_JB outputs
        if (lane < nr) {
            const T* fs = fin + lane * L.rs;
            const T* fa = fs + hsp;
            T* o = cur + lane * L.os;  // the raw row is folded already: reuse it for the output
            for (int jb = 0; jb < hs; jb += GD_JB) {
                T sg[GD_JB], al[GD_JB];
#pragma unroll
                for (int q = 0; q < GD_JB; ++q) { sg[q] = 0; al[q] = 0; }
                for (int k = 0; k < hsp; k += 2) {
                    const V2 x = *reinterpret_cast<const V2*>(fs + k);
#pragma unroll
                    for (int q = 0; q < GD_JB; ++q) {
                        const V2 m = *reinterpret_cast<const V2*>(E + (size_t)(jb + q) * hsp + k);
                        sg[q] = fma(m.x, x.x, sg[q]);
                        sg[q] = fma(m.y, x.y, sg[q]);
                    }
                }
                for (int k = 0; k < hap; k += 2) {
                    const V2 x = *reinterpret_cast<const V2*>(fa + k);
#pragma unroll
                    for (int q = 0; q < GD_JB; ++q) {
                        const V2 m = *reinterpret_cast<const V2*>(F + (size_t)(jb + q) * hap + k);
                        al[q] = fma(m.x, x.x, al[q]);
                        al[q] = fma(m.y, x.y, al[q]);
                    }
                }
#pragma unroll
                for (int q = 0; q < GD_JB; ++q) {
                    const int j = jb + q;
                    if (j < h) {
                        o[j] = sg[q] + al[q];
                        o[P - 1 - j] = sgn * (sg[q] - al[q]);
                    } else if (j == h && L.odd) {
                        o[j] = sg[q] + al[q];
                    }
                }
            }
        }
        __syncwarp();
        const long long my = lane < nr ? gd_row_offset(a, R0 + lane) : 0;
        for (int r = 0; r < nr; ++r) {
            const long long off = __shfl_sync(0xffffffffu, my, r);
            for (int k = lane; k < P; k += 32) out[off + k] = cur[r * L.os + k];
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// FP64 arrays: the two half-size products on the FP64 tensor cores.  Per warp
// tile of 16 rows (two 8-row m-tiles), sigma = S E^T and alpha = A F^T as
// m8n8k4 products.  The raw rows arrive in shared memory by cp.async one tile
// ahead (two buffers per warp); the A operand (folded rows) is built on the fly
// from the mirrored pair (u_k, u_{P-1-k}) of the staged row, the B operands
// (E^T, F^T) sit in shared memory in fragment order (one 8-byte word per lane,
// two wavefronts per warp load), and the outputs go from the accumulators
// straight to global memory.
constexpr int GM_ROWS = 16;  // rows per warp tile

struct GdMmaLayout {
    int h, odd, hs, ks, ka, nt, rs;  // k-steps of the s and a halves, n-tiles, staged row stride
    size_t b_bytes, warp_bytes;
};

static GdMmaLayout gd_mma_layout(int P)
{
    GdMmaLayout L{};
    L.h = P / 2;
    L.odd = P & 1;
    L.hs = L.h + L.odd;
    L.ks = (L.hs + 3) / 4;
    L.ka = (L.h + 3) / 4;
    L.nt = (L.hs + 7) / 8;
    L.rs = P;                           // staged row stride: = 4 mod 16 doubles, so an A fragment
    while ((L.rs & 15) != 4) ++L.rs;    //   (8 rows x 4, and its mirror) is two conflict-free wavefronts
    L.b_bytes = (size_t)(L.ks + L.ka) * L.nt * 32 * sizeof(double);
    L.warp_bytes = (size_t)2 * GM_ROWS * L.rs * sizeof(double);
    return L;
}

template <int NT>
__global__ void gll_deriv_mma_kernel(GllDerivArgs a, GdMmaLayout L)
{
    pdl_enter();
    extern __shared__ __align__(16) unsigned char gm_smem[];
    const int P = a.P, h = L.h, hs = L.hs;
    double* BE = reinterpret_cast<double*>(gm_smem);   // [ks][NT][32]
    double* BF = BE + (size_t)L.ks * NT * 32;          // [ka][NT][32]
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
    double* stage = reinterpret_cast<double*>(gm_smem + L.b_bytes + (size_t)warp * L.warp_bytes);  // [2][16][rs]

    // B fragments: BE[k][t][l] = E[8t + l/4][4k + l%4], BF likewise with F
    for (int e = threadIdx.x; e < L.ks * NT * 32; e += blockDim.x) {
        const int l = e & 31, t = (e >> 5) % NT, k = (e >> 5) / NT;
        const int j = 8 * t + (l >> 2), kk = 4 * k + (l & 3);
        double v = 0.0;
        if (j < hs) {
            if (kk < h) v = 0.5 * (a.M[j * P + kk] + a.M[j * P + P - 1 - kk]);
            else if (kk == h && L.odd) v = a.M[j * P + h];
        }
        BE[e] = v;
    }
    for (int e = threadIdx.x; e < L.ka * NT * 32; e += blockDim.x) {
        const int l = e & 31, t = (e >> 5) % NT, k = (e >> 5) / NT;
        const int j = 8 * t + (l >> 2), kk = 4 * k + (l & 3);
        double v = 0.0;
        if (j < hs && kk < h) v = 0.5 * (a.M[j * P + kk] - a.M[j * P + P - 1 - kk]);
        BF[e] = v;
    }
    __syncthreads();

    const double* in = static_cast<const double*>(a.in);
    double* out = static_cast<double*>(a.out);
    const double sgn = a.order == 1 ? -1.0 : 1.0;
    const long long tiles = (a.nrows + GM_ROWS - 1) / GM_ROWS;
    const long long wstride = (long long)gridDim.x * (blockDim.x >> 5);
    // cp.async of tile t's rows into dst (row r at dst + r rs), all lanes busy
    auto issue = [&](long long t, double* dst) {
        const long long R0 = t * GM_ROWS;
        const int nr = (int)min((long long)GM_ROWS, a.nrows - R0);
        const long long my = lane < nr ? gd_row_offset(a, R0 + lane) : 0;
        // element e = base + lane sits at (r, k) = divmod(e, P), kept incrementally;
        // every lane runs the same trips (the shuffle needs the whole warp)
        int r = 0, k = lane;
        while (k >= P) { k -= P; ++r; }
        for (int base = 0; base < GM_ROWS * P; base += 32) {
            const long long off = __shfl_sync(0xffffffffu, my, r < 31 ? r : 31);
            if (base + lane < GM_ROWS * P && r < nr) cp_async_elem<8>(dst + r * L.rs + k, in + off + k, true);
            k += 32;
            while (k >= P) { k -= P; ++r; }
        }
        cp_async_commit();
    };
    long long t = (long long)warp * gridDim.x + blockIdx.x;  // warp-major: small jobs still reach every SM
    int buf = 0;
    if (t < tiles) issue(t, stage);
    for (; t < tiles; t += wstride, buf ^= 1) {
        const double* cur = stage + (size_t)buf * GM_ROWS * L.rs;
        const long long R0 = t * GM_ROWS;
        const int nr = (int)min((long long)GM_ROWS, a.nrows - R0);
        const long long my = lane < nr ? gd_row_offset(a, R0 + lane) : 0;
        if (t + wstride < tiles) {
            issue(t + wstride, stage + (size_t)(buf ^ 1) * GM_ROWS * L.rs);
            cp_async_wait_prev();
        } else {
            cp_async_wait_all();
        }
        __syncwarp();
#pragma unroll 1
        for (int mt = 0; mt < GM_ROWS / 8; ++mt) {
            if (8 * mt >= nr) break;
            double cs[NT][2], ca[NT][2];
#pragma unroll
            for (int n = 0; n < NT; ++n) { cs[n][0] = cs[n][1] = 0.0; ca[n][0] = ca[n][1] = 0.0; }
            const double* u = cur + (8 * mt + g) * L.rs;
#pragma unroll 2
            for (int kk = 0; kk < L.ks; ++kk) {
                const int k = 4 * kk + q;
                // A fragments of both halves from one mirrored pair
                double sv = 0.0, av = 0.0;
                if (k < h) {
                    const double x = u[k], y = u[P - 1 - k];
                    sv = x + y;
                    av = x - y;
                } else if (k == h && L.odd) {
                    sv = u[h];
                }
                const double* bs = BE + ((size_t)kk * NT) * 32 + lane;
#pragma unroll
                for (int n = 0; n < NT; ++n) dmma_8x8x4(cs[n][0], cs[n][1], sv, bs[n * 32]);
                if (kk < L.ka) {
                    const double* ba = BF + ((size_t)kk * NT) * 32 + lane;
#pragma unroll
                    for (int n = 0; n < NT; ++n) dmma_8x8x4(ca[n][0], ca[n][1], av, ba[n * 32]);
                }
            }
            // du_j = sigma + alpha, du_{P-1-j} = sgn (sigma - alpha), straight to global memory
            const int row = 8 * mt + g;
            const long long off = __shfl_sync(0xffffffffu, my, row);
            if (row < nr) {
                double* o = out + off;
#pragma unroll
                for (int n = 0; n < NT; ++n)
#pragma unroll
                    for (int e2 = 0; e2 < 2; ++e2) {
                        const int j = 8 * n + 2 * q + e2;
                        const double sg = cs[n][e2], al = ca[n][e2];
                        if (j < h) {
                            o[j] = sg + al;
                            o[P - 1 - j] = sgn * (sg - al);
                        } else if (j == h && L.odd) {
                            o[j] = sg + al;
                        }
                    }
            }
        }
        __syncwarp();  // this buffer is refilled by the copy issued in the next iteration
    }
}

// ---------------------------------------------------------------------------
// FP64 arrays whose rows lie back to back (row R at R P, the packed layout):
// tiles of GB_ROWS consecutive rows are one contiguous run of memory, moved by
// untiled bulk copies.  Thread 0 keeps up to `stages` tile loads in flight
// (mbarrier-tracked); each of the GB_WARPS warps multiplies one 8-row m-tile
// of the current tile on the FP64 tensor cores (the folded products of
// gll_deriv_mma_kernel), writes its outputs over its own input rows, and the
// finished tile goes back to global memory as one bulk store.  A tile whose
// byte count is not a multiple of 16 (odd P and an odd row count at the end)
// moves its last 8 bytes with plain loads and stores.
constexpr int GB_WARPS = 8;
constexpr int GB_ROWS = 8 * GB_WARPS;

template <int NT>
__global__ void __launch_bounds__(GB_WARPS * 32, 1) gll_deriv_bulk_kernel(GllDerivArgs a, GdMmaLayout L, int stages)
{
    pdl_enter();
    extern __shared__ __align__(128) unsigned char gb_smem[];
    const int P = a.P, h = L.h, hs = L.hs;
    double* BE = reinterpret_cast<double*>(gb_smem);   // [ks][NT][32]
    double* BF = BE + (size_t)L.ks * NT * 32;          // [ka][NT][32]
    const size_t tile_elems = (size_t)GB_ROWS * P;
    double* stage = reinterpret_cast<double*>(gb_smem + L.b_bytes);          // [stages][GB_ROWS][P]
    uint64_t* full = reinterpret_cast<uint64_t*>(stage + (size_t)stages * tile_elems);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
    const double* in = static_cast<const double*>(a.in);
    double* out = static_cast<double*>(a.out);
    const double sgn = a.order == 1 ? -1.0 : 1.0;
    const long long tiles = (a.nrows + GB_ROWS - 1) / GB_ROWS;
    const int nmine = tiles > blockIdx.x ? (int)((tiles - 1 - blockIdx.x) / gridDim.x + 1) : 0;
    auto tile_of = [&](int i) { return (long long)blockIdx.x + (long long)i * gridDim.x; };
    auto bytes_of = [&](long long t) {
        return (uint32_t)(min((long long)GB_ROWS, a.nrows - t * GB_ROWS) * P * (long long)sizeof(double));
    };
    auto issue = [&](int i) {  // thread 0: tile i of this CTA into stage i % stages
        const long long t = tile_of(i);
        const uint32_t bulk = bytes_of(t) & ~15u;
        uint64_t* bar = &full[i % stages];
        mbar_arrive_expect_tx(bar, bulk);
        bulk_load(stage + (size_t)(i % stages) * tile_elems, in + t * GB_ROWS * P, bulk, bar);
    };
    // the first loads go out before the B fragments are built
    if (threadIdx.x == 0) {
        for (int i = 0; i < stages; ++i) mbar_init(&full[i], 1);
        fence_mbar_init();
        for (int i = 0; i < min(stages, nmine); ++i) issue(i);
    }
    int issued = min(stages, nmine);
    for (int e = threadIdx.x; e < L.ks * NT * 32; e += blockDim.x) {
        const int l = e & 31, t = (e >> 5) % NT, k = (e >> 5) / NT;
        const int j = 8 * t + (l >> 2), kk = 4 * k + (l & 3);
        double v = 0.0;
        if (j < hs) {
            if (kk < h) v = 0.5 * (a.M[j * P + kk] + a.M[j * P + P - 1 - kk]);
            else if (kk == h && L.odd) v = a.M[j * P + h];
        }
        BE[e] = v;
    }
    for (int e = threadIdx.x; e < L.ka * NT * 32; e += blockDim.x) {
        const int l = e & 31, t = (e >> 5) % NT, k = (e >> 5) / NT;
        const int j = 8 * t + (l >> 2), kk = 4 * k + (l & 3);
        double v = 0.0;
        if (j < hs && kk < h) v = 0.5 * (a.M[j * P + kk] - a.M[j * P + P - 1 - kk]);
        BF[e] = v;
    }
    __syncthreads();  // B fragments and the barrier initialisation

    int failed_at = -1;
    for (int i = 0; i < nmine; ++i) {
        const long long t = tile_of(i);
        const uint32_t bytes = bytes_of(t);
        const int nr = (int)(bytes / (P * sizeof(double)));
        double* cur = stage + (size_t)(i % stages) * tile_elems;
        const bool ok = mbar_wait(&full[i % stages], (uint32_t)((i / stages) & 1));
        if (__syncthreads_or(!ok)) {
            failed_at = i;
            break;
        }
        if ((bytes & 15u) && threadIdx.x == 0) cur[(size_t)nr * P - 1] = in[t * GB_ROWS * P + (long long)nr * P - 1];
        __syncthreads();
        if (8 * warp < nr) {
            double cs[NT][2], ca[NT][2];
#pragma unroll
            for (int n = 0; n < NT; ++n) { cs[n][0] = cs[n][1] = 0.0; ca[n][0] = ca[n][1] = 0.0; }
            const int row = 8 * warp + g;
            double* u = cur + (size_t)row * P;
            const bool live = row < nr;
#pragma unroll 2
            for (int kk = 0; kk < L.ks; ++kk) {
                const int k = 4 * kk + q;
                double sv = 0.0, av = 0.0;
                if (live) {
                    if (k < h) {
                        const double x = u[k], y = u[P - 1 - k];
                        sv = x + y;
                        av = x - y;
                    } else if (k == h && L.odd) {
                        sv = u[h];
                    }
                }
                const double* bs = BE + ((size_t)kk * NT) * 32 + lane;
#pragma unroll
                for (int n = 0; n < NT; ++n) dmma_8x8x4(cs[n][0], cs[n][1], sv, bs[n * 32]);
                if (kk < L.ka) {
                    const double* ba = BF + ((size_t)kk * NT) * 32 + lane;
#pragma unroll
                    for (int n = 0; n < NT; ++n) dmma_8x8x4(ca[n][0], ca[n][1], av, ba[n * 32]);
                }
            }
            __syncwarp();  // every lane's reads of the 8 rows are done: overwrite them
            if (live) {
#pragma unroll
                for (int n = 0; n < NT; ++n)
#pragma unroll
                    for (int e2 = 0; e2 < 2; ++e2) {
                        const int j = 8 * n + 2 * q + e2;
                        const double sg = cs[n][e2], al = ca[n][e2];
                        if (j < h) {
                            u[j] = sg + al;
                            u[P - 1 - j] = sgn * (sg - al);
                        } else if (j == h && L.odd) {
                            u[j] = sg + al;
                        }
                    }
            }
        }
        fence_proxy_async_smem();  // the outputs, written through the generic proxy, go out by bulk store
        __syncthreads();
        if (threadIdx.x == 0) {
            bulk_store(out + t * GB_ROWS * P, cur, bytes & ~15u);
            tma_store_commit();
            if (bytes & 15u) out[t * GB_ROWS * P + (long long)nr * P - 1] = cur[(size_t)nr * P - 1];
            // refill the stage of tile i - 1: its store, issued one iteration
            // ago, has read its shared memory once at most this one is pending
            if (i >= 1 && issued < nmine) {
                tma_store_wait_read<1>();
                issue(issued);
                ++issued;
            }
        }
    }
    if (threadIdx.x == 0) {
        if (failed_at >= 0) {
            if (a.err) atomicExch(a.err, 8);
            // loads still in flight (tiles failed_at .. issued - 1, one per
            // stage) land before the CTA's shared memory is released
            for (int i = failed_at; i < issued; ++i) mbar_wait(&full[i % stages], (uint32_t)((i / stages) & 1));
        }
        tma_store_wait_all();
    }
}

template <int NT>
static int run_gll_deriv_bulk(const GllDerivArgs& a, cudaStream_t s)
{
    const GdMmaLayout L = gd_mma_layout(a.P);
    const size_t tile_bytes = (size_t)GB_ROWS * a.P * sizeof(double);
    // two CTAs per SM (16 warps) with two tiles in flight each where they fit,
    // else one CTA with up to five
    constexpr size_t kPerSm = 233472;  // shared memory of an SM, 1 KB of it reserved per CTA
    int per_sm = 2;
    int stages = (int)(((kPerSm / 2 - 1024) - L.b_bytes - 64) / (tile_bytes + sizeof(uint64_t)));
    if (stages < 2) {
        per_sm = 1;
        stages = (int)((kMaxSmemPerBlock - L.b_bytes - 64) / (tile_bytes + sizeof(uint64_t)));
    }
    if (stages > 5) stages = 5;
    if (stages < 2) return -1;  // not this kernel
    const size_t smem = L.b_bytes + (size_t)stages * (tile_bytes + sizeof(uint64_t));
    auto k = gll_deriv_bulk_kernel<NT>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return (int)e;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const long long tiles = (a.nrows + GB_ROWS - 1) / GB_ROWS;
    const long long grid = tiles < (long long)sms * per_sm ? tiles : (long long)sms * per_sm;
    if (grid < 1) return 0;
    return (int)launch_k(k, dim3((unsigned)grid), dim3(GB_WARPS * 32), smem, s, a, L, stages);
}

// The packed layout with 16-byte aligned arrays: the bulk-copy kernel.
static bool gll_deriv_packed(const GllDerivArgs& a)
{
    return a.x_stride == (long long)a.rows_per_x * a.P && a.elem_stride == (long long)a.nx * a.x_stride &&
           (reinterpret_cast<uintptr_t>(a.in) & 15) == 0 && (reinterpret_cast<uintptr_t>(a.out) & 15) == 0;
}

template <int NT>
static int run_gll_deriv_mma(const GllDerivArgs& a, cudaStream_t s)
{
    const GdMmaLayout L = gd_mma_layout(a.P);
    int warps = (int)((kMaxSmemPerBlock - L.b_bytes) / L.warp_bytes);
    if (warps > 16) warps = 16;
    if (warps < 1) return (int)cudaErrorInvalidValue;
    const size_t smem = L.b_bytes + (size_t)warps * L.warp_bytes;
    auto k = gll_deriv_mma_kernel<NT>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return (int)e;
    int dev = 0, sms = 148, per = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k, warps * 32, smem);
    if (per < 1) per = 1;
    const long long tiles = (a.nrows + GM_ROWS - 1) / GM_ROWS;
    long long grid = (long long)sms * per;
    if (grid > tiles) grid = tiles;
    if (grid < 1) return 0;
    return (int)launch_k(k, dim3((unsigned)grid), dim3(warps * 32), smem, s, a, L);
}

static int launch_gll_deriv_bulk(const GllDerivArgs& a, cudaStream_t s)
{
    switch ((a.P / 2 + (a.P & 1) + 7) / 8) {
        case 1: return run_gll_deriv_bulk<1>(a, s);
        case 2: return run_gll_deriv_bulk<2>(a, s);
        case 3: return run_gll_deriv_bulk<3>(a, s);
        case 4: return run_gll_deriv_bulk<4>(a, s);
        case 5: return run_gll_deriv_bulk<5>(a, s);
        case 6: return run_gll_deriv_bulk<6>(a, s);
        case 7: return run_gll_deriv_bulk<7>(a, s);
        case 8: return run_gll_deriv_bulk<8>(a, s);
        case 9: return run_gll_deriv_bulk<9>(a, s);
        default: return -1;
    }
}

static int launch_gll_deriv_mma(const GllDerivArgs& a, cudaStream_t s)
{
    if (gll_deriv_packed(a)) {
        const int e = launch_gll_deriv_bulk(a, s);
        if (e != -1) return e;
    }
    switch ((a.P / 2 + (a.P & 1) + 7) / 8) {
        case 1: return run_gll_deriv_mma<1>(a, s);
        case 2: return run_gll_deriv_mma<2>(a, s);
        case 3: return run_gll_deriv_mma<3>(a, s);
        case 4: return run_gll_deriv_mma<4>(a, s);
        case 5: return run_gll_deriv_mma<5>(a, s);
        case 6: return run_gll_deriv_mma<6>(a, s);
        case 7: return run_gll_deriv_mma<7>(a, s);
        case 8: return run_gll_deriv_mma<8>(a, s);
        case 9: return run_gll_deriv_mma<9>(a, s);
        default: return (int)cudaErrorInvalidValue;
    }
}

template <typename T>
static int run_gll_deriv(const GllDerivArgs& a, cudaStream_t s)
{
    const GdLayout L = gd_layout<T>(a.P);
    int warps = (int)((kMaxSmemPerBlock - L.ef_bytes) / L.warp_bytes);
    if (warps > 8) warps = 8;
    if (warps < 1) return (int)cudaErrorInvalidValue;
    const size_t smem = L.ef_bytes + (size_t)warps * L.warp_bytes;
    auto k = gll_deriv_kernel<T>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return (int)e;
    int dev = 0, sms = 148, per = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k, warps * 32, smem);
    if (per < 1) per = 1;
    const long long tiles = (a.nrows + 31) / 32;
    long long grid = (long long)sms * per;
    if (grid > tiles) grid = tiles;
    if (grid < 1) return 0;
    return (int)launch_k(k, dim3((unsigned)grid), dim3(warps * 32), smem, s, a, L);
}

int launch_gll_deriv(int io_double, const GllDerivArgs& a, cudaStream_t s)
{
    if (a.P < 2 || a.P > 129 || (a.order != 1 && a.order != 2)) return (int)cudaErrorInvalidValue;
    return io_double ? launch_gll_deriv_mma(a, s) : run_gll_deriv<float>(a, s);
}

}  // namespace helm
