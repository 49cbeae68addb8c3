// Device building blocks of the Helmholtz kernels: complex arithmetic on
// float2/double2, in-register power-of-2 DFTs, and one Stockham pass of a
// batched strided-axis FFT held in shared memory.
#pragma once
#include <cstdlib>
#include <cuda_runtime.h>
#include <cstdint>

namespace helm {

template <typename T> struct cplx_of;
template <> struct cplx_of<float> { using type = float2; };
template <> struct cplx_of<double> { using type = double2; };
template <typename T> using cplx_t = typename cplx_of<T>::type;

__device__ __forceinline__ float2 mk(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ double2 mk(double a, double b) { return make_double2(a, b); }
__device__ __forceinline__ float2 operator+(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 operator-(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 operator+(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 operator-(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
template <typename C, typename T> __device__ __forceinline__ C cscale(C a, T s) { return mk(a.x * s, a.y * s); }
// a * b
template <typename C> __device__ __forceinline__ C cmul(C a, C b)
{
    return mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
template <typename C> __device__ __forceinline__ C cmulc(C a, C b)
{
    return mk(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}

// cos and sin of 2*pi*m/16 for m = 0..7 (exact constants of the 16th roots of unity).
__device__ __forceinline__ double root16_cos(int m)
{
    const double c[8] = {1.0, 0.92387953251128675613, 0.70710678118654752440, 0.38268343236508977173,
                         0.0, -0.38268343236508977173, -0.70710678118654752440, -0.92387953251128675613};
    return c[m];
}
__device__ __forceinline__ double root16_sin(int m)
{
    const double s[8] = {0.0, 0.38268343236508977173, 0.70710678118654752440, 0.92387953251128675613,
                         1.0, 0.92387953251128675613, 0.70710678118654752440, 0.38268343236508977173};
    return s[m];
}

// d * exp(DIR * 2 pi i m / 16) for compile-time-foldable m in [0, 8).
template <int DIR, typename T>
__device__ __forceinline__ cplx_t<T> rot16(cplx_t<T> d, int m)
{
    if (m == 0) return d;
    if (m == 4) return DIR < 0 ? mk(d.y, -d.x) : mk(-d.y, d.x);  // * (-i) or * (+i)
    const T c = (T)root16_cos(m), s = (T)(DIR * root16_sin(m));
    return mk(d.x * c - d.y * s, d.x * s + d.y * c);
}

__host__ __device__ constexpr int bitrev(int i, int R)
{
    int r = 0;
    for (int b = 1; b < R; b <<= 1) { r = (r << 1) | (i & 1); i >>= 1; }
    return r;
}

// In-register DFT of R = 2, 4, 8 or 16 points, natural order in and out:
// v_m <- sum_j v_j exp(DIR * 2 pi i j m / R).  Radix-2 decimation in frequency
// with a compile-time bit-reversal at the end.
template <int R, int DIR, typename T>
__device__ __forceinline__ void dft_reg(cplx_t<T> (&v)[R])
{
#pragma unroll
    for (int len = R; len >= 2; len >>= 1) {
        const int h = len >> 1;
#pragma unroll
        for (int s = 0; s < R; s += len) {
#pragma unroll
            for (int k = 0; k < h; ++k) {
                cplx_t<T> a = v[s + k], b = v[s + k + h];
                v[s + k] = a + b;
                v[s + k + h] = rot16<DIR, T>(a - b, k * (16 / len));
            }
        }
    }
#pragma unroll
    for (int i = 0; i < R; ++i) {
        const int j = bitrev(i, R);
        if (j > i) { cplx_t<T> t = v[i]; v[i] = v[j]; v[j] = t; }
    }
}

// Radix schedule of a length-L transform: up to three passes of radix <= 16,
// largest first.  L = 4 .. 4096.
template <int L> struct Radix;
template <> struct Radix<4> { static constexpr int n = 1, r0 = 4, r1 = 1, r2 = 1; };
template <> struct Radix<8> { static constexpr int n = 1, r0 = 8, r1 = 1, r2 = 1; };
template <> struct Radix<16> { static constexpr int n = 1, r0 = 16, r1 = 1, r2 = 1; };
template <> struct Radix<32> { static constexpr int n = 2, r0 = 8, r1 = 4, r2 = 1; };
template <> struct Radix<64> { static constexpr int n = 2, r0 = 8, r1 = 8, r2 = 1; };
template <> struct Radix<128> { static constexpr int n = 2, r0 = 16, r1 = 8, r2 = 1; };
template <> struct Radix<256> { static constexpr int n = 2, r0 = 16, r1 = 16, r2 = 1; };
template <> struct Radix<512> { static constexpr int n = 3, r0 = 8, r1 = 8, r2 = 8; };
template <> struct Radix<1024> { static constexpr int n = 3, r0 = 16, r1 = 8, r2 = 8; };

// Schedule with at most radix 8 per pass where it changes anything (half the
// register tile of the radix-16 passes, so more CTAs fit on an SM).
template <int L, int SMALL> struct RadixV : Radix<L> {};
template <> struct RadixV<128, 1> { static constexpr int n = 3, r0 = 8, r1 = 4, r2 = 4; };
template <> struct RadixV<256, 1> { static constexpr int n = 3, r0 = 8, r1 = 8, r2 = 4; };
template <int L> constexpr bool has_small_radix() { return L == 128 || L == 256; }

// ---- FFT of columns held in shared memory (slab and eigen-basis kernels) ----

template <int R, int NS, int TPC>
__device__ __forceinline__ int slab_out_row(int tc, int t, int r)
{
    const int j = tc + t * TPC;
    return (j / NS) * NS * R + (j % NS) + r * NS;
}

template <int L, int R, int NS, int TPC, int R0>
__device__ __forceinline__ void slab_to_smem(cplx_t<double>* sm, int hs, int tc, int col, const cplx_t<double> (&v)[R0])
{
#pragma unroll
    for (int t = 0; t < R0 / R; ++t)
#pragma unroll
        for (int r = 0; r < R; ++r) sm[slab_out_row<R, NS, TPC>(tc, t, r) * hs + col] = v[t * R + r];
}

template <int L, int R, int NS, int DIR, int TPC, int R0, int TWS = 1>
__device__ __forceinline__ void slab_from_smem(const cplx_t<double>* sm, int hs, const cplx_t<double>* tw, int tc,
                                               int col, cplx_t<double> (&v)[R0])
{
    using C = cplx_t<double>;
#pragma unroll
    for (int t = 0; t < R0 / R; ++t) {
        const int j = tc + t * TPC, jm = j % NS;
        C w8[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            C x = sm[(j + r * (L / R)) * hs + col];
            if (NS > 1 && r > 0) {
                const C w = tw[TWS * r * jm * (L / (NS * R))];
                x = (DIR < 0) ? cmul(x, w) : cmulc(x, w);
            }
            w8[r] = x;
        }
        dft_reg<R, DIR, double>(w8);
#pragma unroll
        for (int r = 0; r < R; ++r) v[t * R + r] = w8[r];
    }
}

// Barrier of the threads that share a slab FFT: the whole CTA (BAR = 0), or
// named barrier BAR of the first THREADS threads (warp-specialised kernels
// whose other warps do not take part).
template <int BAR, int THREADS>
__device__ __forceinline__ void slab_sync()
{
    if constexpr (BAR == 0) __syncthreads();
    else asm volatile("bar.sync %0, %1;\n" ::"n"(BAR), "n"(THREADS) : "memory");
}

// Length-512 schedule with a radix-16 first pass: 32 threads per column
// instead of 64 (twice the columns per round of a slab FFT).
struct Radix512Wide { static constexpr int n = 3, r0 = 16, r1 = 8, r2 = 4; };

// One length-L FFT (direction DIR, unscaled) of each of the ncol columns of the
// [L][hs] complex array sm in shared memory, in place; threads 0 .. THREADS-1
// call it (it synchronises them through slab_sync<BAR, THREADS>).  tw: the
// twiddle table exp(-2 pi i e / (TWS L)), read at every TWS-th entry (TWS = 2:
// the table of a transform twice as long); RS: the radix schedule.
template <int L, int DIR, int THREADS, int BAR = 0, int TWS = 1, class RS = Radix<L>>
__device__ __forceinline__ void slab_fft(cplx_t<double>* sm, int hs, int ncol, const cplx_t<double>* tw)
{
    using C = cplx_t<double>;
    constexpr int R0 = RS::r0, R1 = RS::r1, R2 = RS::r2, NP = RS::n, TPC = L / R0, CPR = THREADS / TPC;
    constexpr int RL = (NP == 1) ? R0 : (NP == 2 ? R1 : R2);
    const int tc = threadIdx.x / CPR, cl = threadIdx.x - tc * CPR;
    for (int c0 = 0; c0 < ncol; c0 += CPR) {
        const int col = c0 + cl;
        const bool on = col < ncol;
        C v[R0];
#pragma unroll
        for (int r = 0; r < R0; ++r) v[r] = on ? sm[(tc + r * TPC) * hs + col] : mk(0.0, 0.0);
        dft_reg<R0, DIR, double>(v);
        if constexpr (NP >= 2) {
            slab_sync<BAR, THREADS>();
            if (on) slab_to_smem<L, R0, 1, TPC, R0>(sm, hs, tc, col, v);
            slab_sync<BAR, THREADS>();
            if (on) slab_from_smem<L, R1, R0, DIR, TPC, R0, TWS>(sm, hs, tw, tc, col, v);
        }
        if constexpr (NP >= 3) {
            slab_sync<BAR, THREADS>();
            if (on) slab_to_smem<L, R1, R0, TPC, R0>(sm, hs, tc, col, v);
            slab_sync<BAR, THREADS>();
            if (on) slab_from_smem<L, R2, R0 * R1, DIR, TPC, R0, TWS>(sm, hs, tw, tc, col, v);
        }
        slab_sync<BAR, THREADS>();
        if (on) slab_to_smem<L, RL, L / RL, TPC, R0>(sm, hs, tc, col, v);
        slab_sync<BAR, THREADS>();
    }
}

// Asynchronous global -> shared copies of one element (cp.async; valid = false
// writes zeros and reads nothing), their commit and wait.
__device__ __forceinline__ void cp_async_bytes4(void* dst, const void* src, bool valid)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(d), "l"(src), "r"(valid ? 4 : 0));
}
__device__ __forceinline__ void cp_async_bytes8(void* dst, const void* src, bool valid)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(valid ? 8 : 0));
}
__device__ __forceinline__ void cp_async_bytes16(void* dst, const void* src, bool valid)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(valid ? 16 : 0));
}
template <int BYTES>
__device__ __forceinline__ void cp_async_elem(void* dst, const void* src, bool valid)
{
    if constexpr (BYTES == 4) cp_async_bytes4(dst, src, valid);
    else if constexpr (BYTES == 8) cp_async_bytes8(dst, src, valid);
    else cp_async_bytes16(dst, src, valid);
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait_prev() { asm volatile("cp.async.wait_group 1;\n" ::); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::); }

// One FP64 tensor-core product C += A B of m8n8k4 (g = lane / 4, q = lane % 4):
// A[g][q], B[q][g], C[g][2 q] and C[g][2 q + 1] per lane.
__device__ __forceinline__ void dmma_8x8x4(double& c0, double& c1, double a, double b)
{
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                 : "+d"(c0), "+d"(c1)
                 : "d"(a), "d"(b));
}

// 1 / sqrt 2, the weight of the orthogonal even/odd fold of the GLL interior.
constexpr double kR2 = 0.70710678118654752440;

// Value of fold `fold` at interior index k of a staged row (interior element
// j at row[1 + j]; rs: the same row of a field to subtract, or NULL):
// (u_{1+k} + u_{n-k}) / sqrt 2 (symmetric fold) or (u_{1+k} - u_{n-k}) /
// sqrt 2 (antisymmetric) for k < m, the middle element for the symmetric fold
// at k = m when n is odd, zero beyond (padding slots).
__device__ __forceinline__ double fold_value(const double* row, const double* rs, int k, int fold, int n, int m, int ms)
{
    if (k < m) {
        double lo = row[1 + k], hi = row[n - k];
        if (rs) {
            lo -= rs[1 + k];
            hi -= rs[n - k];
        }
        return fold ? kR2 * (lo - hi) : kR2 * (lo + hi);
    }
    if (!fold && k < ms) return rs ? row[1 + k] - rs[1 + k] : row[1 + k];
    return 0.0;
}

// Programmatic dependent launch.  Every kernel of a solve is launched with the
// programmatic-serialization attribute, so it may be scheduled while the
// previous kernel in the stream is still finishing; pdl_enter() then waits
// (griddepcontrol.wait) until that kernel has completed and its writes are
// visible, and lets the next kernel in the stream be scheduled in turn.  Call
// it before the first read of anything an earlier kernel wrote.
__device__ __forceinline__ void pdl_enter()
{
    asm volatile("griddepcontrol.wait;\n" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
}

// Host side: launch `k` with the programmatic-serialization attribute
// (environment HELM_PDL=0: ordinary launches).  Returns the launch status.
inline bool pdl_enabled()
{
    static const bool on = [] {
        const char* e = std::getenv("HELM_PDL");
        return !(e && e[0] == '0');
    }();
    return on;
}

template <typename... KArgs, typename... Args>
inline cudaError_t launch_k(void (*k)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args... args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = pdl_enabled() ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, k, ((KArgs)args)...);
}

}  // namespace helm
