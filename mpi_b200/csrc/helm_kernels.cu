// CUDA kernels of the Helmholtz solve (sm_100a):
//   * fft_kernel  -- batched FFT along a strided (non-contiguous) axis, real-to-
//     complex, complex-to-real or complex-to-complex, one tile of columns per
//     CTA with the whole transform length staged in shared memory, radix-8/16
//     Stockham passes in registers.  Replaces FourierTransformX / Y / XY
//     (Fourier_Quadrature.cpp:516-609, 719-926, 1097-1155).
//   * rows_kernel -- the per-wavenumber collocation solves of every spectrum
//     row (ConstructFundamentalSolutions + LUSolve, NonPeriodic2D_MPI.cpp:176-223,
//     LU_Decomposition.cpp:78-108), the element-interface tridiagonal sweep with
//     the Robin ends (NonPeriodic2D_MPI.cpp:265-295, 414-424) and the combination
//     u = phi + zl ul + zr ur (:466-470), fused, one warp per complex row.
#include "helm_device.cuh"
#include "helm_kernels.cuh"

namespace helm {

template <typename T, int L, int THREADS, int SMALL>
struct FftShape {
    using RS = RadixV<L, SMALL>;
    static constexpr int R0 = RS::r0, R1 = RS::r1, R2 = RS::r2, NP = RS::n;
    static constexpr int TPC = L / R0;          // threads per column
    static constexpr int CT = THREADS / TPC;    // columns per tile
    static constexpr size_t smem = (size_t)L * CT * sizeof(cplx_t<T>);
};

template <int R, int DIR, typename T>
__device__ __forceinline__ void dft_sub(cplx_t<T>* v)
{
    cplx_t<T> w[R];
#pragma unroll
    for (int r = 0; r < R; ++r) w[r] = v[r];
    dft_reg<R, DIR, T>(w);
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = w[r];
}

// One Stockham pass (radix R, NS = product of the earlier radices) reading
// shared memory: every thread loads, twiddles and transforms its R0/R items.
template <typename T, int L, int R, int NS, int DIR, int TPC, int CT, int R0>
__device__ __forceinline__ void pass_from_smem(const cplx_t<T>* sm, const cplx_t<T>* tw, int tc, int cl,
                                               cplx_t<T> (&v)[R0])
{
    constexpr int IPT = R0 / R;
#pragma unroll
    for (int t = 0; t < IPT; ++t) {
        const int j = tc + t * TPC;
        const int jm = j % NS;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            cplx_t<T> x = sm[(j + r * (L / R)) * CT + cl];
            if (NS > 1 && r > 0) {
                const cplx_t<T> w = tw[r * jm * (L / (NS * R))];
                x = (DIR < 0) ? cmul(x, w) : cmulc(x, w);
            }
            v[t * R + r] = x;
        }
        dft_sub<R, DIR, T>(&v[t * R]);
    }
}

// Output row of item (t, r) of a pass with radix R and NS.
template <int R, int NS, int TPC>
__device__ __forceinline__ int pass_out_row(int tc, int t, int r)
{
    const int j = tc + t * TPC;
    return (j / NS) * NS * R + (j % NS) + r * NS;
}

template <typename T, int L, int R, int NS, int TPC, int CT, int R0>
__device__ __forceinline__ void pass_to_smem(cplx_t<T>* sm, int tc, int cl, const cplx_t<T> (&v)[R0])
{
#pragma unroll
    for (int t = 0; t < R0 / R; ++t)
#pragma unroll
        for (int r = 0; r < R; ++r) sm[pass_out_row<R, NS, TPC>(tc, t, r) * CT + cl] = v[t * R + r];
}

// The real outputs of one thread of a C2R pass: columns c0 (and c1 when has1)
// at the rows of its last-pass items v[t RL + r], scaled by sc.  In an adjoint
// pass (a.adj_mode) the GLL boundary slots also go to the boundary cotangents
// (first slot of batch a.gl_batch, last slot of batch a.gr_batch: the first and
// last GLL element) and acc gathers the lambda sum; the forward solution values
// it needs are loaded for a whole group of RL rows before any store of that group.
template <bool ADJ, typename T, typename TIO, int R0, int RL, int NSL, int TPC>
__device__ __forceinline__ void c2r_store(const FftArgs& a, TIO* out, long long out_base, int b, int tc, int c0,
                                          int c1, bool has1, const cplx_t<T> (&v)[R0], T sc, double& acc)
{
    if constexpr (!ADJ) {
#pragma unroll
        for (int t = 0; t < R0 / RL; ++t)
#pragma unroll
            for (int r = 0; r < RL; ++r) {
                const long long row = pass_out_row<RL, NSL, TPC>(tc, t, r);
                TIO* o0 = out + row * a.out_row + c0;
                const TIO x0 = (TIO)(v[t * RL + r].x * sc), x1 = (TIO)(v[t * RL + r].y * sc);
                if (a.accumulate) {
                    *o0 += x0;
                    if (has1) o0[c1 - c0] += x1;
                } else {
                    *o0 = x0;
                    if (has1) o0[c1 - c0] = x1;
                }
            }
        return;
    } else {
    const int P = a.adj_P;
    const int k0 = c0 % P, j0 = c0 / P, k1 = c1 % P, j1 = c1 / P;
    const bool b0 = k0 == 0 || k0 == P - 1, b1 = k1 == 0 || k1 == P - 1;
    const bool zero0 = a.adj_mode == 1 && b0, zero1 = a.adj_mode == 1 && b1;
    double* const gbl = b == a.gl_batch ? a.gbar_l : nullptr;
    double* const gbr = b == a.gr_batch ? a.gbar_r : nullptr;
    const double* u = a.lam_u ? a.lam_u + out_base : nullptr;
#pragma unroll
    for (int t = 0; t < R0 / RL; ++t) {
        double u0[RL], u1[RL];
#pragma unroll
        for (int r = 0; r < RL; ++r) {
            const long long row = pass_out_row<RL, NSL, TPC>(tc, t, r);
            u0[r] = (u && !zero0) ? u[row * a.out_row + c0] : 0.0;
            u1[r] = (u && has1 && !zero1) ? u[row * a.out_row + c1] : 0.0;
        }
#pragma unroll
        for (int r = 0; r < RL; ++r) {
            const long long row = pass_out_row<RL, NSL, TPC>(tc, t, r);
            const double x0 = (double)(v[t * RL + r].x * sc), x1 = (double)(v[t * RL + r].y * sc);
            // (accumulate: a refinement sweep adds its correction to fbar and gbar)
            const double keep = a.accumulate ? 1.0 : 0.0;
            if (b0) {
                if (k0 == 0 && gbl) {
                    double* g = &gbl[row * a.bc_row + j0];
                    *g = keep * *g + a.adj_scale_l * x0;
                }
                if (k0 == P - 1 && gbr) {
                    double* g = &gbr[row * a.bc_row + j0];
                    *g = keep * *g + a.adj_scale_r * x0;
                }
            }
            {
                TIO* o = &out[row * a.out_row + c0];
                *o = zero0 ? (TIO)0 : (a.accumulate ? (TIO)(*o + x0) : (TIO)x0);
            }
            acc += x0 * u0[r];
            if (has1) {
                if (b1) {
                    if (k1 == 0 && gbl) {
                        double* g = &gbl[row * a.bc_row + j1];
                        *g = keep * *g + a.adj_scale_l * x1;
                    }
                    if (k1 == P - 1 && gbr) {
                        double* g = &gbr[row * a.bc_row + j1];
                        *g = keep * *g + a.adj_scale_r * x1;
                    }
                }
                TIO* o = &out[row * a.out_row + c1];
                *o = zero1 ? (TIO)0 : (a.accumulate ? (TIO)(*o + x1) : (TIO)x1);
                acc += x1 * u1[r];
            }
        }
    }
    }
}

// Adds every thread's acc into *a.lam_out (one atomic per CTA); all threads call.
__device__ __forceinline__ void c2r_lambda_sum(const FftArgs& a, double acc)
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

// Spectral derivative on the C2R load: multiply half-spectrum row k of both
// real columns by (i w K)^order, K = k below L/2 and K = k - L = -L/2 at L/2
// (FirstDerivativeFourierX / SecondDerivativeFourierX, Fourier_Quadrature.cpp:
// 1400-1407, 1630-1637).  The caller then drops the imaginary parts at k = 0
// and L/2, as the reference's real part of the inverse transform does.
template <typename T, int L>
__device__ __forceinline__ void deriv_mul(const FftArgs& a, int k, cplx_t<T>& A, cplx_t<T>& B)
{
    if (!a.deriv_order) return;
    const double K = (k < L / 2) ? (double)k : (double)(k - L);
    const double wk = a.deriv_w * K;
    if (a.deriv_order == 1) {
        const T m = (T)wk;
        A = mk(-m * A.y, m * A.x);
        B = mk(-m * B.y, m * B.x);
    } else {
        const T m = (T)(-wk * wk);
        A = mk(m * A.x, m * A.y);
        B = mk(m * B.x, m * B.y);
    }
}

// The same multiplication on the full spectrum Z = A + i B of two packed real
// columns: the multiplier is Hermitian (its value at L - k is the conjugate of
// its value at k), so Z_k (i w K)^order is the packed spectrum of the two
// derivatives.  At K = -L/2 the first derivative vanishes (the real part the
// reference keeps) and the second keeps -(w L/2)^2.
template <typename T, int L>
__device__ __forceinline__ cplx_t<T> deriv_mul_packed(int order, double w, int k, cplx_t<T> Z)
{
    const double K = (k < L / 2) ? (double)k : (double)(k - L);
    const double wk = w * K;
    if (order == 1) {
        const T m = (k == L / 2) ? (T)0 : (T)wk;
        return mk(-m * Z.y, m * Z.x);
    }
    const T m = (T)(-wk * wk);
    return mk(m * Z.x, m * Z.y);
}

// Forward (DIR2 = -1) or inverse (+1) Stockham passes of a transform whose
// first-pass inputs v[r] (rows tc + r TPC) are in registers; on return v holds
// the outputs of the last pass (rows pass_out_row).
template <typename T, int L, int DIR2, int TPC, int CT, int R0, int R1, int R2, int NP>
__device__ __forceinline__ void fft_reg_passes(cplx_t<T>* sm, const cplx_t<T>* tw, int tc, int cl, cplx_t<T> (&v)[R0])
{
    dft_reg<R0, DIR2, T>(v);
    if constexpr (NP >= 2) {
        __syncthreads();
        pass_to_smem<T, L, R0, 1, TPC, CT, R0>(sm, tc, cl, v);
        __syncthreads();
        pass_from_smem<T, L, R1, R0, DIR2, TPC, CT, R0>(sm, tw, tc, cl, v);
    }
    if constexpr (NP >= 3) {
        __syncthreads();
        pass_to_smem<T, L, R1, R0, TPC, CT, R0>(sm, tc, cl, v);
        __syncthreads();
        pass_from_smem<T, L, R2, R0 * R1, DIR2, TPC, CT, R0>(sm, tw, tc, cl, v);
    }
}

template <typename T, typename TIO, int L, int DIR, int MODE, int THREADS, int SMALL>
__global__ void __launch_bounds__(THREADS) fft_kernel(FftArgs a, long long total_cols)
{
    pdl_enter();
    if (a.zero_out && blockIdx.x == 0 && threadIdx.x == 0) *a.zero_out = 0.0;
    using C = cplx_t<T>;
    using S = FftShape<T, L, THREADS, SMALL>;
    constexpr int R0 = S::R0, R1 = S::R1, R2 = S::R2, NP = S::NP, TPC = S::TPC, CT = S::CT;
    extern __shared__ __align__(16) unsigned char fft_smem[];
    C* sm = reinterpret_cast<C*>(fft_smem);
    const C* tw = static_cast<const C*>(a.tw);

    const int tc = threadIdx.x / CT;
    const int cl = threadIdx.x - tc * CT;
    const long long g = (long long)blockIdx.x * CT + cl;
    const bool valid = g < total_cols;
    const int ccols = (MODE == FFT_C2C) ? a.ncols : (a.ncols + 1) >> 1;
    const long long gg = valid ? g : 0;
    const int b = (int)(gg / ccols);
    const int c = (int)(gg - (long long)b * ccols);
    const int c0 = 2 * c, c1 = 2 * c + 1;  // real columns of an R2C / C2R pair
    const bool has1 = c1 < a.ncols;
    const long long in_base = a.in_boff ? a.in_boff[b] : (long long)b * a.in_batch;
    const long long out_base = a.out_boff ? a.out_boff[b] : (long long)b * a.out_batch;

    C v[R0];
    // ---------------------------------------------------------- pass 0 --
    if constexpr (MODE == FFT_C2R || MODE == FFT_C2R_ADJ) {
        // Z_k = A_k + i B_k over the full length from the two half spectra
        const C* in = static_cast<const C*>(a.in) + in_base;
        for (int k = tc; k <= L / 2; k += TPC) {
            C A = mk((T)0, (T)0), B = mk((T)0, (T)0);
            if (valid) {
                A = in[(long long)k * a.in_row + c0];
                if (has1) B = in[(long long)k * a.in_row + c1];
            }
            deriv_mul<T, L>(a, k, A, B);
            if (k == 0 || k == L / 2) { A.y = 0; B.y = 0; }
            sm[k * CT + cl] = mk(A.x - B.y, A.y + B.x);
            if (k != 0 && k != L / 2) sm[(L - k) * CT + cl] = mk(A.x + B.y, B.x - A.y);
        }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < R0; ++r) v[r] = sm[(tc + r * TPC) * CT + cl];
    } else if constexpr (MODE == FFT_DERIV) {
        const TIO* in = static_cast<const TIO*>(a.in) + in_base;
#pragma unroll
        for (int r = 0; r < R0; ++r) {
            const long long row = tc + r * TPC;
            T x0 = 0, x1 = 0;
            if (valid) {
                x0 = (T)in[row * a.in_row + c0];
                if (has1) x1 = (T)in[row * a.in_row + c1];
            }
            v[r] = mk(x0, x1);
        }
    } else if constexpr (MODE == FFT_R2C) {
        const TIO* in = static_cast<const TIO*>(a.in) + in_base;
        const TIO* sub = a.in_sub ? static_cast<const TIO*>(a.in_sub) + in_base : nullptr;
        int k0 = -1, k1 = -1, j0 = 0, j1 = 0;  // GLL slot of the two real columns
        if (a.P > 0) { k0 = c0 % a.P; j0 = c0 / a.P; k1 = c1 % a.P; j1 = c1 / a.P; }
        const bool bnd0 = a.P > 0 && (k0 == 0 || k0 == a.P - 1);
        const bool bnd1 = a.P > 0 && (k1 == 0 || k1 == a.P - 1);
        const double* s0 = (k0 == 0) ? (b == a.gl_batch ? a.gl : nullptr) : (b == a.gr_batch ? a.gr : nullptr);
        const double* s1 = (k1 == 0) ? (b == a.gl_batch ? a.gl : nullptr) : (b == a.gr_batch ? a.gr : nullptr);
#pragma unroll
        for (int r = 0; r < R0; ++r) {
            const long long row = tc + r * TPC;
            T x0 = 0, x1 = 0;
            if (valid) {
                if (!bnd0) {
                    x0 = sub ? (T)((double)in[row * a.in_row + c0] - (double)sub[row * a.in_row + c0])
                             : (T)in[row * a.in_row + c0];
                } else if (a.bc_add) {
                    double v = (double)in[row * a.in_row + c0];
                    if (s0) v += (k0 == 0 ? a.bc_scale_l : a.bc_scale_r) * s0[row * a.bc_row + j0];
                    x0 = (T)v;
                } else if (s0) {
                    x0 = (T)s0[row * a.bc_row + j0];
                }
                if (has1) {
                    if (!bnd1) {
                        x1 = sub ? (T)((double)in[row * a.in_row + c1] - (double)sub[row * a.in_row + c1])
                                 : (T)in[row * a.in_row + c1];
                    } else if (a.bc_add) {
                        double v = (double)in[row * a.in_row + c1];
                        if (s1) v += (k1 == 0 ? a.bc_scale_l : a.bc_scale_r) * s1[row * a.bc_row + j1];
                        x1 = (T)v;
                    } else if (s1) {
                        x1 = (T)s1[row * a.bc_row + j1];
                    }
                }
            }
            v[r] = mk(x0, x1);
        }
    } else {
        const C* in = static_cast<const C*>(a.in) + in_base;
#pragma unroll
        for (int r = 0; r < R0; ++r) v[r] = valid ? in[(long long)(tc + r * TPC) * a.in_row + c] : mk((T)0, (T)0);
    }
    dft_reg<R0, DIR, T>(v);

    // --------------------------------------------------- later passes --
    if constexpr (NP >= 2) {
        if constexpr (MODE == FFT_C2R || MODE == FFT_C2R_ADJ) __syncthreads();  // pass 0 read shared memory
        pass_to_smem<T, L, R0, 1, TPC, CT, R0>(sm, tc, cl, v);
        __syncthreads();
        pass_from_smem<T, L, R1, R0, DIR, TPC, CT, R0>(sm, tw, tc, cl, v);
    }
    if constexpr (NP >= 3) {
        __syncthreads();
        pass_to_smem<T, L, R1, R0, TPC, CT, R0>(sm, tc, cl, v);
        __syncthreads();
        pass_from_smem<T, L, R2, R0 * R1, DIR, TPC, CT, R0>(sm, tw, tc, cl, v);
    }
    constexpr int RL = (NP == 1) ? R0 : (NP == 2 ? R1 : R2);   // radix of the last pass
    constexpr int NSL = L / RL;                                 // its NS

    // ---------------------------------------------------------- output --
    const T sc = (T)a.scale;
    if constexpr (MODE == FFT_DERIV) {
        // multiply in place, back to natural row order through shared memory,
        // then the inverse transform and the two real output columns
#pragma unroll
        for (int t = 0; t < R0 / RL; ++t)
#pragma unroll
            for (int r = 0; r < RL; ++r)
                v[t * RL + r] = deriv_mul_packed<T, L>(a.deriv_order, a.deriv_w, pass_out_row<RL, NSL, TPC>(tc, t, r),
                                                       v[t * RL + r]);
        __syncthreads();
        pass_to_smem<T, L, RL, NSL, TPC, CT, R0>(sm, tc, cl, v);
        __syncthreads();
#pragma unroll
        for (int r = 0; r < R0; ++r) v[r] = sm[(tc + r * TPC) * CT + cl];
        fft_reg_passes<T, L, 1, TPC, CT, R0, R1, R2, NP>(sm, tw, tc, cl, v);
        if (valid) {
            TIO* out = static_cast<TIO*>(a.out) + out_base;
#pragma unroll
            for (int t = 0; t < R0 / RL; ++t)
#pragma unroll
                for (int r = 0; r < RL; ++r) {
                    const long long row = pass_out_row<RL, NSL, TPC>(tc, t, r);
                    out[row * a.out_row + c0] = (TIO)(v[t * RL + r].x * sc);
                    if (has1) out[row * a.out_row + c1] = (TIO)(v[t * RL + r].y * sc);
                }
        }
    } else if constexpr (MODE == FFT_C2C) {
        if (valid) {
            C* out = static_cast<C*>(a.out) + out_base;
#pragma unroll
            for (int t = 0; t < R0 / RL; ++t)
#pragma unroll
                for (int r = 0; r < RL; ++r) {
                    const int row = pass_out_row<RL, NSL, TPC>(tc, t, r);
                    out[(long long)row * a.out_row + c] = cscale(v[t * RL + r], sc);
                }
        }
    } else if constexpr (MODE == FFT_C2R || MODE == FFT_C2R_ADJ) {
        double acc = 0.0;
        if (valid)
            c2r_store<MODE == FFT_C2R_ADJ, T, TIO, R0, RL, NSL, TPC>(a, static_cast<TIO*>(a.out) + out_base, out_base, b, tc, c0, c1, has1, v,
                                                sc, acc);
        if constexpr (MODE == FFT_C2R_ADJ)
            if (a.lam_out) c2r_lambda_sum(a, acc);
    } else {  // R2C: separate the two real columns' spectra, keep k = 0 .. L/2
        __syncthreads();
        pass_to_smem<T, L, RL, NSL, TPC, CT, R0>(sm, tc, cl, v);
        __syncthreads();
        if (valid) {
            C* out = static_cast<C*>(a.out) + out_base;
            const T h = (T)0.5 * sc;
            for (int k = tc; k <= L / 2; k += TPC) {
                const C Z = sm[k * CT + cl];
                const C Zm = sm[((L - k) & (L - 1)) * CT + cl];
                out[(long long)k * a.out_row + c0] = mk((Z.x + Zm.x) * h, (Z.y - Zm.y) * h);
                if (has1) out[(long long)k * a.out_row + c1] = mk((Z.y + Zm.y) * h, (Zm.x - Z.x) * h);
            }
        }
    }
}

// ------------------------------------------------ pipelined FFT pass --
// The same transforms as fft_kernel from a persistent grid: every CTA walks
// tiles blockIdx.x, blockIdx.x + gridDim.x, ... and copies the next tile's
// input into shared memory (cp.async, one copy per element) while it
// transforms the current one, so the loads of one tile overlap the butterflies
// and stores of the previous.  Two tile buffers per CTA; the buffer of the
// current tile doubles as the exchange buffer of its passes.


template <typename T, typename TIO, int L, int THREADS, int SMALL>
struct PipeShape {
    using S = FftShape<T, L, THREADS, SMALL>;
    // one tile buffer holds the staged input -- complex values (C2C), pairs of
    // real inputs (R2C), or the pairs A_k, B_k of rows k <= L/2 (C2R) -- and
    // then serves as the exchange buffer of the passes
    static constexpr size_t c2r = (size_t)(L + 2) * S::CT * 2 * sizeof(T);
    static constexpr size_t r2c = (size_t)L * S::CT * 2 * sizeof(TIO);
    static constexpr size_t exch = (size_t)L * S::CT * 2 * sizeof(T);
    static constexpr size_t big = c2r > r2c ? (c2r > exch ? c2r : exch) : (r2c > exch ? r2c : exch);
    static constexpr size_t buf = (big + 15) / 16 * 16;
    static constexpr size_t smem = 2 * buf;
};

// Issue the asynchronous copies of tile `tile` into `stage` (no commit).
template <typename T, typename TIO, int L, int MODE, int THREADS, int SMALL>
__device__ __forceinline__ void pipe_issue(const FftArgs& a, long long total_cols, long long tile,
                                           unsigned char* stage)
{
    using C = cplx_t<T>;
    using S = FftShape<T, L, THREADS, SMALL>;
    constexpr int R0 = S::R0, TPC = S::TPC, CT = S::CT;
    const int tc = threadIdx.x / CT;
    const int cl = threadIdx.x - tc * CT;
    const long long g = tile * CT + cl;
    const bool valid = g < total_cols;
    const int ccols = (MODE == FFT_C2C) ? a.ncols : (a.ncols + 1) >> 1;
    const long long gg = valid ? g : 0;
    const int b = (int)(gg / ccols);
    const int c = (int)(gg - (long long)b * ccols);
    const long long in_base = a.in_boff ? a.in_boff[b] : (long long)b * a.in_batch;
    if constexpr (MODE == FFT_C2C) {
        const C* in = static_cast<const C*>(a.in) + in_base;
        C* st = reinterpret_cast<C*>(stage);
#pragma unroll
        for (int r = 0; r < R0; ++r) {
            const long long row = tc + r * TPC;
            cp_async_elem<sizeof(C)>(&st[row * CT + cl], valid ? &in[row * a.in_row + c] : a.in, valid);
        }
    } else if constexpr (MODE == FFT_R2C || MODE == FFT_DERIV) {
        const TIO* in = static_cast<const TIO*>(a.in) + in_base;
        TIO* st = reinterpret_cast<TIO*>(stage);
        const int c0 = 2 * c, c1 = 2 * c + 1;
        const bool v1 = valid && c1 < a.ncols;
#pragma unroll
        for (int r = 0; r < R0; ++r) {
            const long long row = tc + r * TPC;
            cp_async_elem<sizeof(TIO)>(&st[(row * CT + cl) * 2], valid ? &in[row * a.in_row + c0] : a.in, valid);
            cp_async_elem<sizeof(TIO)>(&st[(row * CT + cl) * 2 + 1], v1 ? &in[row * a.in_row + c1] : a.in, v1);
        }
    } else {  // C2R: A_k, B_k for k = 0 .. L/2
        const C* in = static_cast<const C*>(a.in) + in_base;
        C* st = reinterpret_cast<C*>(stage);
        const int c0 = 2 * c, c1 = 2 * c + 1;
        const bool v1 = valid && c1 < a.ncols;
        for (int k = tc; k <= L / 2; k += TPC) {
            cp_async_elem<sizeof(C)>(&st[((long long)k * CT + cl) * 2], valid ? &in[(long long)k * a.in_row + c0] : a.in,
                                     valid);
            cp_async_elem<sizeof(C)>(&st[((long long)k * CT + cl) * 2 + 1],
                                     v1 ? &in[(long long)k * a.in_row + c1] : a.in, v1);
        }
    }
}

template <typename T, typename TIO, int L, int DIR, int MODE, int THREADS, int SMALL>
__global__ void __launch_bounds__(THREADS) fft_pipe_kernel(FftArgs a, long long total_cols, long long ntiles)
{
    pdl_enter();
    if (a.zero_out && blockIdx.x == 0 && threadIdx.x == 0) *a.zero_out = 0.0;
    using C = cplx_t<T>;
    using S = FftShape<T, L, THREADS, SMALL>;
    using PS = PipeShape<T, TIO, L, THREADS, SMALL>;
    constexpr int R0 = S::R0, R1 = S::R1, R2 = S::R2, NP = S::NP, TPC = S::TPC, CT = S::CT;
    extern __shared__ __align__(16) unsigned char fft_smem[];
    const C* tw = static_cast<const C*>(a.tw);
    const int tc = threadIdx.x / CT;
    const int cl = threadIdx.x - tc * CT;
    const int ccols = (MODE == FFT_C2C) ? a.ncols : (a.ncols + 1) >> 1;

    long long tile = blockIdx.x;
    int cur = 0;
    double lam_acc = 0.0;  // adjoint C2R: this thread's share of the lambda sum
    if (tile < ntiles) pipe_issue<T, TIO, L, MODE, THREADS, SMALL>(a, total_cols, tile, fft_smem);
    cp_async_commit();
    for (; tile < ntiles; tile += gridDim.x, cur ^= 1) {
        unsigned char* buf = fft_smem + (size_t)cur * PS::buf;
        const long long next = tile + gridDim.x;
        if (next < ntiles) pipe_issue<T, TIO, L, MODE, THREADS, SMALL>(a, total_cols, next, fft_smem + (size_t)(cur ^ 1) * PS::buf);
        cp_async_commit();
        cp_async_wait_prev();
        __syncthreads();

        C* sm = reinterpret_cast<C*>(buf);
        const long long g = tile * CT + cl;
        const bool valid = g < total_cols;
        const long long gg = valid ? g : 0;
        const int b = (int)(gg / ccols);
        const int c = (int)(gg - (long long)b * ccols);
        const int c0 = 2 * c, c1 = 2 * c + 1;
        const bool has1 = c1 < a.ncols;
        const long long out_base = a.out_boff ? a.out_boff[b] : (long long)b * a.out_batch;

        C v[R0];
        // ------------------------------------------------ pass 0 input --
        if constexpr (MODE == FFT_C2R || MODE == FFT_C2R_ADJ) {
            constexpr int KPT = (L / 2) / TPC + 1;  // half-spectrum rows per thread (upper bound)
            C A[KPT], B[KPT];
#pragma unroll
            for (int j = 0; j < KPT; ++j) {
                const int k = tc + j * TPC;
                if (k <= L / 2) {
                    A[j] = sm[((size_t)k * CT + cl) * 2];
                    B[j] = sm[((size_t)k * CT + cl) * 2 + 1];
                }
            }
            __syncthreads();
#pragma unroll
            for (int j = 0; j < KPT; ++j) {
                const int k = tc + j * TPC;
                if (k <= L / 2) {
                    C Aj = A[j], Bj = B[j];
                    deriv_mul<T, L>(a, k, Aj, Bj);
                    if (k == 0 || k == L / 2) { Aj.y = 0; Bj.y = 0; }
                    sm[k * CT + cl] = mk(Aj.x - Bj.y, Aj.y + Bj.x);
                    if (k != 0 && k != L / 2) sm[(L - k) * CT + cl] = mk(Aj.x + Bj.y, Bj.x - Aj.y);
                }
            }
            __syncthreads();
#pragma unroll
            for (int r = 0; r < R0; ++r) v[r] = sm[(tc + r * TPC) * CT + cl];
            __syncthreads();
        } else if constexpr (MODE == FFT_R2C || MODE == FFT_DERIV) {
            const TIO* st = reinterpret_cast<const TIO*>(buf);
            int k0 = -1, k1 = -1, j0 = 0, j1 = 0;
            if (a.P > 0) { k0 = c0 % a.P; j0 = c0 / a.P; k1 = c1 % a.P; j1 = c1 / a.P; }
            const bool bnd0 = a.P > 0 && (k0 == 0 || k0 == a.P - 1);
            const bool bnd1 = a.P > 0 && (k1 == 0 || k1 == a.P - 1);
            const double* s0 = (k0 == 0) ? (b == a.gl_batch ? a.gl : nullptr) : (b == a.gr_batch ? a.gr : nullptr);
            const double* s1 = (k1 == 0) ? (b == a.gl_batch ? a.gl : nullptr) : (b == a.gr_batch ? a.gr : nullptr);
#pragma unroll
            for (int r = 0; r < R0; ++r) {
                const long long row = tc + r * TPC;
                const TIO i0 = st[(row * CT + cl) * 2], i1 = st[(row * CT + cl) * 2 + 1];
                T x0 = (T)i0, x1 = (T)i1;
                if (bnd0) {
                    if (a.bc_add) {
                        double vv = (double)i0;
                        if (s0) vv += (k0 == 0 ? a.bc_scale_l : a.bc_scale_r) * s0[row * a.bc_row + j0];
                        x0 = (T)vv;
                    } else {
                        x0 = s0 ? (T)s0[row * a.bc_row + j0] : (T)0;
                    }
                }
                if (has1 && bnd1) {
                    if (a.bc_add) {
                        double vv = (double)i1;
                        if (s1) vv += (k1 == 0 ? a.bc_scale_l : a.bc_scale_r) * s1[row * a.bc_row + j1];
                        x1 = (T)vv;
                    } else {
                        x1 = s1 ? (T)s1[row * a.bc_row + j1] : (T)0;
                    }
                }
                if (!valid) { x0 = 0; x1 = 0; }
                v[r] = mk(x0, x1);
            }
            __syncthreads();  // the stage is the exchange buffer from here on
        } else {
#pragma unroll
            for (int r = 0; r < R0; ++r) v[r] = sm[(tc + r * TPC) * CT + cl];
            __syncthreads();
        }
        dft_reg<R0, DIR, T>(v);

        // ------------------------------------------------ later passes --
        if constexpr (NP >= 2) {
            pass_to_smem<T, L, R0, 1, TPC, CT, R0>(sm, tc, cl, v);
            __syncthreads();
            pass_from_smem<T, L, R1, R0, DIR, TPC, CT, R0>(sm, tw, tc, cl, v);
        }
        if constexpr (NP >= 3) {
            __syncthreads();
            pass_to_smem<T, L, R1, R0, TPC, CT, R0>(sm, tc, cl, v);
            __syncthreads();
            pass_from_smem<T, L, R2, R0 * R1, DIR, TPC, CT, R0>(sm, tw, tc, cl, v);
        }
        constexpr int RL = (NP == 1) ? R0 : (NP == 2 ? R1 : R2);
        constexpr int NSL = L / RL;

        // ------------------------------------------------------ output --
        const T sc = (T)a.scale;
        if constexpr (MODE == FFT_DERIV) {
            // multiplier in registers, natural row order through the tile's
            // buffer, inverse transform, the two real output columns
#pragma unroll
            for (int t = 0; t < R0 / RL; ++t)
#pragma unroll
                for (int r = 0; r < RL; ++r)
                    v[t * RL + r] = deriv_mul_packed<T, L>(a.deriv_order, a.deriv_w,
                                                           pass_out_row<RL, NSL, TPC>(tc, t, r), v[t * RL + r]);
            __syncthreads();
            pass_to_smem<T, L, RL, NSL, TPC, CT, R0>(sm, tc, cl, v);
            __syncthreads();
#pragma unroll
            for (int r = 0; r < R0; ++r) v[r] = sm[(tc + r * TPC) * CT + cl];
            fft_reg_passes<T, L, 1, TPC, CT, R0, R1, R2, NP>(sm, tw, tc, cl, v);
            if (valid) {
                TIO* out = static_cast<TIO*>(a.out) + out_base;
#pragma unroll
                for (int t = 0; t < R0 / RL; ++t)
#pragma unroll
                    for (int r = 0; r < RL; ++r) {
                        const long long row = pass_out_row<RL, NSL, TPC>(tc, t, r);
                        out[row * a.out_row + c0] = (TIO)(v[t * RL + r].x * sc);
                        if (has1) out[row * a.out_row + c1] = (TIO)(v[t * RL + r].y * sc);
                    }
            }
        } else if constexpr (MODE == FFT_C2C) {
            if (valid) {
                C* out = static_cast<C*>(a.out) + out_base;
#pragma unroll
                for (int t = 0; t < R0 / RL; ++t)
#pragma unroll
                    for (int r = 0; r < RL; ++r) {
                        const int row = pass_out_row<RL, NSL, TPC>(tc, t, r);
                        out[(long long)row * a.out_row + c] = cscale(v[t * RL + r], sc);
                    }
            }
        } else if constexpr (MODE == FFT_C2R || MODE == FFT_C2R_ADJ) {
            if (valid)
                c2r_store<MODE == FFT_C2R_ADJ, T, TIO, R0, RL, NSL, TPC>(a, static_cast<TIO*>(a.out) + out_base, out_base, b, tc, c0, c1,
                                                    has1, v, sc, lam_acc);
        } else {
            __syncthreads();
            pass_to_smem<T, L, RL, NSL, TPC, CT, R0>(sm, tc, cl, v);
            __syncthreads();
            if (valid) {
                C* out = static_cast<C*>(a.out) + out_base;
                const T h = (T)0.5 * sc;
                for (int k = tc; k <= L / 2; k += TPC) {
                    const C Z = sm[k * CT + cl];
                    const C Zm = sm[((L - k) & (L - 1)) * CT + cl];
                    out[(long long)k * a.out_row + c0] = mk((Z.x + Zm.x) * h, (Z.y - Zm.y) * h);
                    if (has1) out[(long long)k * a.out_row + c1] = mk((Z.y + Zm.y) * h, (Zm.x - Z.x) * h);
                }
            }
        }
        __syncthreads();  // this buffer is refilled two tiles later
    }
    asm volatile("cp.async.wait_all;\n" ::);
    if constexpr (MODE == FFT_C2R_ADJ)
        if (a.lam_out) c2r_lambda_sum(a, lam_acc);
}

template <typename T, typename TIO, int L, int DIR, int MODE, int THREADS, int SMALL>
static int run_fft_pipe(const FftArgs& a, long long total_cols, cudaStream_t s)
{
    using S = FftShape<T, L, THREADS, SMALL>;
    using PS = PipeShape<T, TIO, L, THREADS, SMALL>;
    auto k = fft_pipe_kernel<T, TIO, L, DIR, MODE, THREADS, SMALL>;
    if (PS::smem > kMaxSmemPerBlock) return (int)cudaErrorInvalidValue;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PS::smem);
    if (e != cudaSuccess) return (int)e;
    const long long tiles = (total_cols + S::CT - 1) / S::CT;
    if (tiles <= 0) return 0;
    int dev = 0, sms = 148, per = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k, THREADS, PS::smem);
    if (per < 1) per = 1;
    long long grid = (long long)sms * per;
    if (grid > tiles) grid = tiles;
    return (int)launch_k(k, dim3((unsigned)grid), dim3(THREADS), PS::smem, s, a, total_cols, tiles);
}

template <typename T, typename TIO, int L, int DIR, int MODE, int THREADS, int SMALL>
static int run_fft(const FftArgs& a, long long total_cols, cudaStream_t s)
{
    using S = FftShape<T, L, THREADS, SMALL>;
    auto k = fft_kernel<T, TIO, L, DIR, MODE, THREADS, SMALL>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::smem);
    if (e != cudaSuccess) return (int)e;
    const long long blocks = (total_cols + S::CT - 1) / S::CT;
    if (blocks <= 0) return 0;
    return (int)launch_k(k, dim3((unsigned)blocks), dim3(THREADS), S::smem, s, a, total_cols);
}

template <typename T, typename TIO, int L, int THREADS, int SMALL>
static int fft_dispatch_mode(int mode, int dir, const FftArgs& a, long long tc, cudaStream_t s, bool pipe)
{
    if (pipe) {
        if (mode == FFT_DERIV) return run_fft_pipe<T, TIO, L, -1, FFT_DERIV, THREADS, SMALL>(a, tc, s);
        if (mode == FFT_C2C)
            return dir < 0 ? run_fft_pipe<T, T, L, -1, FFT_C2C, THREADS, SMALL>(a, tc, s)
                           : run_fft_pipe<T, T, L, 1, FFT_C2C, THREADS, SMALL>(a, tc, s);
        if (mode == FFT_R2C) return run_fft_pipe<T, TIO, L, -1, FFT_R2C, THREADS, SMALL>(a, tc, s);
        if (mode == FFT_C2R_ADJ) {
            if constexpr (sizeof(TIO) == 8) return run_fft_pipe<T, TIO, L, 1, FFT_C2R_ADJ, THREADS, SMALL>(a, tc, s);
            return (int)cudaErrorInvalidValue;  // adjoint outputs are double
        }
        return run_fft_pipe<T, TIO, L, 1, FFT_C2R, THREADS, SMALL>(a, tc, s);
    }
    if (mode == FFT_C2C)
        return dir < 0 ? run_fft<T, T, L, -1, FFT_C2C, THREADS, SMALL>(a, tc, s)
                       : run_fft<T, T, L, 1, FFT_C2C, THREADS, SMALL>(a, tc, s);
    if (mode == FFT_R2C) return run_fft<T, TIO, L, -1, FFT_R2C, THREADS, SMALL>(a, tc, s);
    if (mode == FFT_DERIV) return run_fft<T, TIO, L, -1, FFT_DERIV, THREADS, SMALL>(a, tc, s);
    if (mode == FFT_C2R_ADJ) {
        if constexpr (sizeof(TIO) == 8) return run_fft<T, TIO, L, 1, FFT_C2R_ADJ, THREADS, SMALL>(a, tc, s);
        return (int)cudaErrorInvalidValue;
    }
    return run_fft<T, TIO, L, 1, FFT_C2R, THREADS, SMALL>(a, tc, s);
}

// Launch variants the autotuner chooses from: bit 0 -> 128-thread CTAs (half the
// columns per tile), bit 1 -> radix-8 schedule (lengths 128 and 256), bit 2 ->
// the persistent pipelined kernel, bit 3 -> 512-thread CTAs for lengths 512 and
// 1024 (twice the columns per tile: 128-byte runs of each row instead of 64 on
// the strided x pass); bits 3 and 0 together on an FP32 pass of length 1024:
// 1024-thread CTAs (16 column pairs, whole 128-byte lines of FP32 rows).
template <typename T, typename TIO, int L>
static int fft_dispatch_variant(int variant, int mode, int dir, const FftArgs& a, long long tc, cudaStream_t s)
{
    const bool small_cta = !(variant & 8) && (variant & 1) && (L / Radix<L>::r0 <= 128);
    const bool pipe = (variant & 4) != 0;
    if constexpr (L == 1024 && sizeof(T) == 4) {
        if ((variant & 9) == 9 && !pipe) return fft_dispatch_mode<T, TIO, L, 1024, 0>(mode, dir, a, tc, s, false);
    }
    if constexpr (L >= 512) {
        if (variant & 8) return fft_dispatch_mode<T, TIO, L, 512, 0>(mode, dir, a, tc, s, pipe);
    }
    if constexpr (has_small_radix<L>()) {
        if (variant & 2) {
            if (small_cta) return fft_dispatch_mode<T, TIO, L, 128, 1>(mode, dir, a, tc, s, pipe);
            return fft_dispatch_mode<T, TIO, L, 256, 1>(mode, dir, a, tc, s, pipe);
        }
    }
    if (small_cta) return fft_dispatch_mode<T, TIO, L, 128, 0>(mode, dir, a, tc, s, pipe);
    return fft_dispatch_mode<T, TIO, L, 256, 0>(mode, dir, a, tc, s, pipe);
}

template <typename T, typename TIO>
static int fft_dispatch_len(int L, int variant, int mode, int dir, const FftArgs& a, long long tc, cudaStream_t s)
{
    switch (L) {
        case 4: return fft_dispatch_variant<T, TIO, 4>(variant, mode, dir, a, tc, s);
        case 8: return fft_dispatch_variant<T, TIO, 8>(variant, mode, dir, a, tc, s);
        case 16: return fft_dispatch_variant<T, TIO, 16>(variant, mode, dir, a, tc, s);
        case 32: return fft_dispatch_variant<T, TIO, 32>(variant, mode, dir, a, tc, s);
        case 64: return fft_dispatch_variant<T, TIO, 64>(variant, mode, dir, a, tc, s);
        case 128: return fft_dispatch_variant<T, TIO, 128>(variant, mode, dir, a, tc, s);
        case 256: return fft_dispatch_variant<T, TIO, 256>(variant, mode, dir, a, tc, s);
        case 512: return fft_dispatch_variant<T, TIO, 512>(variant, mode, dir, a, tc, s);
        case 1024: return fft_dispatch_variant<T, TIO, 1024>(variant, mode, dir, a, tc, s);
        default: return (int)cudaErrorInvalidValue;
    }
}

int launch_fft(int L, int mode, int dir, int t_double, int io_bytes, const FftArgs& a, long long total_cols,
               cudaStream_t s, int variant)
{
    if (t_double) return fft_dispatch_len<double, double>(L, variant, mode, dir, a, total_cols, s);
    if (io_bytes == 8) return fft_dispatch_len<float, double>(L, variant, mode, dir, a, total_cols, s);
    return fft_dispatch_len<float, float>(L, variant, mode, dir, a, total_cols, s);
}

// ======================================================== row solves ==

constexpr int ROW_WARPS = 4;
constexpr int ROW_NSMAX = 64;  // max GLL elements per row handled by rows_kernel

__device__ __forceinline__ float shfl(float v, int src) { return __shfl_sync(0xffffffffu, v, src); }
__device__ __forceinline__ double shfl(double v, int src) { return __shfl_sync(0xffffffffu, v, src); }
template <typename T> __device__ __forceinline__ T warp_sum(T v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// x <- (P A)^-1 P x with the combined column-major L\U factor F (unit lower L),
// dinv = 1/U_ii, perm = source row of each position.  Lane l owns rows l + 32 s.
template <typename TF, int NSLOT>
__device__ __forceinline__ void lu_core(const TF* F, int ld, const TF* dinv, const int* perm, int n, TF (&xr)[NSLOT],
                                        TF (&xi)[NSLOT], TF* scr, int lane)
{
#pragma unroll
    for (int s = 0; s < NSLOT; ++s) {
        scr[lane + 32 * s] = xr[s];
        scr[32 * NSLOT + lane + 32 * s] = xi[s];
    }
    __syncwarp();
#pragma unroll
    for (int s = 0; s < NSLOT; ++s) {
        const int i = lane + 32 * s;
        const int p = (i < n) ? perm[i] : i;
        xr[s] = scr[p];
        xi[s] = scr[32 * NSLOT + p];
    }
    __syncwarp();
    // forward substitution with the unit lower factor
#pragma unroll
    for (int ks = 0; ks < NSLOT; ++ks) {
        for (int kl = 0; kl < 32; ++kl) {
            const int k = ks * 32 + kl;
            if (k >= n - 1) break;
            const TF yr = shfl(xr[ks], kl), yi = shfl(xi[ks], kl);
            const TF* col = F + (size_t)k * ld;
#pragma unroll
            for (int s = ks; s < NSLOT; ++s) {
                if (s > ks || lane > kl) {
                    const TF f = col[lane + 32 * s];
                    xr[s] -= f * yr;
                    xi[s] -= f * yi;
                }
            }
        }
    }
    // back substitution with U, column by column
#pragma unroll
    for (int ks = NSLOT - 1; ks >= 0; --ks) {
        for (int kl = 31; kl >= 0; --kl) {
            const int k = ks * 32 + kl;
            if (k >= n) continue;
            const TF di = dinv[k];
            const TF yr = shfl(xr[ks], kl) * di, yi = shfl(xi[ks], kl) * di;
            if (lane == kl) { xr[ks] = yr; xi[ks] = yi; }
            const TF* col = F + (size_t)k * ld;
#pragma unroll
            for (int s = 0; s <= ks; ++s) {
                if (s < ks || lane < kl) {
                    const TF f = col[lane + 32 * s];
                    xr[s] -= f * yr;
                    xi[s] -= f * yi;
                }
            }
        }
    }
}

// x <- V diag(1/(lam - sigma)) V^-1 x (fast diagonalisation of the interior
// operator); vinvT / vT column-major with leading dimension ld.
template <typename TF, int NSLOT>
__device__ __forceinline__ void fdm_core(const TF* vinvT, const TF* vT, int ld, const TF* rdiag, int n,
                                         TF (&xr)[NSLOT], TF (&xi)[NSLOT], cplx_t<TF>* scr, int lane)
{
#pragma unroll
    for (int s = 0; s < NSLOT; ++s) scr[lane + 32 * s] = mk(xr[s], xi[s]);
    __syncwarp();
    TF wr[NSLOT], wi[NSLOT];
#pragma unroll
    for (int s = 0; s < NSLOT; ++s) { wr[s] = 0; wi[s] = 0; }
    for (int k = 0; k < n; ++k) {
        const cplx_t<TF> f = scr[k];
        const TF* col = vinvT + (size_t)k * ld;
#pragma unroll
        for (int s = 0; s < NSLOT; ++s) {
            const TF v = col[lane + 32 * s];
            wr[s] += v * f.x;
            wi[s] += v * f.y;
        }
    }
#pragma unroll
    for (int s = 0; s < NSLOT; ++s) {
        const TF d = rdiag[lane + 32 * s];
        wr[s] *= d;
        wi[s] *= d;
    }
    __syncwarp();
#pragma unroll
    for (int s = 0; s < NSLOT; ++s) scr[lane + 32 * s] = mk(wr[s], wi[s]);
    __syncwarp();
#pragma unroll
    for (int s = 0; s < NSLOT; ++s) { xr[s] = 0; xi[s] = 0; }
    for (int k = 0; k < n; ++k) {
        const cplx_t<TF> w = scr[k];
        const TF* col = vT + (size_t)k * ld;
#pragma unroll
        for (int s = 0; s < NSLOT; ++s) {
            const TF v = col[lane + 32 * s];
            xr[s] += v * w.x;
            xi[s] += v * w.y;
        }
    }
    __syncwarp();
}

// Shared-memory layout of rows_kernel.
struct RowSmem {
    size_t mat, diag, perm, scr, d2, ns, total;
};
__host__ __device__ inline size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }
template <typename TS, typename TF, int METHOD, bool REFINE>
__host__ __device__ inline RowSmem row_smem_layout(int n, int ld)
{
    RowSmem L{};
    size_t o = 0;
    L.mat = o;
    o += (size_t)(METHOD == 1 ? 1 : 2) * n * ld * sizeof(TF);
    o = align_up(o, 16);
    L.diag = o;                                   // LU: 1/U_ii ; FDM: 1/(lam - sigma) per warp
    o += (size_t)(METHOD == 1 ? 1 : ROW_WARPS) * ld * sizeof(TF);
    o = align_up(o, 16);
    L.perm = o;
    o += (size_t)ld * sizeof(int);
    o = align_up(o, 16);
    L.scr = o;  // per warp: 2 * ld values of the widest type, complex-interleaved
    o += (size_t)ROW_WARPS * ld * 2 * (sizeof(TS) > sizeof(TF) ? sizeof(TS) : sizeof(TF));
    o = align_up(o, 16);
    L.ns = o;   // per warp: Ns sweep scalars (rhs re/im, b, c, zl re/im)
    o += (size_t)ROW_WARPS * (ROW_NSMAX + 1) * 6 * sizeof(TS);
    o = align_up(o, 16);
    L.d2 = o;
    if (REFINE) o += (size_t)n * ld * sizeof(double);
    L.total = align_up(o, 16);
    return L;
}

template <typename TS, typename TF, int NSLOT, int METHOD, bool REFINE, bool ADJ = false>
__global__ void __launch_bounds__(ROW_WARPS * 32) rows_kernel(RowArgs a)
{
    pdl_enter();
    using CS = cplx_t<TS>;
    using CF = cplx_t<TF>;
    extern __shared__ __align__(16) unsigned char row_smem[];
    const int n = a.n, P = a.P, ld = a.ldf, Ns = a.Ns;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const RowSmem Lay = row_smem_layout<TS, TF, METHOD, REFINE>(n, ld);
    TF* sMat = reinterpret_cast<TF*>(row_smem + Lay.mat);
    TF* sDiag = reinterpret_cast<TF*>(row_smem + Lay.diag);
    int* sPerm = reinterpret_cast<int*>(row_smem + Lay.perm);
    unsigned char* scrRaw = row_smem + Lay.scr + (size_t)warp * ld * 2 * (sizeof(TS) > sizeof(TF) ? sizeof(TS) : sizeof(TF));
    TS* sNs = reinterpret_cast<TS*>(row_smem + Lay.ns) + (size_t)warp * (ROW_NSMAX + 1) * 6;
    double* sD2 = reinterpret_cast<double*>(row_smem + Lay.d2);

    // shared operator data: the FDM transforms once per CTA; refinement D2
    if (METHOD == 2) {
        const TF* vi = static_cast<const TF*>(a.vinvT);
        const TF* vv = static_cast<const TF*>(a.vT);
        for (int e = threadIdx.x; e < n * ld; e += blockDim.x) { sMat[e] = vi[e]; sMat[(size_t)n * ld + e] = vv[e]; }
    }
    if (REFINE)
        for (int e = threadIdx.x; e < n * ld; e += blockDim.x) sD2[e] = a.d2t[e];
    __syncthreads();

    const bool hom_active = a.hom != nullptr;
    CS* spec = static_cast<CS*>(a.spec);

    // one CTA per group (LU: its factor is staged once); FDM: grid-stride over groups
    for (int grp = blockIdx.x; grp < a.ngroups; grp += gridDim.x) {
        if (METHOD == 1) {
            __syncthreads();
            const TF* fsrc = static_cast<const TF*>(a.fac) + (size_t)grp * a.fac_stride;
            const TF* dsrc = static_cast<const TF*>(a.dinv) + (size_t)grp * ld;
            const uint8_t* psrc = a.perm + (size_t)grp * ld;
            for (int e = threadIdx.x; e < n * ld; e += blockDim.x) sMat[e] = fsrc[e];
            for (int e = threadIdx.x; e < ld; e += blockDim.x) { sDiag[e] = dsrc[e]; sPerm[e] = psrc[e]; }
            __syncthreads();
        }
        const double sig = a.sigma[grp];
        TF* rdiag = sDiag + (size_t)warp * ld;  // FDM: this warp's 1/(lam - sigma)
        if (METHOD == 2) {
            for (int j = lane; j < ld; j += 32) rdiag[j] = (j < n) ? (TF)(1.0 / (a.lam[j] - sig)) : (TF)0;
            __syncwarp();
        }
        const double* ul = hom_active ? a.hom + (size_t)grp * 2 * P : nullptr;
        const double* ur = hom_active ? ul + P : nullptr;
        double d0ul = 0, d0ur = 0, dNul = 0, dNur = 0;
        if (hom_active) {
            d0ul = a.homs[grp * 4 + 0]; d0ur = a.homs[grp * 4 + 1];
            dNul = a.homs[grp * 4 + 2]; dNur = a.homs[grp * 4 + 3];
        }
        // the interior collocation solve of one element (transposed in an
        // adjoint run), with the FP64-residual sweeps of a refined plan
        auto solve_interior = [&](const TS (&fr)[NSLOT], const TS (&fi)[NSLOT], TS (&xr)[NSLOT], TS (&xi)[NSLOT]) {
            TF yr[NSLOT], yi[NSLOT];
#pragma unroll
            for (int s = 0; s < NSLOT; ++s) { yr[s] = (TF)fr[s]; yi[s] = (TF)fi[s]; }
            if (METHOD == 1) lu_core<TF, NSLOT>(sMat, ld, sDiag, sPerm, n, yr, yi, reinterpret_cast<TF*>(scrRaw), lane);
            else fdm_core<TF, NSLOT>(sMat, sMat + (size_t)n * ld, ld, rdiag, n, yr, yi, reinterpret_cast<CF*>(scrRaw), lane);
#pragma unroll
            for (int s = 0; s < NSLOT; ++s) { xr[s] = (TS)yr[s]; xi[s] = (TS)yi[s]; }
            if (REFINE) {
                // FP64 residual r = f - (D2int x - sigma x), then a corrected FP32 solve
                CS* scr = reinterpret_cast<CS*>(scrRaw);
                for (int sw = 0; sw < a.sweeps; ++sw) {
                    __syncwarp();
#pragma unroll
                    for (int s = 0; s < NSLOT; ++s) scr[lane + 32 * s] = mk(xr[s], xi[s]);
                    __syncwarp();
                    TS rr_[NSLOT], ri_[NSLOT];
#pragma unroll
                    for (int s = 0; s < NSLOT; ++s) {
                        rr_[s] = fr[s] + (TS)sig * xr[s];
                        ri_[s] = fi[s] + (TS)sig * xi[s];
                    }
                    for (int k = 0; k < n; ++k) {
                        const CS xk = scr[k];
                        const double* col = sD2 + (size_t)k * ld;
#pragma unroll
                        for (int s = 0; s < NSLOT; ++s) {
                            const double d = col[lane + 32 * s];
                            rr_[s] -= d * xk.x;
                            ri_[s] -= d * xk.y;
                        }
                    }
                    __syncwarp();
#pragma unroll
                    for (int s = 0; s < NSLOT; ++s) { yr[s] = (TF)rr_[s]; yi[s] = (TF)ri_[s]; }
                    if (METHOD == 1) lu_core<TF, NSLOT>(sMat, ld, sDiag, sPerm, n, yr, yi, reinterpret_cast<TF*>(scrRaw), lane);
                    else fdm_core<TF, NSLOT>(sMat, sMat + (size_t)n * ld, ld, rdiag, n, yr, yi, reinterpret_cast<CF*>(scrRaw), lane);
#pragma unroll
                    for (int s = 0; s < NSLOT; ++s) { xr[s] += (TS)yr[s]; xi[s] += (TS)yi[s]; }
                }
            }
        };
        const int r0 = a.grp_start[grp], r1 = a.grp_start[grp + 1];
        for (int rr = r0 + warp; rr < r1; rr += ROW_WARPS) {
            const long long rowoff = (long long)a.grp_rows[rr] * P;
            if (ADJ && Ns > 1) {
                // Transposed map of several elements.  Forward: per row the
                // interface values z_0 .. z_Ns solve T z = h with h_0 = gl +
                // al D0.phi_0, h_j = D0.phi_j - DN.phi_{j-1}, h_Ns = gr - ar
                // DN.phi_{Ns-1}, and element j is u = phi_j + z_j ul + z_{j+1} ur
                // (phi_j = A^-1 f_j).  Transposed: zbar_j gathers ubar at the
                // nodes equal to z_j and ubar . ul / ur of the adjacent
                // elements, w = T^-T zbar (the forward LU factors of T, used
                // transposed), then phibar_j = ubar_j + (d0bar_j D0 + dNbar_j
                // DN) on the interior, fbar_j = A^-T phibar_j, glbar = w_0,
                // grbar = w_Ns (left in the boundary slots for the last pass).
                const double* ul = a.fhom + (size_t)grp * 2 * P;
                const double* ur = ul + P;
                const double D0ul = a.fhoms[grp * 4 + 0], D0ur = a.fhoms[grp * 4 + 1];
                const double DNul = a.fhoms[grp * 4 + 2], DNur = a.fhoms[grp * 4 + 3];
                if (lane == 0)
                    for (int j = 0; j <= Ns; ++j) { sNs[j * 6 + 0] = 0; sNs[j * 6 + 1] = 0; }
                __syncwarp();
                for (int jj = 0; jj < Ns; ++jj) {
                    const CS* row = spec + (long long)jj * a.elem_stride + rowoff;
                    TS slr = 0, sli = 0, srr = 0, sri = 0;
#pragma unroll
                    for (int s = 0; s < NSLOT; ++s) {
                        const int i = lane + 32 * s;
                        if (i < n) {
                            const CS v = row[1 + i];
                            const TS l = (TS)ul[1 + i], r = (TS)ur[1 + i];
                            slr += l * v.x; sli += l * v.y;
                            srr += r * v.x; sri += r * v.y;
                        }
                    }
                    slr = warp_sum(slr); sli = warp_sum(sli);
                    srr = warp_sum(srr); sri = warp_sum(sri);
                    if (lane == 0) {
                        const CS b0 = row[0], bN = row[P - 1];
                        sNs[jj * 6 + 0] += b0.x + slr; sNs[jj * 6 + 1] += b0.y + sli;
                        sNs[(jj + 1) * 6 + 0] += bN.x + srr; sNs[(jj + 1) * 6 + 1] += bN.y + sri;
                    }
                    __syncwarp();
                }
                if (lane == 0) {
                    // T = L U without pivoting, as the forward sweep eliminates:
                    // U diagonal b_j, super c_j; L sub q_j = T[j][j-1] / b_{j-1}.
                    // U^T y = zbar (forward), then L^T w = y (backward).
                    TS bp = 0, cp = 0, yr_ = 0, yi_ = 0;
                    for (int j = 0; j <= Ns; ++j) {
                        TS bj, cj;
                        if (j == 0) {
                            bj = (TS)(a.bl - a.al * D0ul);
                            cj = (TS)(-a.al * D0ur);
                        } else if (j < Ns) {
                            bj = (TS)(DNur - D0ul) - ((TS)DNul / bp) * cp;
                            cj = (TS)(-D0ur);
                        } else {
                            bj = (TS)(a.ar * DNur + a.br) - ((TS)(a.ar * DNul) / bp) * cp;
                            cj = 0;
                        }
                        yr_ = (sNs[j * 6 + 0] - cp * yr_) / bj;
                        yi_ = (sNs[j * 6 + 1] - cp * yi_) / bj;
                        sNs[j * 6 + 2] = yr_; sNs[j * 6 + 3] = yi_; sNs[j * 6 + 4] = bj;
                        bp = bj; cp = cj;
                    }
                    TS wr = sNs[Ns * 6 + 2], wi = sNs[Ns * 6 + 3];
                    for (int j = Ns - 1; j >= 0; --j) {
                        const TS q = (j + 1 < Ns ? (TS)DNul : (TS)(a.ar * DNul)) / sNs[j * 6 + 4];
                        wr = sNs[j * 6 + 2] - q * wr;
                        wi = sNs[j * 6 + 3] - q * wi;
                        sNs[j * 6 + 2] = wr; sNs[j * 6 + 3] = wi;
                    }
                }
                __syncwarp();
                for (int jj = 0; jj < Ns; ++jj) {
                    CS* row = spec + (long long)jj * a.elem_stride + rowoff;
                    const TS w0r = sNs[jj * 6 + 2], w0i = sNs[jj * 6 + 3];
                    const TS w1r = sNs[(jj + 1) * 6 + 2], w1i = sNs[(jj + 1) * 6 + 3];
                    const TS s0 = jj == 0 ? (TS)a.al : (TS)1;           // d0bar = s0 w_jj
                    const TS s1 = jj == Ns - 1 ? (TS)-a.ar : (TS)-1;    // dNbar = s1 w_{jj+1}
                    TS fr[NSLOT], fi[NSLOT], xr[NSLOT], xi[NSLOT];
#pragma unroll
                    for (int s = 0; s < NSLOT; ++s) {
                        const int i = lane + 32 * s;
                        fr[s] = 0; fi[s] = 0;
                        if (i < n) {
                            const CS v = row[1 + i];
                            const TS c0 = (TS)a.fd0[1 + i], cN = (TS)a.fdN[1 + i];
                            fr[s] = v.x + s0 * w0r * c0 + s1 * w1r * cN;
                            fi[s] = v.y + s0 * w0i * c0 + s1 * w1i * cN;
                        }
                    }
                    solve_interior(fr, fi, xr, xi);
#pragma unroll
                    for (int s = 0; s < NSLOT; ++s) {
                        const int i = lane + 32 * s;
                        if (i < n) row[1 + i] = mk(xr[s], xi[s]);
                    }
                    if (lane == 0) {
                        row[0] = jj == 0 ? mk(w0r, w0i) : mk((TS)0, (TS)0);
                        row[P - 1] = jj == Ns - 1 ? mk(w1r, w1i) : mk((TS)0, (TS)0);
                    }
                }
                __syncwarp();
                continue;
            }
            TS pr = 0, pi = 0;                        // running d/dy of the previous element (Ns > 1)
            TS rhs_r = 0, rhs_i = 0, bprev = 0, cprev = 0;
            TS d0r = 0, d0i = 0, dNr = 0, dNi = 0;
            TS xr[NSLOT], xi[NSLOT];
            for (int jj = 0; jj < Ns; ++jj) {
                CS* row = spec + (long long)jj * a.elem_stride + rowoff;
                TS fr[NSLOT], fi[NSLOT];
#pragma unroll
                for (int s = 0; s < NSLOT; ++s) {
                    const int i = lane + 32 * s;
                    CS v = mk((TS)0, (TS)0);
                    if (i < n) v = row[1 + i];
                    fr[s] = v.x;
                    fi[s] = v.y;
                }
                // ---- collocation solve of the interior nodes ----
                solve_interior(fr, fi, xr, xi);
                if (ADJ) {
                    // transposed collocation system: boundary unknowns from the 2x2
                    // system, interior = psi + v0 pl + vN pr (one element)
                    TS a0r = 0, a0i = 0, aNr = 0, aNi = 0;
#pragma unroll
                    for (int s = 0; s < NSLOT; ++s) {
                        const int i = lane + 32 * s;
                        if (i < n) {
                            const TS c0 = (TS)a.d0[1 + i], cN = (TS)a.dN[1 + i];
                            a0r += c0 * xr[s]; a0i += c0 * xi[s];
                            aNr += cN * xr[s]; aNi += cN * xi[s];
                        }
                    }
                    a0r = warp_sum(a0r); a0i = warp_sum(a0i);
                    aNr = warp_sum(aNr); aNi = warp_sum(aNi);
                    const CS w0 = row[0], wN = row[P - 1];
                    const double* m = a.homs + grp * 4;
                    const TS m00 = (TS)m[0], m01 = (TS)m[1], m10 = (TS)m[2], m11 = (TS)m[3];
                    const TS q0r = w0.x - a0r, q0i = w0.y - a0i, qNr = wN.x - aNr, qNi = wN.y - aNi;
                    TS v0r, v0i, vNr, vNi;
                    if (a.periodic) {
                        // periodic: mu = (q0 + qN) / b with the forward b = (D0 - DN).(ul + ur)
                        const TS bb = (TS)((m[0] + m[1]) - (m[2] + m[3]));
                        v0r = (q0r + qNr) / bb; v0i = (q0i + qNi) / bb;
                        vNr = v0r; vNi = v0i;
                    } else {
                        const TS det = m00 * m11 - m01 * m10;
                        v0r = (m11 * q0r - m01 * qNr) / det; v0i = (m11 * q0i - m01 * qNi) / det;
                        vNr = (m00 * qNr - m10 * q0r) / det; vNi = (m00 * qNi - m10 * q0i) / det;
                    }
                    const double* pl = a.hom + (size_t)grp * 2 * P;
                    const double* pr_ = pl + P;
#pragma unroll
                    for (int s = 0; s < NSLOT; ++s) {
                        const int i = lane + 32 * s;
                        if (i < n) {
                            const TS l = (TS)pl[1 + i], r = (TS)pr_[1 + i];
                            row[1 + i] = mk(xr[s] + v0r * l + vNr * r, xi[s] + v0i * l + vNi * r);
                        }
                    }
                    if (lane == 0) { row[0] = mk(v0r, v0i); row[P - 1] = mk(vNr, vNi); }
                    continue;
                }
                if (!hom_active) {
#pragma unroll
                    for (int s = 0; s < NSLOT; ++s) {
                        const int i = lane + 32 * s;
                        if (i < n) row[1 + i] = mk(xr[s], xi[s]);
                    }
                    if (lane == 0) { row[0] = mk((TS)0, (TS)0); row[P - 1] = mk((TS)0, (TS)0); }
                    continue;
                }
                // ---- d/dy of the particular solution at both ends ----
                TS a0r = 0, a0i = 0, aNr = 0, aNi = 0;
#pragma unroll
                for (int s = 0; s < NSLOT; ++s) {
                    const int i = lane + 32 * s;
                    if (i < n) {
                        const TS c0 = (TS)a.d0[1 + i], cN = (TS)a.dN[1 + i];
                        a0r += c0 * xr[s]; a0i += c0 * xi[s];
                        aNr += cN * xr[s]; aNi += cN * xi[s];
                    }
                }
                d0r = warp_sum(a0r); d0i = warp_sum(a0i);
                dNr = warp_sum(aNr); dNi = warp_sum(aNi);
                if (a.periodic) {
                    // the cyclic sweep needs every element's end slopes first
                    if (Ns > 1) {
                        if (lane == 0) {
                            sNs[jj * 6 + 0] = d0r; sNs[jj * 6 + 1] = d0i;
                            sNs[jj * 6 + 2] = dNr; sNs[jj * 6 + 3] = dNi;
                        }
#pragma unroll
                        for (int s = 0; s < NSLOT; ++s) {
                            const int i = lane + 32 * s;
                            if (i < n) row[1 + i] = mk(xr[s], xi[s]);
                        }
                    }
                    continue;
                }
                // ---- forward sweep of the interface system ----
                TS bj, cj;
                if (jj == 0) {
                    bj = (TS)(-a.al * d0ul + a.bl);
                    cj = (TS)(-a.al * d0ur);
                    const CS gl = row[0];
                    rhs_r = gl.x + (TS)a.al * d0r;
                    rhs_i = gl.y + (TS)a.al * d0i;
                } else {
                    const TS q = (TS)dNul / bprev;
                    bj = (TS)dNur - (TS)d0ul - cprev * q;
                    cj = (TS)(-d0ur);
                    rhs_r = d0r - pr - rhs_r * q;
                    rhs_i = d0i - pi - rhs_i * q;
                }
                bprev = bj; cprev = cj; pr = dNr; pi = dNi;
                if (Ns > 1) {
                    if (lane == 0) {
                        sNs[jj * 6 + 0] = rhs_r; sNs[jj * 6 + 1] = rhs_i;
                        sNs[jj * 6 + 2] = bj;    sNs[jj * 6 + 3] = cj;
                    }
#pragma unroll
                    for (int s = 0; s < NSLOT; ++s) {  // park phi of this element in place
                        const int i = lane + 32 * s;
                        if (i < n) row[1 + i] = mk(xr[s], xi[s]);
                    }
                }
            }
            if (ADJ || !hom_active) continue;
            if (a.periodic) {
                if (Ns == 1) {
                    // u(0) = u(L) = zeta, slopes equal (Periodic2D_MPI.cpp:262-266, 524-531)
                    const TS bb = (TS)((d0ul + d0ur) - (dNul + dNur));
                    const TS zr_ = (dNr - d0r) / bb, zi_ = (dNi - d0i) / bb;
                    CS* row = spec + rowoff;
#pragma unroll
                    for (int s = 0; s < NSLOT; ++s) {
                        const int i = lane + 32 * s;
                        if (i < n) {
                            const TS l = (TS)ul[1 + i], r = (TS)ur[1 + i];
                            row[1 + i] = mk(xr[s] + zr_ * l + zr_ * r, xi[s] + zi_ * l + zi_ * r);
                        }
                    }
                    if (lane == 0) { row[0] = mk(zr_, zi_); row[P - 1] = mk(zr_, zi_); }
                    continue;
                }
                // cyclic interface sweep with the rank-one correction (Periodic2D_MPI.cpp:
                // forward 268-293, backward 533-565): slot jj of sNs holds rhs0 (then
                // zeta_l) in [0, 1], b in [2], c in [3], rhs1 (then eta_l) in [4]
                __syncwarp();
                if (lane == 0) {
                    const TS D0ul = (TS)d0ul, D0ur = (TS)d0ur, DNul = (TS)dNul, DNur = (TS)dNur;
                    TS pNr = sNs[(Ns - 1) * 6 + 2], pNi = sNs[(Ns - 1) * 6 + 3];  // DN.phi of the element before
                    TS bp = 0, cp = 0, q0r = 0, q0i = 0, q1 = 0;
                    for (int jj = 0; jj < Ns; ++jj) {
                        const TS e0r = sNs[jj * 6 + 0], e0i = sNs[jj * 6 + 1];
                        const TS eNr = sNs[jj * 6 + 2], eNi = sNs[jj * 6 + 3];
                        TS bj, cj;
                        if (jj == 0) {
                            bj = DNur - DNul - D0ul;
                            cj = -D0ur;
                            q0r = e0r - pNr; q0i = e0i - pNi;
                            q1 = DNul;
                        } else {
                            q0r = e0r - pNr - (q0r / bp) * DNul;
                            q0i = e0i - pNi - (q0i / bp) * DNul;
                            if (jj < Ns - 1) {
                                bj = DNur - D0ul - (cp / bp) * DNul;
                                cj = -D0ur;
                                q1 = -(q1 / bp) * DNul;
                            } else {
                                bj = DNur - D0ul + D0ur - (cp / bp) * DNul;
                                cj = 0;
                                q1 = -D0ur - (q1 / bp) * DNul;
                            }
                        }
                        sNs[jj * 6 + 0] = q0r; sNs[jj * 6 + 1] = q0i;
                        sNs[jj * 6 + 2] = bj;  sNs[jj * 6 + 3] = cj;
                        sNs[jj * 6 + 4] = q1;
                        bp = bj; cp = cj; pNr = eNr; pNi = eNi;
                    }
                    // back sweep: zeta_r(jj) = zeta_l(jj + 1), eta likewise
                    TS zlr = q0r / bp, zli = q0i / bp, el = q1 / bp;
                    sNs[(Ns - 1) * 6 + 0] = zlr; sNs[(Ns - 1) * 6 + 1] = zli; sNs[(Ns - 1) * 6 + 4] = el;
                    const TS zlastr = zlr, zlasti = zli, elast = el;
                    for (int jj = Ns - 2; jj >= 0; --jj) {
                        const TS bj = sNs[jj * 6 + 2], cj = sNs[jj * 6 + 3];
                        zlr = (sNs[jj * 6 + 0] - cj * zlr) / bj;
                        zli = (sNs[jj * 6 + 1] - cj * zli) / bj;
                        el = (sNs[jj * 6 + 4] - cj * el) / bj;
                        sNs[jj * 6 + 0] = zlr; sNs[jj * 6 + 1] = zli; sNs[jj * 6 + 4] = el;
                    }
                    // alpha = -(zeta_l + zeta_r) / (1 + eta_l + eta_r) of the last element,
                    // whose right values are the first element's left ones
                    const TS den = (TS)1 + elast + el;
                    const TS alr = -(zlastr + zlr) / den, ali = -(zlasti + zli) / den;
                    for (int jj = 0; jj < Ns; ++jj) {
                        const TS e = sNs[jj * 6 + 4];
                        sNs[jj * 6 + 0] += alr * e;
                        sNs[jj * 6 + 1] += ali * e;
                    }
                }
                __syncwarp();
                for (int jj = 0; jj < Ns; ++jj) {
                    CS* row = spec + (long long)jj * a.elem_stride + rowoff;
                    const int jn = (jj + 1 == Ns) ? 0 : jj + 1;
                    const TS zl_r = sNs[jj * 6 + 0], zl_i = sNs[jj * 6 + 1];
                    const TS zrr = sNs[jn * 6 + 0], zri = sNs[jn * 6 + 1];
#pragma unroll
                    for (int s = 0; s < NSLOT; ++s) {
                        const int i = lane + 32 * s;
                        if (i < n) {
                            const CS x = row[1 + i];
                            const TS l = (TS)ul[1 + i], r = (TS)ur[1 + i];
                            row[1 + i] = mk(x.x + zl_r * l + zrr * r, x.y + zl_i * l + zri * r);
                        }
                    }
                    if (lane == 0) { row[0] = mk(zl_r, zl_i); row[P - 1] = mk(zrr, zri); }
                }
                __syncwarp();
                continue;
            }
            // ---- right end, back sweep, combination ----
            CS* lastrow = spec + (long long)(Ns - 1) * a.elem_stride + rowoff;
            const CS gr = lastrow[P - 1];
            const TS lb = (TS)(a.ar * dNul);
            const TS bR = (TS)(a.ar * dNur + a.br) - (cprev / bprev) * lb;
            const TS rRr = gr.x - (TS)a.ar * dNr - (rhs_r / bprev) * lb;
            const TS rRi = gr.y - (TS)a.ar * dNi - (rhs_i / bprev) * lb;
            TS zr_r = rRr / bR, zr_i = rRi / bR;
            if (Ns == 1) {
                const TS zl_r = (rhs_r - cprev * zr_r) / bprev, zl_i = (rhs_i - cprev * zr_i) / bprev;
                CS* row = spec + rowoff;
#pragma unroll
                for (int s = 0; s < NSLOT; ++s) {
                    const int i = lane + 32 * s;
                    if (i < n) {
                        const TS l = (TS)ul[1 + i], r = (TS)ur[1 + i];
                        row[1 + i] = mk(xr[s] + zl_r * l + zr_r * r, xi[s] + zl_i * l + zr_i * r);
                    }
                }
                if (lane == 0) { row[0] = mk(zl_r, zl_i); row[P - 1] = mk(zr_r, zr_i); }
            } else {
                __syncwarp();
                if (lane == 0) {
                    for (int jj = Ns - 1; jj >= 0; --jj) {
                        const TS rr_ = sNs[jj * 6 + 0], ri_ = sNs[jj * 6 + 1], bj = sNs[jj * 6 + 2], cj = sNs[jj * 6 + 3];
                        const TS zl_r = (rr_ - cj * zr_r) / bj, zl_i = (ri_ - cj * zr_i) / bj;
                        sNs[jj * 6 + 4] = zl_r; sNs[jj * 6 + 5] = zl_i;
                        sNs[(jj + 1) * 6 + 0] = zr_r; sNs[(jj + 1) * 6 + 1] = zr_i;  // zr of element jj
                        zr_r = zl_r; zr_i = zl_i;
                    }
                }
                __syncwarp();
                for (int jj = 0; jj < Ns; ++jj) {
                    CS* row = spec + (long long)jj * a.elem_stride + rowoff;
                    const TS zl_r = sNs[jj * 6 + 4], zl_i = sNs[jj * 6 + 5];
                    const TS zrr = sNs[(jj + 1) * 6 + 0], zri = sNs[(jj + 1) * 6 + 1];
#pragma unroll
                    for (int s = 0; s < NSLOT; ++s) {
                        const int i = lane + 32 * s;
                        if (i < n) {
                            const CS x = row[1 + i];
                            const TS l = (TS)ul[1 + i], r = (TS)ur[1 + i];
                            row[1 + i] = mk(x.x + zl_r * l + zrr * r, x.y + zl_i * l + zri * r);
                        }
                    }
                    if (lane == 0) { row[0] = mk(zl_r, zl_i); row[P - 1] = mk(zrr, zri); }
                }
                __syncwarp();
            }
        }
    }
}

template <typename TS, typename TF, int NSLOT, int METHOD, bool REFINE, bool ADJ = false>
static int run_rows(const RowArgs& a, cudaStream_t s)
{
    auto k = rows_kernel<TS, TF, NSLOT, METHOD, REFINE, ADJ>;
    const RowSmem L = row_smem_layout<TS, TF, METHOD, REFINE>(a.n, a.ldf);
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.total);
    if (e != cudaSuccess) return (int)e;
    int grid = a.ngroups;
    if (METHOD == 2) {
        int dev = 0, sms = 148, per = 1;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k, ROW_WARPS * 32, L.total);
        if (per < 1) per = 1;
        grid = a.ngroups < sms * per ? a.ngroups : sms * per;
    }
    if (grid <= 0) return 0;
    return (int)launch_k(k, dim3(grid), dim3(ROW_WARPS * 32), L.total, s, a);
}

template <int NSLOT>
static int rows_dispatch_prec(int method, int prec, const RowArgs& a, cudaStream_t s)
{
    if (a.adjoint) {  // transposed solve: FDM only; several elements not periodic
        if (method != 2 || (a.Ns > 1 && (a.periodic || !a.fhom))) return (int)cudaErrorInvalidValue;
        if (prec == 0) return run_rows<double, double, NSLOT, 2, false, true>(a, s);
        if (prec == 1) return run_rows<float, float, NSLOT, 2, false, true>(a, s);
        return run_rows<double, float, NSLOT, 2, true, true>(a, s);
    }
    if (method == 1) {
        if (prec == 0) return run_rows<double, double, NSLOT, 1, false>(a, s);
        if (prec == 1) return run_rows<float, float, NSLOT, 1, false>(a, s);
        return run_rows<double, float, NSLOT, 1, true>(a, s);
    }
    if (prec == 0) return run_rows<double, double, NSLOT, 2, false>(a, s);
    if (prec == 1) return run_rows<float, float, NSLOT, 2, false>(a, s);
    return run_rows<double, float, NSLOT, 2, true>(a, s);
}

// Finite-difference variant (HypreFDM stencil, HelmholtzSolvers/HypreFDM/src/
// Helmholtz3D_MPI.cpp:387-403, periodic x and y turned into the modified
// wavenumbers mx, my): one Thomas solve along z per complex spectrum row, one
// thread per row.  The forward sweep writes the modified right-hand side in
// place and the elimination coefficients to `cprime`; the backward sweep reads
// both.  Consecutive threads take consecutive rows, so every step's loads fall
// on lines the previous step brought into L1.
template <typename T>
__global__ void __launch_bounds__(128) thomas_kernel(ThomasArgs a)
{
    pdl_enter();
    using C = cplx_t<T>;
    const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= a.nrows) return;
    const int Nz = a.Nz;
    const int kx = (int)(r / a.Ny), ky = (int)(r - (long long)kx * a.Ny);
    const double d = -2.0 * a.cz1 - a.lambda - a.mx[kx] - a.my[ky];
    C* x = static_cast<C*>(a.spec) + r * Nz;
    T* cp = static_cast<T*>(a.cprime) + r * Nz;
    const T cz = (T)a.cz1;
    // matrix entries of row k: sub a_k, diagonal b_k, super c_k (transposed: the
    // sub-diagonal of row k is the super-diagonal of row k-1 and vice versa)
    auto diag = [&](int k) -> T {
        double b = d;
        if (k == 0) b += a.d_first;
        if (k == Nz - 1) b += a.d_last;
        return (T)b;
    };
    auto sub = [&](int k) -> T {  // k >= 1
        if (!a.transpose) return (k == Nz - 1) ? (T)a.s_last : cz;
        return (k - 1 == 0) ? (T)a.s_first : cz;
    };
    auto sup = [&](int k) -> T {  // k <= Nz-2
        if (!a.transpose) return (k == 0) ? (T)a.s_first : cz;
        return (k + 1 == Nz - 1) ? (T)a.s_last : cz;
    };
    T cprev = 0;
    C dprev = mk((T)0, (T)0);
    for (int k = 0; k < Nz; ++k) {
        const T ak = (k > 0) ? sub(k) : (T)0;
        const T m = (T)1 / (diag(k) - ak * cprev);
        const T ck = (k < Nz - 1) ? sup(k) * m : (T)0;
        const C f = x[k];
        const C dk = mk((f.x - ak * dprev.x) * m, (f.y - ak * dprev.y) * m);
        x[k] = dk;
        cp[k] = ck;
        cprev = ck;
        dprev = dk;
    }
    C xn = dprev;
    for (int k = Nz - 2; k >= 0; --k) {
        const C dk = x[k];
        const T ck = cp[k];
        xn = mk(dk.x - ck * xn.x, dk.y - ck * xn.y);
        x[k] = xn;
    }
}

// The same tridiagonal solves, one warp per spectrum row (Nz <= 32 M).  Lane p
// owns rows z = p M .. p M + M - 1 (rows beyond Nz are identity rows).  The row
// is read once and written once, both coalesced through a per-warp shared
// buffer; no elimination coefficients go to memory:
//   1. each lane eliminates its interior rows (a Thomas solve of size M - 2
//      with three right-hand sides), leaving two equations that couple its
//      first and last unknowns to the neighbouring lanes' last and first ones;
//   2. the 64 reduced equations (a tridiagonal system in the order first_0,
//      last_0, first_1, ...) are solved by parallel cyclic reduction over warp
//      shuffles, six steps;
//   3. each lane recovers its interior unknowns from its first and last.
// The matrix is diagonally dominant (|diag| >= 2 cz1 + lambda + mx + my), so
// neither elimination pivots.
template <typename T>
struct TriEq {
    T a, b, c;
    cplx_t<T> d;
};

// Shuffles of a whole equation within segments of w lanes.
template <typename T>
__device__ __forceinline__ TriEq<T> tri_shfl_up(const TriEq<T>& e, int k, int w = 32)
{
    TriEq<T> o;
    o.a = __shfl_up_sync(0xffffffffu, e.a, k, w);
    o.b = __shfl_up_sync(0xffffffffu, e.b, k, w);
    o.c = __shfl_up_sync(0xffffffffu, e.c, k, w);
    o.d.x = __shfl_up_sync(0xffffffffu, e.d.x, k, w);
    o.d.y = __shfl_up_sync(0xffffffffu, e.d.y, k, w);
    return o;
}
template <typename T>
__device__ __forceinline__ TriEq<T> tri_shfl_down(const TriEq<T>& e, int k, int w = 32)
{
    TriEq<T> o;
    o.a = __shfl_down_sync(0xffffffffu, e.a, k, w);
    o.b = __shfl_down_sync(0xffffffffu, e.b, k, w);
    o.c = __shfl_down_sync(0xffffffffu, e.c, k, w);
    o.d.x = __shfl_down_sync(0xffffffffu, e.d.x, k, w);
    o.d.y = __shfl_down_sync(0xffffffffu, e.d.y, k, w);
    return o;
}
// One cyclic-reduction update of equation e with its neighbours lo (index - s)
// and hi (index + s), whose b fields hold the reciprocal of their diagonal.
template <typename T>
__device__ __forceinline__ TriEq<T> tri_reduce(const TriEq<T>& e, const TriEq<T>& lo, const TriEq<T>& hi)
{
    const T k1 = e.a * lo.b, k2 = e.c * hi.b;
    TriEq<T> o;
    o.a = -lo.a * k1;
    o.c = -hi.c * k2;
    o.b = e.b - lo.c * k1 - hi.a * k2;
    o.d = mk(e.d.x - lo.d.x * k1 - hi.d.x * k2, e.d.y - lo.d.y * k1 - hi.d.y * k2);
    return o;
}

constexpr int TRI_WARPS = 4;

// Copies row r of the spectrum into the lane-chunked buffer sb of LPR chunks
// of M (asynchronous, coalesced: step j moves elements 32 j .. 32 j + 31);
// elements >= Nz, and every element of a row past the end (live = false), read 0.
template <typename T, int M, int LPR>
__device__ __forceinline__ void tri_issue_row(const ThomasArgs& a, long long r, bool live, cplx_t<T>* sb, int lane)
{
    using C = cplx_t<T>;
    const C* x = static_cast<const C*>(a.spec) + (live ? r : 0) * a.Nz;
#pragma unroll
    for (int j = 0; j < (LPR * M + 31) / 32; ++j) {
        const int e = j * 32 + lane;
        const bool ok = live && e < a.Nz;
        cp_async_elem<sizeof(C)>(&sb[(e / M) * (M + 1) + e % M], ok ? (const void*)&x[e] : a.spec, ok);
    }
}

// LPR = 16: each half-warp solves its own row (two rows per warp, 16 chunks of
// M per row, cyclic reduction over 16-lane segments: one step and half the
// shuffles fewer per row than LPR = 32).
template <typename T, int M, int LPR = 32>
__global__ void __launch_bounds__(TRI_WARPS * 32, (M <= 8 ? 4 : (sizeof(T) == 8 ? 2 : 3))) thomas_warp_kernel(ThomasArgs a)
{
    pdl_enter();
    using C = cplx_t<T>;
    constexpr int RPW = 32 / LPR;            // rows per warp
    constexpr int RB = LPR * (M + 1);        // one row's buffer
    extern __shared__ __align__(16) unsigned char tri_smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int li = lane % LPR, hrow = lane / LPR;  // lane within its row, row within the warp
    C* bufs = reinterpret_cast<C*>(tri_smem) + (size_t)warp * 2 * RPW * RB;
    const int Nz = a.Nz;
    const T cz = (T)a.cz1;
    const TriEq<T> ident{(T)0, (T)1, (T)0, mk((T)0, (T)0)};
    const long long stride = (long long)gridDim.x * TRI_WARPS * RPW;
    long long r0 = ((long long)blockIdx.x * TRI_WARPS + warp) * RPW;  // first row of the warp
    int cur = 0;
    if (r0 < a.nrows)
        for (int hh = 0; hh < RPW; ++hh) tri_issue_row<T, M, LPR>(a, r0 + hh, r0 + hh < a.nrows, bufs + hh * RB, lane);
    cp_async_commit();
    for (; r0 < a.nrows; r0 += stride, cur ^= 1) {
        C* sbw = bufs + (size_t)cur * RPW * RB;
        if (r0 + stride < a.nrows)
            for (int hh = 0; hh < RPW; ++hh)
                tri_issue_row<T, M, LPR>(a, r0 + stride + hh, r0 + stride + hh < a.nrows,
                                         bufs + (size_t)(cur ^ 1) * RPW * RB + hh * RB, lane);
        cp_async_commit();
        cp_async_wait_prev();
        __syncwarp();
        C* sb = sbw + hrow * RB;  // this lane's row
        const long long r = min(r0 + hrow, a.nrows - 1);  // rows past the end solve zeros, unstored
        const int kx = (int)(r / a.Ny), ky = (int)(r - (long long)kx * a.Ny);
        const double dg = -2.0 * a.cz1 - a.lambda - a.mx[kx] - a.my[ky];
        // the lane's chunk is read from the staging buffer where it is used
        // (no register copy: registers for the elimination's arrays)
        const C* dv = sb + li * (M + 1);
        // row k: sub (k >= 1), diagonal, super (k <= Nz - 2); transposed, the sub of
        // row k is the super of row k - 1 and the super of row k the sub of row k + 1.
        // Rows k >= Nz are identity rows.
        auto sub = [&](int k) -> T {
            if (k == 0 || k >= Nz) return (T)0;
            if (!a.transpose) return (k == Nz - 1) ? (T)a.s_last : cz;
            return (k == 1) ? (T)a.s_first : cz;
        };
        auto sup = [&](int k) -> T {
            if (k >= Nz - 1) return (T)0;
            if (!a.transpose) return (k == 0) ? (T)a.s_first : cz;
            return (k + 2 == Nz) ? (T)a.s_last : cz;
        };
        auto dia = [&](int k) -> T {
            if (k >= Nz) return (T)1;
            double b = dg;
            if (k == 0) b += a.d_first;
            if (k == Nz - 1) b += a.d_last;
            return (T)b;
        };
        const int k0 = li * M;
        // ---- 1. eliminate the lane's interior rows ----
        TriEq<T> e0, e1;
        C y[M > 2 ? M - 2 : 1];
        T v[M > 2 ? M - 2 : 1], w[M > 2 ? M - 2 : 1];
        if constexpr (M == 2) {
            e0 = TriEq<T>{sub(k0), dia(k0), sup(k0), dv[0]};
            e1 = TriEq<T>{sub(k0 + 1), dia(k0 + 1), sup(k0 + 1), dv[1]};
        } else {
            constexpr int NI = M - 2;
            T cp[NI];
#pragma unroll
            for (int j = 0; j < NI; ++j) {
                const int k = k0 + j + 1;
                const T al = (j > 0) ? sub(k) : (T)0;
                const T den = (j > 0) ? dia(k) - al * cp[j - 1] : dia(k);
                const T m = (T)1 / den;
                cp[j] = (j < NI - 1) ? sup(k) * m : (T)0;
                const C yp = (j > 0) ? y[j - 1] : mk((T)0, (T)0);
                y[j] = mk((dv[j + 1].x - al * yp.x) * m, (dv[j + 1].y - al * yp.y) * m);
                v[j] = (((j == 0) ? sub(k) : (T)0) - ((j > 0) ? al * v[j - 1] : (T)0)) * m;
                w[j] = (((j == NI - 1) ? sup(k) : (T)0) - ((j > 0) ? al * w[j - 1] : (T)0)) * m;
            }
#pragma unroll
            for (int j = NI - 2; j >= 0; --j) {
                y[j] = mk(y[j].x - cp[j] * y[j + 1].x, y[j].y - cp[j] * y[j + 1].y);
                v[j] -= cp[j] * v[j + 1];
                w[j] -= cp[j] * w[j + 1];
            }
            const T c0 = sup(k0), aM = sub(k0 + M - 1);
            e0 = TriEq<T>{sub(k0), dia(k0) - c0 * v[0], -c0 * w[0],
                          mk(dv[0].x - c0 * y[0].x, dv[0].y - c0 * y[0].y)};
            e1 = TriEq<T>{-aM * v[NI - 1], dia(k0 + M - 1) - aM * w[NI - 1], sup(k0 + M - 1),
                          mk(dv[M - 1].x - aM * y[NI - 1].x, dv[M - 1].y - aM * y[NI - 1].y)};
        }
        // ---- 2. cyclic reduction of the 2 LPR reduced equations (2 li, 2 li + 1) ----
        {
            // stride 1: e0's lower neighbour is lane - 1's e1, e1's upper one lane + 1's e0
            const TriEq<T> q0{e0.a, (T)1 / e0.b, e0.c, e0.d}, q1{e1.a, (T)1 / e1.b, e1.c, e1.d};
            TriEq<T> lo = tri_shfl_up(q1, 1, LPR), hi = tri_shfl_down(q0, 1, LPR);
            if (li == 0) lo = ident;
            if (li == LPR - 1) hi = ident;
            const TriEq<T> n0 = tri_reduce(e0, lo, q1);
            const TriEq<T> n1 = tri_reduce(e1, q0, hi);
            e0 = n0;
            e1 = n1;
        }
#pragma unroll
        for (int k = 1; k < LPR; k <<= 1) {  // strides 2, 4, .., 2 LPR of the reduced index
            const TriEq<T> q0{e0.a, (T)1 / e0.b, e0.c, e0.d}, q1{e1.a, (T)1 / e1.b, e1.c, e1.d};
            TriEq<T> l0 = tri_shfl_up(q0, k, LPR), h0 = tri_shfl_down(q0, k, LPR);
            TriEq<T> l1 = tri_shfl_up(q1, k, LPR), h1 = tri_shfl_down(q1, k, LPR);
            if (li < k) { l0 = ident; l1 = ident; }
            if (li + k > LPR - 1) { h0 = ident; h1 = ident; }
            const TriEq<T> n0 = tri_reduce(e0, l0, h0);
            const TriEq<T> n1 = tri_reduce(e1, l1, h1);
            e0 = n0;
            e1 = n1;
        }
        const C xs = mk(e0.d.x / e0.b, e0.d.y / e0.b);
        const C xe = mk(e1.d.x / e1.b, e1.d.y / e1.b);
        // ---- 3. interior unknowns, coalesced store ----
        __syncwarp();
        sb[li * (M + 1)] = xs;
        sb[li * (M + 1) + M - 1] = xe;
        if constexpr (M > 2) {
#pragma unroll
            for (int j = 0; j < M - 2; ++j)
                sb[li * (M + 1) + j + 1] =
                    mk(y[j].x - xs.x * v[j] - xe.x * w[j], y[j].y - xs.y * v[j] - xe.y * w[j]);
        }
        __syncwarp();
        for (int hh = 0; hh < RPW; ++hh) {
            if (r0 + hh >= a.nrows) break;
            C* x = static_cast<C*>(a.spec) + (r0 + hh) * Nz;
            const C* sr = sbw + hh * RB;
#pragma unroll
            for (int j = 0; j < (LPR * M + 31) / 32; ++j) {
                const int e = j * 32 + lane;
                if (e < Nz) x[e] = sr[(e / M) * (M + 1) + e % M];
            }
        }
        __syncwarp();  // the buffers are refilled by the copies issued in the next iteration
    }
    asm volatile("cp.async.wait_all;\n" ::);
}

template <typename T, int M, int LPR = 32>
static int run_thomas_warp(const ThomasArgs& a, cudaStream_t s)
{
    auto k = thomas_warp_kernel<T, M, LPR>;
    const size_t smem = (size_t)TRI_WARPS * 2 * (32 / LPR) * LPR * (M + 1) * sizeof(cplx_t<T>);
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return (int)e;
    int dev = 0, sms = 148, per = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k, TRI_WARPS * 32, smem);
    if (per < 1) per = 1;
    const long long rows_per_cta = (long long)TRI_WARPS * (32 / LPR);
    long long grid = (a.nrows + rows_per_cta - 1) / rows_per_cta;
    if (grid > (long long)sms * per) grid = (long long)sms * per;
    if (grid <= 0) return 0;
    return (int)launch_k(k, dim3((unsigned)grid), dim3(TRI_WARPS * 32), smem, s, a);
}

template <typename T>
static int thomas_dispatch(const ThomasArgs& a, cudaStream_t s)
{
    if (a.half) {  // a row per half-warp
        if (a.Nz <= 32) return run_thomas_warp<T, 2, 16>(a, s);
        if (a.Nz <= 64) return run_thomas_warp<T, 4, 16>(a, s);
        if (a.Nz <= 128) return run_thomas_warp<T, 8, 16>(a, s);
        if (a.Nz <= 256) return run_thomas_warp<T, 16, 16>(a, s);
    }
    if (a.Nz <= 64) return run_thomas_warp<T, 2>(a, s);
    if (a.Nz <= 128) return run_thomas_warp<T, 4>(a, s);
    if (a.Nz <= 256) return run_thomas_warp<T, 8>(a, s);
    if (a.Nz <= 512) return run_thomas_warp<T, 16>(a, s);
    const long long blocks = (a.nrows + 127) / 128;
    if (blocks <= 0) return 0;
    return (int)launch_k(thomas_kernel<T>, dim3((unsigned)blocks), dim3(128), 0, s, a);
}

int launch_thomas(int prec, const ThomasArgs& a, cudaStream_t s)
{
    return prec == 1 ? thomas_dispatch<float>(a, s) : thomas_dispatch<double>(a, s);
}

size_t rows_smem_bytes(int method, int prec, int n, int ld)
{
    if (method == 1) {
        if (prec == 0) return row_smem_layout<double, double, 1, false>(n, ld).total;
        if (prec == 1) return row_smem_layout<float, float, 1, false>(n, ld).total;
        return row_smem_layout<double, float, 1, true>(n, ld).total;
    }
    if (prec == 0) return row_smem_layout<double, double, 2, false>(n, ld).total;
    if (prec == 1) return row_smem_layout<float, float, 2, false>(n, ld).total;
    return row_smem_layout<double, float, 2, true>(n, ld).total;
}

int launch_rows(int method, int prec, const RowArgs& a, cudaStream_t s)
{
    if (a.Ns > ROW_NSMAX) return (int)cudaErrorInvalidValue;
    switch ((a.n + 31) / 32) {
        case 1: return rows_dispatch_prec<1>(method, prec, a, s);
        case 2: return rows_dispatch_prec<2>(method, prec, a, s);
        case 3: return rows_dispatch_prec<3>(method, prec, a, s);
        case 4: return rows_dispatch_prec<4>(method, prec, a, s);
        default: return (int)cudaErrorInvalidValue;
    }
}

}  // namespace helm
