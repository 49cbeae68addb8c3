// Fast-diagonalisation row solve for one GLL element (Ns = 1), sm_100a.
//
// The interior GLL second-derivative operator D2int (n x n) is centrosymmetric:
// D2int[i][j] = D2int[n-1-i][n-1-j].  The orthogonal even/odd fold Q
//   s_k = (f_k + f_{n-1-k}) / sqrt2,  d_k = (f_k - f_{n-1-k}) / sqrt2  (k < m = n/2),
//   s_m = f_m (odd n)
// block-diagonalises it, Q D2int Q^T = diag(Ms, Ma), and each half-size block
// is diagonalised once at plan time, Ms = Vs diag(ls) Vs^-1, Ma = Va diag(la) Va^-1.
// The solve of (D2int - sigma I) x = f for one spectrum row is then
//   fold -> Vs^-1 s, Va^-1 d -> scale by 1/(l - sigma) -> Vs (.), Va (.) -> unfold,
// n^2 multiply-adds per real right-hand side instead of 2 n^2.  The result is the
// same linear map as the reference's per-wavenumber LU (LU_Decomposition.cpp:78-108
// called from ConstructFundamentalSolutions, NonPeriodic3D_MPI.cpp:184-232),
// followed by the same Robin/interface epilogue (NonPeriodic3D_MPI.cpp:328-369,
// 520-533, 582-587).
//
// Layout of the work: a persistent grid of 8-warp CTAs, the transforms staged
// once per CTA in shared memory, and each warp solving RPW spectrum rows at a
// time (every matrix load feeds RPW rows).  Lane l owns fold index l + 32 t.
#include "helm_device.cuh"
#include "helm_fdm.cuh"

#include <cooperative_groups.h>
#include <cstdint>
#include <cstring>

namespace helm {

constexpr int FDM_WARPS = 8;

__device__ __forceinline__ float fshfl(float v, int s) { return __shfl_sync(0xffffffffu, v, s); }
template <typename T> __device__ __forceinline__ T wsum(T v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

struct FdmSmem {
    size_t mats, d2, stage, total;
};

template <typename TS, typename TF, bool REFINE, int RPW>
__host__ __device__ inline FdmSmem fdm_smem_layout(int ld)
{
    FdmSmem L{};
    size_t o = 0;
    L.mats = o;
    o += (size_t)4 * ld * ld * sizeof(TF);  // Ws^T, Vs^T, Wa^T, Va^T (column-major, padded)
    o = (o + 15) / 16 * 16;
    L.d2 = o;
    if (REFINE) o += (size_t)2 * ld * ld * sizeof(double);  // Ms^T, Ma^T
    o = (o + 15) / 16 * 16;
    L.stage = o;  // per warp, per row: 2*ld complex of the wider type
    const size_t cw = 2 * (sizeof(TS) > sizeof(TF) ? sizeof(TS) : sizeof(TF));
    o += (size_t)FDM_WARPS * RPW * 2 * ld * cw;
    L.total = (o + 15) / 16 * 16;
    return L;
}

// One folded solve: x = (Q^T) diag-solve (Q) applied to the folded input held
// in registers (ins/ind: fold index lane + 32 t), result folded in xs/xd.
template <typename TF, int NSS, int RPW>
__device__ __forceinline__ void fdm_folded_core(const TF* Ws, const TF* Vs, const TF* Wa, const TF* Va, int ld, int ms,
                                                int ma, const TF (&rs)[RPW][NSS], const TF (&ra)[RPW][NSS],
                                                TF (&sr)[RPW][NSS], TF (&si)[RPW][NSS], TF (&dr)[RPW][NSS],
                                                TF (&di)[RPW][NSS], cplx_t<TF>* stg, int lane)
{
    using C = cplx_t<TF>;
    __syncwarp();
#pragma unroll
    for (int r = 0; r < RPW; ++r)
#pragma unroll
        for (int t = 0; t < NSS; ++t) {
            stg[(size_t)r * 2 * ld + lane + 32 * t] = mk(sr[r][t], si[r][t]);
            stg[(size_t)r * 2 * ld + ld + lane + 32 * t] = mk(dr[r][t], di[r][t]);
        }
    __syncwarp();
    TF ar[RPW][NSS], ai[RPW][NSS], br[RPW][NSS], bi[RPW][NSS];
#pragma unroll
    for (int r = 0; r < RPW; ++r)
#pragma unroll
        for (int t = 0; t < NSS; ++t) { ar[r][t] = ai[r][t] = br[r][t] = bi[r][t] = (TF)0; }
    // coefficients: c_s = Vs^-1 s, c_a = Va^-1 d
    for (int k = 0; k < ms; ++k) {
        TF w[NSS], u[NSS];
        const bool anti = k < ma;
#pragma unroll
        for (int t = 0; t < NSS; ++t) {
            w[t] = Ws[(size_t)k * ld + lane + 32 * t];
            u[t] = anti ? Wa[(size_t)k * ld + lane + 32 * t] : (TF)0;
        }
#pragma unroll
        for (int r = 0; r < RPW; ++r) {
            const C s = stg[(size_t)r * 2 * ld + k];
            const C d = stg[(size_t)r * 2 * ld + ld + k];
#pragma unroll
            for (int t = 0; t < NSS; ++t) {
                ar[r][t] += w[t] * s.x;
                ai[r][t] += w[t] * s.y;
                br[r][t] += u[t] * d.x;
                bi[r][t] += u[t] * d.y;
            }
        }
    }
    __syncwarp();
#pragma unroll
    for (int r = 0; r < RPW; ++r)
#pragma unroll
        for (int t = 0; t < NSS; ++t) {
            stg[(size_t)r * 2 * ld + lane + 32 * t] = mk(ar[r][t] * rs[r][t], ai[r][t] * rs[r][t]);
            stg[(size_t)r * 2 * ld + ld + lane + 32 * t] = mk(br[r][t] * ra[r][t], bi[r][t] * ra[r][t]);
        }
    __syncwarp();
#pragma unroll
    for (int r = 0; r < RPW; ++r)
#pragma unroll
        for (int t = 0; t < NSS; ++t) { sr[r][t] = si[r][t] = dr[r][t] = di[r][t] = (TF)0; }
    // back to the folded grid: xs = Vs c_s, xd = Va c_a
    for (int j = 0; j < ms; ++j) {
        TF v[NSS], q[NSS];
        const bool anti = j < ma;
#pragma unroll
        for (int t = 0; t < NSS; ++t) {
            v[t] = Vs[(size_t)j * ld + lane + 32 * t];
            q[t] = anti ? Va[(size_t)j * ld + lane + 32 * t] : (TF)0;
        }
#pragma unroll
        for (int r = 0; r < RPW; ++r) {
            const C cs = stg[(size_t)r * 2 * ld + j];
            const C ca = stg[(size_t)r * 2 * ld + ld + j];
#pragma unroll
            for (int t = 0; t < NSS; ++t) {
                sr[r][t] += v[t] * cs.x;
                si[r][t] += v[t] * cs.y;
                dr[r][t] += q[t] * ca.x;
                di[r][t] += q[t] * ca.y;
            }
        }
    }
}

// Epilogue of a folded solve for RPW rows: boundary values (Robin / interface
// data, or the transposed 2x2 system of the adjoint), unfold, store.  x* hold
// the folded solution, lane l owning fold index l + 32 t.
template <typename TS, int NSS, int RPW, bool ADJ, typename RowOf>
__device__ __forceinline__ void fdm_store_rows_at(const FdmArgs& a, RowOf row_of, const int (&grp)[RPW],
                                                  const bool (&ok)[RPW], const TS (&xsr)[RPW][NSS],
                                                  const TS (&xsi)[RPW][NSS], const TS (&xdr)[RPW][NSS],
                                                  const TS (&xdi)[RPW][NSS], int lane)
{
    using CS = cplx_t<TS>;
    const int ld = a.ld, ms = a.ms, ma = a.ma, m = a.m, n = a.n, P = a.P;
    const TS r2 = (TS)0.70710678118654752440;
#pragma unroll
    for (int r = 0; r < RPW; ++r) {
        if (!ok[r]) continue;  // warp-uniform
        const auto row = row_of(r);
        const int g = grp[r];
        TS zlr = 0, zli = 0, zrr = 0, zri = 0;   // boundary values of the row (weights of hl / hr)
        const bool bnd = a.hvec != nullptr;
        if (bnd) {
            // folded dot products with e0 / eN (forward: D0, DN rows; adjoint: D2 boundary columns)
            TS p0r = 0, p0i = 0, pNr = 0, pNi = 0;
#pragma unroll
            for (int t = 0; t < NSS; ++t) {
                const int k = lane + 32 * t;
                if (k < ms) {
                    const TS e0s = (TS)a.e0f[k], eNs = (TS)a.eNf[k];
                    p0r += e0s * xsr[r][t]; p0i += e0s * xsi[r][t];
                    pNr += eNs * xsr[r][t]; pNi += eNs * xsi[r][t];
                }
                if (k < ma) {
                    const TS e0a = (TS)a.e0f[ld + k], eNa = (TS)a.eNf[ld + k];
                    p0r += e0a * xdr[r][t]; p0i += e0a * xdi[r][t];
                    pNr += eNa * xdr[r][t]; pNi += eNa * xdi[r][t];
                }
            }
            p0r = wsum(p0r); p0i = wsum(p0i); pNr = wsum(pNr); pNi = wsum(pNi);
            const CS wl = row.get(0), wr = row.get(P - 1);
            const double* sc = a.hscal + (size_t)g * 4;
            if (a.periodic) {
                // periodic, one element (Periodic3D_MPI.cpp:322-333, 661-662): forward
                // zeta = (DN - D0).phi / b; adjoint mu = (w0 + wN - c0.s - cN.s) / b,
                // the same b = (D0 - DN).(ul + ur)
                const TS bb = (TS)((sc[0] + sc[1]) - (sc[2] + sc[3]));
                if (!ADJ) {
                    zlr = (pNr - p0r) / bb; zli = (pNi - p0i) / bb;
                } else {
                    zlr = ((wl.x - p0r) + (wr.x - pNr)) / bb; zli = ((wl.y - p0i) + (wr.y - pNi)) / bb;
                }
                zrr = zlr; zri = zli;
            } else if (!ADJ) {
                // Robin ends, one element (NonPeriodic3D_MPI.cpp:334-336, 357-367, 528-529)
                const TS b0 = (TS)(-a.al * sc[0] + a.bl), c0 = (TS)(-a.al * sc[1]);
                const TS lb = (TS)(a.ar * sc[2]);
                const TS bR = (TS)(a.ar * sc[3] + a.br) - (c0 / b0) * lb;
                const TS rhr = wl.x + (TS)a.al * p0r, rhi = wl.y + (TS)a.al * p0i;
                const TS rRr = wr.x - (TS)a.ar * pNr - (rhr / b0) * lb;
                const TS rRi = wr.y - (TS)a.ar * pNi - (rhi / b0) * lb;
                zrr = rRr / bR; zri = rRi / bR;
                zlr = (rhr - c0 * zrr) / b0; zli = (rhi - c0 * zri) / b0;
            } else {
                const TS m00 = (TS)sc[0], m01 = (TS)sc[1], m10 = (TS)sc[2], m11 = (TS)sc[3];
                const TS det = m00 * m11 - m01 * m10;
                const TS q0r = wl.x - p0r, q0i = wl.y - p0i, qNr = wr.x - pNr, qNi = wr.y - pNi;
                zlr = (m11 * q0r - m01 * qNr) / det; zli = (m11 * q0i - m01 * qNi) / det;
                zrr = (m00 * qNr - m10 * q0r) / det; zri = (m00 * qNi - m10 * q0i) / det;
            }
        }
        // the interior correction zl hl + zr hr (skipped when hl = hr = 0: the
        // transposed system of Dirichlet ends)
        const bool hadd = bnd && !a.hzero;
        const double* hl = hadd ? a.hvec + (size_t)g * 2 * P : nullptr;
        const double* hr = hadd ? hl + P : nullptr;
#pragma unroll
        for (int t = 0; t < NSS; ++t) {
            const int k = lane + 32 * t;
            if (k < m) {
                TS lo_r = (TS)r2 * (xsr[r][t] + xdr[r][t]), lo_i = (TS)r2 * (xsi[r][t] + xdi[r][t]);
                TS hi_r = (TS)r2 * (xsr[r][t] - xdr[r][t]), hi_i = (TS)r2 * (xsi[r][t] - xdi[r][t]);
                if (hadd) {
                    const TS l0 = (TS)hl[1 + k], r0 = (TS)hr[1 + k];
                    const TS l1 = (TS)hl[n - k], r1 = (TS)hr[n - k];
                    lo_r += zlr * l0 + zrr * r0; lo_i += zli * l0 + zri * r0;
                    hi_r += zlr * l1 + zrr * r1; hi_i += zli * l1 + zri * r1;
                }
                row.put(1 + k, mk(lo_r, lo_i));
                row.put(n - k, mk(hi_r, hi_i));
            } else if (k < ms) {
                TS mr = xsr[r][t], mi = xsi[r][t];
                if (hadd) {
                    const TS l0 = (TS)hl[1 + k], r0 = (TS)hr[1 + k];
                    mr += zlr * l0 + zrr * r0; mi += zli * l0 + zri * r0;
                }
                row.put(1 + k, mk(mr, mi));
            }
        }
        if (lane == 0) {
            row.put(0, mk(zlr, zli));
            row.put(P - 1, mk(zrr, zri));
        }
    }
}

// One spectrum row in global memory (complex values at GLL slots 0 .. P-1).
template <typename CS>
struct GlobalRow {
    CS* p;
    __device__ __forceinline__ CS get(int k) const { return p[k]; }
    __device__ __forceinline__ void put(int k, CS v) const { p[k] = v; }
};

template <typename TS, int NSS, int RPW, bool ADJ>
__device__ __forceinline__ void fdm_store_rows(const FdmArgs& a, cplx_t<TS>* spec, const int (&rowid)[RPW],
                                               const int (&grp)[RPW], const bool (&ok)[RPW],
                                               const TS (&xsr)[RPW][NSS], const TS (&xsi)[RPW][NSS],
                                               const TS (&xdr)[RPW][NSS], const TS (&xdi)[RPW][NSS], int lane)
{
    fdm_store_rows_at<TS, NSS, RPW, ADJ>(
        a, [&](int r) { return GlobalRow<cplx_t<TS>>{spec + (long long)rowid[r] * a.P}; }, grp, ok, xsr, xsi, xdr, xdi,
        lane);
}

template <typename TS, typename TF, int NSS, int RPW, bool REFINE, bool ADJ>
__global__ void __launch_bounds__(FDM_WARPS * 32, 2) fdm_fast_kernel(FdmArgs a)
{
    using CS = cplx_t<TS>;
    using CF = cplx_t<TF>;
    extern __shared__ __align__(16) unsigned char fsm[];
    const int ld = a.ld, ms = a.ms, ma = a.ma, m = a.m, n = a.n, P = a.P;
    const FdmSmem Lay = fdm_smem_layout<TS, TF, REFINE, RPW>(ld);
    TF* Ws = reinterpret_cast<TF*>(fsm + Lay.mats);
    TF* Vs = Ws + (size_t)ld * ld;
    TF* Wa = Vs + (size_t)ld * ld;
    TF* Va = Wa + (size_t)ld * ld;
    double* Ms = reinterpret_cast<double*>(fsm + Lay.d2);
    double* Ma = Ms + (size_t)ld * ld;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const size_t cw = 2 * (sizeof(TS) > sizeof(TF) ? sizeof(TS) : sizeof(TF));
    unsigned char* stg_raw = fsm + Lay.stage + (size_t)warp * RPW * 2 * ld * cw;

    {
        const TF* src = static_cast<const TF*>(a.mats);
        for (int e = threadIdx.x; e < 4 * ld * ld; e += blockDim.x) Ws[e] = src[e];
        if (REFINE)
            for (int e = threadIdx.x; e < 2 * ld * ld; e += blockDim.x) Ms[e] = a.d2f[e];
    }
    pdl_enter();  // the constants above are plan data; the spectrum comes from the previous pass
    __syncthreads();

    CS* spec = static_cast<CS*>(a.spec);
    const TS r2 = (TS)0.70710678118654752440;  // fold weight, in the storage precision
    const int nrows = a.nrows;
    const long long npacks = (nrows + RPW - 1) / RPW;
    const long long gw0 = (long long)blockIdx.x * FDM_WARPS + warp;
    const long long nw = (long long)gridDim.x * FDM_WARPS;

    for (long long pk = gw0; pk < npacks; pk += nw) {
        int rowid[RPW], grp[RPW];
        bool ok[RPW];
#pragma unroll
        for (int r = 0; r < RPW; ++r) {
            const long long rr = pk * RPW + r;
            ok[r] = rr < nrows;
            rowid[r] = ok[r] ? a.rows[rr] : a.rows[0];
            grp[r] = ok[r] ? a.row_grp[rr] : a.row_grp[0];
        }
        // ---- load the interior of each row and fold it ----
        TS fsr[RPW][NSS], fsi[RPW][NSS], fdr[RPW][NSS], fdi[RPW][NSS];
        {
            CS* stg = reinterpret_cast<CS*>(stg_raw);
            __syncwarp();
#pragma unroll
            for (int r = 0; r < RPW; ++r) {
                const CS* row = spec + (long long)rowid[r] * P;
                for (int i = lane; i < n; i += 32) stg[(size_t)r * 2 * ld + i] = row[1 + i];
            }
            __syncwarp();
#pragma unroll
            for (int r = 0; r < RPW; ++r)
#pragma unroll
                for (int t = 0; t < NSS; ++t) {
                    const int k = lane + 32 * t;
                    TS a0 = 0, a1 = 0, b0 = 0, b1 = 0;
                    if (k < m) {
                        const CS lo = stg[(size_t)r * 2 * ld + k], hi = stg[(size_t)r * 2 * ld + n - 1 - k];
                        a0 = (TS)r2 * (lo.x + hi.x); a1 = (TS)r2 * (lo.y + hi.y);
                        b0 = (TS)r2 * (lo.x - hi.x); b1 = (TS)r2 * (lo.y - hi.y);
                    } else if (k < ms) {  // middle node of an odd n
                        const CS mid = stg[(size_t)r * 2 * ld + k];
                        a0 = mid.x; a1 = mid.y;
                    }
                    fsr[r][t] = a0; fsi[r][t] = a1; fdr[r][t] = b0; fdi[r][t] = b1;
                }
        }
        // ---- reciprocal shifts of each row's group ----
        TF rs[RPW][NSS], ra[RPW][NSS];
#pragma unroll
        for (int r = 0; r < RPW; ++r) {
            const TF* rc = static_cast<const TF*>(a.recip) + (size_t)grp[r] * 2 * ld;
#pragma unroll
            for (int t = 0; t < NSS; ++t) {
                rs[r][t] = rc[lane + 32 * t];
                ra[r][t] = rc[ld + lane + 32 * t];
            }
        }
        // ---- solve (+ FP64-residual refinement) in folded coordinates ----
        TF sr[RPW][NSS], si[RPW][NSS], dr[RPW][NSS], di[RPW][NSS];
#pragma unroll
        for (int r = 0; r < RPW; ++r)
#pragma unroll
            for (int t = 0; t < NSS; ++t) {
                sr[r][t] = (TF)fsr[r][t]; si[r][t] = (TF)fsi[r][t];
                dr[r][t] = (TF)fdr[r][t]; di[r][t] = (TF)fdi[r][t];
            }
        fdm_folded_core<TF, NSS, RPW>(Ws, Vs, Wa, Va, ld, ms, ma, rs, ra, sr, si, dr, di,
                                      reinterpret_cast<CF*>(stg_raw), lane);
        TS xsr[RPW][NSS], xsi[RPW][NSS], xdr[RPW][NSS], xdi[RPW][NSS];
#pragma unroll
        for (int r = 0; r < RPW; ++r)
#pragma unroll
            for (int t = 0; t < NSS; ++t) {
                xsr[r][t] = (TS)sr[r][t]; xsi[r][t] = (TS)si[r][t];
                xdr[r][t] = (TS)dr[r][t]; xdi[r][t] = (TS)di[r][t];
            }
        if (REFINE) {
            CS* stg = reinterpret_cast<CS*>(stg_raw);
            double sg[RPW];
#pragma unroll
            for (int r = 0; r < RPW; ++r) sg[r] = a.sigma[grp[r]];
            for (int sw = 0; sw < a.sweeps; ++sw) {
                // r = f - (M x - sigma x) per folded block, FP64
                __syncwarp();
#pragma unroll
                for (int r = 0; r < RPW; ++r)
#pragma unroll
                    for (int t = 0; t < NSS; ++t) {
                        stg[(size_t)r * 2 * ld + lane + 32 * t] = mk(xsr[r][t], xsi[r][t]);
                        stg[(size_t)r * 2 * ld + ld + lane + 32 * t] = mk(xdr[r][t], xdi[r][t]);
                    }
                __syncwarp();
                TS rsr[RPW][NSS], rsi[RPW][NSS], rdr[RPW][NSS], rdi[RPW][NSS];
#pragma unroll
                for (int r = 0; r < RPW; ++r)
#pragma unroll
                    for (int t = 0; t < NSS; ++t) {
                        rsr[r][t] = fsr[r][t] + (TS)sg[r] * xsr[r][t];
                        rsi[r][t] = fsi[r][t] + (TS)sg[r] * xsi[r][t];
                        rdr[r][t] = fdr[r][t] + (TS)sg[r] * xdr[r][t];
                        rdi[r][t] = fdi[r][t] + (TS)sg[r] * xdi[r][t];
                    }
                for (int k = 0; k < ms; ++k) {
                    double w[NSS], u[NSS];
                    const bool anti = k < ma;
#pragma unroll
                    for (int t = 0; t < NSS; ++t) {
                        w[t] = Ms[(size_t)k * ld + lane + 32 * t];
                        u[t] = anti ? Ma[(size_t)k * ld + lane + 32 * t] : 0.0;
                    }
#pragma unroll
                    for (int r = 0; r < RPW; ++r) {
                        const CS xs = stg[(size_t)r * 2 * ld + k];
                        const CS xd = stg[(size_t)r * 2 * ld + ld + k];
#pragma unroll
                        for (int t = 0; t < NSS; ++t) {
                            rsr[r][t] -= w[t] * xs.x;
                            rsi[r][t] -= w[t] * xs.y;
                            rdr[r][t] -= u[t] * xd.x;
                            rdi[r][t] -= u[t] * xd.y;
                        }
                    }
                }
#pragma unroll
                for (int r = 0; r < RPW; ++r)
#pragma unroll
                    for (int t = 0; t < NSS; ++t) {
                        sr[r][t] = (TF)rsr[r][t]; si[r][t] = (TF)rsi[r][t];
                        dr[r][t] = (TF)rdr[r][t]; di[r][t] = (TF)rdi[r][t];
                    }
                fdm_folded_core<TF, NSS, RPW>(Ws, Vs, Wa, Va, ld, ms, ma, rs, ra, sr, si, dr, di,
                                              reinterpret_cast<CF*>(stg_raw), lane);
#pragma unroll
                for (int r = 0; r < RPW; ++r)
#pragma unroll
                    for (int t = 0; t < NSS; ++t) {
                        xsr[r][t] += (TS)sr[r][t]; xsi[r][t] += (TS)si[r][t];
                        xdr[r][t] += (TS)dr[r][t]; xdi[r][t] += (TS)di[r][t];
                    }
            }
        }
        fdm_store_rows<TS, NSS, RPW, ADJ>(a, spec, rowid, grp, ok, xsr, xsi, xdr, xdi, lane);
    }
}

template <typename TS, typename TF, int NSS, int RPW, bool REFINE, bool ADJ>
static int run_fdm(const FdmArgs& a, cudaStream_t s)
{
    auto k = fdm_fast_kernel<TS, TF, NSS, RPW, REFINE, ADJ>;
    const FdmSmem L = fdm_smem_layout<TS, TF, REFINE, RPW>(a.ld);
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.total);
    if (e != cudaSuccess) return (int)e;
    int dev = 0, sms = 148, per = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k, FDM_WARPS * 32, L.total);
    if (per < 1) per = 1;
    const long long packs = (a.nrows + RPW - 1) / RPW;
    long long grid = (packs + FDM_WARPS - 1) / FDM_WARPS;
    if (grid > (long long)sms * per) grid = (long long)sms * per;
    if (grid <= 0) return 0;
    return (int)launch_k(k, dim3((unsigned)grid), dim3(FDM_WARPS * 32), L.total, s, a);
}

template <int NSS, int RPW>
static int fdm_dispatch(int prec, const FdmArgs& a, cudaStream_t s)
{
    if (a.adjoint) {
        if (prec == 0) return run_fdm<double, double, NSS, RPW, false, true>(a, s);
        if (prec == 1) return run_fdm<float, float, NSS, RPW, false, true>(a, s);
        return run_fdm<double, float, NSS, RPW, true, true>(a, s);
    }
    if (prec == 0) return run_fdm<double, double, NSS, RPW, false, false>(a, s);
    if (prec == 1) return run_fdm<float, float, NSS, RPW, false, false>(a, s);
    return run_fdm<double, float, NSS, RPW, true, false>(a, s);
}

// variant 0: 4 rows per warp (2 for the wide fold); variant 1: half as many.
// Rows per warp keep the accumulators in registers.
int launch_fdm_fast(int prec, const FdmArgs& a, cudaStream_t s, int variant)
{
    switch (a.ld / 32) {
        case 1: return variant ? fdm_dispatch<1, 2>(prec, a, s) : fdm_dispatch<1, 4>(prec, a, s);
        case 2: return variant ? fdm_dispatch<2, 1>(prec, a, s) : fdm_dispatch<2, 2>(prec, a, s);
        default: return (int)cudaErrorInvalidValue;
    }
}

size_t fdm_fast_smem_bytes(int prec, int ld)
{
    if (ld == 32) {
        if (prec == 0) return fdm_smem_layout<double, double, false, 4>(ld).total;
        if (prec == 1) return fdm_smem_layout<float, float, false, 4>(ld).total;
        return fdm_smem_layout<double, float, true, 4>(ld).total;
    }
    if (prec == 0) return fdm_smem_layout<double, double, false, 2>(ld).total;
    if (prec == 1) return fdm_smem_layout<float, float, false, 2>(ld).total;
    return fdm_smem_layout<double, float, true, 2>(ld).total;
}

// ======================================== FP64 tensor-core folded solve ==
//
// The same folded solve as fdm_fast_kernel for FP64 plans, with both
// transforms as products on the FP64 tensor cores (mma.sync m8n8k4 .f64):
// per warp, the folded right-hand sides of RPW = 4 NT spectrum rows form the
// B operand (ld x 8 NT: column 2 r + c is the real (c = 0) or imaginary part of
// row r), the transform is the A operand (ld x ld, i = output fold index,
// k = input fold index), and C accumulates ld x 8 NT in FP64.  The transforms
// sit in shared memory in A-fragment order, so each fragment is one
// conflict-free 8-byte load per lane.  Each row is staged in shared memory
// between the passes (raw interior, scaled coefficients, folded solution) and
// the epilogue is fdm_store_rows.
//
// Fragment layout of m8n8k4 .f64 (g = lane / 4, q = lane % 4):
//   A[g][q];  B[q][g];  C[g][2 q], C[g][2 q + 1].

// dmma_8x8x4: helm_device.cuh

template <int NSS, int NT, int WARPS>
struct MmaShape {
    static constexpr int LD = 32 * NSS;     // padded fold length
    static constexpr int MT = LD / 8;       // 8-row tiles of the output
    static constexpr int KS = LD / 4;       // 4-deep steps of the contraction
    static constexpr int RPW = 4 * NT;      // spectrum rows per warp
    static constexpr int RSD = 4 * LD + 8;  // doubles per staged row (2 LD complex + pad)
    static constexpr size_t mats = (size_t)4 * LD * LD;
    // two staging buffers per warp: the next pack's rows arrive while this one is solved
    static constexpr size_t smem = (mats + (size_t)WARPS * 2 * RPW * RSD) * sizeof(double);
};

// Asynchronous copy of the interiors of pack pk's rows into stg (row r at
// stg + r RSD, complex i at 2 i).
template <int RPW, int RSD>
__device__ __forceinline__ void mma_issue_pack(const FdmArgs& a, long long pk, double* stg, int lane)
{
    const cplx_t<double>* spec = static_cast<const cplx_t<double>*>(a.spec);
#pragma unroll
    for (int r = 0; r < RPW; ++r) {
        const long long rr = pk * RPW + r;
        const int rowid = rr < a.nrows ? a.rows[rr] : a.rows[0];
        const cplx_t<double>* row = spec + (long long)rowid * a.P + 1;
        for (int i = lane; i < a.n; i += 32) cp_async_bytes16(stg + r * RSD + 2 * i, row + i, true);
    }
}

// The folded FP64 solve of RPW = 4 NT rows staged in stg (row r's interior at
// stg + r RSD, complex i at 2 i), both transforms on the FP64 tensor cores
// (mma.sync m8n8k4).  On return stg holds the folded solution: row r's
// symmetric block at stg + r RSD + 2 i, its antisymmetric block at + 2 (LD + i).
// gq[t]: shift group of row 4 t + (lane % 4).
template <int NT, int MT, int KS, int RSD, int LD>
__device__ __forceinline__ void mma_fold_solve(const double* A, const double* recip, double* stg, const int (&gq)[NT],
                                               int n, int m, int ms, int lane)
{
    const int g = lane >> 2, q = lane & 3;
    const double r2 = 0.70710678118654752440;
    const double* As1 = A;                           // first transform, symmetric block
    const double* As2 = A + (size_t)LD * LD;         // second transform, symmetric block
    const double* Aa1 = A + (size_t)2 * LD * LD;     // first transform, antisymmetric block
    const double* Aa2 = A + (size_t)3 * LD * LD;     // second transform, antisymmetric block
    // ---- first transform; B fragments folded on the fly ----
    double cs[NT][MT][2], ca[NT][MT][2];
#pragma unroll
    for (int t = 0; t < NT; ++t)
#pragma unroll
        for (int mt = 0; mt < MT; ++mt) cs[t][mt][0] = cs[t][mt][1] = ca[t][mt][0] = ca[t][mt][1] = 0.0;
#pragma unroll 2
    for (int kk = 0; kk < KS; ++kk) {
        const int k = 4 * kk + q;
        double bs[NT], ba[NT];
#pragma unroll
        for (int t = 0; t < NT; ++t) {
            const double* raw = stg + (4 * t + (g >> 1)) * RSD + (g & 1);
            double vs = 0.0, va = 0.0;
            if (k < m) {
                const double lo = raw[2 * k], hi = raw[2 * (n - 1 - k)];
                vs = r2 * (lo + hi);
                va = r2 * (lo - hi);
            } else if (k < ms) {
                vs = raw[2 * k];
            }
            bs[t] = vs;
            ba[t] = va;
        }
#pragma unroll
        for (int mt = 0; mt < MT; ++mt) {
            const double as = As1[(mt * KS + kk) * 32 + lane];
            const double aa = Aa1[(mt * KS + kk) * 32 + lane];
#pragma unroll
            for (int t = 0; t < NT; ++t) {
                dmma_8x8x4(cs[t][mt][0], cs[t][mt][1], as, bs[t]);
                dmma_8x8x4(ca[t][mt][0], ca[t][mt][1], aa, ba[t]);
            }
        }
    }
    // ---- scale by 1 / (lambda_j - sigma) of each row's shift; stage as the next B ----
    __syncwarp();
#pragma unroll
    for (int t = 0; t < NT; ++t) {
        const int r = 4 * t + q;
        const double* rc = recip + (size_t)gq[t] * 2 * LD;
#pragma unroll
        for (int mt = 0; mt < MT; ++mt) {
            const int i = mt * 8 + g;
            const double s = rc[i], u = rc[LD + i];
            *reinterpret_cast<double2*>(stg + r * RSD + 2 * i) = make_double2(cs[t][mt][0] * s, cs[t][mt][1] * s);
            *reinterpret_cast<double2*>(stg + r * RSD + 2 * (LD + i)) =
                make_double2(ca[t][mt][0] * u, ca[t][mt][1] * u);
            cs[t][mt][0] = cs[t][mt][1] = ca[t][mt][0] = ca[t][mt][1] = 0.0;
        }
    }
    __syncwarp();
    // ---- second transform ----
#pragma unroll 2
    for (int kk = 0; kk < KS; ++kk) {
        const int k = 4 * kk + q;
        double bs[NT], ba[NT];
#pragma unroll
        for (int t = 0; t < NT; ++t) {
            const double* c = stg + (4 * t + (g >> 1)) * RSD + (g & 1);
            bs[t] = c[2 * k];
            ba[t] = c[2 * (LD + k)];
        }
#pragma unroll
        for (int mt = 0; mt < MT; ++mt) {
            const double as = As2[(mt * KS + kk) * 32 + lane];
            const double aa = Aa2[(mt * KS + kk) * 32 + lane];
#pragma unroll
            for (int t = 0; t < NT; ++t) {
                dmma_8x8x4(cs[t][mt][0], cs[t][mt][1], as, bs[t]);
                dmma_8x8x4(ca[t][mt][0], ca[t][mt][1], aa, ba[t]);
            }
        }
    }
    __syncwarp();
#pragma unroll
    for (int t = 0; t < NT; ++t) {
        const int r = 4 * t + q;
#pragma unroll
        for (int mt = 0; mt < MT; ++mt) {
            const int i = mt * 8 + g;
            *reinterpret_cast<double2*>(stg + r * RSD + 2 * i) = make_double2(cs[t][mt][0], cs[t][mt][1]);
            *reinterpret_cast<double2*>(stg + r * RSD + 2 * (LD + i)) = make_double2(ca[t][mt][0], ca[t][mt][1]);
        }
    }
    __syncwarp();
}

template <int NSS, int NT, int WARPS, bool ADJ>
__global__ void __launch_bounds__(WARPS * 32, (NSS == 1 ? 2 : 1)) fdm_mma_kernel(FdmArgs a)
{
    using S = MmaShape<NSS, NT, WARPS>;
    constexpr int LD = S::LD, MT = S::MT, KS = S::KS, RPW = S::RPW, RSD = S::RSD;
    extern __shared__ __align__(16) double dsm[];
    double* A = dsm;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int q = lane & 3;
    double* stg_base = dsm + S::mats + (size_t)warp * 2 * RPW * RSD;
    {
        const double2* src = reinterpret_cast<const double2*>(a.mma_mats);
        double2* dst = reinterpret_cast<double2*>(A);
        for (int e = threadIdx.x; e < (int)(S::mats / 2); e += blockDim.x) dst[e] = src[e];
    }
    pdl_enter();
    __syncthreads();

    cplx_t<double>* spec = static_cast<cplx_t<double>*>(a.spec);
    const int n = a.n, m = a.m, ms = a.ms, nrows = a.nrows;
    const long long npacks = (nrows + RPW - 1) / RPW;

    const long long pstride = (long long)gridDim.x * WARPS;
    long long pk = (long long)blockIdx.x * WARPS + warp;
    int cur = 0;
    if (pk < npacks) mma_issue_pack<RPW, RSD>(a, pk, stg_base, lane);
    cp_async_commit();
    for (; pk < npacks; pk += pstride, cur ^= 1) {
        double* stg = stg_base + (size_t)cur * RPW * RSD;
        if (pk + pstride < npacks) mma_issue_pack<RPW, RSD>(a, pk + pstride, stg_base + (size_t)(cur ^ 1) * RPW * RSD, lane);
        cp_async_commit();
        int rowid[RPW], grp[RPW];
        bool ok[RPW];
#pragma unroll
        for (int r = 0; r < RPW; ++r) {
            const long long rr = pk * RPW + r;
            ok[r] = rr < nrows;
            rowid[r] = ok[r] ? a.rows[rr] : a.rows[0];
            grp[r] = ok[r] ? a.row_grp[rr] : a.row_grp[0];
        }
        // ---- the staged interiors of this pack's rows ----
        cp_async_wait_prev();
        __syncwarp();
        int gq[NT];
#pragma unroll
        for (int t = 0; t < NT; ++t) {
            const long long rr = pk * RPW + 4 * t + q;
            gq[t] = a.row_grp[rr < nrows ? rr : 0];
        }
        mma_fold_solve<NT, MT, KS, RSD, LD>(A, static_cast<const double*>(a.recip), stg, gq, n, m, ms, lane);
        // ---- folded solution to the lane-per-fold-index layout, epilogue ----
        double xsr[RPW][NSS], xsi[RPW][NSS], xdr[RPW][NSS], xdi[RPW][NSS];
#pragma unroll
        for (int r = 0; r < RPW; ++r)
#pragma unroll
            for (int t = 0; t < NSS; ++t) {
                const double2 vs = *reinterpret_cast<const double2*>(stg + r * RSD + 2 * (lane + 32 * t));
                const double2 vd = *reinterpret_cast<const double2*>(stg + r * RSD + 2 * (LD + lane + 32 * t));
                xsr[r][t] = vs.x; xsi[r][t] = vs.y;
                xdr[r][t] = vd.x; xdi[r][t] = vd.y;
            }
        fdm_store_rows<double, NSS, RPW, ADJ>(a, spec, rowid, grp, ok, xsr, xsi, xdr, xdi, lane);
        __syncwarp();  // stg is refilled by the copy issued in the next iteration
    }
    cp_async_wait_all();
}

template <int NSS, int NT, int WARPS, bool ADJ>
static int run_fdm_mma(const FdmArgs& a, cudaStream_t s)
{
    using S = MmaShape<NSS, NT, WARPS>;
    auto k = fdm_mma_kernel<NSS, NT, WARPS, ADJ>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::smem);
    if (e != cudaSuccess) return (int)e;
    int dev = 0, sms = 148, per = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k, WARPS * 32, S::smem);
    if (per < 1) per = 1;
    const long long packs = (a.nrows + S::RPW - 1) / S::RPW;
    long long grid = (packs + WARPS - 1) / WARPS;
    if (grid > (long long)sms * per) grid = (long long)sms * per;
    if (grid <= 0) return 0;
    return (int)launch_k(k, dim3((unsigned)grid), dim3(WARPS * 32), S::smem, s, a);
}

// ---- the same solve with the m16n8k8 .f64 shape (sm_90 and later) ----
// Fragment layout (g = lane / 4, q = lane % 4):
//   A (16 x 8): a0 = A[g][q], a1 = A[g + 8][q], a2 = A[g][q + 4], a3 = A[g + 8][q + 4]
//   B (8 x 8):  b0 = B[q][g], b1 = B[q + 4][g]
//   C (16 x 8): c0, c1 = C[g][2 q], C[g][2 q + 1];  c2, c3 = C[g + 8][2 q], C[g + 8][2 q + 1]
// One product is 1024 multiply-adds (four times m8n8k4), a fragment of A four
// consecutive doubles per lane in the stored order.
__device__ __forceinline__ void dmma_16x8x8(double (&c)[4], const double2& a01, const double2& a23, double b0,
                                            double b1)
{
    asm("mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
                 "{%0, %1, %2, %3};\n"
                 : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
                 : "d"(a01.x), "d"(a01.y), "d"(a23.x), "d"(a23.y), "d"(b0), "d"(b1));
}

template <int NSS, int WARPS, bool ADJ>
__global__ void __launch_bounds__(WARPS * 32, (NSS == 1 ? 2 : 1)) fdm_mma16_kernel(FdmArgs a)
{
    using S = MmaShape<NSS, 1, WARPS>;
    constexpr int LD = S::LD, RPW = S::RPW, RSD = S::RSD;
    constexpr int MT = LD / 16, KS = LD / 8;
    extern __shared__ __align__(16) double dsm[];
    double* A = dsm;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane >> 2, q = lane & 3;
    double* stg_base = dsm + S::mats + (size_t)warp * 2 * RPW * RSD;
    {
        const double2* src = reinterpret_cast<const double2*>(a.mma16_mats);
        double2* dst = reinterpret_cast<double2*>(A);
        for (int e = threadIdx.x; e < (int)(S::mats / 2); e += blockDim.x) dst[e] = src[e];
    }
    pdl_enter();
    __syncthreads();

    cplx_t<double>* spec = static_cast<cplx_t<double>*>(a.spec);
    const int n = a.n, m = a.m, ms = a.ms, nrows = a.nrows;
    const double r2 = 0.70710678118654752440;
    const long long npacks = (nrows + RPW - 1) / RPW;
    // fragment (mt, kk) of transform b: 4 doubles per lane at ((mt KS + kk) 32 + lane) 4
    const double2* Af = reinterpret_cast<const double2*>(A);
    constexpr size_t BLK = (size_t)LD * LD / 2;  // double2 per transform
    const double* rcp = static_cast<const double*>(a.recip);

    const long long pstride = (long long)gridDim.x * WARPS;
    long long pk = (long long)blockIdx.x * WARPS + warp;
    int cur = 0;
    if (pk < npacks) mma_issue_pack<RPW, RSD>(a, pk, stg_base, lane);
    cp_async_commit();
    for (; pk < npacks; pk += pstride, cur ^= 1) {
        double* stg = stg_base + (size_t)cur * RPW * RSD;
        if (pk + pstride < npacks) mma_issue_pack<RPW, RSD>(a, pk + pstride, stg_base + (size_t)(cur ^ 1) * RPW * RSD, lane);
        cp_async_commit();
        int rowid[RPW], grp[RPW];
        bool ok[RPW];
#pragma unroll
        for (int r = 0; r < RPW; ++r) {
            const long long rr = pk * RPW + r;
            ok[r] = rr < nrows;
            rowid[r] = ok[r] ? a.rows[rr] : a.rows[0];
            grp[r] = ok[r] ? a.row_grp[rr] : a.row_grp[0];
        }
        // reciprocal shifts of this lane's accumulator rows (row q), loaded early
        double rs[MT][2], ra[MT][2];
        {
            const int gq = a.row_grp[(pk * RPW + q) < nrows ? pk * RPW + q : 0];
            const double* rc = rcp + (size_t)gq * 2 * LD;
#pragma unroll
            for (int mt = 0; mt < MT; ++mt) {
                rs[mt][0] = rc[mt * 16 + g];
                rs[mt][1] = rc[mt * 16 + g + 8];
                ra[mt][0] = rc[LD + mt * 16 + g];
                ra[mt][1] = rc[LD + mt * 16 + g + 8];
            }
        }
        cp_async_wait_prev();
        __syncwarp();
        // ---- first transform; B fragments folded on the fly ----
        double cs[MT][4], ca[MT][4];
#pragma unroll
        for (int mt = 0; mt < MT; ++mt)
#pragma unroll
            for (int j = 0; j < 4; ++j) cs[mt][j] = ca[mt][j] = 0.0;
        const double* raw = stg + (g >> 1) * RSD + (g & 1);
#pragma unroll 2
        for (int kk = 0; kk < KS; ++kk) {
            double bs[2], ba[2];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int k = 8 * kk + q + 4 * h;
                double vs = 0.0, va = 0.0;
                if (k < m) {
                    const double lo = raw[2 * k], hi = raw[2 * (n - 1 - k)];
                    vs = r2 * (lo + hi);
                    va = r2 * (lo - hi);
                } else if (k < ms) {
                    vs = raw[2 * k];
                }
                bs[h] = vs;
                ba[h] = va;
            }
#pragma unroll
            for (int mt = 0; mt < MT; ++mt) {
                const double2* fs = Af + 0 * BLK + ((size_t)(mt * KS + kk) * 32 + lane) * 2;
                const double2* fa = Af + 2 * BLK + ((size_t)(mt * KS + kk) * 32 + lane) * 2;
                dmma_16x8x8(cs[mt], fs[0], fs[1], bs[0], bs[1]);
                dmma_16x8x8(ca[mt], fa[0], fa[1], ba[0], ba[1]);
            }
        }
        // ---- scale by 1 / (lambda_j - sigma); stage as the next B ----
        __syncwarp();
        {
            double* row = stg + q * RSD;
#pragma unroll
            for (int mt = 0; mt < MT; ++mt) {
                const int i0 = mt * 16 + g, i1 = i0 + 8;
                *reinterpret_cast<double2*>(row + 2 * i0) = make_double2(cs[mt][0] * rs[mt][0], cs[mt][1] * rs[mt][0]);
                *reinterpret_cast<double2*>(row + 2 * i1) = make_double2(cs[mt][2] * rs[mt][1], cs[mt][3] * rs[mt][1]);
                *reinterpret_cast<double2*>(row + 2 * (LD + i0)) =
                    make_double2(ca[mt][0] * ra[mt][0], ca[mt][1] * ra[mt][0]);
                *reinterpret_cast<double2*>(row + 2 * (LD + i1)) =
                    make_double2(ca[mt][2] * ra[mt][1], ca[mt][3] * ra[mt][1]);
#pragma unroll
                for (int j = 0; j < 4; ++j) cs[mt][j] = ca[mt][j] = 0.0;
            }
        }
        __syncwarp();
        // ---- second transform ----
        const double* cf = stg + (g >> 1) * RSD + (g & 1);
#pragma unroll 2
        for (int kk = 0; kk < KS; ++kk) {
            const int k0 = 8 * kk + q, k1 = k0 + 4;
            const double bs0 = cf[2 * k0], bs1 = cf[2 * k1];
            const double ba0 = cf[2 * (LD + k0)], ba1 = cf[2 * (LD + k1)];
#pragma unroll
            for (int mt = 0; mt < MT; ++mt) {
                const double2* fs = Af + 1 * BLK + ((size_t)(mt * KS + kk) * 32 + lane) * 2;
                const double2* fa = Af + 3 * BLK + ((size_t)(mt * KS + kk) * 32 + lane) * 2;
                dmma_16x8x8(cs[mt], fs[0], fs[1], bs0, bs1);
                dmma_16x8x8(ca[mt], fa[0], fa[1], ba0, ba1);
            }
        }
        __syncwarp();
        {
            double* row = stg + q * RSD;
#pragma unroll
            for (int mt = 0; mt < MT; ++mt) {
                const int i0 = mt * 16 + g, i1 = i0 + 8;
                *reinterpret_cast<double2*>(row + 2 * i0) = make_double2(cs[mt][0], cs[mt][1]);
                *reinterpret_cast<double2*>(row + 2 * i1) = make_double2(cs[mt][2], cs[mt][3]);
                *reinterpret_cast<double2*>(row + 2 * (LD + i0)) = make_double2(ca[mt][0], ca[mt][1]);
                *reinterpret_cast<double2*>(row + 2 * (LD + i1)) = make_double2(ca[mt][2], ca[mt][3]);
            }
        }
        __syncwarp();
        double xsr[RPW][NSS], xsi[RPW][NSS], xdr[RPW][NSS], xdi[RPW][NSS];
#pragma unroll
        for (int r = 0; r < RPW; ++r)
#pragma unroll
            for (int t = 0; t < NSS; ++t) {
                const double2 vs = *reinterpret_cast<const double2*>(stg + r * RSD + 2 * (lane + 32 * t));
                const double2 vd = *reinterpret_cast<const double2*>(stg + r * RSD + 2 * (LD + lane + 32 * t));
                xsr[r][t] = vs.x; xsi[r][t] = vs.y;
                xdr[r][t] = vd.x; xdi[r][t] = vd.y;
            }
        fdm_store_rows<double, NSS, RPW, ADJ>(a, spec, rowid, grp, ok, xsr, xsi, xdr, xdi, lane);
        __syncwarp();  // stg is refilled by the copy issued in the next iteration
    }
    cp_async_wait_all();
}

template <int NSS, int WARPS, bool ADJ>
static int run_fdm_mma16(const FdmArgs& a, cudaStream_t s)
{
    using S = MmaShape<NSS, 1, WARPS>;
    auto k = fdm_mma16_kernel<NSS, WARPS, ADJ>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::smem);
    if (e != cudaSuccess) return (int)e;
    int dev = 0, sms = 148, per = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k, WARPS * 32, S::smem);
    if (per < 1) per = 1;
    const long long packs = (a.nrows + S::RPW - 1) / S::RPW;
    long long grid = (packs + WARPS - 1) / WARPS;
    if (grid > (long long)sms * per) grid = (long long)sms * per;
    if (grid <= 0) return 0;
    return (int)launch_k(k, dim3((unsigned)grid), dim3(WARPS * 32), S::smem, s, a);
}

// variant 0: m16n8k8 products; variant 1: m8n8k4 products.  4 rows per warp;
// ld = 64 keeps 4 warps per CTA so the transforms (128 KB) fit.
int launch_fdm_mma(const FdmArgs& a, cudaStream_t s, int variant)
{
    if (!a.mma_mats || !a.mma16_mats) return (int)cudaErrorInvalidValue;
    if (a.ld == 32) {
        if (variant == 0) return a.adjoint ? run_fdm_mma16<1, 8, true>(a, s) : run_fdm_mma16<1, 8, false>(a, s);
        return a.adjoint ? run_fdm_mma<1, 1, 8, true>(a, s) : run_fdm_mma<1, 1, 8, false>(a, s);
    }
    if (a.ld == 64) {
        if (variant == 0) return a.adjoint ? run_fdm_mma16<2, 4, true>(a, s) : run_fdm_mma16<2, 4, false>(a, s);
        return a.adjoint ? run_fdm_mma<2, 1, 4, true>(a, s) : run_fdm_mma<2, 1, 4, false>(a, s);
    }
    return (int)cudaErrorInvalidValue;
}

void fdm_mma16_swizzle(const double* cm, int ld, double* out)
{
    const int MT = ld / 16, KS = ld / 8;
    for (int b = 0; b < 4; ++b) {
        const double* M = cm + (size_t)b * ld * ld;      // column-major: A[i][k] = M[k * ld + i]
        double* O = out + (size_t)b * ld * ld;
        for (int mt = 0; mt < MT; ++mt)
            for (int kk = 0; kk < KS; ++kk)
                for (int l = 0; l < 32; ++l) {
                    const int gg = l >> 2, qq = l & 3;
                    const int i0 = mt * 16 + gg, i1 = i0 + 8, k0 = kk * 8 + qq, k1 = k0 + 4;
                    double* o = O + (((size_t)mt * KS + kk) * 32 + l) * 4;
                    o[0] = M[(size_t)k0 * ld + i0];
                    o[1] = M[(size_t)k0 * ld + i1];
                    o[2] = M[(size_t)k1 * ld + i0];
                    o[3] = M[(size_t)k1 * ld + i1];
                }
    }
}

// ============== fused y-FFT + row solve + inverse y-FFT, one slab per cluster ==
//
// For 3D FP64 plans with one GLL element and up to 65 points: the spectrum
// rows of one kx (a slab [Ny][P] complex, 266 KB at Ny = 256, P = 65) live in
// the shared memory of a cluster of two CTAs, CTA c holding the GLL columns
// [c H0, ...) of every ky.  Each CTA transforms its columns along y in shared
// memory, the pair meets at a cluster barrier, each CTA solves half of the ky
// rows -- gathering a row's two halves through distributed shared memory,
// solving it with mma_fold_solve and writing the result back to both halves --
// and after a second barrier each CTA transforms its columns back and stores
// them.  The spectrum crosses the memory system once instead of three times
// (y pass, row solve, inverse y pass), and two launches disappear.

struct SlabArgs {
    int H0, HS;            // columns of CTA 0; shared-memory row stride of a half (complex)
    const void* tw;        // y twiddles exp(-2 pi i e / Ny), FP64 complex
    const int* grp_of_row; // shift group of each spectrum row kx Ny + ky
};

// A spectrum row split over the two halves of a slab (slots k < h in a, the rest in b).
struct SlabRow {
    cplx_t<double>* a;
    cplx_t<double>* b;
    int h;
    __device__ __forceinline__ cplx_t<double> get(int k) const { return k < h ? a[k] : b[k - h]; }
    __device__ __forceinline__ void put(int k, cplx_t<double> v) const
    {
        if (k < h) a[k] = v;
        else b[k - h] = v;
    }
};

constexpr int SLAB_WARPS = 8, SLAB_LD = 32, SLAB_RSD = 4 * SLAB_LD + 8;

inline size_t slab_smem_bytes(int L, int HS)
{
    return ((size_t)4 * SLAB_LD * SLAB_LD + (size_t)2 * L * HS + (size_t)SLAB_WARPS * 4 * SLAB_RSD) * sizeof(double);
}

template <int L, bool ADJ>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(SLAB_WARPS * 32, 1) slab_kernel(FdmArgs a, SlabArgs sa)
{
    namespace cg = cooperative_groups;
    using C = cplx_t<double>;
    constexpr int RPW = 4, LD = SLAB_LD, MT = LD / 8, KS = LD / 4, RSD = SLAB_RSD;
    extern __shared__ __align__(16) double dsm[];
    double* A = dsm;
    C* slab = reinterpret_cast<C*>(dsm + 4 * LD * LD);
    const int HS = sa.HS, H0 = sa.H0, P = a.P, n = a.n, m = a.m, ms = a.ms;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, q = lane & 3;
    double* stg = dsm + 4 * LD * LD + (size_t)2 * L * HS + (size_t)warp * RPW * RSD;
    {
        const double2* src = reinterpret_cast<const double2*>(a.mma_mats);
        double2* dst = reinterpret_cast<double2*>(A);
        for (int e = threadIdx.x; e < 2 * LD * LD; e += blockDim.x) dst[e] = src[e];
    }
    pdl_enter();
    cg::cluster_group cluster = cg::this_cluster();
    const int c = (int)cluster.block_rank();
    const int kx = blockIdx.x >> 1;
    const int z0 = c ? H0 : 0, nz = c ? P - H0 : H0;
    C* spec = static_cast<C*>(a.spec) + (long long)kx * L * P;
    const C* tw = static_cast<const C*>(sa.tw);
    for (int e = threadIdx.x; e < L * nz; e += blockDim.x) {
        const int ky = e / nz, zc = e - ky * nz;
        cp_async_bytes16(&slab[ky * HS + zc], &spec[(long long)ky * P + z0 + zc], true);
    }
    cp_async_commit();
    cp_async_wait_all();
    __syncthreads();
    slab_fft<L, -1, SLAB_WARPS * 32>(slab, HS, nz, tw);
    cluster.sync();

    // ---- rows ky in [c L/2, (c+1) L/2), 4 per warp at a time ----
    C* s0 = cluster.map_shared_rank(slab, 0);
    C* s1 = cluster.map_shared_rank(slab, 1);
    const int ky0 = c * (L / 2);
    for (int pk = warp; pk < (L / 2) / RPW; pk += SLAB_WARPS) {
        const int kyb = ky0 + pk * RPW;
        __syncwarp();
#pragma unroll
        for (int r = 0; r < RPW; ++r) {
            const SlabRow row{s0 + (kyb + r) * HS, s1 + (kyb + r) * HS, H0};
            for (int i = lane; i < n; i += 32) *reinterpret_cast<C*>(stg + r * RSD + 2 * i) = row.get(i + 1);
        }
        __syncwarp();
        int gq[1] = {sa.grp_of_row[(long long)kx * L + kyb + q]};
        mma_fold_solve<1, MT, KS, RSD, LD>(A, static_cast<const double*>(a.recip), stg, gq, n, m, ms, lane);
        double xsr[RPW][1], xsi[RPW][1], xdr[RPW][1], xdi[RPW][1];
        int grp[RPW];
        bool ok[RPW];
#pragma unroll
        for (int r = 0; r < RPW; ++r) {
            const double2 vs = *reinterpret_cast<const double2*>(stg + r * RSD + 2 * lane);
            const double2 vd = *reinterpret_cast<const double2*>(stg + r * RSD + 2 * (LD + lane));
            xsr[r][0] = vs.x; xsi[r][0] = vs.y;
            xdr[r][0] = vd.x; xdi[r][0] = vd.y;
            grp[r] = sa.grp_of_row[(long long)kx * L + kyb + r];
            ok[r] = true;
        }
        fdm_store_rows_at<double, 1, RPW, ADJ>(
            a, [&](int r) { return SlabRow{s0 + (kyb + r) * HS, s1 + (kyb + r) * HS, H0}; }, grp, ok, xsr, xsi, xdr,
            xdi, lane);
    }
    cluster.sync();
    slab_fft<L, 1, SLAB_WARPS * 32>(slab, HS, nz, tw);
    for (int e = threadIdx.x; e < L * nz; e += blockDim.x) {
        const int ky = e / nz, zc = e - ky * nz;
        spec[(long long)ky * P + z0 + zc] = slab[ky * HS + zc];
    }
}

template <int L>
static int run_slab(const FdmArgs& a, const SlabArgs& sa, int nkx, cudaStream_t s)
{
    auto k = a.adjoint ? slab_kernel<L, true> : slab_kernel<L, false>;
    const size_t smem = slab_smem_bytes(L, sa.HS);
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return (int)e;
    return (int)launch_k(k, dim3(2 * nkx), dim3(SLAB_WARPS * 32), smem, s, a, sa);
}

int launch_slab(const FdmArgs& a, int Ny, int H0, int HS, const void* tw, const int* grp_of_row, int nkx,
                cudaStream_t s)
{
    if (a.ld != SLAB_LD || !a.mma_mats) return (int)cudaErrorInvalidValue;
    const SlabArgs sa{H0, HS, tw, grp_of_row};
    switch (Ny) {
        case 64: return run_slab<64>(a, sa, nkx, s);
        case 128: return run_slab<128>(a, sa, nkx, s);
        case 256: return run_slab<256>(a, sa, nkx, s);
        default: return (int)cudaErrorInvalidValue;
    }
}

bool slab_fits(int Ny, int P, int ld)
{
    if (ld != SLAB_LD || (Ny != 64 && Ny != 128 && Ny != 256)) return false;
    const int H0 = (P + 1) / 2, HS = H0 | 1;
    return slab_smem_bytes(Ny, HS) <= 232448;
}

// ============================== refined solve on the tensor cores ==
//
// The HELM_FP32_REFINE row solve for folds of up to 32 (GLL up to 65 points):
//   x  = S(f)                 S: the folded solve with FP32-accurate products
//   r  = f - (M x - sigma x)  M: the folded blocks of D2int, FP64 tensor cores
//   x += S(r)
// S's two transforms run as three TF32 products each (hi*hi + hi*lo + lo*hi
// with a = hi + lo split at the 10-bit TF32 mantissa; the transforms are split
// once at plan time, the right-hand sides on the fly), accumulated in FP32 --
// the accuracy of an FP32 product at the TF32 tensor rate.  The FP64 residual
// uses mma.sync m16n8k8 .f64.  One warp solves 4 spectrum rows (8 columns:
// re / im) at a time; the TF32 fragment layout of m16n8k8 is that of the f64
// shape (g = lane / 4, q = lane % 4):
//   A: a0 = A[g][q], a1 = A[g + 8][q], a2 = A[g][q + 4], a3 = A[g + 8][q + 4]
//   B: b0 = B[q][g], b1 = B[q + 4][g]
//   C: C[g][2q], C[g][2q + 1], C[g + 8][2q], C[g + 8][2q + 1]
// Per warp a single staging region of 8 columns x 68 doubles holds, in turn,
// the raw rows, the FP32 exchanges between transforms, and the FP64 iterates.

__device__ __forceinline__ uint32_t to_tf32(float x)
{
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(r) : "f"(x));
    return r;
}

__device__ __forceinline__ void mma_tf32(float (&c)[4], const float4& a, uint32_t b0, uint32_t b1)
{
    asm("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, "
                 "{%8, %9}, {%0, %1, %2, %3};\n"
                 : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
                 : "r"(__float_as_uint(a.x)), "r"(__float_as_uint(a.y)), "r"(__float_as_uint(a.z)),
                   "r"(__float_as_uint(a.w)), "r"(b0), "r"(b1));
}

// A B fragment split at the TF32 mantissa: b = hi + lo.
struct Tf32Split {
    uint32_t h0, h1, l0, l1;
};
__device__ __forceinline__ Tf32Split tf32_split(float b0, float b1)
{
    Tf32Split t;
    t.h0 = to_tf32(b0);
    t.h1 = to_tf32(b1);
    t.l0 = to_tf32(b0 - __uint_as_float(t.h0));
    t.l1 = to_tf32(b1 - __uint_as_float(t.h1));
    return t;
}

// c += A (hi + lo) * B (hi + lo), three TF32 products (lo * lo dropped).
__device__ __forceinline__ void mma_3xtf32(float (&c)[4], const float4& ah, const float4& al, const Tf32Split& b)
{
    mma_tf32(c, al, b.h0, b.h1);
    mma_tf32(c, ah, b.l0, b.l1);
    mma_tf32(c, ah, b.h0, b.h1);
}

constexpr int TC_WARPS = 12, TC_LD = 32, TC_MT = 2, TC_KS = 4, TC_S = 68;
constexpr size_t TC_TF32_FLOATS = (size_t)4 * 2 * TC_LD * TC_LD;  // 4 transforms x (hi, lo)
constexpr size_t TC_M_DOUBLES = (size_t)2 * TC_LD * TC_LD;        // Ms, Ma
// per warp two staging regions of 8 columns x 68 doubles: the current pack and the next one arriving
constexpr size_t TC_REG = (size_t)8 * TC_S;  // doubles
constexpr size_t TC_SMEM = TC_TF32_FLOATS * 4 + TC_M_DOUBLES * 8 + (size_t)TC_WARPS * 2 * TC_REG * 8;

// One folded solve S on B columns read by `bread(blk, kk, hf)` (the lane's B
// element of block blk at fold index 8 kk + q + 4 hf, as float; kk and hf are
// compile-time after unrolling, so register arrays stay in registers); result x
// in C layout (FP32).
template <typename BRead>
__device__ __forceinline__ void tc_solve(const float4* Tf, const float (&rs)[TC_MT][2], const float (&ra)[TC_MT][2],
                                         float* X, int g, int q, BRead bread, float (&xs)[TC_MT][4],
                                         float (&xa)[TC_MT][4])
{
    const int lane = g * 4 + q;
    constexpr size_t BLKF = (size_t)2 * TC_LD * TC_LD / 4;  // float4 per transform (hi + lo)
    float cs[TC_MT][4], ca[TC_MT][4];
#pragma unroll
    for (int mt = 0; mt < TC_MT; ++mt)
#pragma unroll
        for (int j = 0; j < 4; ++j) cs[mt][j] = ca[mt][j] = 0.f;
#pragma unroll
    for (int kk = 0; kk < TC_KS; ++kk) {
        const Tf32Split bs = tf32_split(bread(0, kk, 0), bread(0, kk, 1));
        const Tf32Split ba = tf32_split(bread(1, kk, 0), bread(1, kk, 1));
#pragma unroll
        for (int mt = 0; mt < TC_MT; ++mt) {
            const size_t f = (size_t)(mt * TC_KS + kk) * 32 + lane;
            mma_3xtf32(cs[mt], Tf[0 * BLKF + f], Tf[0 * BLKF + BLKF / 2 + f], bs);  // Ws
            mma_3xtf32(ca[mt], Tf[2 * BLKF + f], Tf[2 * BLKF + BLKF / 2 + f], ba);  // Wa
        }
    }
    // scale by 1 / (lambda_j - sigma) and stage as the next B (column 2q + j)
    __syncwarp();
#pragma unroll
    for (int mt = 0; mt < TC_MT; ++mt)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int i = mt * 16 + g + 8 * h;
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                X[(2 * q + j) * TC_S + i] = cs[mt][2 * h + j] * rs[mt][h];
                X[(2 * q + j) * TC_S + TC_LD + i] = ca[mt][2 * h + j] * ra[mt][h];
            }
        }
    __syncwarp();
#pragma unroll
    for (int mt = 0; mt < TC_MT; ++mt)
#pragma unroll
        for (int j = 0; j < 4; ++j) xs[mt][j] = xa[mt][j] = 0.f;
    const float* col = X + g * TC_S;
#pragma unroll
    for (int kk = 0; kk < TC_KS; ++kk) {
        const int k0 = 8 * kk + q, k1 = k0 + 4;
        const Tf32Split bs = tf32_split(col[k0], col[k1]);
        const Tf32Split ba = tf32_split(col[TC_LD + k0], col[TC_LD + k1]);
#pragma unroll
        for (int mt = 0; mt < TC_MT; ++mt) {
            const size_t f = (size_t)(mt * TC_KS + kk) * 32 + lane;
            mma_3xtf32(xs[mt], Tf[1 * BLKF + f], Tf[1 * BLKF + BLKF / 2 + f], bs);  // Vs
            mma_3xtf32(xa[mt], Tf[3 * BLKF + f], Tf[3 * BLKF + BLKF / 2 + f], ba);  // Va
        }
    }
    __syncwarp();  // X is free again
}

template <bool ADJ>
__global__ void __launch_bounds__(TC_WARPS * 32, 1) fdm_tc_refine_kernel(FdmArgs a)
{
    extern __shared__ __align__(16) unsigned char tsm[];
    float4* Tf = reinterpret_cast<float4*>(tsm);
    double* Md = reinterpret_cast<double*>(tsm + TC_TF32_FLOATS * 4);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane >> 2, q = lane & 3;
    double* regions = reinterpret_cast<double*>(tsm + TC_TF32_FLOATS * 4 + TC_M_DOUBLES * 8) + (size_t)warp * 2 * TC_REG;
    {
        const float4* src = static_cast<const float4*>(a.tc_mats);
        for (int e = threadIdx.x; e < (int)(TC_TF32_FLOATS / 4); e += blockDim.x) Tf[e] = src[e];
        const double2* msrc = reinterpret_cast<const double2*>(a.tc_m);
        double2* mdst = reinterpret_cast<double2*>(Md);
        for (int e = threadIdx.x; e < (int)(TC_M_DOUBLES / 2); e += blockDim.x) mdst[e] = msrc[e];
    }
    pdl_enter();
    __syncthreads();

    cplx_t<double>* spec = static_cast<cplx_t<double>*>(a.spec);
    const int n = a.n, m = a.m, ms = a.ms, nrows = a.nrows;
    const double r2 = 0.70710678118654752440;
    constexpr int RPW = 4, RR = 136;  // raw row r at Xd + r RR (complex i at 2 i)
    const long long npacks = (nrows + RPW - 1) / RPW;
    const float* rcp = static_cast<const float*>(a.recip);
    // M fragments in two planes per block: (a0, a1) of every lane, then (a2, a3)
    const double2* Mf = reinterpret_cast<const double2*>(Md);
    constexpr size_t MPLANE = (size_t)TC_LD * TC_LD / 4;  // double2 per plane

    const long long pstride = (long long)gridDim.x * TC_WARPS;
    long long pk = (long long)blockIdx.x * TC_WARPS + warp;
    int cur = 0;
    if (pk < npacks) mma_issue_pack<RPW, RR>(a, pk, regions, lane);
    cp_async_commit();
    for (; pk < npacks; pk += pstride, cur ^= 1) {
        double* Xd = regions + (size_t)cur * TC_REG;
        float* Xf = reinterpret_cast<float*>(Xd);
        if (pk + pstride < npacks) mma_issue_pack<RPW, RR>(a, pk + pstride, regions + (size_t)(cur ^ 1) * TC_REG, lane);
        cp_async_commit();
        int rowid[RPW], grp[RPW];
        bool ok[RPW];
#pragma unroll
        for (int r = 0; r < RPW; ++r) {
            const long long rr = pk * RPW + r;
            ok[r] = rr < nrows;
            rowid[r] = ok[r] ? a.rows[rr] : a.rows[0];
            grp[r] = ok[r] ? a.row_grp[rr] : a.row_grp[0];
        }
        // this lane's C-layout row is q: its shift and reciprocal shifts
        const int gq = a.row_grp[(pk * RPW + q) < nrows ? pk * RPW + q : 0];
        const double sig = a.sigma[gq];
        float rs[TC_MT][2], ra[TC_MT][2];
#pragma unroll
        for (int mt = 0; mt < TC_MT; ++mt)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                rs[mt][h] = rcp[(size_t)gq * 2 * TC_LD + mt * 16 + g + 8 * h];
                ra[mt][h] = rcp[(size_t)gq * 2 * TC_LD + TC_LD + mt * 16 + g + 8 * h];
            }
        // ---- raw interiors of the 4 rows (copied during the previous pack) ----
        cp_async_wait_prev();
        __syncwarp();
        // folded right-hand side at (fold index k, block blk) of column `col` (row col / 2, part col % 2)
        auto fold_at = [&](int col, int blk, int k) -> double {
            const double* raw = Xd + (col >> 1) * RR + (col & 1);
            if (k < m) {
                const double lo = raw[2 * k], hi = raw[2 * (n - 1 - k)];
                return blk == 0 ? r2 * (lo + hi) : r2 * (lo - hi);
            }
            return (blk == 0 && k < ms) ? raw[2 * k] : 0.0;
        };
        // f in C layout (kept for the residual): [blk][mt][h][j]
        double fc[2][TC_MT][2][2];
#pragma unroll
        for (int blk = 0; blk < 2; ++blk)
#pragma unroll
            for (int mt = 0; mt < TC_MT; ++mt)
#pragma unroll
                for (int h = 0; h < 2; ++h)
#pragma unroll
                    for (int j = 0; j < 2; ++j) fc[blk][mt][h][j] = fold_at(2 * q + j, blk, mt * 16 + g + 8 * h);
        // ---- x = S(f) ----
        float xs[TC_MT][4], xa[TC_MT][4];
        {
            float bsave[2][TC_KS][2];  // the lane's B elements of f, read before X is reused
#pragma unroll
            for (int blk = 0; blk < 2; ++blk)
#pragma unroll
                for (int kk = 0; kk < TC_KS; ++kk) {
                    bsave[blk][kk][0] = (float)fold_at(g, blk, 8 * kk + q);
                    bsave[blk][kk][1] = (float)fold_at(g, blk, 8 * kk + q + 4);
                }
            __syncwarp();
            tc_solve(Tf, rs, ra, Xf, g, q,
                     [&](int blk, int kk, int hf) { return bsave[blk][kk][hf]; }, xs, xa);
        }
        // ---- r = f - (M x - sigma x), FP64 ----
#pragma unroll
        for (int mt = 0; mt < TC_MT; ++mt)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int i = mt * 16 + g + 8 * h;
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    Xd[(2 * q + j) * TC_S + i] = (double)xs[mt][2 * h + j];
                    Xd[(2 * q + j) * TC_S + TC_LD + i] = (double)xa[mt][2 * h + j];
                }
            }
        __syncwarp();
        double ys[TC_MT][4], ya[TC_MT][4];
#pragma unroll
        for (int mt = 0; mt < TC_MT; ++mt)
#pragma unroll
            for (int j = 0; j < 4; ++j) ys[mt][j] = ya[mt][j] = 0.0;
        {
            const double* col = Xd + g * TC_S;
#pragma unroll
            for (int kk = 0; kk < TC_KS; ++kk) {
                const int k0 = 8 * kk + q, k1 = k0 + 4;
                const double bs0 = col[k0], bs1 = col[k1], ba0 = col[TC_LD + k0], ba1 = col[TC_LD + k1];
#pragma unroll
                for (int mt = 0; mt < TC_MT; ++mt) {
                    const size_t f = (size_t)(mt * TC_KS + kk) * 32 + lane;
                    dmma_16x8x8(ys[mt], Mf[f], Mf[MPLANE + f], bs0, bs1);
                    dmma_16x8x8(ya[mt], Mf[2 * MPLANE + f], Mf[3 * MPLANE + f], ba0, ba1);
                }
            }
        }
        __syncwarp();  // Xd is reused for the residual below
        float resf[2][TC_KS][2];
        {
            // residual in C layout, staged as FP32 columns, then read back as B elements
#pragma unroll
            for (int mt = 0; mt < TC_MT; ++mt)
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int i = mt * 16 + g + 8 * h;
#pragma unroll
                    for (int j = 0; j < 2; ++j) {
                        const double rsv = fc[0][mt][h][j] - ys[mt][2 * h + j] + sig * (double)xs[mt][2 * h + j];
                        const double rav = fc[1][mt][h][j] - ya[mt][2 * h + j] + sig * (double)xa[mt][2 * h + j];
                        Xf[(2 * q + j) * TC_S + i] = (float)rsv;
                        Xf[(2 * q + j) * TC_S + TC_LD + i] = (float)rav;
                    }
                }
            __syncwarp();
            const float* col = Xf + g * TC_S;
#pragma unroll
            for (int kk = 0; kk < TC_KS; ++kk) {
                resf[0][kk][0] = col[8 * kk + q];
                resf[0][kk][1] = col[8 * kk + q + 4];
                resf[1][kk][0] = col[TC_LD + 8 * kk + q];
                resf[1][kk][1] = col[TC_LD + 8 * kk + q + 4];
            }
            __syncwarp();
        }
        // ---- x += S(r) ----
        float ds[TC_MT][4], da[TC_MT][4];
        tc_solve(Tf, rs, ra, Xf, g, q,
                 [&](int blk, int kk, int hf) { return resf[blk][kk][hf]; }, ds, da);
#pragma unroll
        for (int mt = 0; mt < TC_MT; ++mt)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int i = mt * 16 + g + 8 * h;
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    Xd[(2 * q + j) * TC_S + i] = (double)xs[mt][2 * h + j] + (double)ds[mt][2 * h + j];
                    Xd[(2 * q + j) * TC_S + TC_LD + i] = (double)xa[mt][2 * h + j] + (double)da[mt][2 * h + j];
                }
            }
        __syncwarp();
        double xsr[RPW][1], xsi[RPW][1], xdr[RPW][1], xdi[RPW][1];
#pragma unroll
        for (int r = 0; r < RPW; ++r) {
            xsr[r][0] = Xd[(2 * r) * TC_S + lane];
            xsi[r][0] = Xd[(2 * r + 1) * TC_S + lane];
            xdr[r][0] = Xd[(2 * r) * TC_S + TC_LD + lane];
            xdi[r][0] = Xd[(2 * r + 1) * TC_S + TC_LD + lane];
        }
        fdm_store_rows<double, 1, RPW, ADJ>(a, spec, rowid, grp, ok, xsr, xsi, xdr, xdi, lane);
        __syncwarp();  // this region is refilled by the copy issued in the next iteration
    }
    cp_async_wait_all();
}

int launch_fdm_tc_refine(const FdmArgs& a, cudaStream_t s)
{
    if (a.ld != TC_LD || !a.tc_mats || !a.tc_m || a.sweeps != 1) return (int)cudaErrorInvalidValue;
    auto k = a.adjoint ? fdm_tc_refine_kernel<true> : fdm_tc_refine_kernel<false>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM);
    if (e != cudaSuccess) return (int)e;
    int dev = 0, sms = 148, per = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k, TC_WARPS * 32, TC_SMEM);
    if (per < 1) per = 1;
    const long long packs = (a.nrows + 3) / 4;
    long long grid = (packs + TC_WARPS - 1) / TC_WARPS;
    if (grid > (long long)sms * per) grid = (long long)sms * per;
    if (grid <= 0) return 0;
    return (int)launch_k(k, dim3((unsigned)grid), dim3(TC_WARPS * 32), TC_SMEM, s, a);
}

// The four transforms (column-major ld x ld, A[i][k] = cm[k ld + i]) split into
// TF32 hi + lo, in the m16n8k8 A-fragment order: [4][hi, lo][ld/16][ld/8][32][4].
static float tf32_round(double v)
{
    // round to nearest (ties away from zero) at 10 mantissa bits, like cvt.rna.tf32.f32
    float f = (float)v;
    uint32_t u;
    std::memcpy(&u, &f, 4);
    if ((u & 0x7f800000u) != 0x7f800000u) u = (u + 0x1000u) & 0xffffe000u;
    std::memcpy(&f, &u, 4);
    return f;
}

void fdm_tc_swizzle(const double* cm, int ld, float* out)
{
    const int MT = ld / 16, KS = ld / 8;
    for (int b = 0; b < 4; ++b) {
        const double* M = cm + (size_t)b * ld * ld;
        for (int part = 0; part < 2; ++part) {
            float* O = out + ((size_t)b * 2 + part) * ld * ld;
            for (int mt = 0; mt < MT; ++mt)
                for (int kk = 0; kk < KS; ++kk)
                    for (int l = 0; l < 32; ++l) {
                        const int gg = l >> 2, qq = l & 3;
                        const int i0 = mt * 16 + gg, i1 = i0 + 8, k0 = kk * 8 + qq, k1 = k0 + 4;
                        const double v[4] = {M[(size_t)k0 * ld + i0], M[(size_t)k0 * ld + i1], M[(size_t)k1 * ld + i0],
                                             M[(size_t)k1 * ld + i1]};
                        float* o = O + (((size_t)mt * KS + kk) * 32 + l) * 4;
                        for (int e = 0; e < 4; ++e) {
                            const float hi = tf32_round(v[e]);
                            o[e] = part == 0 ? hi : tf32_round(v[e] - (double)hi);
                        }
                    }
        }
    }
}

// Two FP64 column-major blocks in the m16n8k8 .f64 A-fragment order, each block
// as two planes [2][ld/16][ld/8][32][2]: (a0, a1) of every lane, then (a2, a3),
// so that a warp's 16-byte loads of one plane are contiguous.
void fdm_m16_swizzle2(const double* cm, int ld, double* out)
{
    const int MT = ld / 16, KS = ld / 8;
    const size_t plane = (size_t)ld * ld / 2;
    for (int b = 0; b < 2; ++b) {
        const double* M = cm + (size_t)b * ld * ld;
        double* O = out + (size_t)b * ld * ld;
        for (int mt = 0; mt < MT; ++mt)
            for (int kk = 0; kk < KS; ++kk)
                for (int l = 0; l < 32; ++l) {
                    const int gg = l >> 2, qq = l & 3;
                    const int i0 = mt * 16 + gg, i1 = i0 + 8, k0 = kk * 8 + qq, k1 = k0 + 4;
                    const size_t f = (((size_t)mt * KS + kk) * 32 + l) * 2;
                    O[f] = M[(size_t)k0 * ld + i0];
                    O[f + 1] = M[(size_t)k0 * ld + i1];
                    O[plane + f] = M[(size_t)k1 * ld + i0];
                    O[plane + f + 1] = M[(size_t)k1 * ld + i1];
                }
    }
}

void fdm_mma_swizzle(const double* cm, int ld, double* out)
{
    const int MT = ld / 8, KS = ld / 4;
    for (int b = 0; b < 4; ++b) {
        const double* M = cm + (size_t)b * ld * ld;      // column-major: A[i][k] = M[k * ld + i]
        double* O = out + (size_t)b * ld * ld;
        for (int mt = 0; mt < MT; ++mt)
            for (int kk = 0; kk < KS; ++kk)
                for (int l = 0; l < 32; ++l) {
                    const int i = mt * 8 + (l >> 2), k = kk * 4 + (l & 3);
                    O[((size_t)mt * KS + kk) * 32 + l] = M[(size_t)k * ld + i];
                }
    }
}

}  // namespace helm
