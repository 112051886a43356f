// Batched ACA+ compression of admissible H-matrix blocks, FP64.
//
// One CTA runs the whole ACA+ loop of one (block, slip pass) task, following
// BlockTree.ACA_plus_full_traceS/D (src/Hmatrix.py:581-1011):
//  * reference row set / column set of 3 consecutive rows (cols), restarted by
//    reset_reference_row/col (:620-648) when a pivot falls inside them;
//  * pivots are chosen on the A1 operator only and reused for A2 and B, each
//    with its own pivot value alpha (:718-726);
//  * stops on |alpha| < 1e-4 (:697), on the step-size test (:727-736: absolute
//    ||u_k|| ||v_k/alpha|| < eps, or a relative test against a running
//    Frobenius-norm estimate), when max_iter = min(m, n) is reached, or when a
//    reference set cannot be placed (scan_all).
// Rows/columns are indexed in the block's local order (element ids ascending,
// the order of the reference's row_cluster/col_cluster), so the same starting
// indices give the same pivot sequence.  argmax ties resolve to the highest
// index and NaN ranks above every number, as a stable ascending argsort does.
// The GF entries come from the full-space TD kernel (td_gf.cuh).  Residual
// updates use explicitly rounded products (no FMA contraction) in the order
// of the reference's numpy expressions.
#include <stdio.h>
#include "pq3d_common.cuh"
#include "td_gf.cuh"
#include "td_hs.cuh"
#include "hm_layout.cuh"
#include <cuda_bf16.h>

using namespace pq3d;

struct AcaTask {
    int64_t rows_off, cols_off;  // offsets into the element-id lists
    int64_t ws_off;              // offset (doubles) of this task's workspace
    int32_t m, n, kmax, pass;    // pass 0 = strike slip (Ss=1), 1 = dip slip (Ds=1)
    int32_t iref0, jref0;        // randint(m) - 3 and randint(n) - 3
};

// Workspace of a task (doubles): U[kmax][3][m], V[kmax][3][n], RIref[3][n] (A1),
// RJref[3][m] (A1), RIstar[3][n], RJstar[3][m].
__host__ __device__ inline int64_t aca_ws_doubles(int m, int n, int kmax)
{
    return (int64_t)kmax * 3 * (m + n) + 6 * (int64_t)(m + n);
}

PQ3D_EXPORT int64_t pq3d_aca_ws_doubles(int m, int n, int kmax) { return aca_ws_doubles(m, n, kmax); }
PQ3D_EXPORT size_t pq3d_aca_task_bytes(void) { return sizeof(AcaTask); }

#define ACA_THREADS 256

struct ArgMax {
    double v;
    int i;
};

// "a ranks above b": NaN above numbers, then larger value, then larger index.
__device__ inline bool am_better(double av, int ai, double bv, int bi)
{
    bool an = av != av, bn = bv != bv;
    if (an != bn) return an;
    if (!an && av != bv) return av > bv;
    return ai > bi;
}

__device__ inline double nanmax2(double a, double b)
{
    if (a != a || b != b) return a + b;  // NaN
    return a > b ? a : b;
}

__device__ ArgMax block_argmax(ArgMax loc, ArgMax *red)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        double ov = __shfl_down_sync(0xffffffffu, loc.v, o);
        int oi = __shfl_down_sync(0xffffffffu, loc.i, o);
        if (oi >= 0 && (loc.i < 0 || am_better(ov, oi, loc.v, loc.i))) { loc.v = ov; loc.i = oi; }
    }
    __syncthreads();
    if (lane == 0) red[wid] = loc;
    __syncthreads();
    if (wid == 0) {
        const int nw = blockDim.x >> 5;
        loc = lane < nw ? red[lane] : ArgMax{0.0, -1};
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            double ov = __shfl_down_sync(0xffffffffu, loc.v, o);
            int oi = __shfl_down_sync(0xffffffffu, loc.i, o);
            if (oi >= 0 && (loc.i < 0 || am_better(ov, oi, loc.v, loc.i))) { loc.v = ov; loc.i = oi; }
        }
        if (lane == 0) red[0] = loc;
    }
    __syncthreads();
    ArgMax r = red[0];
    __syncthreads();
    return r;
}

__device__ double block_sum(double v, double *red)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    __syncthreads();
    if (lane == 0) red[wid] = v;
    __syncthreads();
    if (wid == 0) {
        const int nw = blockDim.x >> 5;
        v = lane < nw ? red[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) red[0] = v;
    }
    __syncthreads();
    double r = red[0];
    __syncthreads();
    return r;
}

__device__ inline bool bit_get(const uint32_t *bm, int i) { return (bm[i >> 5] >> (i & 31)) & 1u; }

struct AcaCtx {
    const double *xg, *ev;
    const SrcRec *rec;
    const HsRec *hs;      // half-space records (HS instantiation only)
    int hs_mode;
    const int32_t *rows, *cols;
    double mu, lam, nu;
    int m, n, pass, k;
    double *U, *V;  // U[q][c][m], V[q][c][n]
};

// Residual entries of rows I0..I0+cnt-1 (all columns): out[c][r][j] for comps < ncomp.
template <bool HS>
__device__ void residual_rows(const AcaCtx &C, int I0, int cnt, int ncomp, double *out, int ostride_c)
{
    for (int r = 0; r < cnt; ++r) {
        const int I = I0 + r;
        const int re = C.rows[I];
        double obs[3] = {C.xg[3 * re], C.xg[3 * re + 1], C.xg[3 * re + 2]};
        double f[9];
#pragma unroll
        for (int q = 0; q < 9; ++q) f[q] = C.ev[9 * re + q];
        for (int j = threadIdx.x; j < C.n; j += blockDim.x) {
            double t[3];
            if (HS) gf_traction_one_hs(obs, f, C.rec[C.cols[j]], C.hs[C.cols[j]], C.hs_mode, C.mu, C.lam, C.nu,
                                       C.pass, t);
            else gf_traction_one(obs, f, C.rec[C.cols[j]], C.mu, C.lam, C.nu, C.pass, t);
            for (int c = 0; c < ncomp; ++c) {
                double v = t[c];
                for (int q = 0; q < C.k; ++q)
                    v = __dsub_rn(v, __dmul_rn(C.U[((int64_t)q * 3 + c) * C.m + I], C.V[((int64_t)q * 3 + c) * C.n + j]));
                out[(int64_t)c * ostride_c + (int64_t)r * C.n + j] = v;
            }
        }
    }
}

// Residual entries of columns J0..J0+cnt-1 (all rows): out[c][r][i].
template <bool HS>
__device__ void residual_cols(const AcaCtx &C, int J0, int cnt, int ncomp, double *out, int ostride_c)
{
    for (int r = 0; r < cnt; ++r) {
        const int J = J0 + r;
        const SrcRec s = C.rec[C.cols[J]];
        for (int i = threadIdx.x; i < C.m; i += blockDim.x) {
            const int re = C.rows[i];
            double obs[3] = {C.xg[3 * re], C.xg[3 * re + 1], C.xg[3 * re + 2]};
            double f[9];
#pragma unroll
            for (int q = 0; q < 9; ++q) f[q] = C.ev[9 * re + q];
            double t[3];
            if (HS) gf_traction_one_hs(obs, f, s, C.hs[C.cols[J]], C.hs_mode, C.mu, C.lam, C.nu, C.pass, t);
            else gf_traction_one(obs, f, s, C.mu, C.lam, C.nu, C.pass, t);
            for (int c = 0; c < ncomp; ++c) {
                double v = t[c];
                for (int q = 0; q < C.k; ++q)
                    v = __dsub_rn(v, __dmul_rn(C.V[((int64_t)q * 3 + c) * C.n + J], C.U[((int64_t)q * 3 + c) * C.m + i]));
                out[(int64_t)c * ostride_c + (int64_t)r * C.m + i] = v;
            }
        }
    }
}

// Argmax over len entries of f(x) excluding bitmap members.
template <typename F>
__device__ ArgMax argmax_excl(int len, const uint32_t *bm, F f, ArgMax *red)
{
    ArgMax loc{0.0, -1};
    for (int i = threadIdx.x; i < len; i += blockDim.x) {
        if (bit_get(bm, i)) continue;
        double v = f(i);
        if (loc.i < 0 || am_better(v, i, loc.v, loc.i)) { loc.v = v; loc.i = i; }
    }
    return block_argmax(loc, red);
}

template <bool HS>
__global__ void __launch_bounds__(ACA_THREADS)
k_aca(const double *__restrict__ xg, const double *__restrict__ ev, const SrcRec *__restrict__ rec,
      const int32_t *__restrict__ rowlist, const int32_t *__restrict__ collist, const AcaTask *__restrict__ tasks,
      double *__restrict__ ws, double mu, double lam, double eps, int rel_mode, int32_t *__restrict__ rank_out,
      int32_t *__restrict__ flag_out, const HsRec *__restrict__ hs, int hs_mode, int max_mn)
{
    extern __shared__ uint32_t bits[];
    __shared__ ArgMax red_am[32];
    __shared__ double red_d[32];
    __shared__ int s_scan;

    const AcaTask T = tasks[blockIdx.x];
    if (T.m < 0 || T.n < 0 || T.m > max_mn || T.n > max_mn) {   // the pivot bitmaps are sized for max_mn
        if (threadIdx.x == 0) {
            rank_out[blockIdx.x] = 0;
            flag_out[blockIdx.x] = 8;
        }
        return;
    }
    const int m = T.m, n = T.n;
    uint32_t *prevI = bits;
    uint32_t *prevJ = bits + ((m + 31) >> 5);
    for (int w = threadIdx.x; w < ((m + 31) >> 5) + ((n + 31) >> 5); w += blockDim.x) bits[w] = 0u;

    AcaCtx C;
    C.xg = xg; C.ev = ev; C.rec = rec; C.hs = hs; C.hs_mode = hs_mode;
    C.rows = rowlist + T.rows_off;
    C.cols = collist + T.cols_off;
    C.mu = mu; C.lam = lam; C.nu = 1.0 / (1.0 + lam / mu) / 2.0;
    C.m = m; C.n = n; C.pass = T.pass; C.k = 0;
    double *base = ws + T.ws_off;
    C.U = base;
    C.V = base + (int64_t)T.kmax * 3 * m;
    double *RIref = C.V + (int64_t)T.kmax * 3 * n;  // [3][n] (A1 only)
    double *RJref = RIref + 3 * (int64_t)n;         // [3][m]
    double *RIs = RJref + 3 * (int64_t)m;           // [3][n]
    double *RJs = RIs + 3 * (int64_t)n;             // [3][m]
    __syncthreads();

    const int max_iter = m < n ? m : n;
    int flags = 0;
    double frob2 = 0.0;

    // reset_reference_row / reset_reference_col (src/Hmatrix.py:620-648)
    auto reset_row = [&](int Iref, int &cnt) -> int {
        int attempt = 0;
        const int max_attempts = m / 3 + 1;
        int scan = 0;
        while (true) {
            Iref = ((Iref + 3) % m + m) % m;
            Iref -= Iref % 3;
            attempt++;
            if (!bit_get(prevI, Iref)) break;
            if (attempt > max_attempts) { scan = 1; break; }
        }
        cnt = (Iref + 3 <= m) ? 3 : m - Iref;
        residual_rows<HS>(C, Iref, cnt, 1, RIref, n);
        if (threadIdx.x == 0) s_scan = scan;
        __syncthreads();
        return Iref;
    };
    auto reset_col = [&](int Jref, int &cnt) -> int {
        int attempt = 0;
        const int max_attempts = n / 3 + 1;
        int scan = 0;
        while (true) {
            Jref = ((Jref + 3) % n + n) % n;
            Jref -= Jref % 3;
            attempt++;
            if (!bit_get(prevJ, Jref)) break;
            if (attempt > max_attempts) { scan = 1; break; }
        }
        cnt = (Jref + 3 <= n) ? 3 : n - Jref;
        residual_cols<HS>(C, Jref, cnt, 1, RJref, m);
        if (threadIdx.x == 0) s_scan = scan;
        __syncthreads();
        return Jref;
    };

    int ni = 0, nj = 0;
    int Iref = reset_row(T.iref0, ni);
    int Jref = reset_col(T.jref0, nj);
    int scan_all = s_scan;
    (void)scan_all;

    for (int it = 0; it < max_iter; ++it) {
        // pivot candidates from the reference sets (A1 only)
        ArgMax jc = argmax_excl(n, prevJ, [&](int j) {
            double v = fabs(RIref[j]);
            for (int r = 1; r < ni; ++r) v = nanmax2(v, fabs(RIref[(int64_t)r * n + j]));
            return v;
        }, red_am);
        ArgMax ic = argmax_excl(m, prevI, [&](int i) {
            double v = fabs(RJref[i]);
            for (int r = 1; r < nj; ++r) v = nanmax2(v, fabs(RJref[(int64_t)r * m + i]));
            return v;
        }, red_am);
        int Istar = ic.i, Jstar = jc.i;
        if (Istar < 0 || Jstar < 0) { flags |= 4; break; }  // everything excluded
        if (ic.v > jc.v) {
            residual_rows<HS>(C, Istar, 1, 3, RIs, n);
            __syncthreads();
            Jstar = argmax_excl(n, prevJ, [&](int j) { return fabs(RIs[j]); }, red_am).i;
            residual_cols<HS>(C, Jstar, 1, 3, RJs, m);
        } else {
            residual_cols<HS>(C, Jstar, 1, 3, RJs, m);
            __syncthreads();
            Istar = argmax_excl(m, prevI, [&](int i) { return fabs(RJs[i]); }, red_am).i;
            residual_rows<HS>(C, Istar, 1, 3, RIs, n);
        }
        __syncthreads();
        const double alpha = RIs[Jstar], alpha1 = RIs[(int64_t)n + Jstar], alpha2 = RIs[2 * (int64_t)n + Jstar];
        if (fabs(alpha) < 1e-4) break;
        if (threadIdx.x == 0) {
            prevI[Istar >> 5] |= 1u << (Istar & 31);
            prevJ[Jstar >> 5] |= 1u << (Jstar & 31);
        }
        if (C.k >= T.kmax) { flags |= 1; break; }
        const int q = C.k;
        const double d0 = alpha + 1e-16, d1 = alpha1 + 1e-16, d2 = alpha2 + 1e-16;
        const bool zeroB = fabs(alpha2) < 1e-10;
        for (int i = threadIdx.x; i < m; i += blockDim.x)
            for (int c = 0; c < 3; ++c) C.U[((int64_t)q * 3 + c) * m + i] = RJs[(int64_t)c * m + i];
        for (int j = threadIdx.x; j < n; j += blockDim.x) {
            C.V[((int64_t)q * 3 + 0) * n + j] = RIs[j] / d0;
            C.V[((int64_t)q * 3 + 1) * n + j] = RIs[(int64_t)n + j] / d1;
            C.V[((int64_t)q * 3 + 2) * n + j] = zeroB ? 0.0 : RIs[2 * (int64_t)n + j] / d2;
        }
        // step size ||u_k|| * ||v_k / alpha|| (A1)
        double su = 0.0, sv = 0.0;
        for (int i = threadIdx.x; i < m; i += blockDim.x) su += RJs[i] * RJs[i];
        for (int j = threadIdx.x; j < n; j += blockDim.x) { double w = RIs[j] / alpha; sv += w * w; }
        su = block_sum(su, red_d);
        sv = block_sum(sv, red_d);
        const double step = sqrt(su * sv);
        bool stop;
        if (rel_mode) {
            // ||S_k||_F^2 = ||S_{k-1}||^2 + 2 sum_{p<k} (u_p.u_k)(v_p.v_k) + ||u_k||^2 ||v_k||^2
            double cross = 0.0;
            for (int p = 0; p < q; ++p) {
                double uu = 0.0, vv = 0.0;
                for (int i = threadIdx.x; i < m; i += blockDim.x)
                    uu += C.U[((int64_t)p * 3) * m + i] * RJs[i];
                for (int j = threadIdx.x; j < n; j += blockDim.x)
                    vv += C.V[((int64_t)p * 3) * n + j] * (RIs[j] / alpha);
                uu = block_sum(uu, red_d);
                vv = block_sum(vv, red_d);
                cross += uu * vv;
            }
            frob2 += 2.0 * cross + su * sv;
            stop = step <= eps * sqrt(fabs(frob2));
        } else {
            stop = step < eps;
        }
        C.k = q + 1;
        __syncthreads();
        if (stop) break;
        if (it == max_iter - 1) break;
        if (Iref <= Istar && Istar < Iref + 3) {
            Iref = reset_row(Iref, ni);
            if (s_scan) break;
        } else {
            for (int r = 0; r < ni; ++r) {
                const double ur = C.U[((int64_t)q * 3) * m + Iref + r];
                for (int j = threadIdx.x; j < n; j += blockDim.x)
                    RIref[(int64_t)r * n + j] = __dsub_rn(RIref[(int64_t)r * n + j], __dmul_rn(ur, RIs[j] / alpha));
            }
            __syncthreads();
        }
        if (Jref <= Jstar && Jstar < Jref + 3) {
            Jref = reset_col(Jref, nj);
            if (s_scan) break;
        } else {
            for (int r = 0; r < nj; ++r) {
                const double vr = RIs[Jref + r] / alpha;
                for (int i = threadIdx.x; i < m; i += blockDim.x)
                    RJref[(int64_t)r * m + i] = __dsub_rn(RJref[(int64_t)r * m + i], __dmul_rn(vr, RJs[i]));
            }
            __syncthreads();
        }
    }
    // An all-zero B factor is dropped (src/Hmatrix.py:769-775).
    int nz = 0;
    for (int64_t e = threadIdx.x; e < (int64_t)C.k * m; e += blockDim.x) {
        int q = (int)(e / m), i = (int)(e % m);
        if (C.U[((int64_t)q * 3 + 2) * m + i] != 0.0) { nz = 1; }
    }
    nz = __syncthreads_or(nz);
    if (!nz) flags |= 2;
    if (threadIdx.x == 0) {
        rank_out[blockIdx.x] = C.k;
        flag_out[blockIdx.x] = flags;
    }
}

PQ3D_EXPORT int pq3d_aca_batched(const double *d_xg, const double *d_ev, const void *d_rec,
                                 const int32_t *d_rowlist, const int32_t *d_collist, const void *d_tasks,
                                 int64_t n_tasks, double *d_ws, double mu, double lam, double eps,
                                 int rel_mode, int max_mn, int32_t *d_rank, int32_t *d_flags,
                                 const void *d_hs, int hs_mode, cudaStream_t stream)
{
    if (n_tasks < 0 || max_mn < 0) return PQ3D_ERR_ARG;
    if (hs_mode < 0 || hs_mode > 2 || (hs_mode && !d_hs)) return PQ3D_ERR_ARG;
    if (n_tasks == 0) return PQ3D_OK;
    if (!d_xg || !d_ev || !d_rec || !d_rowlist || !d_collist || !d_tasks || !d_ws || !d_rank || !d_flags)
        return PQ3D_ERR_ARG;
    size_t smem = (size_t)(2 * ((max_mn + 31) / 32) + 2) * sizeof(uint32_t);
    if (smem > 200 * 1024) return PQ3D_ERR_ARG;
    if (smem > 48 * 1024) {
        if (hs_mode) PQ3D_CHECK(cudaFuncSetAttribute(k_aca<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        else PQ3D_CHECK(cudaFuncSetAttribute(k_aca<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    }
    for (int64_t t0 = 0; t0 < n_tasks; t0 += 65535) {
        int64_t nt = n_tasks - t0 < 65535 ? n_tasks - t0 : 65535;
        if (hs_mode)
            k_aca<true><<<(unsigned)nt, ACA_THREADS, smem, stream>>>(
                d_xg, d_ev, (const SrcRec *)d_rec, d_rowlist, d_collist, (const AcaTask *)d_tasks + t0, d_ws, mu,
                lam, eps, rel_mode, d_rank + t0, d_flags + t0, (const HsRec *)d_hs, hs_mode, max_mn);
        else
            k_aca<false><<<(unsigned)nt, ACA_THREADS, smem, stream>>>(
                d_xg, d_ev, (const SrcRec *)d_rec, d_rowlist, d_collist, (const AcaTask *)d_tasks + t0, d_ws, mu,
                lam, eps, rel_mode, d_rank + t0, d_flags + t0, nullptr, 0, max_mn);
    }
    return pq3d_launch_status();
}

// ---------------------------------------------------------------- packing
// Pack one ACA task's factors into the matvec layout (tree order).
struct PackTask {
    int64_t ws_off;      // ACA workspace of this task
    int64_t u_off, v_off; // block offsets in the packed U / V arrays
    int64_t rows_off, cols_off;
    int32_t m, n, kmax, k, pass, kS, kD, K, Q, r0, c0, zeroB;
};

template <typename T>
__device__ inline T cvt(double v);
template <>
__device__ inline double cvt<double>(double v) { return v; }
template <>
__device__ inline float cvt<float>(double v) { return (float)v; }
template <>
__device__ inline __nv_bfloat16 cvt<__nv_bfloat16>(double v) { return __float2bfloat16_rn((float)v); }

template <typename T, int CW>
__global__ void k_aca_pack(const PackTask *__restrict__ tasks, const double *__restrict__ ws,
                           const int32_t *__restrict__ rowlist, const int32_t *__restrict__ collist,
                           const int32_t *__restrict__ iperm, T *__restrict__ Uout, T *__restrict__ Vout)
{
    const PackTask P = tasks[blockIdx.x];
    const double *U = ws + P.ws_off;
    const double *V = U + (int64_t)P.kmax * 3 * P.m;
    const int32_t *rows = rowlist + P.rows_off, *cols = collist + P.cols_off;
    // U: q in this pass's range
    const int qoff = P.pass == 0 ? 0 : P.kS;
    for (int64_t e = threadIdx.x; e < (int64_t)P.k * 3 * P.m; e += blockDim.x) {
        int i = (int)(e % P.m);
        int c = (int)((e / P.m) % 3);
        int q = (int)(e / ((int64_t)3 * P.m));
        double v = (c == 2 && P.zeroB) ? 0.0 : U[((int64_t)q * 3 + c) * P.m + i];
        int it = iperm[rows[i]] - P.r0;
        Uout[P.u_off + u_index(P.m, it, c, qoff + q, CW)] = cvt<T>(v);
    }
    // V rows: S pass rows c*kS + q ; D pass rows 3kS + c*kD + q
    for (int64_t e = threadIdx.x; e < (int64_t)P.k * 3 * P.n; e += blockDim.x) {
        int j = (int)(e % P.n);
        int c = (int)((e / P.n) % 3);
        int q = (int)(e / ((int64_t)3 * P.n));
        double v = (c == 2 && P.zeroB) ? 0.0 : V[((int64_t)q * 3 + c) * P.n + j];
        int jt = iperm[cols[j]] - P.c0;
        int row = P.pass == 0 ? c * P.kS + q : 3 * P.kS + c * P.kD + q;
        Vout[P.v_off + v_index(P.Q, row, P.c0 % CW + jt, CW)] = cvt<T>(v);
    }
}

PQ3D_EXPORT size_t pq3d_pack_task_bytes(void) { return sizeof(PackTask); }

// dtype: 0 = FP64 (CW 2), 1 = FP32 (CW 4), 2 = BF16 (CW 8).  Output arrays must be zeroed.
PQ3D_EXPORT int pq3d_aca_pack(const void *d_tasks, int64_t n_tasks, const double *d_ws, const int32_t *d_rowlist,
                              const int32_t *d_collist, const int32_t *d_iperm, int dtype, void *d_U, void *d_V,
                              cudaStream_t stream)
{
    if (n_tasks < 0) return PQ3D_ERR_ARG;
    if (n_tasks == 0) return PQ3D_OK;
    if (!d_tasks || !d_ws || !d_rowlist || !d_collist || !d_iperm || !d_U || !d_V) return PQ3D_ERR_ARG;
    for (int64_t t0 = 0; t0 < n_tasks; t0 += 65535) {
        unsigned nt = (unsigned)(n_tasks - t0 < 65535 ? n_tasks - t0 : 65535);
        const PackTask *tk = (const PackTask *)d_tasks + t0;
        if (dtype == 0)
            k_aca_pack<double, 2><<<nt, 256, 0, stream>>>(tk, d_ws, d_rowlist, d_collist, d_iperm, (double *)d_U, (double *)d_V);
        else if (dtype == 1)
            k_aca_pack<float, 4><<<nt, 256, 0, stream>>>(tk, d_ws, d_rowlist, d_collist, d_iperm, (float *)d_U, (float *)d_V);
        else if (dtype == 2)
            k_aca_pack<__nv_bfloat16, 8><<<nt, 256, 0, stream>>>(tk, d_ws, d_rowlist, d_collist, d_iperm,
                                                                (__nv_bfloat16 *)d_U, (__nv_bfloat16 *)d_V);
        else
            return PQ3D_ERR_ARG;
    }
    return pq3d_launch_status();
}
