// Batched H-matvec: the six elastic operators applied to the slip-rate
// deficit in one pass (replaces BlockTree.blocks_process_MVM,
// src/Hmatrix.py:1445-1538, called six times per step by QDsim.simu_forward,
// src/QDsim.py:906-917).
//
// Inputs are in cluster-tree order.  x is interleaved, x[2j+s] = deficit of
// element j for slip s (0 strike, 1 dip).  Output y[3i+c] = (A1s x1 + A1d x2,
// A2s x1 + A2d x2, Bs x1 + Bd x2) for c = 0, 1, 2.
//
// Work is split into warp items (hm_layout.cuh).  Lanes run over block rows
// and each lane streams 96 (dense) / 48 (U) / 16 (V) contiguous bytes per
// column group, so every warp load is a contiguous run of the packed operator.
// Each dense (block, column chunk) and each low-rank block writes its own
// per-row partial sums ("slots"); the row reduction adds a row's slots in a
// fixed order, so results are bitwise reproducible (no atomics).
//
// Launch sequence (stream-ordered, no host sync):
//   k_dense_v   dense items and V items (t partials = V x per column chunk)
//   k_treduce   sum t partials per low-rank block -> t[block][3][K]
//   k_u         U items: slot rows += U_c t_c
//   k_rowsum    y[i] = sum of row i's slots (FP64), plus optional loading terms
#include "pq3d_common.cuh"
#include "hm_layout.cuh"
#include <cuda_bf16.h>

using namespace pq3d;

template <typename T>
struct Vec16;  // 16-byte vector of T
template <>
struct Vec16<float> {
    float v[4];
};
template <>
struct Vec16<double> {
    double v[2];
};
template <>
struct Vec16<__nv_bfloat16> {
    __nv_bfloat16 v[8];
};

template <typename T>
__device__ __forceinline__ Vec16<T> ld_stream(const T *p)
{
    // Streamed once per matvec: read-only path, no L1 allocation.
    int4 r;
    asm volatile("ld.global.nc.L1::no_allocate.v4.s32 {%0,%1,%2,%3}, [%4];"
                 : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w)
                 : "l"(p));
    Vec16<T> o;
    memcpy(&o, &r, 16);
    return o;
}

template <typename T>
__device__ __forceinline__ float tof(T v);
template <>
__device__ __forceinline__ float tof<float>(float v) { return v; }
template <>
__device__ __forceinline__ float tof<__nv_bfloat16>(__nv_bfloat16 v) { return __bfloat162float(v); }

template <typename TA, typename T>
__device__ __forceinline__ TA widen(T v)
{
    return (TA)tof(v);
}
template <>
__device__ __forceinline__ double widen<double, double>(double v) { return v; }

// ------------------------------------------------------------------ kernel 1
template <typename TD, typename TL, typename TA>
__global__ void __launch_bounds__(256)
k_dense_v(const DenseItem *__restrict__ ditems, int64_t n_ditems, const VItem *__restrict__ vitems,
          int64_t n_vitems, const TD *__restrict__ D, const TL *__restrict__ Vd, const TA *__restrict__ x,
          TA *__restrict__ slots, TA *__restrict__ tpart)
{
    constexpr int CWD = 16 / sizeof(TD);
    constexpr int CWV = 16 / sizeof(TL);
    const int lane = threadIdx.x & 31;
    const int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    if (w < n_ditems) {
        const DenseItem it = ditems[w];
        const int r = it.r + lane;
        const bool act = r < it.m;
        TA acc[3] = {0, 0, 0};
        const TD *p = D + it.off + (int64_t)r * 6 * CWD;
        const int64_t gstride = (int64_t)it.m * 6 * CWD;
        p += (int64_t)it.g0 * gstride;
        const TA *xp = x + 2 * ((int64_t)it.c0 + (int64_t)it.g0 * CWD);
#pragma unroll 2
        for (int g = it.g0; g < it.g1; ++g) {
            TA xs[2 * CWD];
#pragma unroll
            for (int t = 0; t < 2 * CWD; ++t) xs[t] = xp[t];
            if (act) {
#pragma unroll
                for (int c = 0; c < 3; ++c) {
#pragma unroll
                    for (int s = 0; s < 2; ++s) {
                        Vec16<TD> d = ld_stream(p + (2 * c + s) * CWD);
#pragma unroll
                        for (int t = 0; t < CWD; ++t) acc[c] += widen<TA>(d.v[t]) * xs[2 * t + s];
                    }
                }
            }
            p += gstride;
            xp += 2 * CWD;
        }
        if (act) {
#pragma unroll
            for (int c = 0; c < 3; ++c) slots[3 * ((int64_t)it.slot + r) + c] = acc[c];
        }
        return;
    }
    const int64_t wv = w - n_ditems;
    if (wv >= n_vitems) return;
    const VItem it = vitems[wv];
    const int q = it.q + lane;
    if (q >= it.Q) return;
    const int s = q < 3 * it.kS ? 0 : 1;
    TA acc = 0;
    const TL *p = Vd + it.off + ((int64_t)it.g0 * it.Q + q) * CWV;
    const int64_t gstride = (int64_t)it.Q * CWV;
    const TA *xp = x + 2 * ((int64_t)it.c0 + (int64_t)it.g0 * CWV) + s;
#pragma unroll 4
    for (int g = it.g0; g < it.g1; ++g) {
        Vec16<TL> d = ld_stream(p);
#pragma unroll
        for (int t = 0; t < CWV; ++t) acc += widen<TA>(d.v[t]) * xp[2 * t];
        p += gstride;
        xp += 2 * CWV;
    }
    tpart[it.tp + q] = acc;
}

// ------------------------------------------------------------------ kernel 2
// t[tb + c*K + q] = sum over chunks of the partial V x rows (zero in the K padding).
struct TBlock {
    int32_t kS, kD, K, Q, tp, nch, tb, pad;
};

template <typename TA>
__global__ void k_treduce(const TBlock *__restrict__ tb, int64_t n_blocks, const TA *__restrict__ tpart,
                          TA *__restrict__ t)
{
    const int64_t b = blockIdx.x;
    if (b >= n_blocks) return;
    const TBlock B = tb[b];
    for (int e = threadIdx.x; e < 3 * B.K; e += blockDim.x) {
        const int c = e / B.K, q = e % B.K;
        TA v = 0;
        int row = -1;
        if (q < B.kS) row = c * B.kS + q;
        else if (q < B.kS + B.kD) row = 3 * B.kS + c * B.kD + (q - B.kS);
        if (row >= 0)
            for (int ch = 0; ch < B.nch; ++ch) v += tpart[B.tp + (int64_t)ch * B.Q + row];
        t[B.tb + e] = v;
    }
}

// ------------------------------------------------------------------ kernel 3
template <typename TL, typename TA>
__global__ void __launch_bounds__(256)
k_u(const UItem *__restrict__ items, int64_t n_items, const TL *__restrict__ U, const TA *__restrict__ t,
    TA *__restrict__ slots)
{
    constexpr int CW = 16 / sizeof(TL);
    const int lane = threadIdx.x & 31;
    const int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    if (w >= n_items) return;
    const UItem it = items[w];
    const int r = it.r + lane;
    if (r >= it.m) return;
    TA acc[3] = {0, 0, 0};
    const TL *p = U + it.off + (int64_t)r * 3 * CW;
    const int64_t gstride = (int64_t)it.m * 3 * CW;
    const TA *tp = t + it.tp;  // t[c*K + q]
    const int ng = it.K / CW;
#pragma unroll 2
    for (int g = 0; g < ng; ++g) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            Vec16<TL> d = ld_stream(p + c * CW);
#pragma unroll
            for (int k = 0; k < CW; ++k) acc[c] += widen<TA>(d.v[k]) * tp[c * it.K + g * CW + k];
        }
        p += gstride;
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) slots[3 * ((int64_t)it.slot + r) + c] = acc[c];
}

// ------------------------------------------------------------------ kernel 4
// y[3i+c] = sum of row i's slots (in list order) + add[c][i] (FP64), for rows of leaf clusters.
template <typename TA>
__global__ void k_rowsum(int n, const int32_t *__restrict__ leaf_of_row, const int32_t *__restrict__ leaf_ptr,
                         const int32_t *__restrict__ leaf_off, const TA *__restrict__ slots,
                         const double *__restrict__ add0, const double *__restrict__ add1,
                         const double *__restrict__ add2, double *__restrict__ y)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int l = leaf_of_row[i];
    double a0 = 0, a1 = 0, a2 = 0;
    for (int k = leaf_ptr[l]; k < leaf_ptr[l + 1]; ++k) {
        const int64_t s = 3 * ((int64_t)leaf_off[k] + i);
        a0 += (double)slots[s];
        a1 += (double)slots[s + 1];
        a2 += (double)slots[s + 2];
    }
    if (add0) a0 += add0[i];
    if (add1) a1 += add1[i];
    if (add2) a2 += add2[i];
    y[3 * (int64_t)i] = a0;
    y[3 * (int64_t)i + 1] = a1;
    y[3 * (int64_t)i + 2] = a2;
}

// ------------------------------------------------------------------ host entry
// Packed operator description (device pointers) -- mirrors pq3d_hm_plan in include/pq3d.h.
struct HmPlan {
    int32_t n;             // elements
    int32_t dtype;         // 0: FP64 dense + FP64 low rank; 1: FP32 + FP32; 2: FP32 dense + BF16 low rank
    const void *dense;     // packed dense data
    const void *U;         // packed U factors
    const void *V;         // packed V factors
    const void *ditems;    // DenseItem[n_ditems]
    const void *vitems;    // VItem[n_vitems]
    const void *uitems;    // UItem[n_uitems]
    const void *tblocks;   // TBlock[n_lr]
    const int32_t *leaf_of_row, *leaf_ptr, *leaf_off;
    int64_t n_ditems, n_vitems, n_uitems, n_lr;
    int64_t n_slots, n_tpart, n_t;
};

PQ3D_EXPORT size_t pq3d_item_bytes(int kind)
{
    switch (kind) {
    case 0: return sizeof(DenseItem);
    case 1: return sizeof(VItem);
    case 2: return sizeof(UItem);
    case 3: return sizeof(TBlock);
    case 4: return sizeof(DenseBlock);
    case 5: return sizeof(HmPlan);
    }
    return 0;
}

template <typename TD, typename TL, typename TA>
static int run_matvec(const HmPlan &P, const TA *x, TA *slots, TA *tpart, TA *t, const double *add0,
                      const double *add1, const double *add2, double *y, cudaStream_t st)
{
    const int64_t warps1 = P.n_ditems + P.n_vitems;
    if (warps1 > 0) {
        int64_t blocks = (warps1 * 32 + 255) / 256;
        k_dense_v<TD, TL, TA><<<(unsigned)blocks, 256, 0, st>>>(
            (const DenseItem *)P.ditems, P.n_ditems, (const VItem *)P.vitems, P.n_vitems, (const TD *)P.dense,
            (const TL *)P.V, x, slots, tpart);
    }
    if (P.n_lr > 0) {
        k_treduce<TA><<<(unsigned)P.n_lr, 128, 0, st>>>((const TBlock *)P.tblocks, P.n_lr, tpart, t);
        int64_t blocks = (P.n_uitems * 32 + 255) / 256;
        if (blocks > 0)
            k_u<TL, TA><<<(unsigned)blocks, 256, 0, st>>>((const UItem *)P.uitems, P.n_uitems, (const TL *)P.U, t,
                                                          slots);
    }
    k_rowsum<TA><<<(P.n + 255) / 256, 256, 0, st>>>(P.n, P.leaf_of_row, P.leaf_ptr, P.leaf_off, slots, add0,
                                                     add1, add2, y);
    return pq3d_launch_status();
}

// y (n x 3, FP64, tree order) = K x (+ add_c).  x: interleaved deficit, FP64 for dtype 0 and
// FP32 otherwise, 2*(n + 16) entries with zero padding.  Scratch: slots (3*n_slots),
// tpart (n_tpart), t (n_t) in the accumulation type (FP64 for dtype 0, FP32 otherwise).
PQ3D_EXPORT int pq3d_hmatvec(const void *plan_host, const void *d_x, void *d_slots, void *d_tpart, void *d_t,
                             const double *d_add0, const double *d_add1, const double *d_add2, double *d_y,
                             cudaStream_t stream)
{
    if (!plan_host || !d_x || !d_slots || !d_y) return PQ3D_ERR_ARG;
    const HmPlan &P = *(const HmPlan *)plan_host;
    if (P.n <= 0) return PQ3D_ERR_ARG;
    if (P.n_lr > 0 && (!d_tpart || !d_t)) return PQ3D_ERR_ARG;
    switch (P.dtype) {
    case 0:
        return run_matvec<double, double, double>(P, (const double *)d_x, (double *)d_slots, (double *)d_tpart,
                                                  (double *)d_t, d_add0, d_add1, d_add2, d_y, stream);
    case 1:
        return run_matvec<float, float, float>(P, (const float *)d_x, (float *)d_slots, (float *)d_tpart,
                                               (float *)d_t, d_add0, d_add1, d_add2, d_y, stream);
    case 2:
        return run_matvec<float, __nv_bfloat16, float>(P, (const float *)d_x, (float *)d_slots, (float *)d_tpart,
                                                       (float *)d_t, d_add0, d_add1, d_add2, d_y, stream);
    }
    return PQ3D_ERR_ARG;
}
