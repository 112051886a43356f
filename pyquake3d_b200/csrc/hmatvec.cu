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
// and every warp load instruction reads one contiguous run of the packed
// operator (512 B for dense and U, four 128 B runs for V).
// Each dense (block, column chunk) and each low-rank block writes its own
// per-row partial sums ("slots"); the row reduction adds a row's slots in a
// fixed order, so results are bitwise reproducible (no atomics).
//
// Launch sequence (stream-ordered, no host sync):
//   k_dense_v   V items (t partials = V x per column chunk); in FP64 also the
//               dense items
//   k_du        (FP32 / BF16) the dense items, then per (low-rank block, row
//               range) a U task: t from its chunk partials in shared memory,
//               slot rows = U_c t_c.  Launched with programmatic stream
//               serialization, so its dense items run in k_dense_v's tail; the
//               U tasks wait for k_dense_v.
//   k_u         (FP64) the U tasks as a plain launch after k_dense_v.
//   k_rowsum    y[i] = sum of row i's slots (FP64), plus optional loading terms
//               (skipped when the step kernel sums the slots itself)
#include <algorithm>
#include "pq3d_common.cuh"
#include "hm_layout.cuh"
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <type_traits>

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
template <>
struct Vec16<__half> {
    __half v[8];
};
template <>
struct Vec16<uint8_t> {    // INT8 class: each byte holds b + 128, b in [-127, 127]
    uint32_t w[4];
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

// N values of T from an aligned address (N * sizeof(T) a multiple of 16), read-only path.
template <typename T, int N>
__device__ __forceinline__ void ld_vec(const T *p, T *o)
{
    static_assert((N * sizeof(T)) % 16 == 0, "16-byte multiples");
#pragma unroll
    for (int k = 0; k < (int)(N * sizeof(T) / 16); ++k) {
        const int4 r = __ldg(reinterpret_cast<const int4 *>(p) + k);
        memcpy(o + k * (16 / sizeof(T)), &r, 16);
    }
}

template <typename T>
__device__ __forceinline__ float tof(T v);
template <>
__device__ __forceinline__ float tof<float>(float v) { return v; }
template <>
__device__ __forceinline__ float tof<__nv_bfloat16>(__nv_bfloat16 v) { return __bfloat162float(v); }
template <>
__device__ __forceinline__ float tof<__half>(__half v) { return __half2float(v); }

// Byte k (0..3) of w as the float 2^23 + byte, minus 2^23 + 128: the signed value
// b of an INT8-class entry stored as b + 128, exactly, in one byte permute and one
// add (the integer-to-float conversion instruction issues at a fraction of that rate).
template <int k>
__device__ __forceinline__ float i8_at(uint32_t w)
{
    return __int_as_float((int)__byte_perm(w, 0x4B000000u, 0x7650u + k)) - 8388736.0f;
}

template <typename TA, typename T>
__device__ __forceinline__ TA widen(T v)
{
    return (TA)tof(v);
}
template <>
__device__ __forceinline__ double widen<double, double>(double v) { return v; }

// One V item: rows [q, q+nr) of a block's V (one slip), column groups [g0, g1):
// chunk partials of t = V x.  lane = 8 * jg + rr: rows q + rr + 8u (u < 4),
// column groups g0 + jg, g0 + jg + 4, ...; four rows per lane share each x slice.
template <typename TL, typename TA>
__device__ __forceinline__ void v_item(const VItem &it, int slip, const TL *__restrict__ Vd,
                                       const TA *__restrict__ x, int xstride, TA *__restrict__ tpart)
{
    constexpr int CWV = 16 / sizeof(TL);
    const int lane = threadIdx.x & 31;
    const int rr = lane & 7, jg = lane >> 3;
    TA acc[4] = {0, 0, 0, 0};
    if (rr < it.nr) {
        const TL *p = Vd + it.off + ((int64_t)(it.g0 + jg) * it.Q + it.q + rr) * CWV;
        const int64_t gstride = (int64_t)4 * it.Q * CWV;
        const TA *xp = x + (int64_t)(2 + slip) * xstride + it.c0 + (int64_t)(it.g0 + jg) * CWV;  // CWV-aligned
        const int nu = (it.nr - rr + 7) >> 3;   // rows of this lane (1..4)
#pragma unroll 2
        for (int g = it.g0 + jg; g < it.g1; g += 4) {
            TA xs[CWV];
            ld_vec<TA, CWV>(xp, xs);
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                if (u < nu) {
                    Vec16<TL> d = ld_stream(p + 8 * u * CWV);
                    if constexpr (std::is_same<TL, uint8_t>::value) {
#pragma unroll
                        for (int t = 0; t < 4; ++t) {
                            acc[u] += i8_at<0>(d.w[t]) * xs[4 * t];
                            acc[u] += i8_at<1>(d.w[t]) * xs[4 * t + 1];
                            acc[u] += i8_at<2>(d.w[t]) * xs[4 * t + 2];
                            acc[u] += i8_at<3>(d.w[t]) * xs[4 * t + 3];
                        }
                    } else {
#pragma unroll
                        for (int t = 0; t < CWV; ++t) acc[u] += widen<TA>(d.v[t]) * xs[t];
                    }
                }
            }
            p += gstride;
            xp += 4 * CWV;
        }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        acc[u] += __shfl_xor_sync(0xffffffffu, acc[u], 8);
        acc[u] += __shfl_xor_sync(0xffffffffu, acc[u], 16);
        if (jg == 0 && rr + 8 * u < it.nr) tpart[it.tp + it.q + rr + 8 * u] = acc[u];
    }
}

// ------------------------------------------------------------------ kernel 1
// Work item of warp w: dense items (lanes over block rows) first, then V items (up
// to 32 rows: 8 rows x 4 column groups per warp load, 4 rows per lane, then a
// 2-step shuffle reduction) writing chunk partials of t = V x.
template <typename TD, typename TL, typename TA>
__device__ __forceinline__ void dense_v_item(int64_t w, const DenseItem *__restrict__ ditems, int64_t n_ditems,
                                             const VItem *__restrict__ vitems, int64_t n_vitems,
                                             const TD *__restrict__ D, const TL *__restrict__ Vd,
                                             const TA *__restrict__ x, int xstride, TA *__restrict__ slots,
                                             TA *__restrict__ tpart)
{
    constexpr int CWD = 16 / sizeof(TD);
    const int lane = threadIdx.x & 31;
    if (w < n_ditems) {
        const DenseItem it = ditems[w];
        const int r = it.r + lane;
        const bool act = r < it.m;
        TA acc[3] = {0, 0, 0};
        const TD *p = D + it.off + (int64_t)r * CWD;           // [group][op][row][CW]
        const int64_t ostride = (int64_t)it.m * CWD, gstride = 6 * ostride;
        p += (int64_t)it.g0 * gstride;
        const TA *xp = x + 2 * ((int64_t)it.c0 + (int64_t)it.g0 * CWD);   // c0 is CWD-aligned
#pragma unroll 2
        for (int g = it.g0; g < it.g1; ++g) {
            TA xs[2 * CWD];
            ld_vec<TA, 2 * CWD>(xp, xs);
            if (act) {
#pragma unroll
                for (int c = 0; c < 3; ++c) {
#pragma unroll
                    for (int s = 0; s < 2; ++s) {
                        Vec16<TD> d = ld_stream(p + (2 * c + s) * ostride);
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
    v_item<TL, TA>(vitems[wv], vitems[wv].s, Vd, x, xstride, tpart);
}

// Kernel A: V items (and, in FP64, the dense items), one warp each.  Every CTA
// lets the dependent kernel (k_du) launch as soon as it starts: k_du's dense
// items do not read what this kernel writes and fill the SMs while its last wave
// runs; k_du's U tasks wait for it.
template <typename TD, typename TL, typename TA>
__global__ void __launch_bounds__(256)
k_dense_v(const DenseItem *__restrict__ ditems, int64_t n_ditems, const VItem *__restrict__ vitems,
          int64_t n_vitems, const TD *__restrict__ D, const TL *__restrict__ Vd, const TA *__restrict__ x,
          int xstride, TA *__restrict__ slots, TA *__restrict__ tpart)
{
    asm volatile("griddepcontrol.launch_dependents;");
    const int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    dense_v_item<TD, TL, TA>(w, ditems, n_ditems, vitems, n_vitems, D, Vd, x, xstride, slots, tpart);
}

// Sum of the nch chunk partials of one entry of t = V x (stride Q), in chunk
// order, with four independent loads in flight (a rolled loop waits one L2
// latency per chunk before a U task can start streaming).
template <typename TA>
__device__ __forceinline__ TA sum_partials(const TA *__restrict__ p, int nch, int Q)
{
    TA v = 0;
    int ch = 0;
    for (; ch + 4 <= nch; ch += 4) {
        const TA a0 = p[(int64_t)ch * Q], a1 = p[(int64_t)(ch + 1) * Q], a2 = p[(int64_t)(ch + 2) * Q],
                 a3 = p[(int64_t)(ch + 3) * Q];
        v += a0;
        v += a1;
        v += a2;
        v += a3;
    }
    for (; ch < nch; ++ch) v += p[(int64_t)ch * Q];
    return v;
}

// ------------------------------------------------------------------ kernel 2
// One CTA per (low-rank block, row range): sums the block's chunk partials of
// t = V x into shared memory, then its warps stream U (lanes over rows).
template <typename TA, int CW>
__device__ __forceinline__ void smem_vec(const TA *p, TA *o)
{
#pragma unroll
    for (int k = 0; k < CW; ++k) o[k] = p[k];
}
template <>
__device__ __forceinline__ void smem_vec<float, 8>(const float *p, float *o)
{
    const float4 a = reinterpret_cast<const float4 *>(p)[0], b = reinterpret_cast<const float4 *>(p)[1];
    o[0] = a.x; o[1] = a.y; o[2] = a.z; o[3] = a.w; o[4] = b.x; o[5] = b.y; o[6] = b.z; o[7] = b.w;
}
template <>
__device__ __forceinline__ void smem_vec<float, 4>(const float *p, float *o)
{
    const float4 a = reinterpret_cast<const float4 *>(p)[0];
    o[0] = a.x; o[1] = a.y; o[2] = a.z; o[3] = a.w;
}
template <>
__device__ __forceinline__ void smem_vec<float, 16>(const float *p, float *o)
{
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const float4 a = reinterpret_cast<const float4 *>(p)[k];
        o[4 * k] = a.x; o[4 * k + 1] = a.y; o[4 * k + 2] = a.z; o[4 * k + 3] = a.w;
    }
}
template <>
__device__ __forceinline__ void smem_vec<double, 2>(const double *p, double *o)
{
    const double2 a = reinterpret_cast<const double2 *>(p)[0];
    o[0] = a.x; o[1] = a.y;
}

template <typename TL, typename TA>
__device__ __forceinline__ void u_task(const UTask &T, const TL *__restrict__ U, const TA *__restrict__ tpart,
                                       TA *__restrict__ slots, TA *ts)
{
    constexpr int CW = 16 / sizeof(TL);
    for (int e = threadIdx.x; e < 3 * T.K; e += blockDim.x) {
        const int c = e / T.K, q = e % T.K;
        int row = -1;
        if (q < T.kS) row = c * T.kS + q;
        else if (q < T.kS + T.kD) row = 3 * T.kS + c * T.kD + (q - T.kS);
        TA v = 0;
        if (row >= 0)
            v = sum_partials<TA>(tpart + T.tp + row, T.nch, T.Q);
        ts[e] = v;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int ng = T.K / CW;
    const int64_t gstride = (int64_t)T.m * 3 * CW;   // one column group of U: 3 comps x m rows
    for (int rb = T.r0 + warp * 32; rb < T.r1; rb += blockDim.x) {
        const int r = rb + lane;
        if (r >= T.r1) break;
        TA acc[3] = {0, 0, 0};
        const TL *p = U + T.off + (int64_t)r * CW;             // [group][comp][row][CW]
        const int64_t cstride = (int64_t)T.m * CW;
#pragma unroll 2
        for (int g = 0; g < ng; ++g) {
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                Vec16<TL> d = ld_stream(p + c * cstride);
                TA tv[CW];
                smem_vec<TA, CW>(ts + c * T.K + g * CW, tv);
#pragma unroll
                for (int k = 0; k < CW; ++k) acc[c] += widen<TA>(d.v[k]) * tv[k];
            }
            p += gstride;
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) slots[3 * ((int64_t)T.slot + r) + c] = acc[c];
    }
}

// Kernel B: CTAs [0, n_dblocks) run dense items (eight warps, one item each);
// the remaining CTAs run one U task each.  Launched with programmatic stream
// serialization after k_v: the dense CTAs start while k_v finishes, and a U
// task waits (griddepcontrol.wait: k_v complete, its writes visible) before it
// reads the chunk partials of t.
template <typename TD, typename TL, typename TA>
__global__ void __launch_bounds__(256)
k_du(const DenseItem *__restrict__ ditems, int64_t n_ditems, int64_t n_dblocks, const UTask *__restrict__ tasks,
     const TD *__restrict__ D, const TL *__restrict__ U, const TA *__restrict__ x, TA *__restrict__ slots,
     const TA *__restrict__ tpart)
{
    if (blockIdx.x < n_dblocks) {
        const int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
        dense_v_item<TD, TL, TA>(w, ditems, n_ditems, nullptr, 0, D, nullptr, x, 0, slots, nullptr);
        return;
    }
    asm volatile("griddepcontrol.wait;" ::: "memory");
    extern __shared__ __align__(16) unsigned char smraw[];
    const UTask T = tasks[blockIdx.x - n_dblocks];
    u_task<TL, TA>(T, U, tpart, slots, reinterpret_cast<TA *>(smraw));
}


// FP64 path: the U tasks as their own launch after k_dense_v (dense and V items
// together), which measured faster at this precision than the split launch.
template <typename TL, typename TA>
__global__ void __launch_bounds__(256)
k_u(const UTask *__restrict__ tasks, const TL *__restrict__ U, const TA *__restrict__ tpart, TA *__restrict__ slots)
{
    constexpr int CW = 16 / sizeof(TL);
    extern __shared__ __align__(16) unsigned char smraw[];
    TA *ts = reinterpret_cast<TA *>(smraw);
    const UTask T = tasks[blockIdx.x];
    for (int e = threadIdx.x; e < 3 * T.K; e += blockDim.x) {
        const int c = e / T.K, q = e % T.K;
        int row = -1;
        if (q < T.kS) row = c * T.kS + q;
        else if (q < T.kS + T.kD) row = 3 * T.kS + c * T.kD + (q - T.kS);
        TA v = 0;
        if (row >= 0)
            v = sum_partials<TA>(tpart + T.tp + row, T.nch, T.Q);
        ts[e] = v;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int ng = T.K / CW;
    const int64_t gstride = (int64_t)T.m * 3 * CW;   // one column group of U: 3 comps x m rows
    for (int rb = T.r0 + warp * 32; rb < T.r1; rb += blockDim.x) {
        const int r = rb + lane;
        if (r >= T.r1) break;
        TA acc[3] = {0, 0, 0};
        const TL *p = U + T.off + (int64_t)r * CW;             // [group][comp][row][CW]
        const int64_t cstride = (int64_t)T.m * CW;
#pragma unroll 2
        for (int g = 0; g < ng; ++g) {
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                Vec16<TL> d = ld_stream(p + c * cstride);
                TA tv[CW];
                smem_vec<TA, CW>(ts + c * T.K + g * CW, tv);
#pragma unroll
                for (int k = 0; k < CW; ++k) acc[c] += widen<TA>(d.v[k]) * tv[k];
            }
            p += gstride;
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) slots[3 * ((int64_t)T.slot + r) + c] = acc[c];
    }
}

// ------------------------------------------------------------------ mixed storage
// Resident CTAs per SM the register allocation of k_v_mixed / k_du_mixed is held to
// (measured on B200 at 60k, mixed matvec: 6 and 5 gave 0.483 ms against 0.672 ms for
// the compiler's own choice at one CTA per SM and 0.499 ms for 5 and 5; both kernels are
// latency-bound streams.  With the INT8 V loop below, k_v_mixed at 4 CTAs (64 registers,
// no spill in its loops) beats 5 and 6: 440.9 / 444.6 / 460.1 us per 60k matvec).
#ifndef PQ3D_VMIX_MINB
#define PQ3D_VMIX_MINB 4
#endif
// k_du_mixed at 4 (in 256-thread units: 8 CTAs of 128 threads, 64 registers) with three U
// column groups in flight: 60k 438.0 -> 434.9 us, 20k 94.5 -> 93.8 us against 5 and two
// (its dense items gain, 183 -> 172 us alone, its U tasks lose, 131 -> 138 us).
#ifndef PQ3D_UMIX_MINB
#define PQ3D_UMIX_MINB 4
#endif
#ifndef PQ3D_UMIX_UNROLL
#define PQ3D_UMIX_UNROLL 3
#endif
constexpr int kUmixUnroll = PQ3D_UMIX_UNROLL;     // column groups of a U row in flight
// Storage code 3: FP32 dense near field; each low-rank block's ACA terms split
// into three classes stored as FP32, FP16 and INT8 (class arrays U_c, V_c in
// the layouts of hm_layout.cuh with CW = 4, 8, 16).  FP16 and INT8 columns of U
// and rows of V are stored normalised to their largest magnitude (INT8 as
// round(127 v / max)); the product's scale, one float per V row, multiplies the
// row's sum of chunk partials when a U task gathers t.  FP32 terms are stored
// as in the FP32 plan.  V items carry their class in bits 8+ of VItem::s.
struct UTaskM {
    int64_t off[3];            // block offsets in the FP32 / FP16 / INT8 U arrays
    int32_t m, r0, r1, slot;   // rows [r0, r1) of an m-row block; slot of block row 0
    int32_t K[3], kS[3], kD[3], Q[3], tp[3], nch[3], sb[3];  // per class (sb: scale base)
    int32_t pad;
};

// acc[c] += sum_q U_c[r, q] t_c[q] over one class's column groups.
template <typename TL>
__device__ __forceinline__ void u_row_class(const TL *__restrict__ Ub, int m, int r, int K, const float *ts,
                                            float acc[3])
{
    constexpr int CW = 16 / sizeof(TL);
    const int ng = K / CW;
    const TL *p = Ub + (int64_t)r * CW;                   // [group][comp][row][CW]
    const int64_t cstride = (int64_t)m * CW, gstride = 3 * cstride;
#pragma unroll kUmixUnroll
    for (int g = 0; g < ng; ++g) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            Vec16<TL> d = ld_stream(p + c * cstride);
            const float4 *t4 = reinterpret_cast<const float4 *>(ts + c * K + g * CW);
            if constexpr (std::is_same<TL, uint8_t>::value) {
                // t read four values at a time: 4 live registers instead of 16
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const float4 tv = t4[k];
                    acc[c] += i8_at<0>(d.w[k]) * tv.x;
                    acc[c] += i8_at<1>(d.w[k]) * tv.y;
                    acc[c] += i8_at<2>(d.w[k]) * tv.z;
                    acc[c] += i8_at<3>(d.w[k]) * tv.w;
                }
            } else {
#pragma unroll
                for (int k = 0; k < CW / 4; ++k) {
                    const float4 tv = t4[k];
                    acc[c] += tof(d.v[4 * k]) * tv.x;
                    acc[c] += tof(d.v[4 * k + 1]) * tv.y;
                    acc[c] += tof(d.v[4 * k + 2]) * tv.z;
                    acc[c] += tof(d.v[4 * k + 3]) * tv.w;
                }
            }
        }
        p += gstride;
    }
}

__device__ __forceinline__ void u_task_mixed(const UTaskM &T, const float *__restrict__ U32,
                                             const __half *__restrict__ U16, const uint8_t *__restrict__ U8,
                                             const float *__restrict__ tpart, const float *__restrict__ scales,
                                             float *__restrict__ slots, float *ts)
{
    const int base1 = 3 * T.K[0], base2 = 3 * (T.K[0] + T.K[1]);
#pragma unroll
    for (int cls = 0; cls < 3; ++cls) {
        const int K = T.K[cls], kS = T.kS[cls], kD = T.kD[cls];
        float *tc = ts + (cls == 0 ? 0 : (cls == 1 ? base1 : base2));
        for (int e = threadIdx.x; e < 3 * K; e += blockDim.x) {
            const int c = e / K, q = e % K;
            int row = -1;
            if (q < kS) row = c * kS + q;
            else if (q < kS + kD) row = 3 * kS + c * kD + (q - kS);
            float v = 0.f;
            if (row >= 0) {
                v = sum_partials<float>(tpart + T.tp[cls] + row, T.nch[cls], T.Q[cls]);
                if (cls > 0) v *= scales[T.sb[cls] + row];
            }
            tc[e] = v;
        }
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int rb = T.r0 + warp * 32; rb < T.r1; rb += blockDim.x) {
        const int r = rb + lane;
        if (r >= T.r1) break;
        float acc[3] = {0.f, 0.f, 0.f};
        if (T.K[0]) u_row_class<float>(U32 + T.off[0], T.m, r, T.K[0], ts, acc);
        if (T.K[1]) u_row_class<__half>(U16 + T.off[1], T.m, r, T.K[1], ts + base1, acc);
        if (T.K[2]) u_row_class<uint8_t>(U8 + T.off[2], T.m, r, T.K[2], ts + base2, acc);
#pragma unroll
        for (int c = 0; c < 3; ++c) slots[3 * ((int64_t)T.slot + r) + c] = acc[c];
    }
}

// A merged V item of the mixed storage: up to 32 rows (one class, one slip) taken from
// the low-rank blocks that share one column cluster, so their x slice is loaded once
// for all of them.  Lanes and summation order are those of v_item (8 rows x 4 column
// groups per warp load, up to 4 rows per lane, groups jg, jg + 4, ... per lane, then a
// 2-step shuffle reduction), so each row's sum is the one v_item forms for it.
template <typename TL>
__device__ __forceinline__ void v_item_m(const VItemM &it, int slip, const TL *__restrict__ Vd,
                                         const VRowRec *__restrict__ recs, const float *__restrict__ x, int xstride,
                                         float *__restrict__ tpart)
{
    constexpr int CWV = 16 / sizeof(TL);
    const int lane = threadIdx.x & 31;
    const int rr = lane & 7, jg = lane >> 3;
    const int nu = rr < it.nr ? (it.nr - rr + 7) >> 3 : 0;    // rows of this lane (0..4)
    // element offsets in the class array (the host keeps every class array below 2^32
    // elements), one register per row instead of a pointer's two
    uint32_t off[4];
    int32_t st4[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        off[u] = 0;
        st4[u] = 0;
        if (u < nu) {
            const VRowRec R = recs[it.rows + rr + 8 * u];
            off[u] = (uint32_t)(R.base + (int64_t)(it.g0 + jg) * R.stride);
            st4[u] = 4 * R.stride;
        }
    }
    float acc[4] = {0.f, 0.f, 0.f, 0.f};
    if (nu > 0) {
        const float *xp = x + (int64_t)(2 + slip) * xstride + it.c0 + (int64_t)(it.g0 + jg) * CWV;  // CWV-aligned
#pragma unroll 2
        for (int g = it.g0 + jg; g < it.g1; g += 4) {
            if constexpr (std::is_same<TL, uint8_t>::value) {
                // INT8: the rows' units first, then x four values at a time (4 live registers
                // instead of 16 for the slice); per row the summation order of the other
                // classes' loop (column t, then its four entries).  Units of rows beyond nu
                // hold the byte 128, which decodes to zero, and are never stored.
                // (Measured at 60k: V products 205 -> 153 us, mixed matvec 460 -> 441 us.)
                Vec16<TL> d[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    if (u < nu) d[u] = ld_stream(Vd + off[u]);
                    else d[u].w[0] = d[u].w[1] = d[u].w[2] = d[u].w[3] = 0x80808080u;
                }
                const float4 *x4 = reinterpret_cast<const float4 *>(xp);
#pragma unroll
                for (int t = 0; t < 4; ++t) {
                    const float4 xv = __ldg(x4 + t);
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        acc[u] += i8_at<0>(d[u].w[t]) * xv.x;
                        acc[u] += i8_at<1>(d[u].w[t]) * xv.y;
                        acc[u] += i8_at<2>(d[u].w[t]) * xv.z;
                        acc[u] += i8_at<3>(d[u].w[t]) * xv.w;
                    }
                }
#pragma unroll
                for (int u = 0; u < 4; ++u) off[u] += st4[u];
            } else {
                float xs[CWV];
                ld_vec<float, CWV>(xp, xs);
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    if (u < nu) {
                        Vec16<TL> d = ld_stream(Vd + off[u]);
#pragma unroll
                        for (int t = 0; t < CWV; ++t) acc[u] += widen<float>(d.v[t]) * xs[t];
                        off[u] += st4[u];
                    }
                }
            }
            xp += 4 * CWV;
        }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        acc[u] += __shfl_xor_sync(0xffffffffu, acc[u], 8);
        acc[u] += __shfl_xor_sync(0xffffffffu, acc[u], 16);
        if (jg == 0 && u < nu) tpart[recs[it.rows + rr + 8 * u].out] = acc[u];
    }
}

// V items of all three classes (the class picks the element type).  Persistent: the
// grid is the resident CTAs, and warp w works through its own list of items
// [vwarp[w], vwarp[w + 1]) with no barrier, so a CTA never holds its slot for its
// slowest warp.  The host fills the lists largest item first, each into the least
// loaded warp, so the warps end together.  (One item per warp, as CTAs of 8 items,
// left the SMs busy 64% of the kernel's time at 20k: items differ in size and a CTA
// lives as long as its largest.)
__global__ void __launch_bounds__(256, PQ3D_VMIX_MINB)
k_v_mixed(const VItemM *__restrict__ vitems, const int32_t *__restrict__ vwarp, int n_vwarp,
          const VRowRec *__restrict__ recs, const float *__restrict__ V32, const __half *__restrict__ V16,
          const uint8_t *__restrict__ V8, const float *__restrict__ x, int xstride, float *__restrict__ tpart)
{
    asm volatile("griddepcontrol.launch_dependents;");
    const int w = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5);
    if (w >= n_vwarp) return;
    const int i1 = vwarp[w + 1];
    for (int i = vwarp[w]; i < i1; ++i) {
        const VItemM it = vitems[i];
        const int cls = it.s >> 8, slip = it.s & 255;
        if (cls == 0) v_item_m<float>(it, slip, V32, recs, x, xstride, tpart);
        else if (cls == 1) v_item_m<__half>(it, slip, V16, recs, x, xstride, tpart);
        else v_item_m<uint8_t>(it, slip, V8, recs, x, xstride, tpart);
    }
}

// Resident CTAs of k_v_mixed on the current device (its persistent grid), per device.
static int vmix_ctas()
{
    static int cached[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    if (dev >= 0 && dev < 64 && cached[dev] > 0) return cached[dev];
    int sms = 0, per = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_v_mixed, 256, 0) != cudaSuccess || per <= 0) return 0;
    if (dev >= 0 && dev < 64) cached[dev] = sms * per;
    return sms * per;
}

// Dense items, then the mixed U tasks (programmatic dependent launch after k_v_mixed,
// as k_du after k_dense_v).
// 128 threads per CTA: half of the mixed U tasks cover blocks of 64-127 rows (one row
// per thread), which left most of a 256-thread CTA idle; with the same registers per
// SM, twice the CTAs stay resident (60k mixed matvec 478 -> 461 us, 20k 104 -> 98 us).
#ifndef PQ3D_UMIX_THREADS
#define PQ3D_UMIX_THREADS 128
#endif
__global__ void __launch_bounds__(PQ3D_UMIX_THREADS, PQ3D_UMIX_MINB * 256 / PQ3D_UMIX_THREADS)
k_du_mixed(const DenseItem *__restrict__ ditems, int64_t n_ditems, int64_t n_dblocks,
           const UTaskM *__restrict__ tasks, const float *__restrict__ D, const float *__restrict__ U32,
           const __half *__restrict__ U16, const uint8_t *__restrict__ U8, const float *__restrict__ x,
           float *__restrict__ slots, const float *__restrict__ tpart, const float *__restrict__ scales)
{
    if (blockIdx.x < n_dblocks) {
        const int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
        dense_v_item<float, float, float>(w, ditems, n_ditems, nullptr, 0, D, nullptr, x, 0, slots, nullptr);
        return;
    }
    // The task's U rows do not depend on the V kernel: start bringing them into L2 (one bulk
    // prefetch per class, column group and component: rows [r0, r1), 16 B each) before
    // waiting for the V partials and gathering t.  Measured at 60k: 432.7 -> 420.6 us per
    // mixed matvec, 20k 93.9 -> 90.4 us (the prefetches run during the V kernel's tail).
    const UTaskM T = tasks[blockIdx.x - n_dblocks];
    const int nr = T.r1 - T.r0;
    if (nr > 0) {
        const int n0 = 3 * (T.K[0] / 4), n1 = 3 * (T.K[1] / 8), n2 = 3 * (T.K[2] / 16);
        for (int e = threadIdx.x; e < n0 + n1 + n2; e += blockDim.x) {
            const unsigned char *base;
            int64_t off;
            int q;
            if (e < n0) { base = (const unsigned char *)U32; off = T.off[0] * 4; q = e; }
            else if (e < n0 + n1) { base = (const unsigned char *)U16; off = T.off[1] * 2; q = e - n0; }
            else { base = (const unsigned char *)U8; off = T.off[2]; q = e - n0 - n1; }
            // run q = 3 g + c (column group g, component c) starts at unit (3 g + c) m + r0
            const unsigned char *p = base + off + ((int64_t)q * T.m + T.r0) * 16;
            asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(nr * 16) : "memory");
        }
    }
    asm volatile("griddepcontrol.wait;" ::: "memory");
    extern __shared__ __align__(16) unsigned char smraw[];
    u_task_mixed(T, U32, U16, U8, tpart, scales, slots, reinterpret_cast<float *>(smraw));
}

// ------------------------------------------------------------------ mixed storage, streamed
// The products of k_v_mixed / k_du_mixed with every byte of the packed operator
// moved by bulk copies.  Each task reads contiguous runs, so in every CTA one
// producer thread streams them with 1-D cp.async.bulk (global -> shared,
// completion counted in bytes on the stage's "full" mbarrier) into a ring of
// ST_STAGES stages, while eight consumer warps compute from shared memory and
// release each stage on its "empty" mbarrier.  The CTAs are persistent: each
// works through its own task list (balanced by bytes on the host), and the ring
// runs on across task boundaries, so a small task costs no pipeline start-up.
// The first piece of every task is what its consumers need besides the operator
// (the x slices of its columns, or the block's t), so no task waits on a load.
//   phase A, k_stream (kind 0 dense, kind 1 V):
//     dense task: rows [r0, r1) (<= 128) of a dense block, column groups [g0, g1);
//       x piece: the interleaved (strike, dip) deficit of its columns; data
//       pieces: whole column groups, [group][6 operators][rows][16 B].
//     V task: all Q rows of one term class of one low-rank block over column
//       groups [g0, g1); x piece: the strike and dip planes of its columns; data
//       pieces: whole groups, [group][Q][16 B].
//   k_t_gather: per low-rank block, t of every class (sum of the V partials over
//     the column chunks, times the FP16 / INT8 scales) into one contiguous run.
//   phase B, k_stream (kind 2 U): rows [r0, r1) (<= 256) of a low-rank block; t
//     piece, then per class and column group the three components' row runs.
// A piece is a flat array of 16-byte units; consumer thread tid owns units tid,
// tid + 256 and tid + 512 of every piece, whose (group offset, operator or
// component, row) are the same in all full pieces of a task, so it accumulates
// in registers, and the owned partial sums are reduced per row in shared memory
// at the end of the task (fixed order: results are reproducible).  All waits are
// bounded (ST_SPIN polls); a timeout stores 1 in *status, a task of a size the
// plan builder never produces stores 2 and is skipped by producer and consumers
// alike, and the producer waits (bounded) for the copies it issued before exit.
constexpr int ST_STAGES = 4;
constexpr int ST_STAGE_BYTES = 12288;
constexpr int ST_CONSUMERS = 256;
constexpr int ST_THREADS = ST_CONSUMERS + 32;
constexpr int ST_BUF = 3072;              // floats of a task's x slices or t in shared memory
constexpr long long ST_SPIN = 1ll << 22;

struct StreamTask {
    int64_t off, off1, off2;   // dense: float offset of the block in D; V: element offset of the block in the
                               // class's V array; U: element offsets in the FP32 / FP16 / INT8 U arrays
    int32_t kind, cls;         // 0 dense, 1 V, 2 U; V: term class
    int32_t m, r0, r1;         // dense / U: block rows and the task's row range; V: Q rows of the class
    int32_t g0, g1, c0;        // dense / V: column groups, the block's aligned first column
    int32_t out;               // dense / U: slot of block row 0; V: tpart offset of this chunk
    int32_t kS3;               // V: rows below kS3 use the strike plane
    int32_t K0, K1, K2, tb;    // U: class column counts, offset of the block's t in tfull
};

struct TGather {               // one low-rank block: its classes' V rows, partials, scales, t offset
    int32_t K[3], kS[3], kD[3], Q[3], tp[3], nch[3], sb[3], tb, pad;
};

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *b, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *b, unsigned bytes)
{
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}"
                 ::"r"(smem_addr(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *b)
{
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}"
                 ::"r"(smem_addr(b)) : "memory");
}
// Bounded wait for the phase of parity `parity` to complete; false on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t *b, unsigned parity)
{
    const uint32_t a = smem_addr(b);
    for (long long i = 0; i < ST_SPIN; ++i) {
        uint32_t ok;
        asm volatile("{\n\t.reg .pred p;\n\t"
                     "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}"
                     : "=r"(ok) : "r"(a), "r"(parity) : "memory");
        if (ok) return true;
    }
    return false;
}
// 1-D bulk copy global -> this CTA's shared memory; completion counted on `bar`.
// dst, src 16-byte aligned, bytes a multiple of 16 (the layouts guarantee both).
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, uint64_t *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ void consumers_sync() { asm volatile("bar.sync 1, %0;" ::"n"(ST_CONSUMERS) : "memory"); }

// dot of one 16-byte unit of class element type TL with CW floats
template <typename TL>
__device__ __forceinline__ float dot16(const unsigned char *u, const float *xv)
{
    const int4 r = *reinterpret_cast<const int4 *>(u);
    Vec16<TL> d;
    memcpy(&d, &r, 16);
    float a = 0.f;
    if constexpr (std::is_same<TL, uint8_t>::value) {
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            a += i8_at<0>(d.w[t]) * xv[4 * t];
            a += i8_at<1>(d.w[t]) * xv[4 * t + 1];
            a += i8_at<2>(d.w[t]) * xv[4 * t + 2];
            a += i8_at<3>(d.w[t]) * xv[4 * t + 3];
        }
    } else {
        constexpr int CW = 16 / sizeof(TL);
#pragma unroll
        for (int t = 0; t < CW; ++t) a += tof(d.v[t]) * xv[t];
    }
    return a;
}

__device__ __forceinline__ int cw_of(int cls) { return cls == 0 ? 4 : (cls == 1 ? 8 : 16); }

// Sizes the plan builder produces; anything else is skipped (status 2).
__device__ __forceinline__ bool task_ok(const StreamTask &T)
{
    const int G = T.g1 - T.g0;
    if (T.kind == 0) {
        const int R = T.r1 - T.r0;
        return R >= 1 && R <= 128 && T.r0 >= 0 && T.r1 <= T.m && G >= 1 && 8 * G <= ST_BUF;
    }
    if (T.kind == 1)
        return T.cls >= 0 && T.cls <= 2 && T.m >= 1 && T.m * 16 <= ST_STAGE_BYTES && G >= 1 &&
               2 * G * cw_of(T.cls) <= ST_BUF && T.kS3 >= 0 && T.kS3 <= T.m;
    if (T.kind == 2) {
        const int R = T.r1 - T.r0;
        return R >= 1 && R <= ST_CONSUMERS && T.r0 >= 0 && T.r1 <= T.m && T.K0 >= 0 && T.K1 >= 0 && T.K2 >= 0 &&
               T.K0 % 4 == 0 && T.K1 % 8 == 0 && T.K2 % 16 == 0 && 3 * (T.K0 + T.K1 + T.K2) <= ST_BUF;
    }
    return false;
}

// Groups per data piece of dense (R rows) and V (Q rows) tasks.
__device__ __forceinline__ int dense_gp(int R) { return ST_STAGE_BYTES / (6 * R * 16); }
__device__ __forceinline__ int v_gp(int Q) { return ST_STAGE_BYTES / (Q * 16); }

__device__ __forceinline__ int task_pieces(const StreamTask &T)
{
    const int G = T.g1 - T.g0;
    if (T.kind == 0) { const int gp = dense_gp(T.r1 - T.r0); return 1 + (G + gp - 1) / gp; }
    if (T.kind == 1) { const int gp = v_gp(T.m); return 1 + (G + gp - 1) / gp; }
    return 1 + T.K0 / 4 + T.K1 / 8 + T.K2 / 16;
}

struct StreamArgs {
    const StreamTask *tasks;
    const int32_t *cta_ptr;    // tasks [cta_ptr[b], cta_ptr[b + 1]) belong to CTA b
    const float *D;            // FP32 dense blocks
    const void *V[3], *U[3];   // class arrays (FP32, FP16, INT8)
    const float *x;            // deficit (hm_layout.cuh)
    int xstride;
    float *tpart, *slots;
    const float *tfull;
    int *status;
};

// Producer: issue the copies of piece `p` of task T into stage s.
__device__ __forceinline__ void issue_piece(const StreamArgs &A, const StreamTask &T, int p, unsigned char *dst,
                                            uint64_t *bar)
{
    const int G = T.g1 - T.g0;
    if (T.kind == 0) {
        const int R = T.r1 - T.r0;
        if (p == 0) {
            const unsigned nb = (unsigned)(32 * G);
            mbar_expect_tx(bar, nb);
            bulk_g2s(dst, A.x + 2 * ((int64_t)T.c0 + (int64_t)T.g0 * 4), nb, bar);
            return;
        }
        const int gp = dense_gp(R), ga = (p - 1) * gp, gb = min(G, ga + gp);
        if (R == T.m) {                                   // whole rows: the piece is one run
            const unsigned nb = (unsigned)((gb - ga) * 6 * R * 16);
            mbar_expect_tx(bar, nb);
            bulk_g2s(dst, A.D + T.off + ((int64_t)(T.g0 + ga) * 6 * T.m) * 4, nb, bar);
        } else {
            mbar_expect_tx(bar, (unsigned)((gb - ga) * 6 * R * 16));
            for (int g = ga; g < gb; ++g)
                for (int op = 0; op < 6; ++op)
                    bulk_g2s(dst + ((size_t)(g - ga) * 6 + op) * R * 16,
                             A.D + T.off + (((int64_t)(T.g0 + g) * 6 + op) * T.m + T.r0) * 4, (unsigned)(R * 16), bar);
        }
        return;
    }
    if (T.kind == 1) {
        const int CW = cw_of(T.cls), Q = T.m;
        if (p == 0) {
            const unsigned nb = (unsigned)(G * CW * 4);
            mbar_expect_tx(bar, 2 * nb);
            const float *xs = A.x + T.c0 + (int64_t)T.g0 * CW;
            bulk_g2s(dst, xs + 2 * (int64_t)A.xstride, nb, bar);
            bulk_g2s(dst + nb, xs + 3 * (int64_t)A.xstride, nb, bar);
            return;
        }
        const int gp = v_gp(Q), ga = (p - 1) * gp, gb = min(G, ga + gp);
        const unsigned nb = (unsigned)((gb - ga) * Q * 16);
        mbar_expect_tx(bar, nb);
        const void *Vc = T.cls == 0 ? A.V[0] : (T.cls == 1 ? A.V[1] : A.V[2]);
        bulk_g2s(dst, reinterpret_cast<const unsigned char *>(Vc) + (T.off + (int64_t)(T.g0 + ga) * Q * CW) * (16 / CW),
                 nb, bar);
        return;
    }
    const int R = T.r1 - T.r0;
    if (p == 0) {
        const unsigned nb = (unsigned)(3 * (T.K0 + T.K1 + T.K2) * 4);
        mbar_expect_tx(bar, nb);
        bulk_g2s(dst, A.tfull + T.tb, nb, bar);
        return;
    }
    int q = p - 1, cls = 0;
    const int n0 = T.K0 / 4, n1 = T.K1 / 8;
    if (q >= n0) { q -= n0; cls = 1; if (q >= n1) { q -= n1; cls = 2; } }
    const int64_t off = cls == 0 ? T.off : (cls == 1 ? T.off1 : T.off2);
    const void *Uc = cls == 0 ? A.U[0] : (cls == 1 ? A.U[1] : A.U[2]);
    const unsigned char *base = reinterpret_cast<const unsigned char *>(Uc) + off * (cls == 0 ? 4 : (cls == 1 ? 2 : 1));
    mbar_expect_tx(bar, (unsigned)(3 * R * 16));
    for (int c = 0; c < 3; ++c)
        bulk_g2s(dst + (size_t)c * R * 16, base + (((int64_t)q * 3 + c) * T.m + T.r0) * 16, (unsigned)(R * 16), bar);
}

__global__ void __launch_bounds__(ST_THREADS, 1) k_stream(StreamArgs A)
{
    extern __shared__ __align__(128) unsigned char sm[];
    uint64_t *full = reinterpret_cast<uint64_t *>(sm), *empty = full + ST_STAGES;
    float *buf = reinterpret_cast<float *>(sm + 128);                    // x slices or t
    float *red = buf + ST_BUF;                                           // 3 x ST_CONSUMERS
    unsigned char *stage = reinterpret_cast<unsigned char *>(red + 3 * ST_CONSUMERS);
    const int tid = threadIdx.x;
    if (tid == 0) {
        for (int s = 0; s < ST_STAGES; ++s) {
            mbar_init(full + s, 1);                         // the producer's arrive.expect_tx
            mbar_init(empty + s, ST_CONSUMERS / 32);        // one arrive per consumer warp
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    const int t0 = A.cta_ptr[blockIdx.x], t1 = A.cta_ptr[blockIdx.x + 1];
    if (tid >= ST_CONSUMERS) {
        // ---------------------------------------------------------- producer
        if (tid != ST_CONSUMERS) return;
        int i = 0;
        bool stop = false;
        for (int t = t0; t < t1 && !stop; ++t) {
            const StreamTask T = A.tasks[t];
            if (!task_ok(T)) { atomicExch(A.status, 2); continue; }
            const int np = task_pieces(T);
            for (int p = 0; p < np; ++p, ++i) {
                const int s = i % ST_STAGES;
                if (i >= ST_STAGES && !mbar_wait(empty + s, (unsigned)(i / ST_STAGES - 1) & 1u)) {
                    atomicExch(A.status, 1);
                    stop = true;
                    break;
                }
                issue_piece(A, T, p, stage + (size_t)s * ST_STAGE_BYTES, full + s);
            }
        }
        for (int k = i > ST_STAGES ? i - ST_STAGES : 0; k < i; ++k)      // the copies still in flight
            if (!mbar_wait(full + k % ST_STAGES, (unsigned)(k / ST_STAGES) & 1u)) atomicExch(A.status, 1);
        return;
    }
    // -------------------------------------------------------------- consumers
    int i = 0;
    for (int t = t0; t < t1; ++t) {
        const StreamTask T = A.tasks[t];
        if (!task_ok(T)) continue;
        const int np = task_pieces(T), G = T.g1 - T.g0;
        // piece 0: x slices / t into buf
        {
            const int s = i % ST_STAGES;
            const bool ok = mbar_wait(full + s, (unsigned)(i / ST_STAGES) & 1u);
            if (!ok) atomicExch(A.status, 1);
            const float *st = reinterpret_cast<const float *>(stage + (size_t)s * ST_STAGE_BYTES);
            if (T.kind == 0) {
                for (int e = tid; e < 8 * G; e += ST_CONSUMERS) buf[e] = ok ? st[e] : 0.f;
            } else if (T.kind == 1) {
                const int w = G * cw_of(T.cls);
                for (int e = tid; e < w; e += ST_CONSUMERS) {
                    buf[e] = ok ? st[e] : 0.f;
                    buf[ST_BUF / 2 + e] = ok ? st[w + e] : 0.f;
                }
            } else {
                for (int e = tid; e < 3 * (T.K0 + T.K1 + T.K2); e += ST_CONSUMERS) buf[e] = ok ? st[e] : 0.f;
            }
            __syncwarp();
            if ((tid & 31) == 0) mbar_arrive(empty + s);
            ++i;
            consumers_sync();
        }
        if (T.kind == 0) {
            // ---- dense: a piece is [gp groups][6 operators][R rows] 16-byte units (the last
            // piece may hold fewer groups); thread tid owns units tid, tid + 256, tid + 512 of
            // every piece, so its (group offset, operator, row) are the same in all pieces
            const int R = T.r1 - T.r0, gp = dense_gp(R), per = 6 * R;
            float acc[3] = {0.f, 0.f, 0.f};
            int ug[3], uop[3];
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const int u = tid + k * ST_CONSUMERS;
                ug[k] = u / per;
                uop[k] = (u % per) / R;
            }
            for (int p = 1; p < np; ++p, ++i) {
                const int s = i % ST_STAGES;
                const bool ok = mbar_wait(full + s, (unsigned)(i / ST_STAGES) & 1u);
                if (!ok) atomicExch(A.status, 1);
                const int ga = (p - 1) * gp, nu = (min(G, ga + gp) - ga) * per;
                if (ok) {
                    const unsigned char *st = stage + (size_t)s * ST_STAGE_BYTES;
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        const int u = tid + k * ST_CONSUMERS;
                        if (u < nu) {
                            const float4 d = *reinterpret_cast<const float4 *>(st + (size_t)u * 16);
                            const float *xv = buf + 8 * (ga + ug[k]) + (uop[k] & 1);
                            acc[k] += d.x * xv[0] + d.y * xv[2] + d.z * xv[4] + d.w * xv[6];
                        }
                    }
                }
                __syncwarp();
                if ((tid & 31) == 0) mbar_arrive(empty + s);
            }
            // per (component, row): the sum over group offsets and slips of the owned units
            const int full_units = min(G, gp) * per;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const int u = tid + k * ST_CONSUMERS;
                if (u < full_units) red[u] = acc[k];
            }
            consumers_sync();
            for (int e = tid; e < 3 * R; e += ST_CONSUMERS) {
                const int c = e / R, r = e % R;
                float v = 0.f;
                for (int g = 0; g < min(G, gp); ++g)
                    v += red[(g * 6 + 2 * c) * R + r] + red[(g * 6 + 2 * c + 1) * R + r];
                A.slots[3 * ((int64_t)T.out + T.r0 + r) + c] = v;
            }
        } else if (T.kind == 1) {
            // ---- V: a piece is [gp groups][Q rows] units; thread tid owns units tid + 256 k
            const int Q = T.m, gp = v_gp(Q), CW = cw_of(T.cls);
            float acc[3] = {0.f, 0.f, 0.f};
            int ug[3], uq[3];
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const int u = tid + k * ST_CONSUMERS;
                ug[k] = u / Q;
                uq[k] = u % Q;
            }
            for (int p = 1; p < np; ++p, ++i) {
                const int s = i % ST_STAGES;
                const bool ok = mbar_wait(full + s, (unsigned)(i / ST_STAGES) & 1u);
                if (!ok) atomicExch(A.status, 1);
                const int ga = (p - 1) * gp, nu = (min(G, ga + gp) - ga) * Q;
                if (ok) {
                    const unsigned char *st = stage + (size_t)s * ST_STAGE_BYTES;
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        const int u = tid + k * ST_CONSUMERS;
                        if (u < nu) {
                            const float *xv = buf + (uq[k] < T.kS3 ? 0 : ST_BUF / 2) + (ga + ug[k]) * CW;
                            if (T.cls == 0) acc[k] += dot16<float>(st + (size_t)u * 16, xv);
                            else if (T.cls == 1) acc[k] += dot16<__half>(st + (size_t)u * 16, xv);
                            else acc[k] += dot16<uint8_t>(st + (size_t)u * 16, xv);
                        }
                    }
                }
                __syncwarp();
                if ((tid & 31) == 0) mbar_arrive(empty + s);
            }
            const int full_units = min(G, gp) * Q;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const int u = tid + k * ST_CONSUMERS;
                if (u < full_units) red[u] = acc[k];
            }
            consumers_sync();
            for (int q = tid; q < Q; q += ST_CONSUMERS) {
                float v = 0.f;
                for (int g = 0; g < min(G, gp); ++g) v += red[g * Q + q];
                A.tpart[T.out + q] = v;
            }
        } else {
            // ---- U: a piece is [3 components][R rows] units; thread tid owns units tid + 256 k
            const int R = T.r1 - T.r0;
            float acc[3] = {0.f, 0.f, 0.f};
            int uc[3], ur[3];
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const int u = tid + k * ST_CONSUMERS;
                uc[k] = u / R;
                ur[k] = u % R;
            }
            const int n0 = T.K0 / 4, n1 = T.K1 / 8;
            for (int p = 1; p < np; ++p, ++i) {
                const int s = i % ST_STAGES;
                const bool ok = mbar_wait(full + s, (unsigned)(i / ST_STAGES) & 1u);
                if (!ok) atomicExch(A.status, 1);
                if (ok) {
                    const unsigned char *st = stage + (size_t)s * ST_STAGE_BYTES;
                    const int q = p - 1;
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        const int u = tid + k * ST_CONSUMERS;
                        if (u < 3 * R) {
                            if (q < n0) acc[k] += dot16<float>(st + (size_t)u * 16, buf + uc[k] * T.K0 + q * 4);
                            else if (q < n0 + n1)
                                acc[k] += dot16<__half>(st + (size_t)u * 16, buf + 3 * T.K0 + uc[k] * T.K1 + (q - n0) * 8);
                            else
                                acc[k] += dot16<uint8_t>(st + (size_t)u * 16,
                                                         buf + 3 * (T.K0 + T.K1) + uc[k] * T.K2 + (q - n0 - n1) * 16);
                        }
                    }
                }
                __syncwarp();
                if ((tid & 31) == 0) mbar_arrive(empty + s);
            }
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const int u = tid + k * ST_CONSUMERS;
                if (u < 3 * R) A.slots[3 * ((int64_t)T.out + T.r0 + ur[k]) + uc[k]] = acc[k];
            }
        }
        consumers_sync();      // buf and red are reused by the next task
    }
}

// t of every class of every low-rank block (as the U tasks of k_du_mixed gather it):
// one CTA per block, t_c[c][q] = scale * sum over chunks of the V partials.
__global__ void __launch_bounds__(128) k_t_gather(const TGather *__restrict__ gs, const float *__restrict__ tpart,
                                                  const float *__restrict__ scales, float *__restrict__ tfull)
{
    const TGather T = gs[blockIdx.x];
    float *o = tfull + T.tb;
#pragma unroll
    for (int cls = 0; cls < 3; ++cls) {
        const int K = T.K[cls], kS = T.kS[cls], kD = T.kD[cls];
        for (int e = threadIdx.x; e < 3 * K; e += blockDim.x) {
            const int c = e / K, q = e % K;
            int row = -1;
            if (q < kS) row = c * kS + q;
            else if (q < kS + kD) row = 3 * kS + c * kD + (q - kS);
            float v = 0.f;
            if (row >= 0) {
                v = sum_partials<float>(tpart + T.tp[cls] + row, T.nch[cls], T.Q[cls]);
                if (cls > 0) v *= scales[T.sb[cls] + row];
            }
            o[e] = v;
        }
        o += 3 * K;
    }
}

// ------------------------------------------------------------------ kernel 3
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
    const int k0 = leaf_ptr[l], k1 = leaf_ptr[l + 1];
    int k = k0;
    // four slots per iteration: independent loads in flight, summed in list order
    for (; k + 4 <= k1; k += 4) {
        TA v[12];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int64_t s = 3 * ((int64_t)leaf_off[k + u] + i);
            v[3 * u] = slots[s];
            v[3 * u + 1] = slots[s + 1];
            v[3 * u + 2] = slots[s + 2];
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            a0 += (double)v[3 * u];
            a1 += (double)v[3 * u + 1];
            a2 += (double)v[3 * u + 2];
        }
    }
    for (; k < k1; ++k) {
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
// Packed operator description (device pointers) -- mirrors the Python HM_PLAN record.
struct HmPlan {
    int32_t n;             // elements
    int32_t dtype;         // 0: FP64 dense + FP64 low rank; 1: FP32 + FP32; 2: FP32 dense + BF16 low rank;
                           // 3: FP32 dense + FP32/FP16/INT8 low-rank term classes
    const void *dense;     // packed dense data
    const void *U;         // packed U factors
    const void *V;         // packed V factors
    const void *ditems;    // DenseItem[n_ditems]
    const void *vitems;    // VItem[n_vitems] (storage code 3, plain kernels: VItemM)
    const void *utasks;    // UTask[n_utasks]
    const int32_t *leaf_of_row, *leaf_ptr, *leaf_off;
    int64_t n_ditems, n_vitems, n_utasks, n_slots, n_tpart;
    int32_t kmax, pad;     // largest K of a low-rank block (shared memory of k_u); mixed: of K0+K1+K2
    // storage code 3 only (U, V above are the FP32 class arrays)
    const void *U16, *V16, *U8, *V8;   // FP16 and INT8 class arrays
    const float *scales;               // per-V-row scales of the FP16 and INT8 classes
    int32_t *status;                   // streamed kernels: 1 after a timed-out wait, 2 after a skipped task
    int32_t stream, pad2;              // 1: the streamed kernels (k_stream, k_t_gather) run the plan
    const void *tasks_a, *tasks_b;     // StreamTask lists: phase A (dense, V), phase B (U), grouped by CTA
    const int32_t *cta_a, *cta_b;      // per-CTA ranges of the task lists (ncta + 1 entries)
    const void *gather;                // TGather per low-rank block
    float *tfull;                      // the blocks' t, written by k_t_gather
    int64_t n_gather;
    int32_t ncta_a, ncta_b;
    const void *vrows;                 // storage code 3, plain kernels: VRowRec list of the VItemM items
    const int32_t *vwarp;              // k_v_mixed's per-warp item lists (n_vwarp + 1 offsets)
    int32_t n_vwarp, pad3;
};

PQ3D_EXPORT size_t pq3d_item_bytes(int kind)
{
    switch (kind) {
    case 0: return sizeof(DenseItem);
    case 1: return sizeof(VItem);
    case 2: return sizeof(UTask);
    case 4: return sizeof(DenseBlock);
    case 5: return sizeof(HmPlan);
    case 6: return sizeof(UTaskM);
    case 7: return sizeof(StreamTask);
    case 8: return sizeof(TGather);
    case 9: return sizeof(VItemM);
    case 10: return sizeof(VRowRec);
    }
    return 0;
}

template <typename TD, typename TL, typename TA>
static int run_matvec(const HmPlan &P, const TA *x, TA *slots, TA *tpart, const double *add0,
                      const double *add1, const double *add2, double *y, cudaStream_t st)
{
    // FP32 / BF16: V items first, dense items and U tasks in the dependent launch (the
    // dense items fill the first launch's tail).  FP64: dense and V items together,
    // then the U tasks (measured faster at this precision).
    const bool split = !std::is_same<TD, double>::value;
    const int64_t nd_a = split ? 0 : P.n_ditems, nd_b = split ? P.n_ditems : 0;
    if (P.n_vitems + nd_a > 0) {
        const int64_t blocks = ((P.n_vitems + nd_a) * 32 + 255) / 256;
        k_dense_v<TD, TL, TA><<<(unsigned)blocks, 256, 0, st>>>((const DenseItem *)P.ditems, nd_a,
                                                                (const VItem *)P.vitems, P.n_vitems,
                                                                (const TD *)P.dense, (const TL *)P.V, x,
                                                                x_stride(P.n), slots, tpart);
    }
    if (!split) {
        if (P.n_utasks > 0) {
            const size_t smem = (size_t)3 * P.kmax * sizeof(TA);
            if (smem > 200 * 1024) return PQ3D_ERR_ARG;
            if (smem > 48 * 1024)
                PQ3D_CHECK(cudaFuncSetAttribute(k_u<TL, TA>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            k_u<TL, TA><<<(unsigned)P.n_utasks, 256, smem, st>>>((const UTask *)P.utasks, (const TL *)P.U, tpart,
                                                                 slots);
        }
    } else {
        const int64_t n_dblocks = (nd_b * 32 + 255) / 256;
        const int64_t grid = n_dblocks + P.n_utasks;
        if (grid > 0) {
            const size_t smem = P.n_utasks > 0 ? (size_t)3 * P.kmax * sizeof(TA) : 0;
            if (smem > 200 * 1024) return PQ3D_ERR_ARG;
            if (smem > 48 * 1024)
                PQ3D_CHECK(cudaFuncSetAttribute(k_du<TD, TL, TA>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3((unsigned)grid);
            cfg.blockDim = dim3(256);
            cfg.dynamicSmemBytes = smem;
            cfg.stream = st;
            cudaLaunchAttribute attr[1];
            attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
            attr[0].val.programmaticStreamSerializationAllowed = 1;
            cfg.attrs = attr;
            cfg.numAttrs = (P.n_vitems + nd_a) > 0 ? 1 : 0;
            PQ3D_CHECK(cudaLaunchKernelEx(&cfg, k_du<TD, TL, TA>, (const DenseItem *)P.ditems, nd_b, n_dblocks,
                                          (const UTask *)P.utasks, (const TD *)P.dense, (const TL *)P.U, x, slots,
                                          (const TA *)tpart));
        }
    }
    if (y)
        k_rowsum<TA><<<(P.n + 255) / 256, 256, 0, st>>>(P.n, P.leaf_of_row, P.leaf_ptr, P.leaf_off, slots, add0,
                                                         add1, add2, y);
    return pq3d_launch_status();
}

// Storage code 3: k_v_mixed (V items of every class), then k_du_mixed (dense items in
// its tail, then the U tasks), then the optional row sum.
static int run_matvec_mixed(const HmPlan &P, const float *x, float *slots, float *tpart, const double *add0,
                            const double *add1, const double *add2, double *y, cudaStream_t st)
{
    if (P.n_vitems > 0) {
        if (!P.vrows || !P.vwarp || P.n_vwarp <= 0) return PQ3D_ERR_ARG;
        const int blocks = (P.n_vwarp + 7) / 8;
        k_v_mixed<<<(unsigned)blocks, 256, 0, st>>>((const VItemM *)P.vitems, P.vwarp, P.n_vwarp,
                                                    (const VRowRec *)P.vrows, (const float *)P.V,
                                                    (const __half *)P.V16, (const uint8_t *)P.V8, x, x_stride(P.n),
                                                    tpart);
    }
    const int64_t n_dblocks = (P.n_ditems * 32 + PQ3D_UMIX_THREADS - 1) / PQ3D_UMIX_THREADS;
    const int64_t grid = n_dblocks + P.n_utasks;
    if (grid > 0) {
        const size_t smem = P.n_utasks > 0 ? (size_t)3 * P.kmax * sizeof(float) : 0;
        if (smem > 200 * 1024) return PQ3D_ERR_ARG;
        if (smem > 48 * 1024)
            PQ3D_CHECK(cudaFuncSetAttribute(k_du_mixed, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)grid);
        cfg.blockDim = dim3(PQ3D_UMIX_THREADS);
        cfg.dynamicSmemBytes = smem;
        cfg.stream = st;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = attr;
        cfg.numAttrs = P.n_vitems > 0 ? 1 : 0;
        PQ3D_CHECK(cudaLaunchKernelEx(&cfg, k_du_mixed, (const DenseItem *)P.ditems, P.n_ditems, n_dblocks,
                                      (const UTaskM *)P.utasks, (const float *)P.dense, (const float *)P.U,
                                      (const __half *)P.U16, (const uint8_t *)P.U8, x, slots, (const float *)tpart,
                                      P.scales));
    }
    if (y)
        k_rowsum<float><<<(P.n + 255) / 256, 256, 0, st>>>(P.n, P.leaf_of_row, P.leaf_ptr, P.leaf_off, slots, add0,
                                                           add1, add2, y);
    return pq3d_launch_status();
}

// Storage code 3, streamed: phase A (dense and V tasks), the t gather, phase B (U tasks).
static size_t stream_smem() { return 128 + (size_t)(ST_BUF + 3 * ST_CONSUMERS) * 4 + (size_t)ST_STAGES * ST_STAGE_BYTES; }

static int run_matvec_stream(const HmPlan &P, const float *x, float *slots, float *tpart, const double *add0,
                             const double *add1, const double *add2, double *y, cudaStream_t st)
{
    if (!P.status || (P.ncta_a > 0 && (!P.tasks_a || !P.cta_a)) || (P.ncta_b > 0 && (!P.tasks_b || !P.cta_b)) ||
        (P.n_gather > 0 && (!P.gather || !P.tfull)))
        return PQ3D_ERR_ARG;
    const size_t sm = stream_smem();
    PQ3D_CHECK(cudaFuncSetAttribute(k_stream, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    StreamArgs A;
    A.D = (const float *)P.dense;
    A.V[0] = P.V; A.V[1] = P.V16; A.V[2] = P.V8;
    A.U[0] = P.U; A.U[1] = P.U16; A.U[2] = P.U8;
    A.x = x;
    A.xstride = x_stride(P.n);
    A.tpart = tpart;
    A.slots = slots;
    A.tfull = P.tfull;
    A.status = P.status;
    if (P.ncta_a > 0) {
        A.tasks = (const StreamTask *)P.tasks_a;
        A.cta_ptr = P.cta_a;
        k_stream<<<(unsigned)P.ncta_a, ST_THREADS, sm, st>>>(A);
    }
    if (P.n_gather > 0) {
        if (P.n_gather > 0x7fffffff) return PQ3D_ERR_ARG;
        k_t_gather<<<(unsigned)P.n_gather, 128, 0, st>>>((const TGather *)P.gather, tpart, P.scales, P.tfull);
    }
    if (P.ncta_b > 0) {
        A.tasks = (const StreamTask *)P.tasks_b;
        A.cta_ptr = P.cta_b;
        k_stream<<<(unsigned)P.ncta_b, ST_THREADS, sm, st>>>(A);
    }
    if (y)
        k_rowsum<float><<<(P.n + 255) / 256, 256, 0, st>>>(P.n, P.leaf_of_row, P.leaf_ptr, P.leaf_off, slots, add0,
                                                           add1, add2, y);
    return pq3d_launch_status();
}

// Resident CTAs of k_v_mixed on this device: its plans' per-warp lists are made for
// 8 warps per resident CTA.
PQ3D_EXPORT int pq3d_vmix_ctas(void)
{
    const int v = vmix_ctas();
    return v > 0 ? v : PQ3D_ERR_CUDA;
}

// Resident CTAs of the streamed kernel on this device (persistent grid size).
PQ3D_EXPORT int pq3d_stream_ctas(void)
{
    int dev = 0, sms = 0, per = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return PQ3D_ERR_CUDA;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return PQ3D_ERR_CUDA;
    const size_t sm = stream_smem();
    if (cudaFuncSetAttribute(k_stream, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) != cudaSuccess)
        return PQ3D_ERR_CUDA;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_stream, ST_THREADS, sm) != cudaSuccess || per <= 0)
        return PQ3D_ERR_CUDA;
    return sms * per;
}

// y (n x 3, FP64, tree order) = K x (+ add_c).  x: deficit in the layout of hm_layout.cuh
// (4 * x_stride(n) entries: interleaved, strike plane, dip plane), FP64 for dtype 0 and
// FP32 otherwise.  Scratch: slots (3*n_slots) and
// tpart (n_tpart) in the accumulation type (FP64 for dtype 0, FP32 otherwise).  With
// d_y == NULL only the per-row slots are written (the step kernel sums them itself).
PQ3D_EXPORT int pq3d_hmatvec(const void *plan_host, const void *d_x, void *d_slots, void *d_tpart,
                             const double *d_add0, const double *d_add1, const double *d_add2, double *d_y,
                             cudaStream_t stream)
{
    if (!plan_host || !d_x || !d_slots) return PQ3D_ERR_ARG;
    const HmPlan &P = *(const HmPlan *)plan_host;
    if (P.n <= 0) return PQ3D_ERR_ARG;
    if (P.n_vitems > 0 && !d_tpart) return PQ3D_ERR_ARG;
    switch (P.dtype) {
    case 0:
        return run_matvec<double, double, double>(P, (const double *)d_x, (double *)d_slots, (double *)d_tpart,
                                                  d_add0, d_add1, d_add2, d_y, stream);
    case 1:
        return run_matvec<float, float, float>(P, (const float *)d_x, (float *)d_slots, (float *)d_tpart, d_add0,
                                               d_add1, d_add2, d_y, stream);
    case 2:
        return run_matvec<float, __nv_bfloat16, float>(P, (const float *)d_x, (float *)d_slots, (float *)d_tpart,
                                                       d_add0, d_add1, d_add2, d_y, stream);
    case 3:
        if (P.n_utasks > 0 && (!P.U || !P.U16 || !P.U8 || !P.V || !P.V16 || !P.V8 || !P.scales)) return PQ3D_ERR_ARG;
        if (P.stream)
            return run_matvec_stream(P, (const float *)d_x, (float *)d_slots, (float *)d_tpart, d_add0, d_add1,
                                     d_add2, d_y, stream);
        return run_matvec_mixed(P, (const float *)d_x, (float *)d_slots, (float *)d_tpart, d_add0, d_add1, d_add2,
                                d_y, stream);
    }
    return PQ3D_ERR_ARG;
}
