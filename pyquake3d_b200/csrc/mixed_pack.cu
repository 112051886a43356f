// Packing of the ACA factors into the mixed storage (storage code 3 of the
// H-matvec, hmatvec.cu): each ACA term of a low-rank block is stored as FP32,
// FP16 or INT8 according to how much of its rows' products it can carry.
//
// The reference applies every block in FP64 (blocks_process_MVM,
// src/Hmatrix.py:1445-1538); this storage is the project's own.  The
// classification rests on the size of the error a term can put into a row:
// quantising the term u v^T with a relative error e moves row i of the product
// by about e |u_i| ||v||_1 ||x||_inf, while FP32 storage of the row's operator
// entries already rounds at 2^-24 sum_j |K_ij| ||x||_inf.  The weight of a term is
//     w = max_i (|u_i| / R_i) * ||v||_1 ,   R_i = sum over the near-field (dense)
// blocks of row i of |K_ij| (both slips, largest of the three components), a
// lower bound of the row's absolute sum.  The host picks the class from w and a
// tolerance (hmatrix.py).
//
//   k_nearfield_rowabs   R3[c][i] += sum_j |K^c_ij| over the dense blocks
//   k_term_weights       w per (task, term): max over the three components
//   k_pack_mixed         normalised, quantised factors and per-row scales; an INT8
//                        entry b = round(127 v / max|v|) is stored as the byte b + 128
#include "pq3d_common.cuh"
#include "hm_layout.cuh"
#include <cuda_fp16.h>

using namespace pq3d;

namespace {

// One ACA task (block, slip pass) of the mixed packing.  tmap[tmap_off + q]
// holds the class of term q (bits 0-1) and its position among this pass's
// terms of that class (bits 2+).
struct PackTaskM {
    int64_t ws_off, rows_off, cols_off, tmap_off;
    int64_t u_off[3], v_off[3];    // block offsets in the FP32 / FP16 / INT8 arrays
    int32_t m, n, kmax, k, pass, r0, c0, zeroB;
    int32_t kS[3], kD[3], Q[3], K[3], sb[3];
    int32_t pad;
};

__device__ double block_max(double v, double *red)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    __syncthreads();
    if (lane == 0) red[wid] = v;
    __syncthreads();
    if (wid == 0) {
        v = lane < (int)(blockDim.x >> 5) ? red[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
        if (lane == 0) red[0] = v;
    }
    __syncthreads();
    const double r = red[0];
    __syncthreads();
    return r;
}

__device__ double block_add(double v, double *red)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    __syncthreads();
    if (lane == 0) red[wid] = v;
    __syncthreads();
    if (wid == 0) {
        v = lane < (int)(blockDim.x >> 5) ? red[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) red[0] = v;
    }
    __syncthreads();
    const double r = red[0];
    __syncthreads();
    return r;
}

// One CTA per dense block: threads over rows, each summing |K| over the block's
// columns for the three components (both slips).
__global__ void k_nearfield_rowabs(const float *__restrict__ D, const DenseBlock *__restrict__ blocks, int n,
                                   double *__restrict__ R3)
{
    const DenseBlock b = blocks[blockIdx.x];
    const int ng = (b.n + b.c0 % kCW32 + kCW32 - 1) / kCW32;
    for (int i = threadIdx.x; i < b.m; i += blockDim.x) {
        double a[3] = {0.0, 0.0, 0.0};
        for (int g = 0; g < ng; ++g)
            for (int c = 0; c < 3; ++c)
                for (int s = 0; s < 2; ++s) {
                    const float *p = D + b.off32 + (((int64_t)g * 6 + 2 * c + s) * b.m + i) * kCW32;
#pragma unroll
                    for (int t = 0; t < kCW32; ++t) a[c] += fabs((double)p[t]);
                }
        for (int c = 0; c < 3; ++c) atomicAdd(&R3[(int64_t)c * n + b.r0 + i], a[c]);
    }
}

// One CTA per task: w for every term (largest over the components; the B factor is
// skipped when the packing drops it).
__global__ void k_term_weights(const PackTaskM *__restrict__ tasks, const double *__restrict__ ws,
                               const int32_t *__restrict__ rowlist, const int32_t *__restrict__ iperm,
                               const double *__restrict__ R, double *__restrict__ w_out)
{
    __shared__ double red[32];
    const PackTaskM P = tasks[blockIdx.x];
    const double *U = ws + P.ws_off;
    const double *V = U + (int64_t)P.kmax * 3 * P.m;
    const int32_t *rows = rowlist + P.rows_off;
    for (int q = 0; q < P.k; ++q) {
        double w = 0.0;
        for (int c = 0; c < (P.zeroB ? 2 : 3); ++c) {
            double um = 0.0, vs = 0.0;
            for (int i = threadIdx.x; i < P.m; i += blockDim.x) {
                const double r = R[iperm[rows[i]]];
                const double u = fabs(U[((int64_t)q * 3 + c) * P.m + i]);
                um = fmax(um, r > 0.0 ? u / r : (u > 0.0 ? INFINITY : 0.0));
            }
            for (int j = threadIdx.x; j < P.n; j += blockDim.x) vs += fabs(V[((int64_t)q * 3 + c) * P.n + j]);
            um = block_max(um, red);
            vs = block_add(vs, red);
            w = fmax(w, um * vs);
        }
        if (threadIdx.x == 0) w_out[P.tmap_off + q] = w;
    }
}

__global__ void k_pack_mixed(const PackTaskM *__restrict__ tasks, const double *__restrict__ ws,
                             const int32_t *__restrict__ rowlist, const int32_t *__restrict__ collist,
                             const int32_t *__restrict__ iperm, const int32_t *__restrict__ tmap,
                             float *__restrict__ U32, __half *__restrict__ U16, uint8_t *__restrict__ U8,
                             float *__restrict__ V32, __half *__restrict__ V16, uint8_t *__restrict__ V8,
                             float *__restrict__ scales)
{
    __shared__ double red[32];
    const PackTaskM P = tasks[blockIdx.x];
    const double *U = ws + P.ws_off;
    const double *V = U + (int64_t)P.kmax * 3 * P.m;
    const int32_t *rows = rowlist + P.rows_off, *cols = collist + P.cols_off;
    for (int q = 0; q < P.k; ++q) {
        const int code = tmap[P.tmap_off + q];
        const int cls = code & 3, pos = code >> 2;
        const int col = P.pass == 0 ? pos : P.kS[cls] + pos;                 // U column within the class
        for (int c = 0; c < 3; ++c) {
            if (c == 2 && P.zeroB) continue;                                  // dropped B factor: zeros
            const int row = P.pass == 0 ? c * P.kS[cls] + pos : 3 * P.kS[cls] + c * P.kD[cls] + pos;  // V row
            const double *u = U + ((int64_t)q * 3 + c) * P.m;
            const double *v = V + ((int64_t)q * 3 + c) * P.n;
            if (cls == 0) {
                for (int i = threadIdx.x; i < P.m; i += blockDim.x)
                    U32[P.u_off[0] + u_index(P.m, iperm[rows[i]] - P.r0, c, col, 4)] = (float)u[i];
                for (int j = threadIdx.x; j < P.n; j += blockDim.x)
                    V32[P.v_off[0] + v_index(P.Q[0], row, P.c0 % 4 + iperm[cols[j]] - P.c0, 4)] = (float)v[j];
                continue;
            }
            double su = 0.0, sv = 0.0;
            for (int i = threadIdx.x; i < P.m; i += blockDim.x) su = fmax(su, fabs(u[i]));
            for (int j = threadIdx.x; j < P.n; j += blockDim.x) sv = fmax(sv, fabs(v[j]));
            su = block_max(su, red);
            sv = block_max(sv, red);
            if (!(su > 0.0) || !(sv > 0.0)) continue;                         // an all-zero term stays zero
            if (cls == 1) {
                for (int i = threadIdx.x; i < P.m; i += blockDim.x)
                    U16[P.u_off[1] + u_index(P.m, iperm[rows[i]] - P.r0, c, col, 8)] = __float2half_rn((float)(u[i] / su));
                for (int j = threadIdx.x; j < P.n; j += blockDim.x)
                    V16[P.v_off[1] + v_index(P.Q[1], row, P.c0 % 8 + iperm[cols[j]] - P.c0, 8)] =
                        __float2half_rn((float)(v[j] / sv));
                if (threadIdx.x == 0) scales[P.sb[1] + row] = (float)(su * sv);
            } else {
                for (int i = threadIdx.x; i < P.m; i += blockDim.x) {
                    const double t = fmin(127.0, fmax(-127.0, rint(127.0 * u[i] / su)));
                    U8[P.u_off[2] + u_index(P.m, iperm[rows[i]] - P.r0, c, col, 16)] = (uint8_t)(t + 128.0);
                }
                for (int j = threadIdx.x; j < P.n; j += blockDim.x) {
                    const double t = fmin(127.0, fmax(-127.0, rint(127.0 * v[j] / sv)));
                    V8[P.v_off[2] + v_index(P.Q[2], row, P.c0 % 16 + iperm[cols[j]] - P.c0, 16)] = (uint8_t)(t + 128.0);
                }
                if (threadIdx.x == 0) scales[P.sb[2] + row] = (float)(su * sv / (127.0 * 127.0));
            }
        }
    }
}

}  // namespace

PQ3D_EXPORT size_t pq3d_pack_mixed_task_bytes(void) { return sizeof(PackTaskM); }

PQ3D_EXPORT int pq3d_nearfield_rowabs(const float *d_dense32, const void *d_blocks, int64_t n_blocks, int n,
                                      double *d_R3, cudaStream_t stream)
{
    if (n_blocks < 0 || n <= 0) return PQ3D_ERR_ARG;
    if (n_blocks == 0) return PQ3D_OK;
    if (!d_dense32 || !d_blocks || !d_R3) return PQ3D_ERR_ARG;
    for (int64_t b0 = 0; b0 < n_blocks; b0 += 65535) {
        const unsigned nb = (unsigned)(n_blocks - b0 < 65535 ? n_blocks - b0 : 65535);
        k_nearfield_rowabs<<<nb, 128, 0, stream>>>(d_dense32, (const DenseBlock *)d_blocks + b0, n, d_R3);
    }
    return pq3d_launch_status();
}

PQ3D_EXPORT int pq3d_aca_term_weights(const void *d_tasks, int64_t n_tasks, const double *d_ws,
                                      const int32_t *d_rowlist, const int32_t *d_iperm, const double *d_R,
                                      double *d_w, cudaStream_t stream)
{
    if (n_tasks < 0) return PQ3D_ERR_ARG;
    if (n_tasks == 0) return PQ3D_OK;
    if (!d_tasks || !d_ws || !d_rowlist || !d_iperm || !d_R || !d_w) return PQ3D_ERR_ARG;
    for (int64_t t0 = 0; t0 < n_tasks; t0 += 65535) {
        const unsigned nt = (unsigned)(n_tasks - t0 < 65535 ? n_tasks - t0 : 65535);
        k_term_weights<<<nt, 256, 0, stream>>>((const PackTaskM *)d_tasks + t0, d_ws, d_rowlist, d_iperm, d_R, d_w);
    }
    return pq3d_launch_status();
}

PQ3D_EXPORT int pq3d_aca_pack_mixed(const void *d_tasks, int64_t n_tasks, const double *d_ws,
                                    const int32_t *d_rowlist, const int32_t *d_collist, const int32_t *d_iperm,
                                    const int32_t *d_tmap, float *d_U32, void *d_U16, void *d_U8, float *d_V32,
                                    void *d_V16, void *d_V8, float *d_scales, cudaStream_t stream)
{
    if (n_tasks < 0) return PQ3D_ERR_ARG;
    if (n_tasks == 0) return PQ3D_OK;
    if (!d_tasks || !d_ws || !d_rowlist || !d_collist || !d_iperm || !d_tmap || !d_U32 || !d_U16 || !d_U8 ||
        !d_V32 || !d_V16 || !d_V8 || !d_scales)
        return PQ3D_ERR_ARG;
    for (int64_t t0 = 0; t0 < n_tasks; t0 += 65535) {
        const unsigned nt = (unsigned)(n_tasks - t0 < 65535 ? n_tasks - t0 : 65535);
        k_pack_mixed<<<nt, 256, 0, stream>>>((const PackTaskM *)d_tasks + t0, d_ws, d_rowlist, d_collist, d_iperm,
                                             d_tmap, d_U32, (__half *)d_U16, (uint8_t *)d_U8, d_V32, (__half *)d_V16,
                                             (uint8_t *)d_V8, d_scales);
    }
    return pq3d_launch_status();
}
