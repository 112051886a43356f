// Green's-function kernels: per-source records, pair evaluations, dense
// near-field block assembly, and the two host-pointer drop-ins with the
// reference's C signatures (src/TDstressFS_C.cpp:2048-2143).
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <mutex>

#include "pq3d_common.cuh"
#include "td_gf.cuh"
#include "td_hs.cuh"
#include "hm_layout.cuh"

using namespace pq3d;

// ---------------------------------------------------------------- records
__global__ void k_src_records(const double *__restrict__ nodes, const int64_t *__restrict__ tri,
                              int64_t n_elem, SrcRec *__restrict__ rec)
{
    int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= n_elem) return;
    const double *P1 = nodes + 3 * (tri[3 * e + 0] - 1);
    const double *P2 = nodes + 3 * (tri[3 * e + 1] - 1);
    const double *P3 = nodes + 3 * (tri[3 * e + 2] - 1);
    SrcRec s;
    make_src_rec(P1, P2, P3, s);
    rec[e] = s;
}

PQ3D_EXPORT size_t pq3d_src_record_bytes(void) { return sizeof(SrcRec); }

PQ3D_EXPORT int pq3d_src_records(const double *d_nodes, const int64_t *d_tri, int64_t n_elem,
                                 void *d_rec, cudaStream_t stream)
{
    if (n_elem < 0 || (n_elem > 0 && (!d_nodes || !d_tri || !d_rec))) return PQ3D_ERR_ARG;
    if (n_elem == 0) return PQ3D_OK;
    int th = 128;
    k_src_records<<<(unsigned)((n_elem + th - 1) / th), th, 0, stream>>>(d_nodes, d_tri, n_elem, (SrcRec *)d_rec);
    return pq3d_launch_status();
}

__global__ void k_hs_records(const double *__restrict__ nodes, const int64_t *__restrict__ tri, int64_t n_elem,
                             HsRec *__restrict__ hs)
{
    int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= n_elem) return;
    HsRec h;
    make_hs_rec(nodes + 3 * (tri[3 * e + 0] - 1), nodes + 3 * (tri[3 * e + 1] - 1), nodes + 3 * (tri[3 * e + 2] - 1), h);
    hs[e] = h;
}

PQ3D_EXPORT size_t pq3d_hs_record_bytes(void) { return sizeof(HsRec); }

PQ3D_EXPORT int pq3d_hs_records(const double *d_nodes, const int64_t *d_tri, int64_t n_elem, void *d_hs,
                                cudaStream_t stream)
{
    if (n_elem < 0 || (n_elem > 0 && (!d_nodes || !d_tri || !d_hs))) return PQ3D_ERR_ARG;
    if (n_elem == 0) return PQ3D_OK;
    k_hs_records<<<(unsigned)((n_elem + 127) / 128), 128, 0, stream>>>(d_nodes, d_tri, n_elem, (HsRec *)d_hs);
    return pq3d_launch_status();
}

static bool hs_args_ok(const void *hs, int mode) { return mode == 0 || ((mode == 1 || mode == 2) && hs); }

// ---------------------------------------------------------------- traction pairs
// out[p*6 + 0..5] = (A1s, A2s, Bs, A1d, A2d, Bd) for receiver rows[p], source cols[p].
template <bool HS>
__global__ void k_traction_pairs(const double *__restrict__ xg, const double *__restrict__ ev,
                                 const SrcRec *__restrict__ rec, const int64_t *__restrict__ rows,
                                 const int64_t *__restrict__ cols, int64_t npairs, double mu, double lam,
                                 double *__restrict__ out, const HsRec *__restrict__ hs, int hs_mode)
{
    int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (p >= npairs) return;
    int64_t r = rows[p], c = cols[p];
    double nu = 1.0 / (1.0 + lam / mu) / 2.0;
    double obs[3] = {xg[3 * r], xg[3 * r + 1], xg[3 * r + 2]};
    double f[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) f[k] = ev[9 * r + k];
    double t[6];
    if (HS) gf_traction_sd_hs(obs, f, rec[c], hs[c], hs_mode, mu, lam, nu, t);
    else gf_traction_sd(obs, f, rec[c], mu, lam, nu, t);
#pragma unroll
    for (int k = 0; k < 6; ++k) out[6 * p + k] = t[k];
}

PQ3D_EXPORT int pq3d_traction_pairs(const double *d_xg, const double *d_ev, const void *d_rec,
                                    const int64_t *d_rows, const int64_t *d_cols, int64_t npairs,
                                    double mu, double lam, double *d_out, const void *d_hs, int hs_mode,
                                    cudaStream_t stream)
{
    if (npairs < 0 || !hs_args_ok(d_hs, hs_mode)) return PQ3D_ERR_ARG;
    if (npairs == 0) return PQ3D_OK;
    if (!d_xg || !d_ev || !d_rec || !d_rows || !d_cols || !d_out) return PQ3D_ERR_ARG;
    int th = 128;
    const unsigned g = (unsigned)((npairs + th - 1) / th);
    if (hs_mode)
        k_traction_pairs<true><<<g, th, 0, stream>>>(d_xg, d_ev, (const SrcRec *)d_rec, d_rows, d_cols, npairs, mu,
                                                     lam, d_out, (const HsRec *)d_hs, hs_mode);
    else
        k_traction_pairs<false><<<g, th, 0, stream>>>(d_xg, d_ev, (const SrcRec *)d_rec, d_rows, d_cols, npairs, mu,
                                                      lam, d_out, nullptr, 0);
    return pq3d_launch_status();
}

// ---------------------------------------------------------------- stress at points
// Full stress/strain tensors for receivers (X,Y,Z) and sources rec[src[p]], general
// Burgers vector (Ts, Ss, Ds); half-space adds the image and free-surface terms.
template <bool HS>
__global__ void k_stress_points(const double *__restrict__ X, const double *__restrict__ Y,
                                const double *__restrict__ Z, int64_t xstride,
                                const double *__restrict__ P, int64_t pstride, int64_t npairs,
                                double Ss, double Ds, double Ts, double mu, double lam, int halfspace,
                                double *__restrict__ stress, double *__restrict__ strain)
{
    int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (p >= npairs) return;
    int64_t xi = p * xstride, si = p * pstride;
    double obs[3] = {X[xi], Y[xi], Z[xi]};
    const double *P1 = P + 9 * si, *P2 = P + 9 * si + 3, *P3 = P + 9 * si + 6;
    double e[6], sig[6];
    {
        SrcRec s;
        make_src_rec(P1, P2, P3, s);
        double X1[3];
        to_td_frame(obs, s, X1);
        double nu = 1.0 / (1.0 + lam / mu) / 2.0;
        const double b[1][3] = {{Ts, Ss, Ds}};
        double ee[1][6];
        td_strain_multi<1, true>(X1, s, nu, b, ee);
        if (HS) {
            HsRec h;
            make_hs_rec(P1, P2, P3, h);
            hs_add_strain<1, true>(obs, s, h, nu, b, halfspace, ee);
        }
        for (int c = 0; c < 6; ++c) e[c] = ee[0][c];
        hooke(e, mu, lam, sig);
    }
#pragma unroll
    for (int c = 0; c < 6; ++c) {
        stress[6 * p + c] = sig[c];
        if (strain) strain[6 * p + c] = e[c];
    }
}

// Device-pointer form of both reference entry points.  n_pts receivers and
// n_src sources, one of which is 1 (xstride/pstride 0 broadcast the single one).
PQ3D_EXPORT int pq3d_stress_points(const double *d_X, const double *d_Y, const double *d_Z, int64_t n_pts,
                                   const double *d_P /* n_src x 9: P1,P2,P3 */, int64_t n_src,
                                   double Ss, double Ds, double Ts, double mu, double lam, int halfspace,
                                   double *d_stress, double *d_strain, cudaStream_t stream)
{
    if (n_pts < 0 || n_src < 0) return PQ3D_ERR_ARG;
    if (n_pts != 1 && n_src != 1 && n_pts != n_src) return PQ3D_ERR_ARG;
    int64_t np = n_pts > n_src ? n_pts : n_src;
    if (n_pts == 0 || n_src == 0) return PQ3D_OK;
    if (!d_X || !d_Y || !d_Z || !d_P || !d_stress) return PQ3D_ERR_ARG;
    if (halfspace < 0 || halfspace > 2) return PQ3D_ERR_ARG;
    int th = 128;
    const unsigned g = (unsigned)((np + th - 1) / th);
    if (halfspace)
        k_stress_points<true><<<g, th, 0, stream>>>(d_X, d_Y, d_Z, n_pts == 1 ? 0 : 1, d_P, n_src == 1 ? 0 : 1, np,
                                                    Ss, Ds, Ts, mu, lam, halfspace, d_stress, d_strain);
    else
        k_stress_points<false><<<g, th, 0, stream>>>(d_X, d_Y, d_Z, n_pts == 1 ? 0 : 1, d_P, n_src == 1 ? 0 : 1, np,
                                                     Ss, Ds, Ts, mu, lam, 0, d_stress, d_strain);
    return pq3d_launch_status();
}

// Host-pointer drop-ins.  Same signature, argument meaning and output layout as
// the reference (no return value); inputs are staged to the device, the pair
// kernel runs, outputs come back before return.  A CUDA failure is reported on
// stderr and the outputs are filled with NaN (the reference has no error channel).
static void fill_nan(double *a, size_t n)
{
    if (!a) return;
    for (size_t i = 0; i < n; ++i) a[i] = __builtin_nan("");
}

// Staging of the drop-ins: per device, one device buffer and one pinned host
// buffer, grown to the largest call and kept until exit, and one stream.  The
// reference calls its entry points for every row and column of small blocks,
// so per-call allocations and several pageable copies would cost more than the
// work: small calls pack their inputs into the pinned buffer and cross in one
// copy each way.  Calls on a device are serialised by a mutex (the buffers are
// shared).
namespace {
constexpr int kDropinDevices = 64;
struct DropinStage {
    double *buf = nullptr, *hbuf = nullptr;
    size_t cap = 0, hcap = 0;
    cudaStream_t st = nullptr;
};
std::mutex g_dropin_mu[kDropinDevices];
DropinStage g_dropin[kDropinDevices];

int grow(double *&p, size_t &cap, size_t need, bool host)
{
    if (cap >= need) return PQ3D_OK;
    const size_t c = need > 2 * cap ? need : 2 * cap;
    if (p) {
        if (host) cudaFreeHost(p);
        else cudaFree(p);
    }
    p = nullptr;
    cap = 0;
    const cudaError_t e = host ? cudaHostAlloc((void **)&p, c * sizeof(double), cudaHostAllocDefault)
                               : cudaMalloc((void **)&p, c * sizeof(double));
    if (e != cudaSuccess) {
        p = nullptr;
        return PQ3D_ERR_CUDA;
    }
    cap = c;
    return PQ3D_OK;
}
}  // namespace

static int stress_host(const double *X, const double *Y, const double *Z, size_t npt,
                       const double *P9, size_t nsrc, double Ss, double Ds, double Ts, double mu,
                       double lam, bool hs, double *stress, double *strain)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kDropinDevices) return PQ3D_ERR_CUDA;
    std::lock_guard<std::mutex> lk(g_dropin_mu[dev]);
    DropinStage &S = g_dropin[dev];
    const size_t np = npt > nsrc ? npt : nsrc;
    const size_t nin = 3 * npt + 9 * nsrc, need = nin + 12 * np;   // inputs, then stress + strain
    if (!S.st && cudaStreamCreateWithFlags(&S.st, cudaStreamNonBlocking) != cudaSuccess) {
        S.st = nullptr;
        return PQ3D_ERR_CUDA;
    }
    // small calls: pack into pinned memory, one copy each way; large calls (over
    // 1 MB) copy the caller's arrays directly, where packing would cost more
    const bool packed = need * sizeof(double) <= (size_t(1) << 20);
    if (grow(S.buf, S.cap, need, false) != PQ3D_OK || (packed && grow(S.hbuf, S.hcap, need, true) != PQ3D_OK))
        return PQ3D_ERR_CUDA;
    double *h = S.hbuf, *d = S.buf, *dS = d + nin;
    const cudaStream_t st = S.st;
    const size_t b = npt * sizeof(double), bp = 9 * nsrc * sizeof(double);
    if (packed) {
        memcpy(h, X, b);
        memcpy(h + npt, Y, b);
        memcpy(h + 2 * npt, Z, b);
        memcpy(h + 3 * npt, P9, bp);
        if (cudaMemcpyAsync(d, h, nin * sizeof(double), cudaMemcpyHostToDevice, st) != cudaSuccess)
            return PQ3D_ERR_CUDA;
    } else if (cudaMemcpyAsync(d, X, b, cudaMemcpyHostToDevice, st) != cudaSuccess ||
               cudaMemcpyAsync(d + npt, Y, b, cudaMemcpyHostToDevice, st) != cudaSuccess ||
               cudaMemcpyAsync(d + 2 * npt, Z, b, cudaMemcpyHostToDevice, st) != cudaSuccess ||
               cudaMemcpyAsync(d + 3 * npt, P9, bp, cudaMemcpyHostToDevice, st) != cudaSuccess) {
        return PQ3D_ERR_CUDA;
    }
    int rc = pq3d_stress_points(d, d + npt, d + 2 * npt, (int64_t)npt, d + 3 * npt, (int64_t)nsrc, Ss, Ds, Ts, mu,
                                lam, hs ? 2 : 0, dS, dS + 6 * np, st);
    if (rc != PQ3D_OK) return rc;
    const size_t bs = 6 * np * sizeof(double);
    if (packed) {
        if (cudaMemcpyAsync(h + nin, dS, (strain ? 2 : 1) * bs, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
            return PQ3D_ERR_CUDA;
        memcpy(stress, h + nin, bs);
        if (strain) memcpy(strain, h + nin + 6 * np, bs);
        return PQ3D_OK;
    }
    if (cudaMemcpyAsync(stress, dS, bs, cudaMemcpyDeviceToHost, st) != cudaSuccess) return PQ3D_ERR_CUDA;
    if (strain && cudaMemcpyAsync(strain, dS + 6 * np, bs, cudaMemcpyDeviceToHost, st) != cudaSuccess)
        return PQ3D_ERR_CUDA;
    return cudaStreamSynchronize(st) == cudaSuccess ? PQ3D_OK : PQ3D_ERR_CUDA;
}

// Replaces TDstressFS_C (src/TDstressFS_C.cpp:2048-2095): one source triangle, n receivers.
PQ3D_EXPORT void TDstressFS_C(const double *X, const double *Y, const double *Z, size_t n,
                              const double *P1, const double *P2, const double *P3, double Ss,
                              double Ds, double Ts, double mu, double lambda_, bool jud_halfspace,
                              double *stress, double *strain)
{
    if (n == 0) return;
    if (jud_halfspace) {
        double zmax = Z[0];
        for (size_t i = 1; i < n; ++i) zmax = Z[i] > zmax ? Z[i] : zmax;
        if (zmax > 0 || P1[2] > 0 || P2[2] > 0 || P3[2] > 0)
            printf("Half-space solution: Z coordinates must be negative!\n");
    }
    double P9[9] = {P1[0], P1[1], P1[2], P2[0], P2[1], P2[2], P3[0], P3[1], P3[2]};
    int rc = stress_host(X, Y, Z, n, P9, 1, Ss, Ds, Ts, mu, lambda_, jud_halfspace, stress, strain);
    if (rc != PQ3D_OK) {
        fprintf(stderr, "pq3d TDstressFS_C: CUDA failure %d\n", rc);
        fill_nan(stress, 6 * n);
        fill_nan(strain, 6 * n);
    }
}

// Replaces TDstressEachSourceAtReceiver_C (src/TDstressFS_C.cpp:2098-2143): one
// receiver, n_sources triangles given as flat xyz triplets.
PQ3D_EXPORT void TDstressEachSourceAtReceiver_C(double x, double y, double z, const double *P1_flat,
                                                const double *P2_flat, const double *P3_flat,
                                                size_t n_sources, double Ss, double Ds, double Ts,
                                                double mu, double lambda_, bool jud_halfspace,
                                                double *stress_out, double *strain_out)
{
    if (n_sources == 0) return;
    double *P9 = (double *)malloc(9 * n_sources * sizeof(double));
    if (!P9) {
        fill_nan(stress_out, 6 * n_sources);
        fill_nan(strain_out, 6 * n_sources);
        return;
    }
    for (size_t i = 0; i < n_sources; ++i) {
        for (int k = 0; k < 3; ++k) {
            P9[9 * i + k] = P1_flat[3 * i + k];
            P9[9 * i + 3 + k] = P2_flat[3 * i + k];
            P9[9 * i + 6 + k] = P3_flat[3 * i + k];
        }
        // the reference's warning, once per offending source (its TDstressHS runs per source)
        if (jud_halfspace && (z > 0 || P9[9 * i + 2] > 0 || P9[9 * i + 5] > 0 || P9[9 * i + 8] > 0))
            printf("Half-space solution: Z coordinates must be negative!\n");
    }
    int rc = stress_host(&x, &y, &z, 1, P9, n_sources, Ss, Ds, Ts, mu, lambda_, jud_halfspace, stress_out,
                         strain_out);
    free(P9);
    if (rc != PQ3D_OK) {
        fprintf(stderr, "pq3d TDstressEachSourceAtReceiver_C: CUDA failure %d\n", rc);
        fill_nan(stress_out, 6 * n_sources);
        fill_nan(strain_out, 6 * n_sources);
    }
}

// ---------------------------------------------------------------- dense near-field assembly
// One CTA per dense block (blocks listed largest first).  Entry (i, j) of block b is the
// traction at the element in tree position r0+i due to the element in tree position c0+j,
// written straight into the packed matvec layout (FP64 and/or FP32 copies).
template <bool HS>
__global__ void k_dense_assemble(const double *__restrict__ xg, const double *__restrict__ ev,
                                 const SrcRec *__restrict__ rec, const int32_t *__restrict__ perm,
                                 const DenseBlock *__restrict__ blocks, double mu, double lam,
                                 double *__restrict__ out64, float *__restrict__ out32,
                                 const HsRec *__restrict__ hs, int hs_mode)
{
    const DenseBlock B = blocks[blockIdx.x];
    const double nu = 1.0 / (1.0 + lam / mu) / 2.0;
    const int64_t npairs = (int64_t)B.m * B.n;
    for (int64_t p = threadIdx.x; p < npairs; p += blockDim.x) {
        int i = (int)(p % B.m), j = (int)(p / B.m);
        int r = perm[B.r0 + i], c = perm[B.c0 + j];
        double obs[3] = {xg[3 * r], xg[3 * r + 1], xg[3 * r + 2]};
        double f[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) f[k] = ev[9 * r + k];
        double t[6];
        if (HS) gf_traction_sd_hs(obs, f, rec[c], hs[c], hs_mode, mu, lam, nu, t);
        else gf_traction_sd(obs, f, rec[c], mu, lam, nu, t);
#pragma unroll
        for (int slip = 0; slip < 2; ++slip)
#pragma unroll
            for (int comp = 0; comp < 3; ++comp) {
                double v = t[3 * slip + comp];
                if (out64) out64[B.off64 + dense_index(B.m, i, j + B.c0 % kCW64, comp, slip, kCW64)] = v;
                if (out32) out32[B.off32 + dense_index(B.m, i, j + B.c0 % kCW32, comp, slip, kCW32)] = (float)v;
            }
    }
}

PQ3D_EXPORT int pq3d_dense_assemble(const double *d_xg, const double *d_ev, const void *d_rec,
                                    const int32_t *d_perm, const void *d_blocks, int64_t n_blocks,
                                    double mu, double lam, double *d_out64, float *d_out32,
                                    const void *d_hs, int hs_mode, cudaStream_t stream)
{
    if (n_blocks < 0 || !hs_args_ok(d_hs, hs_mode)) return PQ3D_ERR_ARG;
    if (n_blocks == 0) return PQ3D_OK;
    if (!d_xg || !d_ev || !d_rec || !d_perm || !d_blocks || (!d_out64 && !d_out32)) return PQ3D_ERR_ARG;
    for (int64_t b0 = 0; b0 < n_blocks; b0 += 65535) {
        int64_t nb = n_blocks - b0 < 65535 ? n_blocks - b0 : 65535;
        if (hs_mode)
            k_dense_assemble<true><<<(unsigned)nb, 256, 0, stream>>>(d_xg, d_ev, (const SrcRec *)d_rec, d_perm,
                                                                    (const DenseBlock *)d_blocks + b0, mu, lam,
                                                                    d_out64, d_out32, (const HsRec *)d_hs, hs_mode);
        else
            k_dense_assemble<false><<<(unsigned)nb, 256, 0, stream>>>(d_xg, d_ev, (const SrcRec *)d_rec, d_perm,
                                                                     (const DenseBlock *)d_blocks + b0, mu, lam,
                                                                     d_out64, d_out32, nullptr, 0);
    }
    return pq3d_launch_status();
}
