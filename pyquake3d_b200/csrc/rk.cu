// Fused rate-and-state Dormand-Prince 5(4) step, FP64, reference formulation.
//
// One cooperative launch performs one time step of QDsim.simu_forward
// (src/QDsim.py:892-996) after the elastic load has been applied:
//  * the load (AdotV1, AdotV2, dsigma/dt) and the start-of-step slip rate are
//    frozen for all stages and retries, as in the reference (:906-922, :803);
//  * every attempt runs the 7 stages of RungeKutte_solve_Dormand_Prince
//    (:1001-1134) element-wise with derivative (:760-813), reduces the max
//    relative errors over all elements, and applies the reference's
//    accept/reject controller (:931-958) identically in every CTA;
//  * the accepted step updates slip rates, rake, slip and friction (:960-993)
//    and writes the next slip-rate deficit (:902-903) for the next matvec.
// Python min()/max() semantics (including their NaN behaviour) are kept.
// Optional dt replay (hforce) takes a given step size and accepts it, so two
// runs (e.g. FP64 and mixed-precision operators) can be compared at equal times.
// Grid-wide barriers are bounded spins; a timeout sets PQ3D_ERR_TIMEOUT.
#include "pq3d_common.cuh"

namespace {

struct RkArgs {
    double *Tno, *Tt1o, *Tt2o, *psi;                        // state (MPa, MPa, MPa, -)
    double *slip1, *slip2, *slipv1, *slipv2, *slipv, *rake, *Tt, *fric, *slip;
    const double *a, *b, *dc, *f0, *shear_loading, *normal_loading, *vplc, *cr0, *sr0;
    double *y;           // elastic load rates (n x 3): A1 x, A2 x, B x  (Pa/s)
    double *cand;        // 4n scratch
    double *blk;         // 10 * gridDim scratch: per-CTA maxima [0,4G), [4G,6G); reduced result at 6G
    void *x;             // next deficit, interleaved (2n + padding), FP32 or FP64
    double *ctrl;        // control block (see pq3d.h)
    double *hist;        // per-step history, 6 doubles per step (may be null)
    const double *hforce; // dt replay: if non-null, step s uses h = hforce[s] and is accepted
    unsigned *bar;       // bar[0] arrivals, bar[1] generation, bar[2] end-of-step count (zeroed once)
    const void *slots;   // when fuse_rowsum: per-row partial sums of the H-matvec
    const int32_t *leaf_of_row, *leaf_ptr, *leaf_off;
    int n, fix_tn, x_fp32, step_index, fuse_rowsum, slots_fp32;
    double V0, eta, reltol;
};

__device__ __forceinline__ double py_min(double a, double b) { return (b < a) ? b : a; }
__device__ __forceinline__ double py_max(double a, double b) { return (b > a) ? b : a; }
__device__ __forceinline__ double nanmax(double a, double b)
{
    if (a != a || b != b) return __longlong_as_double(0x7ff8000000000000ULL);
    return a > b ? a : b;
}

// Grid-wide NaN-propagating max of four values.  Every CTA reduces its own
// values and posts them to blk; the CTA that arrives last at the barrier reduces
// the posted values with all its threads, publishes the result in res and then
// releases the others (bounded spin: on timeout ctrl[4] = PQ3D_ERR_TIMEOUT and
// false is returned).  All CTAs return the same four values.
// bar[0]: arrival count, bar[1]: generation, bar[2]: end-of-step count.
template <int NT>
__device__ bool grid_max4(double *v, double *blk, double *res, unsigned *bar, double *ctrl)
{
    __shared__ double wred[NT / 32][4];
    __shared__ int s_last;
    __shared__ unsigned s_gen;
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[q] = nanmax(v[q], __shfl_down_sync(0xffffffffu, v[q], o));
    if ((threadIdx.x & 31) == 0)
#pragma unroll
        for (int q = 0; q < 4; ++q) wred[threadIdx.x >> 5][q] = v[q];
    __syncthreads();
    if (threadIdx.x == 0) {
        double w[4] = {wred[0][0], wred[0][1], wred[0][2], wred[0][3]};
        for (int k = 1; k < NT / 32; ++k)
            for (int q = 0; q < 4; ++q) w[q] = nanmax(w[q], wred[k][q]);
        for (int q = 0; q < 4; ++q) blk[(int64_t)q * gridDim.x + blockIdx.x] = w[q];
        s_gen = *(volatile unsigned *)(bar + 1);
        __threadfence();
        s_last = atomicAdd(bar, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    bool ok = true;
    if (s_last) {
        __threadfence();
        double m[4] = {0, 0, 0, 0};
        for (unsigned k = threadIdx.x; k < gridDim.x; k += NT)
#pragma unroll
            for (int q = 0; q < 4; ++q) m[q] = nanmax(m[q], __ldcg(blk + (int64_t)q * gridDim.x + k));
#pragma unroll
        for (int q = 0; q < 4; ++q)
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) m[q] = nanmax(m[q], __shfl_down_sync(0xffffffffu, m[q], o));
        __syncthreads();
        if ((threadIdx.x & 31) == 0)
#pragma unroll
            for (int q = 0; q < 4; ++q) wred[threadIdx.x >> 5][q] = m[q];
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int q = 0; q < 4; ++q) {
                double w = wred[0][q];
                for (int k = 1; k < NT / 32; ++k) w = nanmax(w, wred[k][q]);
                __stcg(res + q, w);
            }
            __threadfence();
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(bar + 1, 1u);
        }
    } else if (threadIdx.x == 0) {
        long long it = 0;
        while (*(volatile unsigned *)(bar + 1) == s_gen) {
            if (++it > (1LL << 24)) {
                ctrl[4] = (double)PQ3D_ERR_TIMEOUT;
                ok = false;
                break;
            }
            __nanosleep(64);
        }
        __threadfence();
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 4; ++q) v[q] = __ldcg(res + q);
    return __syncthreads_and(ok);
}

#ifndef PQ3D_RK_THREADS
#define PQ3D_RK_THREADS 256
#endif
constexpr int RK_THREADS = PQ3D_RK_THREADS;   // CTA size of the step kernel

struct Deriv {
    double dpsi, dsig, dt1, dt2;
};

// derivative (src/QDsim.py:760-813); Tno, Tt in MPa, loads in Pa/s.  The same
// expressions, with the quotients shared through per-element (ia = 1/a,
// ib = 1/b, bdc = b/dc) and per-stage (1/(a Tno)) reciprocals.
__device__ __forceinline__ Deriv derivative(double Tno, double Tt1o, double Tt2o, double state, double ia,
                                            double ib, double bdc, double f0, double V0, double slipv,
                                            double AdotV1, double AdotV2, double dsigmadt, double shear,
                                            double eta)
{
    Tno = Tno * 1e6;
    Tt1o = Tt1o * 1e6;
    Tt2o = Tt2o * 1e6;
    const double iaT = ia / Tno;                  // 1 / (a Tno)
    const double sa = -state * ia;
    const double e1p = exp(sa + Tt1o * iaT), e1m = exp(sa - Tt1o * iaT);
    const double e2p = exp(sa + Tt2o * iaT), e2m = exp(sa - Tt2o * iaT);
    const double g1 = V0 * iaT * (e1p + e1m);     // 2 V0/(a Tno) * cosh-term
    const double g2 = V0 * iaT * (e2p + e2m);
    const double dV1dtau = g1, dV2dtau = g2;
    const double iTno = 1.0 / Tno;
    const double dV1dsigma = -g1 * Tt1o * iTno;
    const double dV2dsigma = -g2 * Tt2o * iTno;
    const double dV1dstate = -V0 * ia * (e1p - e1m);
    const double dV2dstate = -V0 * ia * (e2p - e2m);
    double arg = (f0 - state) * ib;
    arg = arg > 700.0 ? 700.0 : (arg < -700.0 ? -700.0 : arg);
    const double dstatedt = bdc * (V0 * exp(arg) - slipv);
    const double dtau1dt = (-AdotV1 + shear - eta * (dV1dsigma * dsigmadt + dV1dstate * dstatedt)) / (1.0 + eta * dV1dtau);
    const double dtau2dt = (-AdotV2 + shear - eta * (dV2dsigma * dsigmadt + dV2dstate * dstatedt)) / (1.0 + eta * dV2dtau);
    return Deriv{dstatedt, dsigmadt * 1e-6, dtau1dt * 1e-6, dtau2dt * 1e-6};
}

// Dormand-Prince 5(4) tableau (src/QDsim.py:1002-1032).
constexpr double B21 = .2;
constexpr double B31 = 3. / 40, B32 = 9. / 40.;
constexpr double B41 = 44. / 45., B42 = -56. / 15, B43 = 32. / 9;
constexpr double B51 = 19372. / 6561., B52 = -25360 / 2187., B53 = 64448. / 6561., B54 = -212. / 729.;
constexpr double B61 = 9017. / 3168., B62 = -355. / 33., B63 = -46732. / 5247., B64 = 49. / 176., B65 = -5103. / 18656.;
constexpr double B71 = 35. / 384., B73 = 500. / 1113., B74 = 125. / 192., B75 = -2187. / 6784., B76 = 11. / 84.;
constexpr double B81 = 5179. / 57600., B83 = 7571. / 16695., B84 = 393. / 640., B85 = -92097. / 339200.,
                 B86 = 187. / 2100., B87 = 1. / 40.;

__global__ void __launch_bounds__(RK_THREADS) k_rk_step(RkArgs A)
{
    const int n = A.n;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t tid0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (A.fuse_rowsum) {
        // the H-matvec's row reduction (k_rowsum) done here: y[i] = sum of row i's slots
        for (int64_t i = tid0; i < n; i += stride) {
            const int l = A.leaf_of_row[i];
            double a0 = 0, a1 = 0, a2 = 0;
            const int k0 = A.leaf_ptr[l], k1 = A.leaf_ptr[l + 1];
            if (A.slots_fp32) {
                const float *sl = (const float *)A.slots;
                int k = k0;
                for (; k + 4 <= k1; k += 4) {   // four independent loads in flight, list-order sums
                    float v[12];
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const int64_t s = 3 * ((int64_t)A.leaf_off[k + u] + i);
                        v[3 * u] = sl[s]; v[3 * u + 1] = sl[s + 1]; v[3 * u + 2] = sl[s + 2];
                    }
#pragma unroll
                    for (int u = 0; u < 4; ++u) { a0 += (double)v[3 * u]; a1 += (double)v[3 * u + 1]; a2 += (double)v[3 * u + 2]; }
                }
                for (; k < k1; ++k) {
                    const int64_t s = 3 * ((int64_t)A.leaf_off[k] + i);
                    a0 += (double)sl[s]; a1 += (double)sl[s + 1]; a2 += (double)sl[s + 2];
                }
            } else {
                const double *sl = (const double *)A.slots;
                int k = k0;
                for (; k + 4 <= k1; k += 4) {
                    double v[12];
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const int64_t s = 3 * ((int64_t)A.leaf_off[k + u] + i);
                        v[3 * u] = sl[s]; v[3 * u + 1] = sl[s + 1]; v[3 * u + 2] = sl[s + 2];
                    }
#pragma unroll
                    for (int u = 0; u < 4; ++u) { a0 += v[3 * u]; a1 += v[3 * u + 1]; a2 += v[3 * u + 2]; }
                }
                for (; k < k1; ++k) {
                    const int64_t s = 3 * ((int64_t)A.leaf_off[k] + i);
                    a0 += sl[s]; a1 += sl[s + 1]; a2 += sl[s + 2];
                }
            }
            A.y[3 * i] = a0;
            A.y[3 * i + 1] = a1;
            A.y[3 * i + 2] = a2;
        }
    }
    const bool forced = A.hforce != nullptr;
    double h = forced ? A.hforce[A.step_index] : A.ctrl[0];
    int nrjct = 0, attempt = 0;
    bool accepted = false;
    double dtnext = h;

    while (true) {
        double m1 = 0.0, g1 = 0.0, g2 = 0.0, g3 = 0.0;  // max relative errors, NaN-propagating
        for (int64_t i = tid0; i < n; i += stride) {
            const double a = A.a[i], b = A.b[i], dc = A.dc[i], f0 = A.f0[i], sh = A.shear_loading[i];
            const double ia = 1.0 / a, ib = 1.0 / b, bdc = b / dc;
            const double sv = A.slipv[i];
            const double L1 = A.y[3 * i], L2 = A.y[3 * i + 1];
            const double dsg = A.fix_tn ? A.normal_loading[i] : A.y[3 * i + 2] + A.normal_loading[i];
            const double Tn = A.Tno[i], T1 = A.Tt1o[i], T2 = A.Tt2o[i], ps = A.psi[i];
#define DER(tn, t1, t2, p) derivative(tn, t1, t2, p, ia, ib, bdc, f0, A.V0, sv, L1, L2, dsg, sh, A.eta)
            const Deriv k1 = DER(Tn, T1, T2, ps);
            const Deriv k2 = DER(Tn + h * B21 * k1.dsig, T1 + h * B21 * k1.dt1, T2 + h * B21 * k1.dt2, ps + h * B21 * k1.dpsi);
            const Deriv k3 = DER(Tn + h * (B31 * k1.dsig + B32 * k2.dsig), T1 + h * (B31 * k1.dt1 + B32 * k2.dt1),
                                 T2 + h * (B31 * k1.dt2 + B32 * k2.dt2), ps + h * (B31 * k1.dpsi + B32 * k2.dpsi));
            const Deriv k4 = DER(Tn + h * (B41 * k1.dsig + B42 * k2.dsig + B43 * k3.dsig),
                                 T1 + h * (B41 * k1.dt1 + B42 * k2.dt1 + B43 * k3.dt1),
                                 T2 + h * (B41 * k1.dt2 + B42 * k2.dt2 + B43 * k3.dt2),
                                 ps + h * (B41 * k1.dpsi + B42 * k2.dpsi + B43 * k3.dpsi));
            const Deriv k5 = DER(Tn + h * (B51 * k1.dsig + B52 * k2.dsig + B53 * k3.dsig + B54 * k4.dsig),
                                 T1 + h * (B51 * k1.dt1 + B52 * k2.dt1 + B53 * k3.dt1 + B54 * k4.dt1),
                                 T2 + h * (B51 * k1.dt2 + B52 * k2.dt2 + B53 * k3.dt2 + B54 * k4.dt2),
                                 ps + h * (B51 * k1.dpsi + B52 * k2.dpsi + B53 * k3.dpsi + B54 * k4.dpsi));
            const Deriv k6 = DER(Tn + h * (B61 * k1.dsig + B62 * k2.dsig + B63 * k3.dsig + B64 * k4.dsig + B65 * k5.dsig),
                                 T1 + h * (B61 * k1.dt1 + B62 * k2.dt1 + B63 * k3.dt1 + B64 * k4.dt1 + B65 * k5.dt1),
                                 T2 + h * (B61 * k1.dt2 + B62 * k2.dt2 + B63 * k3.dt2 + B64 * k4.dt2 + B65 * k5.dt2),
                                 ps + h * (B61 * k1.dpsi + B62 * k2.dpsi + B63 * k3.dpsi + B64 * k4.dpsi + B65 * k5.dpsi));
            const double y5n = Tn + h * (B71 * k1.dsig + B73 * k3.dsig + B74 * k4.dsig + B75 * k5.dsig + B76 * k6.dsig);
            const double y51 = T1 + h * (B71 * k1.dt1 + B73 * k3.dt1 + B74 * k4.dt1 + B75 * k5.dt1 + B76 * k6.dt1);
            const double y52 = T2 + h * (B71 * k1.dt2 + B73 * k3.dt2 + B74 * k4.dt2 + B75 * k5.dt2 + B76 * k6.dt2);
            const double y5p = ps + h * (B71 * k1.dpsi + B73 * k3.dpsi + B74 * k4.dpsi + B75 * k5.dpsi + B76 * k6.dpsi);
            const Deriv k7 = DER(y5n, y51, y52, y5p);
#undef DER
            const double y8n = Tn + h * (B81 * k1.dsig + B83 * k3.dsig + B84 * k4.dsig + B85 * k5.dsig + B86 * k6.dsig + B87 * k7.dsig);
            const double y81 = T1 + h * (B81 * k1.dt1 + B83 * k3.dt1 + B84 * k4.dt1 + B85 * k5.dt1 + B86 * k6.dt1 + B87 * k7.dt1);
            const double y82 = T2 + h * (B81 * k1.dt2 + B83 * k3.dt2 + B84 * k4.dt2 + B85 * k5.dt2 + B86 * k6.dt2 + B87 * k7.dt2);
            const double y8p = ps + h * (B81 * k1.dpsi + B83 * k3.dpsi + B84 * k4.dpsi + B85 * k5.dpsi + B86 * k6.dpsi + B87 * k7.dpsi);
            A.cand[i] = y5n;
            A.cand[n + i] = y51;
            A.cand[2 * (int64_t)n + i] = y52;
            A.cand[3 * (int64_t)n + i] = y5p;
            m1 = nanmax(m1, fabs(fabs(y8p - y5p) / y8p));
            // Relerrormax2 = max(max|dTt1/Tt1|, max|dTt2/Tt2|, max|dTno/Tno|): the three
            // maxima are reduced separately and combined with Python max() afterwards.
            g1 = nanmax(g1, fabs(fabs(y81 - y51) / y81));
            g2 = nanmax(g2, fabs(fabs(y82 - y52) / y82));
            g3 = nanmax(g3, fabs(fabs(y8n - y5n) / y8n));
        }
        // grid-wide maxima of (m1, g1, g2, g3); identical in every CTA
        double E[4] = {m1, g1, g2, g3};
        if (!grid_max4<RK_THREADS>(E, A.blk, A.blk + 6 * (int64_t)gridDim.x, A.bar, A.ctrl)) return;
        const double R1 = E[0] + 1e-10;
        const double R2 = py_max(py_max(E[1], E[2]), E[3]) + 1e-10;
        const double c1 = R1 / A.reltol, c2 = R2 / A.reltol;
        const double hnew1 = h * 0.9 * pow(A.reltol / R1, 0.2);
        const double hnew2 = h * 0.9 * pow(A.reltol / R2, 0.2);
        attempt++;
        if (forced || (py_max(c1, c2) < 1.0 && !(c1 != c1 || c2 != c2))) {
            dtnext = py_min(hnew1, hnew2);
            dtnext = py_min(1.5 * h, dtnext);
            accepted = true;
            break;
        }
        nrjct++;
        dtnext = py_min(hnew1, hnew2);
        h = py_max(0.5 * h, dtnext);
        if (h < 1.e-15 || nrjct > 20) break;
    }

    // accepted step: state update (src/QDsim.py:960-993) and next deficit (:902-903)
    double mv1 = 0.0, mv2 = 0.0;
    if (accepted) {
        for (int64_t i = tid0; i < n; i += stride) {
            const double Tn = A.cand[i], T1 = A.cand[n + i], T2 = A.cand[2 * (int64_t)n + i],
                         ps = A.cand[3 * (int64_t)n + i];
            const double a = A.a[i];
            A.Tno[i] = Tn; A.Tt1o[i] = T1; A.Tt2o[i] = T2; A.psi[i] = ps;
            A.Tt[i] = sqrt(T1 * T1 + T2 * T2);
            const double ex = exp(-ps / a);
            const double v1 = (2.0 * A.V0) * ex * sinh(T1 / Tn / a);
            const double v2 = (2.0 * A.V0) * ex * sinh(T2 / Tn / a);
            A.slipv1[i] = v1;
            A.slipv2[i] = v2;
            double vv = sqrt(v1 * v1 + v2 * v2);
            A.rake[i] = atan2(T2, T1);
            if (vv < 1e-30) vv = 1e-30;
            A.slipv[i] = vv;
            const double s1 = A.slip1[i] + v1 * h, s2 = A.slip2[i] + v2 * h;
            A.slip1[i] = s1; A.slip2[i] = s2;
            A.slip[i] = sqrt(s1 * s1 + s2 * s2);
            A.fric[i] = A.Tt[i] / Tn;
            const double x1 = v1 - A.vplc[i] * A.cr0[i];
            const double x2 = v2 - A.vplc[i] * A.sr0[i];
            // interleaved copy (dense blocks) and strike / dip planes (V rows)
            const int64_t P = ((n + 16 + 7) / 8) * 8;
            if (A.x_fp32) {
                float *xf = (float *)A.x;
                xf[2 * i] = (float)x1;
                xf[2 * i + 1] = (float)x2;
                xf[2 * P + i] = (float)x1;
                xf[3 * P + i] = (float)x2;
            } else {
                double *xd = (double *)A.x;
                xd[2 * i] = x1;
                xd[2 * i + 1] = x2;
                xd[2 * P + i] = x1;
                xd[3 * P + i] = x2;
            }
            mv1 = fmax(mv1, fabs(v1));
            mv2 = fmax(mv2, fabs(v2));
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mv1 = fmax(mv1, __shfl_down_sync(0xffffffffu, mv1, o));
        mv2 = fmax(mv2, __shfl_down_sync(0xffffffffu, mv2, o));
    }
    __shared__ double vred[RK_THREADS / 32][2];
    __shared__ int s_done;
    if ((threadIdx.x & 31) == 0) { vred[threadIdx.x >> 5][0] = mv1; vred[threadIdx.x >> 5][1] = mv2; }
    __syncthreads();
    // the last CTA to finish the step reduces the slip-rate maxima and updates ctrl
    if (threadIdx.x == 0) {
        double w1 = vred[0][0], w2 = vred[0][1];
        for (int k = 1; k < RK_THREADS / 32; ++k) { w1 = fmax(w1, vred[k][0]); w2 = fmax(w2, vred[k][1]); }
        A.blk[(int64_t)4 * gridDim.x + blockIdx.x] = w1;
        A.blk[(int64_t)5 * gridDim.x + blockIdx.x] = w2;
        __threadfence();
        s_done = atomicAdd(A.bar + 2, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_done) return;
    __threadfence();
    double w1 = 0, w2 = 0;
    for (unsigned k = threadIdx.x; k < gridDim.x; k += RK_THREADS) {
        w1 = fmax(w1, __ldcg(A.blk + (int64_t)4 * gridDim.x + k));
        w2 = fmax(w2, __ldcg(A.blk + (int64_t)5 * gridDim.x + k));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        w1 = fmax(w1, __shfl_down_sync(0xffffffffu, w1, o));
        w2 = fmax(w2, __shfl_down_sync(0xffffffffu, w2, o));
    }
    __syncthreads();
    if ((threadIdx.x & 31) == 0) { vred[threadIdx.x >> 5][0] = w1; vred[threadIdx.x >> 5][1] = w2; }
    __syncthreads();
    if (threadIdx.x == 0) {
        w1 = vred[0][0];
        w2 = vred[0][1];
        for (int k = 1; k < RK_THREADS / 32; ++k) { w1 = fmax(w1, vred[k][0]); w2 = fmax(w2, vred[k][1]); }
        A.bar[2] = 0u;
        if (accepted) {
            const double t = A.ctrl[2] + h;
            A.ctrl[2] = t;
            A.ctrl[0] = dtnext;   // next dttry
            A.ctrl[1] = h;        // accepted step
            A.ctrl[3] = nrjct;
            A.ctrl[5] = w1;
            A.ctrl[6] = w2;
            A.ctrl[8] += 1.0;
            A.ctrl[9] += nrjct;
            A.ctrl[10] += attempt;
            if (A.hist) {
                double *hh = A.hist + 6 * (int64_t)A.step_index;
                hh[0] = h; hh[1] = dtnext; hh[2] = t; hh[3] = w1; hh[4] = w2; hh[5] = nrjct;
            }
        } else {
            A.ctrl[1] = h;
            A.ctrl[3] = nrjct;
            if (A.ctrl[4] == 0.0) A.ctrl[4] = (double)PQ3D_ERR_DT;
        }
    }
}

}  // namespace

PQ3D_EXPORT size_t pq3d_rk_args_bytes(void) { return sizeof(RkArgs); }

// Largest co-resident grid for the step kernel on the current device.
PQ3D_EXPORT int pq3d_rk_grid(int n)
{
    int dev = 0, sms = 0, per = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return -1;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return -1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_rk_step, RK_THREADS, 0) != cudaSuccess) return -1;
    int need = (n + RK_THREADS - 1) / RK_THREADS;
    int cap = sms * per;
    return need < cap ? need : cap;
}

// One reference-mode step.  args: host copy of RkArgs; grid from pq3d_rk_grid.
// The launch is cooperative, so all CTAs are co-resident and the barriers complete.
PQ3D_EXPORT int pq3d_rk_step(const void *args, int grid, cudaStream_t stream)
{
    if (!args || grid <= 0) return PQ3D_ERR_ARG;
    RkArgs A = *(const RkArgs *)args;
    if (A.n <= 0 || !A.ctrl || !A.bar || !A.blk || !A.cand || !A.y || !A.x) return PQ3D_ERR_ARG;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3(RK_THREADS);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    PQ3D_CHECK(cudaLaunchKernelEx(&cfg, k_rk_step, A));
    return PQ3D_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free variant of pq3d_rk_step.
//
// Some callers cannot allocate device memory: code that runs inside another
// framework's memory pool or under a host-side allocation policy, embedded
// solvers that only receive pre-allocated state vectors, and callers that
// must not call cudaMalloc in their time loop.  For them the step's scratch
// (candidate state, per-CTA error maxima, grid-barrier counter) lives in the
// file-scope array below, reserved in device memory when the library is
// loaded and held by every GPU that loads it until the process exits.
// Limits: n <= PQ3D_NOALLOC_MAX_N elements and grid <= PQ3D_NOALLOC_MAX_GRID
// CTAs (about 4.5 MB per device).  All calls share the array: the barrier
// counter is cleared on the stream before each launch, and calls that overlap
// on the GPU (different streams, or several threads) race on it.
#define PQ3D_NOALLOC_MAX_N 131072
#define PQ3D_NOALLOC_MAX_GRID 4096   // CTAs of RK_THREADS threads

static __device__ __align__(256) double g_rk_scratch[4 * PQ3D_NOALLOC_MAX_N + 10 * PQ3D_NOALLOC_MAX_GRID + 2];

#include <mutex>
#include <stdio.h>

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
double *g_scratch_dev[kMaxDevices] = {nullptr};

// Device address of g_rk_scratch on the current device.  The name is only a
// host-side stand-in, so the address is looked up once per device (with that
// device current) and cached.
int scratch_address(double **out)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return PQ3D_ERR_CUDA;
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    if (!g_scratch_dev[dev]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_rk_scratch) != cudaSuccess || !p) return PQ3D_ERR_CUDA;
        g_scratch_dev[dev] = (double *)p;
    }
    *out = g_scratch_dev[dev];
    return PQ3D_OK;
}
}  // namespace

// Same step as pq3d_rk_step; the cand, blk and bar members of args are ignored.
// The first call on a device looks up the scratch address (make that call
// before any stream capture).  Allocates nothing.
PQ3D_EXPORT int pq3d_rk_step_noalloc(const void *args, int grid, cudaStream_t stream)
{
    if (!args || grid <= 0) return PQ3D_ERR_ARG;
    RkArgs A = *(const RkArgs *)args;
    if (A.n <= 0 || !A.ctrl || !A.y || !A.x) return PQ3D_ERR_ARG;
    if (A.n > PQ3D_NOALLOC_MAX_N || grid > PQ3D_NOALLOC_MAX_GRID) {
        fprintf(stderr, "pq3d_rk_step_noalloc: n=%d, grid=%d exceed the static scratch (n <= %d, grid <= %d)\n",
                A.n, grid, PQ3D_NOALLOC_MAX_N, PQ3D_NOALLOC_MAX_GRID);
        return PQ3D_ERR_NOMEM;
    }
    double *s = nullptr;
    int rc = scratch_address(&s);
    if (rc != PQ3D_OK) return rc;
    A.cand = s;
    A.blk = s + 4 * (size_t)PQ3D_NOALLOC_MAX_N;
    A.bar = (unsigned *)(s + 4 * (size_t)PQ3D_NOALLOC_MAX_N + 10 * (size_t)PQ3D_NOALLOC_MAX_GRID);
    // the barrier counters must start at zero; the rest is written before it is read
    PQ3D_CHECK(cudaMemsetAsync(A.bar, 0, 4 * sizeof(unsigned), stream));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3(RK_THREADS);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    PQ3D_CHECK(cudaLaunchKernelEx(&cfg, k_rk_step, A));
    return PQ3D_OK;
}
