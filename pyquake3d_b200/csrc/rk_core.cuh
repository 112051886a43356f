// Element-wise pieces of the reference's rate-and-state DP5(4) step, shared by
// the single-fault step kernel (rk.cu) and the ensemble step kernel (ensemble.cu).
#pragma once
#include "pq3d_common.cuh"

namespace pq3d_rk {

__device__ __forceinline__ double py_min(double a, double b) { return (b < a) ? b : a; }
__device__ __forceinline__ double py_max(double a, double b) { return (b > a) ? b : a; }
__device__ __forceinline__ double nanmax(double a, double b)
{
    if (a != a || b != b) return __longlong_as_double(0x7ff8000000000000ULL);
    return a > b ? a : b;
}

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


// The H-matvec's row reduction (k_rowsum) fused into the step kernels:
// y[i] = sum of row i's slots, in the per-leaf list order, for the CTA's rows
// [base, min(base + NT, end)), with all NT threads of the CTA taking part (call
// from every thread).  The leaf_off range of the CTA's leaves is contiguous
// (leaves are numbered in row order), so it is staged in shared memory once;
// then every thread sums its row's slots with eight list entries of loads in
// flight.
constexpr int RS_STAGE = 2048;   // staged leaf_off entries per CTA (larger ranges read them from global)

template <int NT, class A>
__device__ __forceinline__ void rowsum_cta(const A &S, int64_t base, int64_t end)
{
    __shared__ int s_off[RS_STAGE];
    __shared__ int s_kb, s_ke;
    const int64_t n = end;
    const int64_t i = base + threadIdx.x;
    const int64_t last = (base + NT < n ? base + NT : n) - 1;
    int k0 = 0, k1 = 0;
    if (i < n) {
        const int l = S.leaf_of_row[i];
        k0 = S.leaf_ptr[l];
        k1 = S.leaf_ptr[l + 1];
    }
    if (threadIdx.x == 0) s_kb = k0;
    if (i == last) s_ke = k1;
    __syncthreads();
    const int kb = s_kb, ke = s_ke;
    const bool staged = ke - kb <= RS_STAGE;
    if (staged)
        for (int k = kb + (int)threadIdx.x; k < ke; k += NT) s_off[k - kb] = __ldg(S.leaf_off + k);
    __syncthreads();
    if (i < n) {
        double a0 = 0, a1 = 0, a2 = 0;
        int k = k0;
        if (S.slots_fp32) {
            const float *sl = (const float *)S.slots;
            for (; k + 8 <= k1; k += 8) {
                float v[24];
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    const int off = staged ? s_off[k + u - kb] : __ldg(S.leaf_off + k + u);
                    const int64_t s = 3 * ((int64_t)off + i);
                    v[3 * u] = __ldcg(sl + s); v[3 * u + 1] = __ldcg(sl + s + 1); v[3 * u + 2] = __ldcg(sl + s + 2);
                }
#pragma unroll
                for (int u = 0; u < 8; ++u) { a0 += (double)v[3 * u]; a1 += (double)v[3 * u + 1]; a2 += (double)v[3 * u + 2]; }
            }
            for (; k < k1; ++k) {
                const int off = staged ? s_off[k - kb] : __ldg(S.leaf_off + k);
                const int64_t s = 3 * ((int64_t)off + i);
                a0 += (double)__ldcg(sl + s); a1 += (double)__ldcg(sl + s + 1); a2 += (double)__ldcg(sl + s + 2);
            }
        } else {
            const double *sl = (const double *)S.slots;
            for (; k + 8 <= k1; k += 8) {
                double v[24];
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    const int off = staged ? s_off[k + u - kb] : __ldg(S.leaf_off + k + u);
                    const int64_t s = 3 * ((int64_t)off + i);
                    v[3 * u] = __ldcg(sl + s); v[3 * u + 1] = __ldcg(sl + s + 1); v[3 * u + 2] = __ldcg(sl + s + 2);
                }
#pragma unroll
                for (int u = 0; u < 8; ++u) { a0 += v[3 * u]; a1 += v[3 * u + 1]; a2 += v[3 * u + 2]; }
            }
            for (; k < k1; ++k) {
                const int off = staged ? s_off[k - kb] : __ldg(S.leaf_off + k);
                const int64_t s = 3 * ((int64_t)off + i);
                a0 += __ldcg(sl + s); a1 += __ldcg(sl + s + 1); a2 += __ldcg(sl + s + 2);
            }
        }
        S.y[3 * i] = a0;
        S.y[3 * i + 1] = a1;
        S.y[3 * i + 2] = a2;
    }
    __syncthreads();   // s_off is reused for the CTA's next rows
}

// One DP5(4) attempt of size h for element i (RungeKutte_solve_Dormand_Prince,
// src/QDsim.py:1001-1134) with the frozen load y[i] and start-of-step slip rate:
// the 5th-order candidate goes to cand (Tno, Tt1o, Tt2o, psi planes of n), the
// relative error terms |dpsi/psi8|, |dTt1/Tt1_8|, |dTt2/Tt2_8|, |dTno/Tno8| to err.
template <class A>
__device__ __forceinline__ void dp54_element(const A &S, int64_t i, double h, double err[4])
{
    const int64_t n = S.n;
    const double a = S.a[i], b = S.b[i], dc = S.dc[i], f0 = S.f0[i], sh = S.shear_loading[i];
    const double ia = 1.0 / a, ib = 1.0 / b, bdc = b / dc;
    const double sv = S.slipv[i];
    const double L1 = S.y[3 * i], L2 = S.y[3 * i + 1];
    const double dsg = S.fix_tn ? S.normal_loading[i] : S.y[3 * i + 2] + S.normal_loading[i];
    const double Tn = S.Tno[i], T1 = S.Tt1o[i], T2 = S.Tt2o[i], ps = S.psi[i];
#define DER(tn, t1, t2, p) derivative(tn, t1, t2, p, ia, ib, bdc, f0, S.V0, sv, L1, L2, dsg, sh, S.eta)
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
    S.cand[i] = y5n;
    S.cand[n + i] = y51;
    S.cand[2 * (int64_t)n + i] = y52;
    S.cand[3 * (int64_t)n + i] = y5p;
    err[0] = fabs(fabs(y8p - y5p) / y8p);
    // Relerrormax2 = max(max|dTt1/Tt1|, max|dTt2/Tt2|, max|dTno/Tno|): the three
    // maxima are reduced separately and combined with Python max() afterwards.
    err[1] = fabs(fabs(y81 - y51) / y81);
    err[2] = fabs(fabs(y82 - y52) / y82);
    err[3] = fabs(fabs(y8n - y5n) / y8n);
}

// Accepted step for element i (src/QDsim.py:960-993): state from cand, slip
// rates, rake, slip, friction, and the next slip-rate deficit in both x layouts
// (:902-903).  Returns the new slip rates (v1o, v2o).
template <class A>
__device__ __forceinline__ void accept_element(const A &S, int64_t i, double h, double &v1o, double &v2o)
{
    const int64_t n = S.n;
    const double Tn = S.cand[i], T1 = S.cand[n + i], T2 = S.cand[2 * (int64_t)n + i],
                 ps = S.cand[3 * (int64_t)n + i];
    const double a = S.a[i];
    S.Tno[i] = Tn; S.Tt1o[i] = T1; S.Tt2o[i] = T2; S.psi[i] = ps;
    S.Tt[i] = sqrt(T1 * T1 + T2 * T2);
    const double ex = exp(-ps / a);
    const double v1 = (2.0 * S.V0) * ex * sinh(T1 / Tn / a);
    const double v2 = (2.0 * S.V0) * ex * sinh(T2 / Tn / a);
    S.slipv1[i] = v1;
    S.slipv2[i] = v2;
    double vv = sqrt(v1 * v1 + v2 * v2);
    S.rake[i] = atan2(T2, T1);
    if (vv < 1e-30) vv = 1e-30;
    S.slipv[i] = vv;
    const double s1 = S.slip1[i] + v1 * h, s2 = S.slip2[i] + v2 * h;
    S.slip1[i] = s1; S.slip2[i] = s2;
    S.slip[i] = sqrt(s1 * s1 + s2 * s2);
    S.fric[i] = S.Tt[i] / Tn;
    const double x1 = v1 - S.vplc[i] * S.cr0[i];
    const double x2 = v2 - S.vplc[i] * S.sr0[i];
    // interleaved copy (dense blocks) and strike / dip planes (V rows)
    const int64_t P = ((n + 16 + 7) / 8) * 8;
    if (S.x_fp32) {
        float *xf = (float *)S.x;
        xf[2 * i] = (float)x1;
        xf[2 * i + 1] = (float)x2;
        xf[2 * P + i] = (float)x1;
        xf[3 * P + i] = (float)x2;
    } else {
        double *xd = (double *)S.x;
        xd[2 * i] = x1;
        xd[2 * i + 1] = x2;
        xd[2 * P + i] = x1;
        xd[3 * P + i] = x2;
    }
    v1o = v1;
    v2o = v2;
}

// Step-size controller of the reference (src/QDsim.py:931-958) for one attempt
// with error maxima E (psi, Tt1, Tt2, Tno).  Returns true when the attempt ends
// the step (accepted, or given up: h < 1e-15 or more than 20 rejections).
struct StepCtl {
    double h, dtnext;
    int nrjct, attempt;
    bool accepted;
};

__device__ __forceinline__ bool controller(StepCtl &c, const double E[4], double reltol, bool forced)
{
    const double R1 = E[0] + 1e-10;
    const double R2 = py_max(py_max(E[1], E[2]), E[3]) + 1e-10;
    const double c1 = R1 / reltol, c2 = R2 / reltol;
    const double hnew1 = c.h * 0.9 * pow(reltol / R1, 0.2);
    const double hnew2 = c.h * 0.9 * pow(reltol / R2, 0.2);
    c.attempt++;
    if (forced || (py_max(c1, c2) < 1.0 && !(c1 != c1 || c2 != c2))) {
        c.dtnext = py_min(py_min(hnew1, hnew2), 1.5 * c.h);
        c.accepted = true;
        return true;
    }
    c.nrjct++;
    c.dtnext = py_min(hnew1, hnew2);
    c.h = py_max(0.5 * c.h, c.dtnext);
    return c.h < 1.e-15 || c.nrjct > 20;
}

}  // namespace pq3d_rk
