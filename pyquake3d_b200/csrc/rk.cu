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
    const double *y;     // elastic load rates (n x 3): A1 x, A2 x, B x  (Pa/s)
    double *cand;        // 4n scratch
    double *blk;         // 4 * gridDim scratch (two attempt parities x two maxima) + 2*gridDim
    void *x;             // next deficit, interleaved (2n + padding), FP32 or FP64
    double *ctrl;        // control block (see pq3d.h)
    double *hist;        // per-step history, 6 doubles per step (may be null)
    const double *hforce; // dt replay: if non-null, step s uses h = hforce[s] and is accepted
    unsigned *bar;       // barrier counter + generation
    int n, fix_tn, x_fp32, step_index;
    double V0, eta, reltol;
};

__device__ __forceinline__ double py_min(double a, double b) { return (b < a) ? b : a; }
__device__ __forceinline__ double py_max(double a, double b) { return (b > a) ? b : a; }
__device__ __forceinline__ double nanmax(double a, double b)
{
    if (a != a || b != b) return __longlong_as_double(0x7ff8000000000000ULL);
    return a > b ? a : b;
}

__device__ bool grid_sync(unsigned *bar, double *ctrl)
{
    __syncthreads();
    bool ok = true;
    if (threadIdx.x == 0) {
        volatile unsigned *vgen = bar + 1;
        const unsigned gen = *vgen;
        __threadfence();
        const unsigned arrived = atomicAdd(bar, 1u);
        if (arrived == gridDim.x - 1) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(bar + 1, 1u);
        } else {
            long long it = 0;
            while (*vgen == gen) {
                if (++it > (1LL << 24)) {
                    ctrl[4] = (double)PQ3D_ERR_TIMEOUT;
                    ok = false;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return ok;
}

struct Deriv {
    double dpsi, dsig, dt1, dt2;
};

// derivative (src/QDsim.py:760-813); Tno, Tt in MPa, loads in Pa/s.
__device__ __forceinline__ Deriv derivative(double Tno, double Tt1o, double Tt2o, double state, double a,
                                            double b, double dc, double f0, double V0, double slipv,
                                            double AdotV1, double AdotV2, double dsigmadt, double shear,
                                            double eta)
{
    Tno = Tno * 1e6;
    Tt1o = Tt1o * 1e6;
    Tt2o = Tt2o * 1e6;
    const double aT = a * Tno;
    const double sa = -state / a;
    const double e1p = exp(sa + Tt1o / aT), e1m = exp(sa - Tt1o / aT);
    const double e2p = exp(sa + Tt2o / aT), e2m = exp(sa - Tt2o / aT);
    const double dV1dtau = 2 * V0 / aT * 0.5 * (e1p + e1m);
    const double dV2dtau = 2 * V0 / aT * 0.5 * (e2p + e2m);
    const double aT2 = a * (Tno * Tno);
    const double dV1dsigma = -2 * V0 * Tt1o / aT2 * 0.5 * (e1p + e1m);
    const double dV2dsigma = -2 * V0 * Tt2o / aT2 * 0.5 * (e2p + e2m);
    const double dV1dstate = -2 * V0 / a * 0.5 * (e1p - e1m);
    const double dV2dstate = -2 * V0 / a * 0.5 * (e2p - e2m);
    double arg = (f0 - state) / b;
    arg = arg > 700.0 ? 700.0 : (arg < -700.0 ? -700.0 : arg);
    const double dstatedt = b / dc * (V0 * exp(arg) - slipv);
    const double dtau1dt = (-AdotV1 + shear - eta * (dV1dsigma * dsigmadt + dV1dstate * dstatedt)) / (1.0 + eta * dV1dtau);
    const double dtau2dt = (-AdotV2 + shear - eta * (dV2dsigma * dsigmadt + dV2dstate * dstatedt)) / (1.0 + eta * dV2dtau);
    return Deriv{dstatedt, dsigmadt / 1e6, dtau1dt / 1e6, dtau2dt / 1e6};
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

__global__ void __launch_bounds__(256) k_rk_step(RkArgs A)
{
    const int n = A.n;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t tid0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool forced = A.hforce != nullptr;
    double h = forced ? A.hforce[A.step_index] : A.ctrl[0];
    int nrjct = 0, attempt = 0;
    bool accepted = false;
    double dtnext = h;

    while (true) {
        double m1 = 0.0, g1 = 0.0, g2 = 0.0, g3 = 0.0;  // max relative errors, NaN-propagating
        for (int64_t i = tid0; i < n; i += stride) {
            const double a = A.a[i], b = A.b[i], dc = A.dc[i], f0 = A.f0[i], sh = A.shear_loading[i];
            const double sv = A.slipv[i];
            const double L1 = A.y[3 * i], L2 = A.y[3 * i + 1];
            const double dsg = A.fix_tn ? A.normal_loading[i] : A.y[3 * i + 2] + A.normal_loading[i];
            const double Tn = A.Tno[i], T1 = A.Tt1o[i], T2 = A.Tt2o[i], ps = A.psi[i];
#define DER(tn, t1, t2, p) derivative(tn, t1, t2, p, a, b, dc, f0, A.V0, sv, L1, L2, dsg, sh, A.eta)
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
        // block reduction of (m1, g1, g2, g3)
        double v[4] = {m1, g1, g2, g3};
#pragma unroll
        for (int q = 0; q < 4; ++q)
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v[q] = nanmax(v[q], __shfl_down_sync(0xffffffffu, v[q], o));
        __shared__ double wred[8][4];
        if ((threadIdx.x & 31) == 0)
#pragma unroll
            for (int q = 0; q < 4; ++q) wred[threadIdx.x >> 5][q] = v[q];
        __syncthreads();
        const int par = attempt & 1;
        if (threadIdx.x == 0) {
            double w[4] = {wred[0][0], wred[0][1], wred[0][2], wred[0][3]};
            for (int k = 1; k < (int)(blockDim.x >> 5); ++k)
                for (int q = 0; q < 4; ++q) w[q] = nanmax(w[q], wred[k][q]);
            for (int q = 0; q < 4; ++q) A.blk[(int64_t)(par * 4 + q) * gridDim.x + blockIdx.x] = w[q];
        }
        if (!grid_sync(A.bar, A.ctrl)) return;
        // every CTA reduces the per-CTA maxima in the same order -> identical decision
        double E[4] = {0, 0, 0, 0};
        for (unsigned k = 0; k < gridDim.x; ++k)
#pragma unroll
            for (int q = 0; q < 4; ++q) E[q] = nanmax(E[q], A.blk[(int64_t)(par * 4 + q) * gridDim.x + k]);
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
            if (A.x_fp32) {
                ((float *)A.x)[2 * i] = (float)x1;
                ((float *)A.x)[2 * i + 1] = (float)x2;
            } else {
                ((double *)A.x)[2 * i] = x1;
                ((double *)A.x)[2 * i + 1] = x2;
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
    __shared__ double vred[8][2];
    if ((threadIdx.x & 31) == 0) { vred[threadIdx.x >> 5][0] = mv1; vred[threadIdx.x >> 5][1] = mv2; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double w1 = vred[0][0], w2 = vred[0][1];
        for (int k = 1; k < (int)(blockDim.x >> 5); ++k) { w1 = fmax(w1, vred[k][0]); w2 = fmax(w2, vred[k][1]); }
        A.blk[(int64_t)8 * gridDim.x + blockIdx.x] = w1;
        A.blk[(int64_t)9 * gridDim.x + blockIdx.x] = w2;
    }
    if (!grid_sync(A.bar, A.ctrl)) return;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        double w1 = 0, w2 = 0;
        for (unsigned k = 0; k < gridDim.x; ++k) {
            w1 = fmax(w1, A.blk[(int64_t)8 * gridDim.x + k]);
            w2 = fmax(w2, A.blk[(int64_t)9 * gridDim.x + k]);
        }
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
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_rk_step, 256, 0) != cudaSuccess) return -1;
    int need = (n + 255) / 256;
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
    cfg.blockDim = dim3(256);
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
#define PQ3D_NOALLOC_MAX_GRID 4096

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
    // the barrier counter must start at zero; the rest is written before it is read
    PQ3D_CHECK(cudaMemsetAsync(A.bar, 0, 2 * sizeof(unsigned), stream));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3(256);
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
