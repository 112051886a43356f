// V-mode stepper: slip, state and normal stress integrated with DP5(4) and one
// H-matvec per stage; the slip rate of each element and traction component
// solves the radiation-damped friction law with Newton, seeded by the
// previous stage's rate, by the undamped bound, or by a small MLP.
//
// No counterpart in the reference (its stepper integrates tractions with a
// frozen elastic load, src/QDsim.py:892-1134).  The formulation uses the
// reference's friction law, aging law, loading and elastic operators
// (src/QDsim.py:760-813):
//   deficit d(t) = slip - Vpl (cos r0, sin r0) t
//   tq_c(t) = tq_c(0) - (A_c d)(t) + shear_loading t,   sig(t) = sig(0) + (B d)(t) + normal_loading t
//   tq_c - eta V_c = a sig asinh(V_c e^{psi/a} / (2 V0))
//   z = asinh(|V_c| e^{psi/a} / (2 V0)):  F(z) = z + kappa sinh z - S = 0,
//   S = |tq_c| / (a sig), kappa = 2 V0 eta e^{-psi/a} / (a sig), root in [0, S]
//   d slip_c/dt = V_c,  d psi/dt = (b/Dc)(V0 exp((f0 - psi)/b) - |V|)
// Error: E = max_i max(|dpsi|/|psi|, |dslip_c|/(|slip_c| + atol)) / RelTol; the
// reference's controller constants (0.9, exponent 0.2, growth 1.5, 20 rejects).
//
// One attempt = stages 2..7, each an H-matvec of the stage's deficit followed
// by pq3d_vmode_stage, then pq3d_vmode_finalize.  FSAL: k1 of the next step is
// k7.  The accept/reject decision is taken by the last CTA of stage 7 and read
// by the finalize kernel, so attempts chain on the device with no host sync.
#include "pq3d_common.cuh"
#include <math.h>

namespace {

struct VArgs {
    double *y0;           // 3 x n: slip1, slip2 (m), psi at step start (tree order)
    double *k;            // 7 x 3 x n stage derivatives
    double *y5;           // 3 x n: fifth-order solution (stage-7 input)
    const double *mv;     // n x 3 H-matvec of this stage's deficit: A1 d, A2 d, B d (Pa)
    const double *tq1, *tq2, *sig0;   // quasi-static tractions and normal stress at t = 0 (Pa)
    const double *a, *b, *dc, *f0, *shear_loading, *normal_loading, *vplc, *cr0, *sr0;
    double *V;            // 2 x n: latest slip rates (previous-rate seed)
    void *x;              // deficit of the next matvec (device layout of hm_layout.cuh)
    double *ctrl;         // control block (pq3d.h)
    double *blk;          // 2 * grid scratch
    unsigned *bar;        // bar[0]: stage-7 completion count (zeroed once)
    unsigned long long *stats;  // [0] Newton iterations, [1] solves, [2] max iterations, [3] fallbacks
    const float *mlp;     // MLP parameters (4609 floats) or null
    float *log_x;         // training samples: 5 features + 1 target per sample, or null
    unsigned long long *log_n;
    long long log_cap;
    int n, x_fp32, seed_mode, newton_max;
    double V0, eta, reltol, atol, newton_tol;
    double mlp_gate;      // seed 3: first-step correction (in z) above which the MLP is consulted
};

__device__ const double kC[7] = {0.0, 1.0 / 5, 3.0 / 10, 4.0 / 5, 8.0 / 9, 1.0, 1.0};
__device__ const double kA[7][6] = {
    {0, 0, 0, 0, 0, 0},
    {1.0 / 5, 0, 0, 0, 0, 0},
    {3.0 / 40, 9.0 / 40, 0, 0, 0, 0},
    {44.0 / 45, -56.0 / 15, 32.0 / 9, 0, 0, 0},
    {19372.0 / 6561, -25360.0 / 2187, 64448.0 / 6561, -212.0 / 729, 0, 0},
    {9017.0 / 3168, -355.0 / 33, -46732.0 / 5247, 49.0 / 176, -5103.0 / 18656, 0},
    {35.0 / 384, 0.0, 500.0 / 1113, 125.0 / 192, -2187.0 / 6784, 11.0 / 84}};
__device__ const double kB4[7] = {5179.0 / 57600, 0.0, 7571.0 / 16695, 393.0 / 640, -92097.0 / 339200,
                                  187.0 / 2100, 1.0 / 40};

constexpr int VM_THREADS = 128;
constexpr int MLP_H = 64;
// parameter layout: W1[64][5], b1[64], W2[64][64], b2[64], W3[64], b3[1]
constexpr int OFF_W1 = 0, OFF_B1 = 320, OFF_W2 = 384, OFF_B2 = 4480, OFF_W3 = 4544, OFF_B3 = 4608;

// MLP features of one solve: (log1p S, log10 kappa, a, b, log10 sigma), scaled to O(1).
__device__ inline void mlp_features(double S, double lk, double a, double b, double sig, float *f)
{
    f[0] = (float)(log1p(S) / 5.0);
    f[1] = (float)(lk / 2.302585092994046 / 20.0);
    f[2] = (float)(a * 50.0);
    f[3] = (float)(b * 50.0);
    f[4] = (float)(log10(sig / 1e6) / 2.0);
}

// 5 -> 64 -> 64 -> 1 tanh network, FP32 (parameters read through the read-only cache).
// Both loops over the hidden layer are unrolled completely, so the 64 hidden
// values stay in registers (indexed by constants) instead of local memory.
__device__ inline float mlp_eval(const float *__restrict__ P, const float *f)
{
    float h1[MLP_H];
#pragma unroll
    for (int j = 0; j < MLP_H; ++j) {
        float s = __ldg(P + OFF_B1 + j);
#pragma unroll
        for (int i = 0; i < 5; ++i) s += __ldg(P + OFF_W1 + 5 * j + i) * f[i];
        h1[j] = tanhf(s);
    }
    float out = __ldg(P + OFF_B3);
#pragma unroll 1
    for (int j = 0; j < MLP_H; ++j) {
        float s = __ldg(P + OFF_B2 + j);
        const float4 *w = reinterpret_cast<const float4 *>(P + OFF_W2 + MLP_H * j);
#pragma unroll
        for (int i = 0; i < MLP_H / 4; ++i) {
            const float4 q = __ldg(w + i);
            s += q.x * h1[4 * i];       // the same products in the same order as a scalar loop
            s += q.y * h1[4 * i + 1];
            s += q.z * h1[4 * i + 2];
            s += q.w * h1[4 * i + 3];
        }
        out += __ldg(P + OFF_W3 + j) * tanhf(s);
    }
    return out;
}

struct Solve {
    double V;
    int iters;
    bool fallback;
};

// Newton on F(z) = z + kappa sinh z - S over [0, S]; kappa sinh z, kappa cosh z
// evaluated as exp(lk + z)(1 -/+ e^{-2z})/2 (no overflow).
__device__ inline bool newton(double S, double lk, double tol, int maxit, double &z, int &it)
{
    for (int k = 0; k < maxit; ++k) {
        const double e = exp(lk + z), q = exp(-2.0 * z);
        const double F = z + 0.5 * e * (1.0 - q) - S;
        const double dz = F / (1.0 + 0.5 * e * (1.0 + q));
        double zn = z - dz;
        zn = zn < 0.0 ? 0.0 : (zn > S ? S : zn);
        const bool conv = fabs(zn - z) <= tol * fmax(1.0, z);
        z = zn;
        ++it;
        if (conv) return true;
    }
    return false;
}

__device__ inline Solve vsolve(double tq, double sig, double psi, double a, double b, double V0, double eta,
                               double Vprev, int mode, const float *P, double gate, double tol, int maxit, float *logx,
                               unsigned long long *logn, long long logcap)
{
    const double S = fabs(tq) / (a * sig);
    const double lk = log(2.0 * V0 * eta / (a * sig)) - psi / a;
    double z;
    Solve r{0.0, 0, false};
    bool ok;
    // Undamped start z = S: one Newton step decides whether it is already the root (slow
    // slip, negligible damping); the MLP is consulted only when it is not.
    bool easy = false;
    if (mode == 2 && P) {
        const double e = exp(lk + S), q = exp(-2.0 * S);
        const double dz = 0.5 * e * (1.0 - q) / (1.0 + 0.5 * e * (1.0 + q));
        easy = dz <= tol * fmax(1.0, S);
    }
    if (mode == 3 && P) {
        // Gated network start.  The undamped start z = S takes its first Newton step
        // (the "easy" test above); when that step's correction is at most `gate` in z
        // the solve goes on with plain Newton from there -- the usual case away from
        // nucleation, where it converges in a step or two -- and only a larger
        // correction (strong radiation damping) evaluates the network, whose start Newton
        // then refines.  The step from z = S counts as an iteration either way; the
        // bracketed solve stays the fallback.
        const double e0 = exp(lk + S), q0 = exp(-2.0 * S);
        const double dz0 = 0.5 * e0 * (1.0 - q0) / (1.0 + 0.5 * e0 * (1.0 + q0));
        r.iters = 1;
        double z1 = S - dz0;
        z1 = z1 < 0.0 ? 0.0 : z1;
        if (dz0 <= tol * fmax(1.0, S)) {
            z = S;
        } else {
            if (dz0 > gate) {
                float f[5];
                mlp_features(S, lk, a, b, sig, f);
                z = S / (1.0 + exp(-(double)mlp_eval(P, f)));
            } else {
                z = z1;
            }
            ok = newton(S, lk, tol, maxit, z, r.iters);
            const double e = exp(lk + z), res = fabs(z + 0.5 * e * (1.0 - exp(-2.0 * z)) - S);
            if (!ok || res > 1e-10 * (1.0 + S)) {
                r.fallback = true;
                z = S;
                ok = newton(S, lk, tol, maxit, z, r.iters);
            }
        }
    } else if (mode == 2 && P && easy) {
        z = S;
        r.iters = 1;
    } else if (mode == 2 && P) {
        float f[5];
        mlp_features(S, lk, a, b, sig, f);
        const float q = mlp_eval(P, f);
        z = S / (1.0 + exp(-(double)q));
        // the MLP only proposes the start: a few Newton steps, judged by the residual
        ok = newton(S, lk, tol, 8, z, r.iters);
        const double e = exp(lk + z), res = fabs(z + 0.5 * e * (1.0 - exp(-2.0 * z)) - S);
        if (!ok || res > 1e-10 * (1.0 + S)) {
            r.fallback = true;
            z = S;
            ok = newton(S, lk, tol, maxit, z, r.iters);
        }
    } else {
        if (mode == 0 && Vprev != 0.0) {
            const double L = log(fabs(Vprev) / (2.0 * V0)) + psi / a;
            z = L > 20.0 ? L + 0.6931471805599453 : asinh(exp(L));
            z = z < 0.0 ? 0.0 : (z > S ? S : z);
        } else {
            z = S;
        }
        ok = newton(S, lk, tol, maxit, z, r.iters);
        if (ok && logx && S > 0.0) {
            const unsigned long long slot = atomicAdd(logn, 1ull);
            if ((long long)slot < logcap) {
                float *o = logx + 6 * slot;
                mlp_features(S, lk, a, b, sig, o);
                double ratio = z / S;
                ratio = ratio < 1e-6 ? 1e-6 : (ratio > 1.0 - 1e-6 ? 1.0 - 1e-6 : ratio);
                o[5] = (float)log(ratio / (1.0 - ratio));
            }
        }
    }
    (void)ok;
    const double V = 2.0 * V0 * exp(-psi / a + z) * 0.5 * (1.0 - exp(-2.0 * z));
    r.V = tq < 0.0 ? -V : V;
    return r;
}

__device__ inline void write_x(const VArgs &A, int64_t i, double d1, double d2)
{
    const int64_t P = ((A.n + 16 + 7) / 8) * 8;
    if (A.x_fp32) {
        float *x = (float *)A.x;
        x[2 * i] = (float)d1; x[2 * i + 1] = (float)d2; x[2 * P + i] = (float)d1; x[3 * P + i] = (float)d2;
    } else {
        double *x = (double *)A.x;
        x[2 * i] = d1; x[2 * i + 1] = d2; x[2 * P + i] = d1; x[3 * P + i] = d2;
    }
}

__global__ void __launch_bounds__(VM_THREADS) k_vmode_stage(VArgs A, int s)
{
    __shared__ double red[VM_THREADS / 32][2];
    __shared__ int s_last;
    // MLP parameters are read in place through the read-only cache: only solves that
    // fail the undamped-start test touch them, and a warp's lanes read the same weight.
    const bool use_mlp = (A.seed_mode == 2 || A.seed_mode == 3) && A.mlp;
    const float *__restrict__ P = A.mlp;
    const int n = A.n;
    const double h = A.ctrl[0], t0 = A.ctrl[2];
    const double ts = t0 + kC[s - 1] * h;
    double Emax = 0.0;
    unsigned long long its = 0, solves = 0, itmax = 0, fb = 0;
    const int64_t i = (int64_t)blockIdx.x * VM_THREADS + threadIdx.x;
    if (i < n) {
        double *k = A.k;
        // stage state
        double ys[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            double acc = 0.0;
            for (int j = 0; j < s - 1; ++j) acc += kA[s - 1][j] * k[((int64_t)j * 3 + c) * n + i];
            ys[c] = A.y0[(int64_t)c * n + i] + h * acc;
        }
        const double a = A.a[i], b = A.b[i];
        const double tq1 = A.tq1[i] - A.mv[3 * i] + A.shear_loading[i] * ts;
        const double tq2 = A.tq2[i] - A.mv[3 * i + 1] + A.shear_loading[i] * ts;
        const double sig = A.sig0[i] + A.mv[3 * i + 2] + A.normal_loading[i] * ts;
        const Solve r1 = vsolve(tq1, sig, ys[2], a, b, A.V0, A.eta, A.V[i], A.seed_mode, use_mlp ? P : nullptr,
                                A.mlp_gate, A.newton_tol, A.newton_max, A.log_x, A.log_n, A.log_cap);
        const Solve r2 = vsolve(tq2, sig, ys[2], a, b, A.V0, A.eta, A.V[n + i], A.seed_mode, use_mlp ? P : nullptr,
                                A.mlp_gate, A.newton_tol, A.newton_max, A.log_x, A.log_n, A.log_cap);
        A.V[i] = r1.V;
        A.V[n + i] = r2.V;
        its = r1.iters + r2.iters;
        solves = 2;
        itmax = r1.iters > r2.iters ? r1.iters : r2.iters;
        fb = (r1.fallback ? 1 : 0) + (r2.fallback ? 1 : 0);
        const double Vm = sqrt(r1.V * r1.V + r2.V * r2.V);
        double arg = (A.f0[i] - ys[2]) / b;
        arg = arg > 700.0 ? 700.0 : (arg < -700.0 ? -700.0 : arg);
        const double dpsi = b / A.dc[i] * (A.V0 * exp(arg) - Vm);
        k[((int64_t)(s - 1) * 3 + 0) * n + i] = r1.V;
        k[((int64_t)(s - 1) * 3 + 1) * n + i] = r2.V;
        k[((int64_t)(s - 1) * 3 + 2) * n + i] = dpsi;
        if (s < 7) {
            // next stage state and its deficit for the next matvec
            double yn[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                double acc = 0.0;
                for (int j = 0; j < s; ++j) acc += kA[s][j] * k[((int64_t)j * 3 + c) * n + i];
                yn[c] = A.y0[(int64_t)c * n + i] + h * acc;
            }
            if (s == 6)
#pragma unroll
                for (int c = 0; c < 3; ++c) A.y5[(int64_t)c * n + i] = yn[c];
            const double tn = t0 + kC[s] * h;
            write_x(A, i, yn[0] - A.vplc[i] * A.cr0[i] * tn, yn[1] - A.vplc[i] * A.sr0[i] * tn);
        } else {
            double e[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                double acc = 0.0;
                for (int j = 0; j < 7; ++j) acc += kB4[j] * k[((int64_t)j * 3 + c) * n + i];
                const double y4 = A.y0[(int64_t)c * n + i] + h * acc;
                e[c] = fabs(A.y5[(int64_t)c * n + i] - y4);
            }
            const double y51 = A.y5[i], y52 = A.y5[n + i], y5p = A.y5[2 * (int64_t)n + i];
            Emax = fmax(fmax(e[2] / fabs(y5p), e[0] / (fabs(y51) + A.atol)), e[1] / (fabs(y52) + A.atol));
            if (Emax != Emax) Emax = INFINITY;
        }
    }
    // Newton statistics
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        its += __shfl_down_sync(0xffffffffu, its, o);
        solves += __shfl_down_sync(0xffffffffu, solves, o);
        fb += __shfl_down_sync(0xffffffffu, fb, o);
        const unsigned long long om = __shfl_down_sync(0xffffffffu, itmax, o);
        itmax = om > itmax ? om : itmax;
    }
    if ((threadIdx.x & 31) == 0 && solves) {
        atomicAdd(A.stats, its);
        atomicAdd(A.stats + 1, solves);
        atomicMax(A.stats + 2, itmax);
        if (fb) atomicAdd(A.stats + 3, fb);
    }
    if (s < 7) return;
    // stage 7: grid max of the error ratio; the last CTA decides (accept / reject)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) Emax = fmax(Emax, __shfl_down_sync(0xffffffffu, Emax, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5][0] = Emax;
    __syncthreads();
    if (threadIdx.x == 0) {
        double w = red[0][0];
        for (int q = 1; q < VM_THREADS / 32; ++q) w = fmax(w, red[q][0]);
        A.blk[blockIdx.x] = w;
        __threadfence();
        s_last = atomicAdd(A.bar, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    double w = 0.0;
    for (unsigned q = threadIdx.x; q < gridDim.x; q += VM_THREADS) w = fmax(w, __ldcg(A.blk + q));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) w = fmax(w, __shfl_down_sync(0xffffffffu, w, o));
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5][0] = w;
    __syncthreads();
    if (threadIdx.x == 0) {
        w = red[0][0];
        for (int q = 1; q < VM_THREADS / 32; ++q) w = fmax(w, red[q][0]);
        A.bar[0] = 0u;
        const double E = w / A.reltol;
        const double hnew = E > 0.0 ? 0.9 * h * pow(E, -0.2) : 1.5 * h;
        double *c = A.ctrl;
        c[10] += 1.0;
        c[13] = E;
        if (E < 1.0) {
            c[11] = 1.0;
            c[1] = h;
            c[2] = t0 + h;
            c[0] = fmin(hnew, 1.5 * h);
            c[12] = c[0];
            c[8] += 1.0;
            c[3] = 0.0;
        } else {
            c[11] = 0.0;
            c[3] += 1.0;
            c[9] += 1.0;
            c[0] = fmax(0.5 * h, hnew);
            if (c[0] < 1e-15 || c[3] > 20.0) c[4] = (double)PQ3D_ERR_DT;
        }
    }
}

// After stage 7: accept (y0 <- y5, k1 <- k7) or keep; then the deficit of stage 2
// of the next attempt at the new step size.
__global__ void k_vmode_finalize(VArgs A)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int n = A.n;
    if (i >= n) return;
    const bool acc = A.ctrl[11] != 0.0;
    double *k = A.k;
    if (acc) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            A.y0[(int64_t)c * n + i] = A.y5[(int64_t)c * n + i];
            k[(int64_t)c * n + i] = k[((int64_t)6 * 3 + c) * n + i];
        }
    }
    const double h = A.ctrl[0], t0 = A.ctrl[2];
    const double tn = t0 + kC[1] * h;
    const double y1 = A.y0[i] + h * kA[1][0] * k[i];
    const double y2 = A.y0[n + i] + h * kA[1][0] * k[(int64_t)n + i];
    write_x(A, i, y1 - A.vplc[i] * A.cr0[i] * tn, y2 - A.vplc[i] * A.sr0[i] * tn);
}

// Deficit of the current step-start state (before the stage-1 matvec).
__global__ void k_vmode_deficit(VArgs A)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int n = A.n;
    if (i >= n) return;
    const double t0 = A.ctrl[2];
    write_x(A, i, A.y0[i] - A.vplc[i] * A.cr0[i] * t0, A.y0[n + i] - A.vplc[i] * A.sr0[i] * t0);
}

}  // namespace

PQ3D_EXPORT size_t pq3d_vmode_args_bytes(void) { return sizeof(VArgs); }

// stage 1..7 of the current attempt (stage 1 only at start-up, after a matvec of the
// step-start deficit); -1: write the step-start deficit; 0: finalize the attempt.
PQ3D_EXPORT int pq3d_vmode_stage(const void *args, int stage, cudaStream_t stream)
{
    if (!args || stage < -1 || stage > 7) return PQ3D_ERR_ARG;
    const VArgs &A = *(const VArgs *)args;
    if (A.n <= 0 || !A.ctrl || !A.k || !A.y0 || !A.x || !A.V) return PQ3D_ERR_ARG;
    const unsigned grid = (unsigned)((A.n + VM_THREADS - 1) / VM_THREADS);
    if (stage == -1) {
        k_vmode_deficit<<<grid, VM_THREADS, 0, stream>>>(A);
    } else if (stage == 0) {
        k_vmode_finalize<<<grid, VM_THREADS, 0, stream>>>(A);
    } else {
        if (!A.mv || !A.y5 || !A.blk || !A.bar || !A.stats) return PQ3D_ERR_ARG;
        k_vmode_stage<<<grid, VM_THREADS, 0, stream>>>(A, stage);
    }
    return pq3d_launch_status();
}

PQ3D_EXPORT int pq3d_vmode_grid(int n) { return (n + VM_THREADS - 1) / VM_THREADS; }
