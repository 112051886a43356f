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
#include "rk_core.cuh"

namespace {
using namespace pq3d_rk;

struct RkArgs {
    double *Tno, *Tt1o, *Tt2o, *psi;                        // state (MPa, MPa, MPa, -)
    double *slip1, *slip2, *slipv1, *slipv2, *slipv, *rake, *Tt, *fric, *slip;
    const double *a, *b, *dc, *f0, *shear_loading, *normal_loading, *vplc, *cr0, *sr0;
    double *y;           // elastic load rates (n x 3): A1 x, A2 x, B x  (Pa/s)
    double *cand;        // 4n scratch
    double *blk;         // 10 * gridDim + 16 scratch: per-CTA slip-rate maxima at [4G, 6G), the
                         // grid maxima's three result slots (12 x u64) at 10G
    void *x;             // next deficit, interleaved (2n + padding), FP32 or FP64
    double *ctrl;        // control block (see pq3d.h)
    double *hist;        // per-step history, 6 doubles per step (may be null)
    const double *hforce; // dt replay: if non-null, step s uses h = hforce[s] and is accepted
    unsigned *bar;       // bar[0] arrivals, bar[2] end-of-step count (zeroed once; cleared by each step)
    const void *slots;   // when fuse_rowsum: per-row partial sums of the H-matvec
    const int32_t *leaf_of_row, *leaf_ptr, *leaf_off;
    double *ctrl_host;   // mapped host memory (may be null): ctrl[0..11) after the step, then
                         // ctrl_host[15] = step_index + 1 once those are stored
    int n, fix_tn, x_fp32, step_index, fuse_rowsum, slots_fp32;
    double V0, eta, reltol;
    double h_in;         // > 0: the step's trial size (instead of ctrl[0])
};

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned *p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ unsigned atom_add_acq_rel_u32(unsigned *p, unsigned x)
{
    unsigned old;
    asm volatile("atom.add.acq_rel.gpu.global.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(x) : "memory");
    return old;
}

// Grid-wide NaN-propagating max of four values that are >= 0 or +NaN, in one
// phase.  Every CTA folds its block maximum into a result slot with 64-bit
// atomicMax on the bit patterns (for such values the unsigned order of the
// bits is the order of the values, and +NaN lies above +inf, so the fold is
// nanmax), then arrives on bar[0] with acquire-release semantics; a CTA goes on
// once bar[0] reaches (attempt + 1) * gridDim.x and reads the slot.  Attempts
// rotate over three slots of four: the CTA that arrives last at attempt a
// clears slot (a + 2) % 3, which every CTA finished reading before it arrived
// at a and which no CTA touches before the next barrier.  The last CTA to
// finish the step clears bar[0] and the slots.  All CTAs return the same four
// values.  Bounded spin: on timeout ctrl[4] = PQ3D_ERR_TIMEOUT and false is
// returned.
template <int NT>
__device__ bool grid_max4(double *v, unsigned long long *slots3, unsigned *bar, int attempt, double *ctrl)
{
    __shared__ double wred[NT / 32][4];
    __shared__ double s_res[4];
    __shared__ int s_ok;
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[q] = nanmax(v[q], __shfl_down_sync(0xffffffffu, v[q], o));
    if ((threadIdx.x & 31) == 0)
#pragma unroll
        for (int q = 0; q < 4; ++q) wred[threadIdx.x >> 5][q] = v[q];
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long *r = slots3 + 4 * (attempt % 3);
        double w[4] = {wred[0][0], wred[0][1], wred[0][2], wred[0][3]};
        for (int k = 1; k < NT / 32; ++k)
            for (int q = 0; q < 4; ++q) w[q] = nanmax(w[q], wred[k][q]);
        for (int q = 0; q < 4; ++q) atomicMax(r + q, (unsigned long long)__double_as_longlong(w[q]));
        const unsigned target = (unsigned)(attempt + 1) * gridDim.x;
        int ok = 1;
        if (atom_add_acq_rel_u32(bar, 1u) + 1u == target) {
            unsigned long long *z = slots3 + 4 * ((attempt + 2) % 3);
            for (int q = 0; q < 4; ++q) __stcg(z + q, 0ull);
        } else {
            long long it = 0;
            while (ld_acquire_u32(bar) < target) {
                if (++it > (1LL << 24)) {
                    ctrl[4] = (double)PQ3D_ERR_TIMEOUT;
                    ok = 0;
                    break;
                }
                __nanosleep(32);
            }
        }
        for (int q = 0; q < 4; ++q) s_res[q] = __longlong_as_double((long long)__ldcg(r + q));
        s_ok = ok;
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 4; ++q) v[q] = s_res[q];
    return s_ok != 0;
}

#ifndef PQ3D_RK_THREADS
#define PQ3D_RK_THREADS 256
#endif
// Two 256-thread CTAs per SM (registers capped at 128, ~84 B spilled): at 60k
// elements the co-resident grid then covers every element with one thread,
// instead of two elements in half the threads at one CTA per SM (measured on
// B200 at 60k: 49 us per step kernel instead of 61 us).
#ifndef PQ3D_RK_MINB
#define PQ3D_RK_MINB 2
#endif
constexpr int RK_THREADS = PQ3D_RK_THREADS;   // CTA size of the step kernel

__global__ void __launch_bounds__(RK_THREADS, PQ3D_RK_MINB) k_rk_step(RkArgs A)
{
    const int n = A.n;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t tid0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (A.fuse_rowsum) {
        // the H-matvec's row reduction (k_rowsum) done here: y[i] = sum of row i's slots
        for (int64_t base = (int64_t)blockIdx.x * RK_THREADS; base < n; base += stride) rowsum_cta<RK_THREADS>(A, base, n);
    }
    unsigned long long *slots3 = (unsigned long long *)(A.blk + 10 * (int64_t)gridDim.x);
    const bool forced = A.hforce != nullptr;
    StepCtl c{forced ? A.hforce[A.step_index] : (A.h_in > 0.0 ? A.h_in : A.ctrl[0]), 0.0, 0, 0, false};
    c.dtnext = c.h;

    while (true) {
        double m1 = 0.0, g1 = 0.0, g2 = 0.0, g3 = 0.0;  // max relative errors, NaN-propagating
        for (int64_t i = tid0; i < n; i += stride) {
            double e[4];
            dp54_element(A, i, c.h, e);
            m1 = nanmax(m1, e[0]);
            g1 = nanmax(g1, e[1]);
            g2 = nanmax(g2, e[2]);
            g3 = nanmax(g3, e[3]);
        }
        // grid-wide maxima of (m1, g1, g2, g3); identical in every CTA
        double E[4] = {m1, g1, g2, g3};
        if (!grid_max4<RK_THREADS>(E, slots3, A.bar, c.attempt, A.ctrl)) return;
        if (controller(c, E, A.reltol, forced)) break;
    }
    const double h = c.h, dtnext = c.dtnext;
    const bool accepted = c.accepted;
    const int nrjct = c.nrjct, attempt = c.attempt;

    // accepted step: state update (src/QDsim.py:960-993) and next deficit (:902-903)
    double mv1 = 0.0, mv2 = 0.0;
    if (accepted) {
        for (int64_t i = tid0; i < n; i += stride) {
            double v1, v2;
            accept_element(A, i, h, v1, v2);
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
        A.bar[0] = 0u;
        for (int q = 0; q < 12; ++q) slots3[q] = 0ull;
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
        if (A.ctrl_host) {
            // the host's copy, sequence number last (a step that ended early leaves it stale)
            for (int k = 0; k < 11; ++k) A.ctrl_host[k] = A.ctrl[k];
            __threadfence_system();
            A.ctrl_host[15] = (double)A.step_index + 1.0;
        }
    }
}

// Row-range kernels of the row-partitioned (multi-GPU) step: the same element
// work as k_rk_step on rows [r0, r1) only, as plain launches; the host applies
// the controller to maxima reduced over all ranks.  Per-CTA maxima go to blk;
// the last CTA to finish (bar[2] count, no waiting) reduces them into out:
// out[0..4) values with NaN replaced by 0, out[4..8) NaN flags.
template <int NT>
__device__ void rows_finish(const RkArgs &A, double *v, double *out)
{
    __shared__ double wred[NT / 32][4];
    __shared__ int s_done;
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[q] = nanmax(v[q], __shfl_down_sync(0xffffffffu, v[q], o));
    if ((threadIdx.x & 31) == 0)
#pragma unroll
        for (int q = 0; q < 4; ++q) wred[threadIdx.x >> 5][q] = v[q];
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int q = 0; q < 4; ++q) {
            double w = wred[0][q];
            for (int k = 1; k < NT / 32; ++k) w = nanmax(w, wred[k][q]);
            A.blk[(int64_t)q * gridDim.x + blockIdx.x] = w;
        }
        __threadfence();
        s_done = atomicAdd(A.bar + 2, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_done || threadIdx.x != 0) return;
    __threadfence();
    for (int q = 0; q < 4; ++q) {
        double w = 0.0;
        for (unsigned k = 0; k < gridDim.x; ++k) w = nanmax(w, __ldcg(A.blk + (int64_t)q * gridDim.x + k));
        const bool isnan_w = w != w;
        out[q] = isnan_w ? 0.0 : w;
        out[4 + q] = isnan_w ? 1.0 : 0.0;
    }
    A.bar[2] = 0u;
}

__global__ void __launch_bounds__(RK_THREADS) k_rk_rows_attempt(RkArgs A, int r0, int r1, double h, int first,
                                                                double *out)
{
    double e4[4] = {0.0, 0.0, 0.0, 0.0};
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    if (first && A.fuse_rowsum)   // the H-matvec's row sums, staged per CTA (same rows per thread as below)
        for (int64_t base = r0 + (int64_t)blockIdx.x * RK_THREADS; base < r1; base += stride)
            rowsum_cta<RK_THREADS>(A, base, r1);
    for (int64_t i = r0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < r1; i += stride) {
        double e[4];
        dp54_element(A, i, h, e);
#pragma unroll
        for (int q = 0; q < 4; ++q) e4[q] = nanmax(e4[q], e[q]);
    }
    rows_finish<RK_THREADS>(A, e4, out);
}

__global__ void __launch_bounds__(RK_THREADS) k_rk_rows_accept(RkArgs A, int r0, int r1, double h, double *out)
{
    double v4[4] = {0.0, 0.0, 0.0, 0.0};
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = r0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < r1; i += stride) {
        double v1, v2;
        accept_element(A, i, h, v1, v2);
        v4[0] = fmax(v4[0], fabs(v1));
        v4[1] = fmax(v4[1], fabs(v2));
    }
    rows_finish<RK_THREADS>(A, v4, out);
}

// ---------------------------------------------------------------------------
// Row-partitioned step with the controller on the device.  Every rank keeps the
// same control block pc (PC_* below) and applies the same controller to the same
// maxima reduced over ranks, so all ranks take identical decisions without the
// host: a step is a fixed launch sequence (gather, matvec, R x [attempt, reduce,
// control], accept, reduce, finish) that can be enqueued or captured ahead.  An
// attempt after acceptance, or anything after a halt, returns at once.  A step
// that needs more than R attempts halts (status 0): the host finishes it.
enum {
    PC_H = 0,        // trial size of the next attempt
    PC_DTNEXT = 1,   // the controller's next size
    PC_TIME = 2,
    PC_NRJCT = 3,    // rejections in this step
    PC_STATUS = 4,   // PQ3D_ERR_DT when the step was given up
    PC_ACC = 5,      // this step's attempt was accepted
    PC_V1 = 6, PC_V2 = 7,   // max |V1|, max |V2| after the last accepted step
    PC_STEPS = 8, PC_REJ = 9,
    PC_HALT = 10,    // no further work until the host resumes
    PC_FIRST = 11,   // the next attempt is the step's first (sums the matvec slots)
    PC_ATT = 12,     // attempts in this step
    PC_LASTH = 13    // accepted h of the last step
};

__global__ void __launch_bounds__(RK_THREADS) k_rk_rows_attempt_dev(RkArgs A, int r0, int r1, const double *pc,
                                                                    double *out)
{
    if (pc[PC_HALT] != 0.0 || pc[PC_ACC] != 0.0) return;     // the same for every CTA
    const double h = pc[PC_H];
    const bool first = pc[PC_FIRST] != 0.0;
    double e4[4] = {0.0, 0.0, 0.0, 0.0};
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    if (first && A.fuse_rowsum)
        for (int64_t base = r0 + (int64_t)blockIdx.x * RK_THREADS; base < r1; base += stride)
            rowsum_cta<RK_THREADS>(A, base, r1);
    for (int64_t i = r0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < r1; i += stride) {
        double e[4];
        dp54_element(A, i, h, e);
#pragma unroll
        for (int q = 0; q < 4; ++q) e4[q] = nanmax(e4[q], e[q]);
    }
    rows_finish<RK_THREADS>(A, e4, out);
}

// The reference's controller on the reduced maxima E8 (values with NaN -> 0, then
// NaN flags), one thread.
__global__ void k_rk_rows_control(double *pc, const double *E8, double reltol, int max_attempts)
{
    if (pc[PC_HALT] != 0.0 || pc[PC_ACC] != 0.0) return;
    double E[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) E[q] = E8[4 + q] > 0.0 ? __longlong_as_double(0x7ff8000000000000ll) : E8[q];
    StepCtl c{pc[PC_H], 0.0, (int)pc[PC_NRJCT], (int)pc[PC_ATT], false};
    const bool done = controller(c, E, reltol, false);
    pc[PC_ATT] = c.attempt;
    pc[PC_FIRST] = 0.0;
    pc[PC_DTNEXT] = c.dtnext;
    if (c.accepted) {
        pc[PC_ACC] = 1.0;
        return;
    }
    pc[PC_NRJCT] = c.nrjct;
    pc[PC_H] = c.h;
    if (done) {
        pc[PC_STATUS] = (double)PQ3D_ERR_DT;
        pc[PC_HALT] = 1.0;
    } else if (c.attempt >= max_attempts) {
        pc[PC_HALT] = 1.0;                 // more attempts than launched: the host continues
    }
}

__global__ void __launch_bounds__(RK_THREADS) k_rk_rows_accept_dev(RkArgs A, int r0, int r1, const double *pc,
                                                                   double *out)
{
    if (pc[PC_HALT] != 0.0 || pc[PC_ACC] == 0.0) return;
    const double h = pc[PC_H];
    double v4[4] = {0.0, 0.0, 0.0, 0.0};
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = r0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < r1; i += stride) {
        double v1, v2;
        accept_element(A, i, h, v1, v2);
        v4[0] = fmax(v4[0], fabs(v1));
        v4[1] = fmax(v4[1], fabs(v2));
    }
    rows_finish<RK_THREADS>(A, v4, out);
}

// After the accepted step (maxima V8 reduced over ranks): time, counters, and the
// next step's trial size.
__global__ void k_rk_rows_finish(double *pc, const double *V8)
{
    if (pc[PC_HALT] != 0.0 || pc[PC_ACC] == 0.0) return;
    pc[PC_TIME] += pc[PC_H];
    pc[PC_STEPS] += 1.0;
    pc[PC_REJ] += pc[PC_NRJCT];
    pc[PC_V1] = V8[0];
    pc[PC_V2] = V8[1];
    pc[PC_LASTH] = pc[PC_H];
    pc[PC_H] = pc[PC_DTNEXT];
    pc[PC_NRJCT] = 0.0;
    pc[PC_ACC] = 0.0;
    pc[PC_ATT] = 0.0;
    pc[PC_FIRST] = 1.0;
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

static int rows_check(const RkArgs &A, int grid, int r0, int r1, const double *out)
{
    if (grid <= 0 || r0 < 0 || r1 < r0 || r1 > A.n || !out || !A.blk || !A.bar || !A.cand || !A.y || !A.x) return PQ3D_ERR_ARG;
    return PQ3D_OK;
}

// One DP5(4) attempt of size h on rows [r0, r1) (row-partitioned step); out: 8
// doubles (error maxima psi, Tt1, Tt2, Tno with NaN -> 0, then NaN flags).  blk
// must hold 4 * grid doubles; bar[2] must be zero before the first call.
PQ3D_EXPORT int pq3d_rk_rows_attempt(const void *args, int grid, int r0, int r1, double h, int first, double *d_out,
                                     cudaStream_t stream)
{
    if (!args) return PQ3D_ERR_ARG;
    const RkArgs A = *(const RkArgs *)args;
    const int rc = rows_check(A, grid, r0, r1, d_out);
    if (rc != PQ3D_OK) return rc;
    if (first && A.fuse_rowsum && (!A.slots || !A.leaf_of_row || !A.leaf_ptr || !A.leaf_off)) return PQ3D_ERR_ARG;
    k_rk_rows_attempt<<<grid, RK_THREADS, 0, stream>>>(A, r0, r1, h, first, d_out);
    return pq3d_launch_status();
}

// Device-controlled forms (control block pc, 16 doubles, see PC_* in this file).
PQ3D_EXPORT int pq3d_rk_rows_attempt_dev(const void *args, int grid, int r0, int r1, const double *d_pc,
                                         double *d_out, cudaStream_t stream)
{
    if (!args || !d_pc) return PQ3D_ERR_ARG;
    const RkArgs A = *(const RkArgs *)args;
    const int rc = rows_check(A, grid, r0, r1, d_out);
    if (rc != PQ3D_OK) return rc;
    if (A.fuse_rowsum && (!A.slots || !A.leaf_of_row || !A.leaf_ptr || !A.leaf_off)) return PQ3D_ERR_ARG;
    k_rk_rows_attempt_dev<<<grid, RK_THREADS, 0, stream>>>(A, r0, r1, d_pc, d_out);
    return pq3d_launch_status();
}

PQ3D_EXPORT int pq3d_rk_rows_control(double *d_pc, const double *d_E8, double reltol, int max_attempts,
                                     cudaStream_t stream)
{
    if (!d_pc || !d_E8 || max_attempts < 1 || !(reltol > 0.0)) return PQ3D_ERR_ARG;
    k_rk_rows_control<<<1, 1, 0, stream>>>(d_pc, d_E8, reltol, max_attempts);
    return pq3d_launch_status();
}

PQ3D_EXPORT int pq3d_rk_rows_accept_dev(const void *args, int grid, int r0, int r1, const double *d_pc,
                                        double *d_out, cudaStream_t stream)
{
    if (!args || !d_pc) return PQ3D_ERR_ARG;
    const RkArgs A = *(const RkArgs *)args;
    const int rc = rows_check(A, grid, r0, r1, d_out);
    if (rc != PQ3D_OK) return rc;
    k_rk_rows_accept_dev<<<grid, RK_THREADS, 0, stream>>>(A, r0, r1, d_pc, d_out);
    return pq3d_launch_status();
}

PQ3D_EXPORT int pq3d_rk_rows_finish(double *d_pc, const double *d_V8, cudaStream_t stream)
{
    if (!d_pc || !d_V8) return PQ3D_ERR_ARG;
    k_rk_rows_finish<<<1, 1, 0, stream>>>(d_pc, d_V8);
    return pq3d_launch_status();
}

// Accepted step of size h on rows [r0, r1): state, slip, and the rows' deficit in
// args.x; out[0], out[1] = max |V1|, max |V2| over the rows.
PQ3D_EXPORT int pq3d_rk_rows_accept(const void *args, int grid, int r0, int r1, double h, double *d_out,
                                    cudaStream_t stream)
{
    if (!args) return PQ3D_ERR_ARG;
    const RkArgs A = *(const RkArgs *)args;
    const int rc = rows_check(A, grid, r0, r1, d_out);
    if (rc != PQ3D_OK) return rc;
    k_rk_rows_accept<<<grid, RK_THREADS, 0, stream>>>(A, r0, r1, h, d_out);
    return pq3d_launch_status();
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

static __device__ __align__(256) double g_rk_scratch[4 * PQ3D_NOALLOC_MAX_N + 10 * PQ3D_NOALLOC_MAX_GRID + 16 + 2];

#include <mutex>
#include <stdio.h>

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
double *g_scratch_dev[kMaxDevices] = {nullptr};

// Device address of g_rk_scratch on the current device.  The name is only a
// host-side stand-in, so the address is looked up with that device current
// and cached per device.  Every call checks that the cached address is still
// device memory of this device: after cudaDeviceReset (or any teardown of the
// context) the module is loaded again and the address is looked up afresh.
int scratch_address(double **out)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return PQ3D_ERR_CUDA;
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    if (g_scratch_dev[dev]) {
        cudaPointerAttributes at = {};
        const cudaError_t e = cudaPointerGetAttributes(&at, g_scratch_dev[dev]);
        if (e != cudaSuccess || at.type != cudaMemoryTypeDevice || at.device != dev) {
            (void)cudaGetLastError();   // the failed query must not linger as a sticky launch status
            g_scratch_dev[dev] = nullptr;
        }
    }
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
    A.bar = (unsigned *)(s + 4 * (size_t)PQ3D_NOALLOC_MAX_N + 10 * (size_t)PQ3D_NOALLOC_MAX_GRID + 16);
    // the barrier counters and the grid maxima's result slots (at blk + 10 * grid)
    // must start at zero; the rest is written before it is read
    PQ3D_CHECK(cudaMemsetAsync(A.bar, 0, 4 * sizeof(unsigned), stream));
    PQ3D_CHECK(cudaMemsetAsync(A.blk + 10 * (size_t)grid, 0, 12 * sizeof(unsigned long long), stream));
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
