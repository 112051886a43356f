// Ensemble of independent faults stepped together: one cooperative launch per
// time step covers every fault, each with its own step-size controller.
//
// The faults share one block-diagonal H-matrix (one matvec launch for all), and
// rows of fault s are the contiguous tree-order range [fault_row[s], fault_row[s+1]).
// The step kernel does, per fault, exactly what k_rk_step does for one fault
// (the reference's simu_forward after the load, src/QDsim.py:892-996): DP5(4)
// attempts with the frozen load, NaN-propagating error maxima over the fault's
// elements, the reference controller, and the accepted-step update.  Faults
// advance in lock-step attempts: a fault whose step is accepted (or given up)
// is skipped by the later attempts of the others.
//
// Work is split into CTA tasks of at most ENS_THREADS rows of one fault; the
// fused row sums of a task's rows are done by its CTA before its first attempt
// (staged slot lists, rowsum_cta).  After
// each attempt the last CTA to arrive reduces the per-task maxima of every
// running fault, applies the controller, publishes the per-fault state and
// releases the others (bounded spins; PQ3D_ERR_TIMEOUT in every fault's status).
#include "pq3d_common.cuh"
#include "rk_core.cuh"

namespace {
using namespace pq3d_rk;

constexpr int ENS_THREADS = 256;
constexpr int ENS_CTRL = 16;    // doubles of per-fault control (layout of the single-fault ctrl)
constexpr int ENS_FSTATE = 8;   // doubles of per-fault attempt state
constexpr int ENS_MAX_ATTEMPTS = 64;

struct EnsArgs {
    double *Tno, *Tt1o, *Tt2o, *psi;
    double *slip1, *slip2, *slipv1, *slipv2, *slipv, *rake, *Tt, *fric, *slip;
    const double *a, *b, *dc, *f0, *shear_loading, *normal_loading, *vplc, *cr0, *sr0;
    double *y;                 // elastic load rates (n x 3)
    double *cand;              // 4n scratch
    void *x;                   // next deficit (both layouts), FP32 or FP64
    const void *slots;         // per-row partial sums of the H-matvec (fused row sum)
    const int32_t *leaf_of_row, *leaf_ptr, *leaf_off;
    const int32_t *task_row;   // task t: rows [task_row[t], task_row[t+1])
    const int32_t *task_fault; // fault of task t
    const int32_t *fault_task; // tasks of fault s: [fault_task[s], fault_task[s+1])
    double *tmax;              // 4 doubles per task
    double *ctrl;              // ENS_CTRL doubles per fault
    double *fstate;            // ENS_FSTATE doubles per fault: h, dtnext, nrjct, attempt, phase
    double *hist;              // 6 doubles per (step, fault), may be null
    const double *hforce;      // dt replay: step s of fault f takes hforce[s * n_faults + f]
    unsigned *bar;             // [0] arrivals, [1] generation, [2] end-of-step count, [3] all-done flag
    int n, n_faults, n_tasks, fix_tn, x_fp32, step_index, fuse_rowsum, slots_fp32;
    double V0, eta, reltol;
};

// Bounded grid barrier: returns true in the last CTA to arrive, which must do its
// work and then call release(); the others wait for the release.
__device__ bool arrive(unsigned *bar, unsigned *s_gen, int *s_last)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        *s_gen = *(volatile unsigned *)(bar + 1);
        __threadfence();
        *s_last = atomicAdd(bar, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (*s_last) __threadfence();
    return *s_last;
}

__device__ void release(unsigned *bar)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        atomicExch(bar, 0u);
        __threadfence();
        atomicAdd(bar + 1, 1u);
    }
    __syncthreads();
}

__device__ bool wait_release(const EnsArgs &A, unsigned gen)
{
    __shared__ int s_ok;
    if (threadIdx.x == 0) {
        long long it = 0;
        s_ok = 1;
        while (*(volatile unsigned *)(A.bar + 1) == gen) {
            if (++it > (1LL << 24)) {
                for (int s = 0; s < A.n_faults; ++s) A.ctrl[(int64_t)ENS_CTRL * s + 4] = (double)PQ3D_ERR_TIMEOUT;
                s_ok = 0;
                break;
            }
            __nanosleep(64);
        }
        __threadfence();
    }
    __syncthreads();
    return s_ok != 0;
}

template <int NT>
__device__ void cta_max4(double *v, double *out)
{
    __shared__ double wred[NT / 32][4];
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
            out[q] = w;
        }
    }
    __syncthreads();
}

__global__ void __launch_bounds__(ENS_THREADS) k_rk_ensemble(EnsArgs A)
{
    __shared__ unsigned s_gen;
    __shared__ int s_last;
    const bool forced = A.hforce != nullptr;
    const int M = A.n_faults;

    for (int k = 0; k < ENS_MAX_ATTEMPTS; ++k) {
        // one attempt of every running fault
        for (int t = blockIdx.x; t < A.n_tasks; t += gridDim.x) {
            const int s = A.task_fault[t];
            double h;
            if (k == 0) {
                h = forced ? A.hforce[(int64_t)A.step_index * M + s] : A.ctrl[(int64_t)ENS_CTRL * s];
            } else {
                if (__ldcg(A.fstate + (int64_t)ENS_FSTATE * s + 4) != 0.0) continue;
                h = __ldcg(A.fstate + (int64_t)ENS_FSTATE * s);
            }
            // the H-matvec's row sums of the task's rows (one task is at most ENS_THREADS rows)
            if (k == 0 && A.fuse_rowsum) rowsum_cta<ENS_THREADS>(A, A.task_row[t], A.task_row[t + 1]);
            double e4[4] = {0.0, 0.0, 0.0, 0.0};
            for (int64_t i = A.task_row[t] + threadIdx.x; i < A.task_row[t + 1]; i += ENS_THREADS) {
                double e[4];
                dp54_element(A, i, h, e);
#pragma unroll
                for (int q = 0; q < 4; ++q) e4[q] = nanmax(e4[q], e[q]);
            }
            __shared__ double red[4];
            cta_max4<ENS_THREADS>(e4, red);
            if (threadIdx.x < 4) A.tmax[4 * (int64_t)t + threadIdx.x] = red[threadIdx.x];
        }
        // last CTA: per-fault maxima and controller
        if (arrive(A.bar, &s_gen, &s_last)) {
            const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
            for (int s = warp; s < M; s += ENS_THREADS / 32) {
                double *fs = A.fstate + (int64_t)ENS_FSTATE * s;
                StepCtl c;
                if (k == 0) {
                    c.h = forced ? A.hforce[(int64_t)A.step_index * M + s] : A.ctrl[(int64_t)ENS_CTRL * s];
                    c.dtnext = c.h;
                    c.nrjct = 0;
                    c.attempt = 0;
                } else {
                    if (__ldcg(fs + 4) != 0.0) continue;
                    c.h = __ldcg(fs);
                    c.dtnext = __ldcg(fs + 1);
                    c.nrjct = (int)__ldcg(fs + 2);
                    c.attempt = (int)__ldcg(fs + 3);
                }
                c.accepted = false;
                double E[4] = {0.0, 0.0, 0.0, 0.0};
                for (int t = A.fault_task[s] + lane; t < A.fault_task[s + 1]; t += 32)
#pragma unroll
                    for (int q = 0; q < 4; ++q) E[q] = nanmax(E[q], __ldcg(A.tmax + 4 * (int64_t)t + q));
#pragma unroll
                for (int q = 0; q < 4; ++q)
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) E[q] = nanmax(E[q], __shfl_xor_sync(0xffffffffu, E[q], o));
                const bool done = controller(c, E, A.reltol, forced);
                if (lane == 0) {
                    fs[0] = c.h;
                    fs[1] = c.dtnext;
                    fs[2] = c.nrjct;
                    fs[3] = c.attempt;
                    fs[4] = done ? (c.accepted ? 1.0 : 2.0) : 0.0;
                }
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                __threadfence();
                unsigned running = 0;
                for (int s = 0; s < M; ++s) running += A.fstate[(int64_t)ENS_FSTATE * s + 4] == 0.0;
                A.bar[3] = running == 0 ? 1u : 0u;
            }
            release(A.bar);
        } else if (!wait_release(A, s_gen)) {
            return;
        }
        if (__ldcg(A.bar + 3) != 0u) break;
    }

    // accepted faults: state update, next deficit, slip-rate maxima per task
    for (int t = blockIdx.x; t < A.n_tasks; t += gridDim.x) {
        const int s = A.task_fault[t];
        const bool acc = __ldcg(A.fstate + (int64_t)ENS_FSTATE * s + 4) == 1.0;
        const double h = __ldcg(A.fstate + (int64_t)ENS_FSTATE * s);
        double v4[4] = {0.0, 0.0, 0.0, 0.0};
        if (acc) {
            for (int64_t i = A.task_row[t] + threadIdx.x; i < A.task_row[t + 1]; i += ENS_THREADS) {
                double v1, v2;
                accept_element(A, i, h, v1, v2);
                v4[0] = fmax(v4[0], fabs(v1));
                v4[1] = fmax(v4[1], fabs(v2));
            }
        }
        __shared__ double red[4];
        cta_max4<ENS_THREADS>(v4, red);
        if (threadIdx.x < 2) A.tmax[4 * (int64_t)t + threadIdx.x] = red[threadIdx.x];
    }
    // the last CTA to finish writes every fault's control block and history row
    __shared__ int s_done;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        s_done = atomicAdd(A.bar + 2, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_done) return;
    __threadfence();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int s = warp; s < M; s += ENS_THREADS / 32) {
        double w1 = 0.0, w2 = 0.0;
        for (int t = A.fault_task[s] + lane; t < A.fault_task[s + 1]; t += 32) {
            w1 = fmax(w1, __ldcg(A.tmax + 4 * (int64_t)t));
            w2 = fmax(w2, __ldcg(A.tmax + 4 * (int64_t)t + 1));
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            w1 = fmax(w1, __shfl_xor_sync(0xffffffffu, w1, o));
            w2 = fmax(w2, __shfl_xor_sync(0xffffffffu, w2, o));
        }
        if (lane != 0) continue;
        const double *fs = A.fstate + (int64_t)ENS_FSTATE * s;
        double *C = A.ctrl + (int64_t)ENS_CTRL * s;
        const double h = fs[0], dtnext = fs[1], nrjct = fs[2], attempt = fs[3];
        if (fs[4] == 1.0) {
            const double tt = C[2] + h;
            C[2] = tt;
            C[0] = dtnext;
            C[1] = h;
            C[3] = nrjct;
            C[5] = w1;
            C[6] = w2;
            C[8] += 1.0;
            C[9] += nrjct;
            C[10] += attempt;
            if (A.hist) {
                double *hh = A.hist + 6 * ((int64_t)A.step_index * M + s);
                hh[0] = h; hh[1] = dtnext; hh[2] = tt; hh[3] = w1; hh[4] = w2; hh[5] = nrjct;
            }
        } else {
            C[1] = h;
            C[3] = nrjct;
            if (C[4] == 0.0) C[4] = (double)PQ3D_ERR_DT;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        A.bar[2] = 0u;
        A.bar[3] = 0u;
    }
}

}  // namespace

PQ3D_EXPORT size_t pq3d_ens_args_bytes(void) { return sizeof(EnsArgs); }

// Largest co-resident grid of the ensemble step kernel for n_tasks tasks.
PQ3D_EXPORT int pq3d_ens_grid(int n_tasks)
{
    int dev = 0, sms = 0, per = 0;
    if (n_tasks <= 0) return -1;
    if (cudaGetDevice(&dev) != cudaSuccess) return -1;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return -1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_rk_ensemble, ENS_THREADS, 0) != cudaSuccess) return -1;
    const int cap = sms * per;
    return n_tasks < cap ? n_tasks : cap;
}

// Rows per ensemble task (tasks never span two faults).
PQ3D_EXPORT int pq3d_ens_task_rows(void) { return ENS_THREADS; }

// One time step of every fault of the ensemble (cooperative launch).
PQ3D_EXPORT int pq3d_ens_step(const void *args, int grid, cudaStream_t stream)
{
    if (!args || grid <= 0) return PQ3D_ERR_ARG;
    EnsArgs A = *(const EnsArgs *)args;
    if (A.n <= 0 || A.n_faults <= 0 || A.n_tasks <= 0 || !A.task_row || !A.task_fault || !A.fault_task ||
        !A.tmax || !A.ctrl || !A.fstate || !A.bar || !A.y || !A.cand || !A.x)
        return PQ3D_ERR_ARG;
    if (A.fuse_rowsum && (!A.slots || !A.leaf_of_row || !A.leaf_ptr || !A.leaf_off)) return PQ3D_ERR_ARG;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(ENS_THREADS);
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    PQ3D_CHECK(cudaLaunchKernelEx(&cfg, k_rk_ensemble, A));
    return PQ3D_OK;
}
