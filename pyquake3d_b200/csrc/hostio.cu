// Host-visible results of the host-driven step: QDsim.simu_forward's return
// values (src/QDsim.py:892-1134) and the reference main loop's per-step output,
// which reads max |V1|, max |V2|, the slip rate and the shear traction after
// every step (src/main.py:161-184).
//
// The host waits for one small control block per step and, for output, reads
// state vectors in element order.  The step kernel's last CTA stores the control
// block in pinned host memory mapped into the device address space, so no copy
// operation enters the compute stream.  Snapshots are gathered from tree order
// on a side stream (high priority, so the gather runs between the waves of the
// H-matvec enqueued before it) and moved to the host by the copy engine; the
// compute stream waits only for the gather, before the next step kernel
// overwrites the state being read.
#include "pq3d_common.cuh"

namespace {

constexpr int SNAP_MAX_FIELDS = 8;
constexpr int SNAP_THREADS = 256;

struct SnapFields {
    const double *f[SNAP_MAX_FIELDS];
};

// out[j * n + e] = field_j[iperm[e]]: element order from tree order
// (consecutive threads write consecutive elements).
__global__ void __launch_bounds__(SNAP_THREADS) k_snapshot(SnapFields F, int nf, const int64_t *__restrict__ iperm,
                                                           int64_t n, double *__restrict__ out)
{
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += stride) {
        const int64_t t = __ldg(iperm + e);
#pragma unroll
        for (int j = 0; j < SNAP_MAX_FIELDS; ++j)      // constant indices: F stays in parameter space
            if (j < nf) out[j * n + e] = __ldg(F.f[j] + t);
    }
}

}  // namespace

// Pinned host memory mapped into every device's address space.  *host is the
// host pointer, *dev the pointer kernels use (the same value under unified
// addressing).
PQ3D_EXPORT int pq3d_host_map_alloc(size_t bytes, void **host, void **dev)
{
    if (!host || !dev || bytes == 0) return PQ3D_ERR_ARG;
    *host = *dev = nullptr;
    void *h = nullptr;
    PQ3D_CHECK(cudaHostAlloc(&h, bytes, cudaHostAllocMapped | cudaHostAllocPortable));
    void *d = nullptr;
    if (cudaHostGetDevicePointer(&d, h, 0) != cudaSuccess) {
        cudaFreeHost(h);
        return PQ3D_ERR_CUDA;
    }
    *host = h;
    *dev = d;
    return PQ3D_OK;
}

PQ3D_EXPORT int pq3d_host_map_free(void *host)
{
    if (!host) return PQ3D_OK;
    PQ3D_CHECK(cudaFreeHost(host));
    return PQ3D_OK;
}

// Events without timing (the cheapest kind to record and wait on).
PQ3D_EXPORT int pq3d_event_create(void **ev)
{
    if (!ev) return PQ3D_ERR_ARG;
    cudaEvent_t e;
    PQ3D_CHECK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    *ev = (void *)e;
    return PQ3D_OK;
}

PQ3D_EXPORT int pq3d_event_destroy(void *ev)
{
    if (!ev) return PQ3D_OK;
    PQ3D_CHECK(cudaEventDestroy((cudaEvent_t)ev));
    return PQ3D_OK;
}

PQ3D_EXPORT int pq3d_event_record(void *ev, cudaStream_t stream)
{
    if (!ev) return PQ3D_ERR_ARG;
    PQ3D_CHECK(cudaEventRecord((cudaEvent_t)ev, stream));
    return PQ3D_OK;
}

PQ3D_EXPORT int pq3d_event_sync(void *ev)
{
    if (!ev) return PQ3D_ERR_ARG;
    PQ3D_CHECK(cudaEventSynchronize((cudaEvent_t)ev));
    return PQ3D_OK;
}

// 1 if the work before the event has finished, 0 if not, < 0 on error.
PQ3D_EXPORT int pq3d_event_query(void *ev)
{
    if (!ev) return PQ3D_ERR_ARG;
    const cudaError_t e = cudaEventQuery((cudaEvent_t)ev);
    if (e == cudaSuccess) return 1;
    if (e == cudaErrorNotReady) {
        cudaGetLastError();
        return 0;
    }
    return PQ3D_ERR_CUDA;
}

// Snapshot of nf device state vectors (tree order, n doubles each) into host
// memory (nf x n, element order: host_out[j][e] = field_j[iperm[e]]).  On `side`,
// after `ready` (recorded by the caller after the step that produced the state):
// the gather kernel writes the device staging buffer d_stage (nf x n), `gathered`
// is recorded and `compute` waits for it, so the next step kernel on `compute`
// cannot overwrite the state before it is read, but does not wait for the
// transfer; the copy engine then moves d_stage to host_out and `done` is
// recorded.  host_out is complete once `done` has completed.  d_stage and
// host_out must not be reused before `done`.  With compute_waits = 0 the caller
// makes `compute` wait for `gathered` itself (pq3d_stream_wait_event), e.g. after
// enqueueing work that does not write the gathered vectors.
PQ3D_EXPORT int pq3d_snapshot(int nf, const double *const *fields, const int64_t *iperm, int64_t n, double *d_stage,
                              double *host_out, void *ready, void *gathered, void *done, cudaStream_t compute,
                              cudaStream_t side, int compute_waits)
{
    if (nf <= 0 || nf > SNAP_MAX_FIELDS || !fields || !iperm || n <= 0 || !d_stage || !host_out || !gathered || !done)
        return PQ3D_ERR_ARG;
    SnapFields F = {};
    for (int j = 0; j < nf; ++j) {
        if (!fields[j]) return PQ3D_ERR_ARG;
        F.f[j] = fields[j];
    }
    if (ready) PQ3D_CHECK(cudaStreamWaitEvent(side, (cudaEvent_t)ready, 0));
    int dev = 0, sms = 0;
    PQ3D_CHECK(cudaGetDevice(&dev));
    PQ3D_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int64_t need = (n + SNAP_THREADS - 1) / SNAP_THREADS;
    const int grid = (int)(need < (int64_t)sms ? need : (int64_t)sms);
    k_snapshot<<<grid, SNAP_THREADS, 0, side>>>(F, nf, iperm, n, d_stage);
    PQ3D_CHECK(cudaGetLastError());
    PQ3D_CHECK(cudaEventRecord((cudaEvent_t)gathered, side));
    if (compute_waits) PQ3D_CHECK(cudaStreamWaitEvent(compute, (cudaEvent_t)gathered, 0));
    PQ3D_CHECK(cudaMemcpyAsync(host_out, d_stage, (size_t)nf * (size_t)n * sizeof(double), cudaMemcpyDeviceToHost,
                               side));
    PQ3D_CHECK(cudaEventRecord((cudaEvent_t)done, side));
    return PQ3D_OK;
}

PQ3D_EXPORT int pq3d_stream_wait_event(cudaStream_t stream, void *ev)
{
    if (!ev) return PQ3D_ERR_ARG;
    PQ3D_CHECK(cudaStreamWaitEvent(stream, (cudaEvent_t)ev, 0));
    return PQ3D_OK;
}
