/*
 * pq3d: B200 (sm_100a) kernels for PyQuake3D's quasi-dynamic SEAS hot path.
 *
 * C ABI of libpq3d.so (pyquake3d_b200/libpq3d.so).  Plain pointers and sizes only.
 * Two groups of entry points:
 *
 *  1. Host-pointer drop-ins with the exact signatures the reference binds with
 *     ctypes (src/Hmatrix.py:22-49).  They stage the inputs to the GPU, run the
 *     FP64 Green's-function kernel and copy the result back before returning.
 *
 *  2. Device entry points (prefix pq3d_): device pointers + a cudaStream_t,
 *     return 0 (PQ3D_OK) or a negative error code, never exit or trap.  They
 *     are stream-ordered and do not synchronize the host.
 *
 * All element vectors handed to the H-matrix and stepper entry points are in
 * cluster-tree order (depth-first, left-first walk of the geometric cluster
 * tree of src/Hmatrix.py:143-182), so every H-matrix block covers contiguous
 * index ranges.
 */
#ifndef PQ3D_H
#define PQ3D_H

#include <stddef.h>
#include <stdint.h>
#include <stdbool.h>
#include <cuda_runtime_api.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PQ3D_OK 0
#define PQ3D_ERR_ARG -1
#define PQ3D_ERR_CUDA -2
#define PQ3D_ERR_RANK -3
#define PQ3D_ERR_DT -4
#define PQ3D_ERR_TIMEOUT -5
#define PQ3D_ERR_NOMEM -6

/* ---------------------------------------------------------------- drop-ins */

/* Replaces TDstressFS_C (src/TDstressFS_C.cpp:2048-2095): stress and strain
 * (xx,yy,zz,xy,xz,yz per receiver, stress[i*6+c]) at n receivers (X,Y,Z) from one
 * triangular dislocation P1,P2,P3 with Burgers components (Ss strike, Ds dip,
 * Ts tensile).  jud_halfspace=true gives the half-space solution with the
 * reference library's side handling (hs_mode 2 below), and prints the
 * reference's warning when a z coordinate is positive. */
void TDstressFS_C(const double *X, const double *Y, const double *Z, size_t n,
                  const double *P1, const double *P2, const double *P3,
                  double Ss, double Ds, double Ts, double mu, double lambda_,
                  bool jud_halfspace, double *stress, double *strain);

/* Replaces TDstressEachSourceAtReceiver_C (src/TDstressFS_C.cpp:2098-2143): one
 * receiver (x,y,z), n_sources triangles given as flat xyz triplets. */
void TDstressEachSourceAtReceiver_C(double x, double y, double z,
                                    const double *P1_flat, const double *P2_flat,
                                    const double *P3_flat, size_t n_sources,
                                    double Ss, double Ds, double Ts, double mu,
                                    double lambda_, bool jud_halfspace,
                                    double *stress_out, double *strain_out);

/* ---------------------------------------------------------------- Green's function */

/* Bytes of one per-element source record. */
size_t pq3d_src_record_bytes(void);

/* Per-element source records (TD frame, local vertices, angles) for n_elem
 * triangles; d_tri holds 1-based node ids (n_elem x 3), d_nodes xyz in metres.
 * Replaces the per-call setup inside TDstressFS (src/TDstressFS_C.cpp:294-385). */
int pq3d_src_records(const double *d_nodes, const int64_t *d_tri, int64_t n_elem,
                     void *d_rec, cudaStream_t stream);

/* Half space (TDstressHS, src/TDstressFS_C.cpp:1911-2000): per-element records of
 * the image triangle and the three sides' free-surface-correction frames.
 * hs_mode of the entry points below: 0 full space (d_hs may be NULL); 1 half
 * space, a triangle side along z adds no free-surface term (the reference's
 * numpy TDstressHS, src/SH_greenfunction.py:734-888); 2 half space as the
 * reference's compiled library, which lets such a side repeat the term of the
 * side before it (src/TDstressFS_C.cpp:1517-1522) -- the values the reference's
 * H-matrix assembly uses. */
size_t pq3d_hs_record_bytes(void);
int pq3d_hs_records(const double *d_nodes, const int64_t *d_tri, int64_t n_elem, void *d_hs,
                    cudaStream_t stream);

/* Tractions (A1s,A2s,Bs,A1d,A2d,Bd) for npairs (receiver, source) element pairs:
 * the entries BlockTree.calc_stressfunc_fromCS/CD compute (src/Hmatrix.py:425-511). */
int pq3d_traction_pairs(const double *d_xg, const double *d_ev, const void *d_rec,
                        const int64_t *d_rows, const int64_t *d_cols, int64_t npairs,
                        double mu, double lam, double *d_out, const void *d_hs, int hs_mode,
                        cudaStream_t stream);

/* Device form of both drop-ins: n_pts receivers x n_src sources, one of which is 1
 * (or both equal: pairwise).  d_P is n_src x 9 (P1,P2,P3).  halfspace: hs_mode
 * (0, 1, 2 as above; the drop-ins use 2). */
int pq3d_stress_points(const double *d_X, const double *d_Y, const double *d_Z, int64_t n_pts,
                       const double *d_P, int64_t n_src, double Ss, double Ds, double Ts,
                       double mu, double lam, int halfspace, double *d_stress,
                       double *d_strain, cudaStream_t stream);

/* ---------------------------------------------------------------- H-matrix assembly */

/* Dense near-field blocks (the Mf_* matrices of BlockTree.ACA_worker,
 * src/Hmatrix.py:1050-1063) written straight into the packed matvec layout.
 * d_blocks: array of DenseBlock {int64 off64, off32; int32 m, n, r0, c0}. */
int pq3d_dense_assemble(const double *d_xg, const double *d_ev, const void *d_rec,
                        const int32_t *d_perm, const void *d_blocks, int64_t n_blocks,
                        double mu, double lam, double *d_out64, float *d_out32,
                        const void *d_hs, int hs_mode, cudaStream_t stream);

/* Workspace (doubles) of one ACA task with rank cap kmax. */
int64_t pq3d_aca_ws_doubles(int m, int n, int kmax);
size_t pq3d_aca_task_bytes(void);
size_t pq3d_pack_task_bytes(void);

/* Batched ACA+ (BlockTree.ACA_plus_full_traceS/D, src/Hmatrix.py:581-1011), one
 * CTA per (block, slip pass).  eps: absolute step-size tolerance (rel_mode 0, the
 * reference's 0.01) or relative Frobenius tolerance (rel_mode 1).  Writes the
 * rank and a flag word (1 rank cap reached, 2 B factor all zero, 4 the pivot
 * search found every remaining row or column excluded, 8 the task is larger
 * than max_mn rows or columns and was not run) per task. */
int pq3d_aca_batched(const double *d_xg, const double *d_ev, const void *d_rec,
                     const int32_t *d_rowlist, const int32_t *d_collist,
                     const void *d_tasks, int64_t n_tasks, double *d_ws, double mu,
                     double lam, double eps, int rel_mode, int max_mn, int32_t *d_rank,
                     int32_t *d_flags, const void *d_hs, int hs_mode, cudaStream_t stream);

/* Pack ACA factors into the matvec layout; dtype 0 FP64, 1 FP32, 2 BF16. */
int pq3d_aca_pack(const void *d_tasks, int64_t n_tasks, const double *d_ws,
                  const int32_t *d_rowlist, const int32_t *d_collist, const int32_t *d_iperm,
                  int dtype, void *d_U, void *d_V, cudaStream_t stream);

/* Mixed storage of the low-rank factors (storage code 3 of pq3d_hmatvec; no
 * counterpart in the reference, which applies every block in FP64,
 * src/Hmatrix.py:1445-1538).  Each ACA term u v^T is stored as FP32, FP16 or
 * INT8 according to its weight w = max_i(|u_i| / R_i) * ||v||_1, R_i the
 * near-field absolute row sum of row i (largest component): the size of the
 * row error a quantised term can cause, against the scale at which FP32
 * storage of the row already rounds.
 *  pq3d_nearfield_rowabs: R3[c * n + i] += sum over dense blocks of |K^c_ij|
 *    (both slips); d_blocks are the DenseBlock records (off32 used), R3 zeroed.
 *  pq3d_aca_term_weights: w per (task, term) into d_w[tmap_off + q].
 *  pq3d_aca_pack_mixed: the factors in the class arrays (zeroed beforehand) and
 *    the FP16 / INT8 per-V-row scales.  Task records: pq3d_pack_mixed_task_bytes(). */
size_t pq3d_pack_mixed_task_bytes(void);
int pq3d_nearfield_rowabs(const float *d_dense32, const void *d_blocks, int64_t n_blocks, int n, double *d_R3,
                          cudaStream_t stream);
int pq3d_aca_term_weights(const void *d_tasks, int64_t n_tasks, const double *d_ws, const int32_t *d_rowlist,
                          const int32_t *d_iperm, const double *d_R, double *d_w, cudaStream_t stream);
int pq3d_aca_pack_mixed(const void *d_tasks, int64_t n_tasks, const double *d_ws, const int32_t *d_rowlist,
                        const int32_t *d_collist, const int32_t *d_iperm, const int32_t *d_tmap, float *d_U32,
                        void *d_U16, void *d_U8, float *d_V32, void *d_V16, void *d_V8, float *d_scales,
                        cudaStream_t stream);

/* ---------------------------------------------------------------- H-matvec */

/* Sizes of the work-item records: kind 0 DenseItem, 1 VItem, 2 UTask,
 * 4 DenseBlock, 5 the plan struct, 6 the mixed-storage U task, 7 and 8 the
 * streamed kernels' task and t-gather records, 9 the mixed-storage V item (rows
 * of the blocks that share a column cluster), 10 its row record. */
size_t pq3d_item_bytes(int kind);

/* y (n x 3, FP64) = [A1s A1d; A2s A2d; Bs Bd] x (+ add0/add1/add2 per component).
 * Replaces the six BlockTree.blocks_process_MVM calls of QDsim.simu_forward
 * (src/Hmatrix.py:1445-1538, src/QDsim.py:906-917).  plan_host is a host copy of
 * the plan (device pointers inside); x interleaved strike/dip deficit.  Plan
 * dtype: 0 FP64, 1 FP32, 2 FP32 dense + BF16 low rank, 3 FP32 dense + mixed low
 * rank (FP32 / FP16 / INT8 term classes, the class arrays and scales in the
 * plan's trailing fields).  d_y may be
 * NULL: then only the per-row partial sums (d_slots) are written, for the step
 * kernel to reduce. */
int pq3d_hmatvec(const void *plan_host, const void *d_x, void *d_slots, void *d_tpart,
                 const double *d_add0, const double *d_add1,
                 const double *d_add2, double *d_y, cudaStream_t stream);
/* Resident CTAs of the bulk-copy (streamed) mixed-storage kernel on the current
 * device: the persistent grid its task lists are balanced for. */
int pq3d_stream_ctas(void);
/* Resident CTAs of the mixed storage's V kernel on the current device: a plan's
 * per-warp V item lists are made for 8 warps per resident CTA. */
int pq3d_vmix_ctas(void);

/* ---------------------------------------------------------------- stepper */

size_t pq3d_rk_args_bytes(void);
/* Co-resident grid size for the step kernel, for n elements. */
int pq3d_rk_grid(int n);
/* One DP5(4) step with frozen load (QDsim.simu_forward after the matvec and
 * RungeKutte_solve_Dormand_Prince, src/QDsim.py:892-1134), cooperative launch.
 * Control block ctrl: [0] dttry in / dtnext out, [1] accepted h, [2] time,
 * [3] rejects this step, [4] status, [5] max|V1|, [6] max|V2|, [8] steps,
 * [9] total rejects, [10] total attempts.  A positive args.h_in is the trial
 * size instead of ctrl[0] (the host's dttry without a write to device memory).
 * Scratch in args: cand 4n doubles, blk 10 * grid + 16 doubles and bar 4
 * unsigned (blk and bar zeroed once, before the first step; every step leaves
 * them cleared). */
int pq3d_rk_step(const void *args, int grid, cudaStream_t stream);

/* Row-partitioned step (one fault over several GPUs, each rank owning tree-order
 * rows [r0, r1); replaces the reference's MPI block split with its reduce of the
 * products, src/QDsim.py:906-922).  Plain launches on the rank's rows; the host
 * reduces the returned maxima over ranks and applies the controller.
 * attempt: one DP5(4) attempt of size h (first = 1 also sums the matvec slots
 * into y); d_out[8] = error maxima (psi, Tt1, Tt2, Tno) with NaN -> 0, then NaN
 * flags.  accept: the accepted-step update of the rows, the rows' deficit into
 * args.x; d_out[0..1] = max|V1|, max|V2|.  args.blk: 4 * grid doubles;
 * args.bar[2] zero before the first call (the kernels leave it zero). */
int pq3d_rk_rows_attempt(const void *args, int grid, int r0, int r1, double h, int first, double *d_out,
                         cudaStream_t stream);
int pq3d_rk_rows_accept(const void *args, int grid, int r0, int r1, double h, double *d_out, cudaStream_t stream);
/* The same step with the controller on the device (the controller of
 * src/QDsim.py:931-958, as the host form applies it): every rank keeps a control
 * block pc (16 doubles: [0] h of the next attempt, [1] dtnext, [2] time, [3]
 * rejects this step, [4] status, [5] accepted, [6] max|V1|, [7] max|V2|, [8]
 * steps, [9] total rejects, [10] halt, [11] first attempt pending, [12] attempts
 * this step, [13] accepted h of the last step) and receives the same maxima reduced over ranks, so all ranks decide
 * alike without the host.  A step is the fixed sequence attempt_dev -> reduce ->
 * control (max_attempts times), accept_dev -> reduce -> finish; kernels skip
 * their work once the step is accepted or halted.  control halts with status 0
 * after max_attempts rejected attempts (the host then finishes the step) and with
 * PQ3D_ERR_DT when the step is given up; finish prepares the next step
 * (h = dtnext, counters). */
int pq3d_rk_rows_attempt_dev(const void *args, int grid, int r0, int r1, const double *d_pc, double *d_out,
                             cudaStream_t stream);
int pq3d_rk_rows_control(double *d_pc, const double *d_E8, double reltol, int max_attempts, cudaStream_t stream);
int pq3d_rk_rows_accept_dev(const void *args, int grid, int r0, int r1, const double *d_pc, double *d_out,
                            cudaStream_t stream);
int pq3d_rk_rows_finish(double *d_pc, const double *d_V8, cudaStream_t stream);

/* ---------------------------------------------------------------- ensemble
 * Many independent faults stepped together (the reference runs one fault per
 * process; this is the batched form of its simu_forward, src/QDsim.py:892-996):
 * one block-diagonal H-matvec for all faults, then one cooperative launch that
 * performs, for every fault, the step of pq3d_rk_step with the fault's own
 * controller.  Rows of a fault are a contiguous tree-order range; CTA tasks of
 * at most pq3d_ens_task_rows() rows never span two faults.  ctrl holds 16
 * doubles per fault (layout of the pq3d_rk_step control block), hist 6 doubles
 * per (step, fault). */
size_t pq3d_ens_args_bytes(void);
int pq3d_ens_task_rows(void);
int pq3d_ens_grid(int n_tasks);
int pq3d_ens_step(const void *args, int grid, cudaStream_t stream);

/* ---------------------------------------------------------------- V-mode and MLP
 * No counterpart in the reference: slip and state integrated with DP5(4), one
 * H-matvec per stage, the slip rate from a radiation-damped Newton solve per
 * element seeded by the previous rate, the undamped bound or an MLP
 * (formulation in pyquake3d_b200/csrc/vmode.cu; parity unpinned by the reference). */
size_t pq3d_vmode_args_bytes(void);
int pq3d_vmode_grid(int n);
/* stage 1..7 after a matvec of that stage's deficit; -1 writes the step-start deficit;
 * 0 finalizes an attempt (accept/reject decided on the device). */
int pq3d_vmode_stage(const void *args, int stage, cudaStream_t stream);
/* 5-64-64-1 tanh MLP, FP32, 4609 parameters: forward, gradient of the mean squared
 * error, and one Adam step; scratch of pq3d_mlp_scratch_floats(B) floats. */
int pq3d_mlp_param_count(void);
int64_t pq3d_mlp_scratch_floats(int B);
int pq3d_mlp_forward(const float *d_P, const float *d_X, int xstride, int B, float *d_Y, cudaStream_t stream);
int pq3d_mlp_grad(const float *d_P, const float *d_X, int xstride, const float *d_T, int tstride, int B,
                  float *d_scratch, float *d_G, float *d_loss, cudaStream_t stream);
int pq3d_mlp_train_step(float *d_P, float *d_M, float *d_V, const float *d_X, int xstride, const float *d_T,
                        int tstride, int B, float *d_scratch, float *d_G, float lr, float beta1, float beta2,
                        float eps, int step, float *d_loss, cudaStream_t stream);

/* No counterpart in the reference.  The same step as pq3d_rk_step for callers
 * that cannot allocate device memory (a host framework that owns every device
 * buffer, an embedded solver handed only its state vectors, a time loop that
 * must not call cudaMalloc).  The scratch of args (cand, blk, bar) is ignored:
 * the step uses a static array inside libpq3d.so (about 4.5 MB, held by every
 * GPU that loads the library until exit).  Limits: n <= 131072 elements and
 * grid <= 4096 CTAs; larger sizes return PQ3D_ERR_NOMEM without launching.
 * The first call on a device looks up the array's device address; make it
 * before any stream capture.  All calls share the array (its barrier counter
 * is cleared on the stream before each launch), so calls that overlap on the
 * GPU race.  Allocates nothing. */
int pq3d_rk_step_noalloc(const void *args, int grid, cudaStream_t stream);

/* ------------------------------------------------------- host-visible results */

/* The host side of QDsim.simu_forward and of the reference main loop's per-step
 * output (src/QDsim.py:892-1134, src/main.py:161-184: dtnext, max |V1|, max |V2|,
 * slip rate and traction after every step), without copy operations on the
 * compute stream.  Pinned host memory mapped into the device address space:
 * *host for the host, *dev for kernels. */
int pq3d_host_map_alloc(size_t bytes, void **host, void **dev);
int pq3d_host_map_free(void *host);
/* Events without timing; query returns 1 when complete, 0 when not. */
int pq3d_event_create(void **ev);
int pq3d_event_destroy(void *ev);
int pq3d_event_record(void *ev, cudaStream_t stream);
int pq3d_event_sync(void *ev);
int pq3d_event_query(void *ev);
/* Gather nf <= 8 tree-order state vectors (fields: host array of device
 * pointers, n doubles each) into host memory host_out (nf x n, element order:
 * host_out[j][e] = fields[j][iperm[e]]) through the device staging buffer
 * d_stage (nf x n).  On `side`, after `ready` (may be NULL): gather, record
 * `gathered` (and, when compute_waits, make `compute` wait for it, so a step
 * enqueued later on `compute` cannot overwrite the vectors before they are
 * read; otherwise the caller does so with pq3d_stream_wait_event), copy to
 * host_out, record `done`.  With RkArgs.ctrl_host set (mapped memory, 16
 * doubles), pq3d_rk_step also stores ctrl[0..11) there and then
 * ctrl_host[15] = step_index + 1. */
int pq3d_snapshot(int nf, const double *const *fields, const int64_t *iperm, int64_t n, double *d_stage,
                  double *host_out, void *ready, void *gathered, void *done, cudaStream_t compute,
                  cudaStream_t side, int compute_waits);
int pq3d_stream_wait_event(cudaStream_t stream, void *ev);

#ifdef __cplusplus
}
#endif
#endif /* PQ3D_H */
