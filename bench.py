"""Benchmark: RK steps/s of the quasi-dynamic SEAS step at ~60k triangles.

Workload ("curved60k"): 150 km rough vertical strike-slip fault + 40 km branch
at 20 degrees, 59,696 triangles, H-matrix leaf 64, eta 2, ACA relative tol 1e-5;
operator stored mixed (FP32 near field, low-rank ACA terms in FP32 / FP16 / INT8
by weight; FP32, BF16 low rank and FP64 also timed), FP64 state and slip;
reference-mode DP5(4) stepping (one H-matvec per step, frozen load).

A step = one H-matvec of the slip-rate deficit + one fused DP5(4) step kernel
(accept/reject loop on the device).  The printed JSON line reports:
  value       steps/s of the mixed path (mixed operator storage, FP64 state:
              meets the 1e-5 slip target), state resident in HBM; FP32, BF16 low
              rank and FP64 plain are timed beside it (all_precisions)
  e2e         steps/s through QDsim.simu_forward (the reference call), with the
              per-step host traffic of the reference main loop (dttry in; h,
              dtnext and max slip rates out; slip-rate and traction vectors out)
  plain_fp64  the same step with the FP64 operator (the plain GPU path)
  roofline    H-matvec algorithmic bytes / measured duration vs measured HBM peak
  cpu_baseline the reference's CPU step (six block-loop MVMs + DP5(4), oracle
              port) on the same operator, bounded sample, on the host cores
--impl reference runs only that CPU arm (all host cores, the reference's MPI
block split emulated with worker processes) and prints its own line.
Multi-GPU (torchrun): the one fault row-partitioned over the ranks (strong
scaling; run_partition: one all-gather of the deficit per step, one max
all-reduce per attempt, the controller on the device, CUDA-graph replays);
value = steps of that fault per second.  --parallelism replicas runs one fault
per rank instead (value = sum over ranks).  --parallelism partition on one GPU
runs the partitioned path with a single rank.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "oracle"))

CASE = "curved60k"
METRIC = "RK steps/s and H-matvec HBM GB/s at 60k tris, mixed vs FP64 plain @1e-5 slip"


def peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def fp64_peak_tflops(n=8192, reps=3):
    """Measured FP64 peak of this GPU: a cuBLAS DGEMM (n^3, FP64), CUDA-event timed."""
    import torch
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    torch.matmul(a, b)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        torch.matmul(a, b)
    e1.record()
    torch.cuda.synchronize()
    t = e0.elapsed_time(e1) / 1e3 / reps
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / t / 1e12


def gf_roofline(op, struct):
    """Dense near-field assembly as a Green's-function roofline: (receiver, source)
    pairs, pair-evaluations per second (strike and dip slip counted separately),
    and, with the FP64 operations per pair counted by ncu on the same kernel
    (profiles/gf_flops.json), the achieved FP64 rate against a measured DGEMM."""
    import torch
    pairs = int(struct.stats()["dense_entries"])
    recs = op.dense_recs
    from pyquake3d_b200._lib import check, ptr
    order = np.argsort(-(recs["m"].astype(np.int64) * recs["n"]), kind="stable")
    d_recs = torch.from_numpy(recs[order].view(np.uint8)).to(op.dev)
    out32 = torch.empty_like(op.dense32) if op.dense32 is not None else None
    out64 = None if out32 is not None else torch.empty_like(op.dense64)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def run():
        check(op.L.pq3d_dense_assemble(ptr(op.xg), ptr(op.ev), ptr(op.rec), ptr(op.perm), ptr(d_recs), len(recs), op.mu,
                                       op.lam, ptr(out64), ptr(out32), ptr(op.hs), op.halfspace, op._stream),
              "pq3d_dense_assemble")
    run()
    torch.cuda.synchronize()
    e0.record()
    run()
    e1.record()
    torch.cuda.synchronize()
    t = e0.elapsed_time(e1) / 1e3
    del out32, out64
    out = {"kernel": "k_dense_assemble (full space)", "pairs": pairs, "ms": 1e3 * t,
           "pair_evals_per_s": 2 * pairs / t}
    # ACA (k_aca): every iteration of a slip pass evaluates one residual row (n
    # sources) and one column (m receivers) of the block's Green's function, so a pass
    # of rank k costs at least k (m + n) single-slip pair evaluations (reference-set
    # resets add more): a lower bound on its rate, against the dense assembly's
    kS, kD = op.ranks()
    mn = np.array([len(b.row.indices) + len(b.col.indices) for b in struct.blocks if b.aca], dtype=np.float64)
    aca_pairs = float(np.sum((kS + kD) * mn))
    aca_s = op.timings.get("aca_s")
    if aca_s:
        out["aca"] = {"pair_evals_min": aca_pairs, "s": aca_s, "pair_evals_per_s_min": aca_pairs / aca_s,
                      "vs_dense_rate_min": aca_pairs / aca_s / (2 * pairs / t),
                      "note": "lower bound: k (m + n) single-slip evaluations per pass of rank k"}
    fp = os.path.join(REPO, "profiles", "gf_flops.json")
    if os.path.exists(fp):
        f = json.load(open(fp))
        peak = fp64_peak_tflops()
        ach = f["fp64_flops_per_pair"] * pairs / t / 1e12
        out.update({"fp64_flops_per_pair": f["fp64_flops_per_pair"], "achieved_tflops": ach, "peak_tflops": peak,
                    "peak_source": "cuBLAS DGEMM 8192^3 measured in this run", "frac": ach / peak})
    return out


def set_case(name):
    global CASE
    CASE = name


def make_case(rank=0):
    from pyquake3d_b200 import meshgen
    d = os.path.join(tempfile.gettempdir(), "pq3d_bench_%s_r%d" % (CASE, rank))
    msh = os.path.join(d, CASE + ".msh")
    para = os.path.join(d, "parameter.txt")
    if not (os.path.exists(msh) and os.path.exists(para)):
        meshgen.make_case(CASE, d)
    return msh, para


class Clocks:
    """nvidia-smi samples during the timed region."""

    def __init__(self, gpu_index):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", "--query-gpu=" + q, "--format=csv,noheader,nounits", "-lms", "200",
                                       "-i", str(gpu_index)], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
        # the sampler's first row before the timed region starts (nvidia-smi takes a
        # few hundred ms to come up); rows from then on are the region's
        self.n0 = 0
        t0 = time.time()
        while self.p is not None and time.time() - t0 < 5.0 and self.p.poll() is None:
            self.n0 = len(self._rows())
            if self.n0:
                break
            time.sleep(0.05)

    def _rows(self):
        self.f.flush()
        return [l.strip().split(", ") for l in open(self.f.name) if l.strip()]

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        self.p.wait()
        rows = self._rows()
        os.unlink(self.f.name)
        # samples taken during the region; the last one before it when the region was
        # shorter than the 200 ms sampling period
        rows = rows[self.n0:] or rows[-1:]
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if len(r) > 5 + k and r[5 + k] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def export_host_operator(op):
    import qd_oracle
    from pyquake3d_b200.hmatrix import export_blocks
    ho = object.__new__(qd_oracle.OracleOperator)
    ho.blocks = export_blocks(op)
    return ho


def cpu_reference_steps(ho, state, V0, mu, Cs, budget_s, max_steps=20, dttry=1e-3, reltol=1e-4, fix_tn=False):
    """The reference's step (oracle port) on the host: returns (steps/s, steps, seconds,
    the oracle stepper, its accepted step sizes)."""
    import qd_oracle
    st = qd_oracle.OracleStepper(state, qd_oracle.operator_mvm(ho), V0, mu, Cs, reltol, fix_tn)
    t0 = time.perf_counter()
    k = 0
    hs = []
    while k < max_steps:
        h, dttry = st.simu_forward(dttry)
        hs.append(h)
        k += 1
        if time.perf_counter() - t0 > budget_s:
            break
    dt = time.perf_counter() - t0
    return k / dt, k, dt, st, hs


def pin_fp64_to_oracle(sim, op, ost, hs):
    """The device FP64 stepper from the same initial state, stepped adaptively as
    many steps as the oracle took: relative differences of h and of the state."""
    from pyquake3d_b200.qdsim import DeviceStepper
    d = DeviceStepper(sim, op, "fp64")
    dt = sim.htry
    hd = []
    for _ in hs:
        h, dt = d.step(dt)
        hd.append(h)
    out = {"steps": len(hs), "h_max_rel_diff": float(np.max(np.abs(np.array(hd) - hs) / np.array(hs)))}
    for name, dev in (("slip1", "slip1"), ("state", "psi"), ("Tt1o", "Tt1o"), ("Tno", "Tno"), ("slipv", "slipv")):
        r = getattr(ost, name)
        out[name + "_max_rel_diff"] = float(np.abs(d.get(dev) - r).max() / np.abs(r).max())
    return out


def accuracy_study(sim, op, nrep, precisions=("bf16",), marks=(50, 100, 200, 500)):
    """Relative L2 errors of slip, V, psi and theta of each precision against the FP64
    operator at equal times (dt replay of the FP64 run), after each mark; plus the FP64
    chaos floor: the same errors between two FP64 runs whose initial shear tractions
    (both components) differ by a relative 1e-12, and the same with a relative 2^-24
    (FP32 unit roundoff: how far the fault's own dynamics carry a difference of the
    size FP32 storage makes).  The FP64 device path itself is pinned to the oracle's
    simu_forward on the same operator (the cpu_baseline leg and the GPU tests)."""
    import torch
    from pyquake3d_b200.qdsim import DeviceStepper

    def theta(st):
        # state variable theta = (Dc / V0) exp((psi - f0) / b) of the log-state psi
        return st.t["dc"] / st.V0 * torch.exp((st.t["psi"] - st.t["f0"]) / st.t["b"])

    def errs(a, b):
        sa = torch.sqrt(a.t["slip1"] ** 2 + a.t["slip2"] ** 2)
        sb = torch.sqrt(b.t["slip1"] ** 2 + b.t["slip2"] ** 2)
        r = lambda u, v: float(torch.linalg.norm(u - v) / torch.linalg.norm(v))
        return {"slip": r(sa, sb), "V": r(a.t["slipv"], b.t["slipv"]), "psi": r(a.t["psi"], b.t["psi"]),
                "theta": r(theta(a), theta(b))}

    marks = [m for m in marks if m <= nrep] or [nrep]
    ref = DeviceStepper(sim, op, "fp64")
    others = {p: DeviceStepper(sim, op, p) for p in precisions if p in op.plans}
    perts = {}
    for name, eps in (("fp64_perturbed_1e-12", 1e-12), ("fp64_perturbed_2^-24", 2.0 ** -24)):
        st = DeviceStepper(sim, op, "fp64")
        st.t["Tt1o"].mul_(1.0 + eps)           # both shear components: a pure-dip or pure-strike
        st.t["Tt2o"].mul_(1.0 + eps)           # fault has one of them zero
        perts[name] = st
    for st in [ref] + list(perts.values()) + list(others.values()):
        st.ctrl[0] = sim.htry
    ref.set_history(nrep)
    out = {p: [] for p in list(others) + list(perts)}
    done = 0
    for mk in marks:
        for i in range(done, mk):
            ref.launch(i)
        torch.cuda.synchronize()
        h = ref.hist.view(-1, 6)[:, 0]
        for name, st in list(others.items()) + list(perts.items()):
            st.set_replay(h)
            for i in range(done, mk):
                st.launch(i)
        torch.cuda.synchronize()
        for name, st in list(others.items()) + list(perts.items()):
            e = errs(st, ref)
            e["steps"] = mk
            out[name].append(e)
        done = mk
    out["method"] = "dt replay of the FP64 run; relative L2 over elements"
    out["sim_time_s"] = float(ref.hist.view(-1, 6)[done - 1, 2])
    return out


def accuracy_common_times(sim, op, prec, nrep, marks=(100, 200, 500)):
    """The second parity measure: FP64 and `prec` each step with their own controller;
    at the FP64 run's times after each mark the `prec` run's slip, V and theta are
    interpolated linearly in time between its two bracketing steps, and relative L2
    errors over elements are formed against the FP64 state at that time."""
    import torch
    from pyquake3d_b200.qdsim import DeviceStepper

    def fields(st):
        return {"slip": torch.sqrt(st.t["slip1"] ** 2 + st.t["slip2"] ** 2), "V": st.t["slipv"].clone(),
                "theta": st.t["dc"] / st.V0 * torch.exp((st.t["psi"] - st.t["f0"]) / st.t["b"])}

    marks = [m for m in marks if m <= nrep] or [nrep]
    ref = DeviceStepper(sim, op, "fp64")
    ref.ctrl[0] = sim.htry
    targets = []
    done = 0
    for mk in marks:
        for i in range(done, mk):
            ref.launch(i)
        done = mk
        targets.append((mk, float(ref.ctrl[2].item()), fields(ref)))
    st = DeviceStepper(sim, op, prec)
    st.ctrl[0] = sim.htry
    prev_t, prev_f = 0.0, fields(st)
    out = []
    i = 0
    for mk, t_ref, f_ref in targets:
        while True:
            t_now = float(st.ctrl[2].item())
            if t_now >= t_ref:
                break
            prev_t, prev_f = t_now, fields(st)
            st.launch(i)
            i += 1
            if i > 10 * nrep:
                raise RuntimeError("the %s run fell behind the FP64 run's time" % prec)
        cur = fields(st)
        w = (t_ref - prev_t) / (t_now - prev_t) if t_now > prev_t else 1.0
        e = {k: float(torch.linalg.norm(prev_f[k] + w * (cur[k] - prev_f[k]) - f_ref[k]) / torch.linalg.norm(f_ref[k]))
             for k in f_ref}
        e.update(steps_fp64=mk, steps=i, time_s=t_ref)
        out.append(e)
    return out


def time_stepper(stepper, k, dttry, G=100):
    """k device-controlled steps (CUDA-graph replays of G steps when k is a multiple
    of G): seconds by CUDA events, and the next trial size."""
    import torch
    g = stepper.capture(G) if k % G == 0 and k >= G else None
    if g is None:
        stepper.set_history(k)
    stepper.ctrl[0] = dttry
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    if g is not None:
        for _ in range(k // G):
            g.replay()
    else:
        for i in range(k):
            stepper.launch(i)
    e1.record()
    torch.cuda.synchronize()
    c = stepper.ctrl.cpu().numpy()
    if c[4] != 0:
        raise RuntimeError("step failed with status %d" % int(c[4]))
    return e0.elapsed_time(e1) / 1e3, float(c[0]), g is not None


def config_study(case, prec, nsteps, cpu_budget, marks, extra=()):
    """One of the smaller benchmark configurations at its full step count: steps/s of
    `prec` and of the FP64 plain path, the H-matvec roofline, errors against the FP64
    path (dt replay) at the marks, the FP64 path pinned to the oracle's simu_forward
    on the same operator over the oracle's steps, and the oracle's CPU step rate."""
    import torch
    from pyquake3d_b200 import QDsim, meshgen, read_mshV2
    from pyquake3d_b200.qdsim import DeviceStepper
    import qd_oracle
    d = os.path.join(tempfile.gettempdir(), "pq3d_bench_cfg_%s" % case)
    msh, para = meshgen.make_case(case, d)
    nodes, tris = read_mshV2(msh)
    sim = QDsim(tris, nodes, para, precision=prec)
    precs = tuple(dict.fromkeys((prec,) + tuple(extra) + ("fp64",)))
    sim.tree_block.want = precs
    op = sim.tree_block.op()
    hbm, _ = peaks()
    out = {"workload": case, "triangles": int(sim.xg.shape[0]), "precision": prec, "steps": nsteps,
           "aca": "%s %s" % ("relative" if sim.Para0.get("ACA relative tolerance") == "True" else "absolute",
                             sim.Para0.get("ACA tolerance")),
           "dense_only": int(sum(1 for b in sim.tree_block.struct.blocks if b.aca)) == 0}
    for p in precs:
        st = DeviceStepper(sim, op, p)
        _, dt, _ = time_stepper(st, 5, sim.htry)
        t, _, graph = time_stepper(st, nsteps, dt)
        x = st.x
        for _ in range(5):
            op.matvec(x, p, slots_only=True)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(50):
            op.matvec(x, p, slots_only=True)
        e1.record()
        torch.cuda.synchronize()
        tm = e0.elapsed_time(e1) / 1e3 / 50
        ab = op.plan(p)["alg_bytes"]
        out[p] = {"steps_per_s": nsteps / t, "ms_per_step": 1e3 * t / nsteps, "cuda_graph": graph,
                  "hmatvec": {"ms": 1e3 * tm, "alg_bytes": int(ab), "GBs": ab / tm / 1e9, "frac": ab / tm / 1e9 / hbm},
                  "sim_time_s": float(st.ctrl[2].item())}
        del st
    out["vs_fp64"] = {p: out[p]["steps_per_s"] / out["fp64"]["steps_per_s"] for p in precs}
    low = [p for p in precs if p != "fp64"]
    if low:
        acc = accuracy_study(sim, op, nsteps, precisions=tuple(low), marks=marks)
        out["err_vs_fp64"] = {p: acc[p] for p in low}
        out["fp64_chaos_floor"] = acc["fp64_perturbed_1e-12"]
        out["fp64_perturbed_fp32_roundoff"] = acc["fp64_perturbed_2^-24"]
    ho = export_host_operator(op)
    crate, k, secs, ost, hs = cpu_reference_steps(ho, qd_oracle.sim_state(sim), sim.V0, sim.mu, sim.Cs, cpu_budget,
                                                  max_steps=200, dttry=sim.htry, reltol=sim.RelTol, fix_tn=sim.fix_Tn)
    out["cpu_baseline"] = {"value": crate, "unit": "steps/s", "cores": 1, "kind": "port",
                           "sample": "%d steps (%.1f s): six block-loop MVMs + DP5(4), numpy FP64" % (k, secs)}
    out["fp64_pinned_to_oracle"] = pin_fp64_to_oracle(sim, op, ost, hs)
    out["vs_cpu"] = out[prec]["steps_per_s"] / crate
    del ho, op
    torch.cuda.empty_cache()
    return out


def vmode_study(sim, op, nsteps, prec="fp32"):
    """V-mode steps/s and Newton iteration counts for every start of the slip-rate
    solve -- the previous rate (seed 0), the undamped bound (seed 1), the MLP (seed 2)
    and the gated MLP (seed 3) -- with the `prec` operator, and plain Newton with the
    FP64 operator.  The MLP is trained first on solves logged from a short plain run
    of the same fault."""
    import torch
    from pyquake3d_b200.vmode import MLPTrainer, VStepper
    out = {}
    logger = VStepper(sim, op, prec, seed_mode=1, log_cap=1 << 20)
    logger.run(20, chunk=4)
    data = logger.samples()
    t0 = time.perf_counter()
    tr = MLPTrainer(seed=0)
    hist = tr.fit(data, epochs=15, batch=8192, lr=3e-3)
    torch.cuda.synchronize()
    out["mlp"] = {"samples": int(data.shape[0]), "epochs": 15, "train_s": round(time.perf_counter() - t0, 2),
                  "loss_first": hist[0], "loss_last": hist[-1]}
    del logger
    names = {0: "prev", 1: "newton", 2: "mlp", 3: "mlp_gated"}
    for prc, mode in ((prec, 0), (prec, 1), (prec, 2), (prec, 3), ("fp64", 1)):
        st = VStepper(sim, op, prc, seed_mode=mode, mlp_params=tr.P if mode >= 2 else None)
        st.run(5, chunk=2)                      # warm-up steps
        st.reset_stats()
        c0 = st.ctrl.cpu().numpy().copy()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        c = st.run(nsteps, chunk=4)
        e1.record()
        torch.cuda.synchronize()
        secs = e0.elapsed_time(e1) / 1e3
        steps = int(c[8] - c0[8])
        out["%s_%s" % (prc, names[mode])] = {
            "steps_per_s": steps / secs, "steps": steps, "attempts": int(c[10] - c0[10]),
            "matvecs_per_step": 6 * (c[10] - c0[10]) / max(steps, 1), "sim_time_s": float(c[2]),
            "newton": st.newton_stats()}
        del st
    out["mixed_mlp_vs_fp64_newton"] = out["%s_mlp_gated" % prec]["steps_per_s"] / out["fp64_newton"]["steps_per_s"]
    best = max(out["%s_prev" % prec]["steps_per_s"], out["%s_newton" % prec]["steps_per_s"])
    out["mlp_gated_vs_best_classical"] = out["%s_mlp_gated" % prec]["steps_per_s"] / best
    return out


def vmode_config3(nsteps):
    """Config 3: curved120k (the 60k geometry refined, a - b from a seeded Gaussian field
    in [-0.006, 0.006], sigma_n in [20, 80] MPa) in V-mode with the gated MLP start:
    steps/s and Newton statistics against the classical starts."""
    import gc
    import torch
    from pyquake3d_b200 import QDsim, read_mshV2
    set_case("curved120k")
    msh, para = make_case(0)
    set_case("curved60k")
    nodes, tris = read_mshV2(msh)
    sim = QDsim(tris, nodes, para, precision="mixed")
    sim.tree_block.want = ("fp64", "mixed")
    op = sim.tree_block.op()
    out = vmode_study(sim, op, nsteps, prec="mixed")
    out["triangles"] = int(op.n)
    del op, sim
    gc.collect()
    torch.cuda.empty_cache()
    return out


# --------------------------------------------------------------------- reference arm (CPU)
_W = {}


def ensemble_study(nsteps, nrep, faults=32):
    """Batched ensemble: `faults` independent planar faults of uneven size (seeded
    U[2000, 20000] triangles, dips U[20, 90] degrees, seeded friction), one
    block-diagonal matvec and one cooperative step launch per step for all.
    Aggregate fault-steps/s for the FP32 and FP64 operators, matvec bandwidth, and
    per-fault slip error of the FP32 run against the FP64 run on the FP64 step
    sizes (dt replay)."""
    import torch
    from pyquake3d_b200 import QDsim, read_mshV2
    from pyquake3d_b200.ensemble import Ensemble
    from pyquake3d_b200.meshgen import ensemble_faults
    d = os.path.join(tempfile.gettempdir(), "pq3d_bench_ensemble%d" % faults)
    if not os.path.exists(os.path.join(d, "fault%02d" % (faults - 1), "parameter.txt")):
        ensemble_faults(d, n_faults=faults, seed=4, lo=2000, hi=20000, edge=0.5)
    t0 = time.perf_counter()
    sims = []
    for f in range(faults):
        fd = os.path.join(d, "fault%02d" % f)
        nodes, tris = read_mshV2(os.path.join(fd, "fault%02d.msh" % f))
        sims.append(QDsim(tris, nodes, os.path.join(fd, "parameter.txt"), precision="fp32"))
    t_host = time.perf_counter() - t0
    E64 = Ensemble(sims, precision="fp64", want=("fp64", "fp32", "mixed"))
    torch.cuda.synchronize()
    t_asm = time.perf_counter() - t0 - t_host
    E32 = Ensemble(sims, precision="fp32", share=E64)
    EMX = Ensemble(sims, precision="mixed", share=E64)
    hbm, _ = peaks()
    out = {"faults": faults, "triangles": int(E64.n), "sizes": [int(s) for s in E64.struct.sizes],
           "host_setup_s": round(t_host, 2), "assembly_s": round(t_asm, 2)}
    h0 = [s.htry for s in sims]
    G = 50
    for name, E in (("mixed", EMX), ("fp32", E32), ("fp64", E64)):
        E.run(5, h0)                                  # warm-up (and the first steps of the run)
        E.set_history(G)
        g = E.capture(G)
        reps = max(1, nsteps // G)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            g.replay()
        e1.record()
        torch.cuda.synchronize()
        E._status()
        t = e0.elapsed_time(e1) / 1e3
        P = E.op.plan(name)
        for _ in range(3):
            E.op.matvec(E.x, name, slots_only=True)
        torch.cuda.synchronize()
        m0, m1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        m0.record()
        for _ in range(20):
            E.op.matvec(E.x, name, slots_only=True)
        m1.record()
        torch.cuda.synchronize()
        tm = m0.elapsed_time(m1) / 1e3 / 20
        out[name] = {"ensemble_steps_per_s": reps * G / t, "fault_steps_per_s": faults * reps * G / t,
                     "ms_per_step": 1e3 * t / (reps * G), "steps": reps * G,
                     "hmatvec": {"ms": 1e3 * tm, "GBs": P["alg_bytes"] / tm / 1e9, "frac": P["alg_bytes"] / tm / 1e9 / hbm,
                                 "alg_bytes": int(P["alg_bytes"])}}
        del g
    out["fp32_vs_fp64"] = out["fp32"]["fault_steps_per_s"] / out["fp64"]["fault_steps_per_s"]
    out["mixed_vs_fp64"] = out["mixed"]["fault_steps_per_s"] / out["fp64"]["fault_steps_per_s"]
    # per-fault error: fresh ensembles from the initial state, FP32 on the FP64 step sizes;
    # beside it each fault's FP64 chaos floor (an FP64 run whose initial shear tractions
    # differ by a relative 1e-12, on the same step sizes)
    R64 = Ensemble(sims, precision="fp64", share=E64)
    R32 = Ensemble(sims, precision="fp32", share=E64)
    RMX = Ensemble(sims, precision="mixed", share=E64)
    RP = Ensemble(sims, precision="fp64", share=E64)
    RP.t["Tt1o"].mul_(1.0 + 1e-12)
    RP.t["Tt2o"].mul_(1.0 + 1e-12)
    h = R64.run(nrep, h0)
    for R in (R32, RMX, RP):
        R.set_replay(torch.tensor(h[:, :, 0], device=R.op.dev))
        R.run(nrep, h0)
    rel = lambda R, f, b: float(np.linalg.norm(R.get("slip", f) - b) / np.linalg.norm(b))
    errs, errm, floor = [], [], []
    for f in range(faults):
        b = R64.get("slip", f)
        errs.append(rel(R32, f, b))
        errm.append(rel(RMX, f, b))
        floor.append(rel(RP, f, b))
    above = [f for f in range(faults) if max(errs[f], errm[f]) > 1e-5]
    out["slip_rel_err_vs_fp64"] = {"steps": nrep, "max": max(errs), "median": float(np.median(errs)),
                                   "mixed_max": max(errm), "mixed_median": float(np.median(errm)),
                                   "per_fault": errs, "mixed_per_fault": errm, "chaos_floor_per_fault": floor,
                                   "above_1e-5": {str(f): {"fp32": errs[f], "mixed": errm[f], "chaos_floor": floor[f]}
                                                  for f in above},
                                   "method": "dt replay of the FP64 ensemble; chaos floor: FP64 with initial shear "
                                             "tractions perturbed by a relative 1e-12"}
    del E32, E64, EMX, R32, R64, RMX, RP
    torch.cuda.empty_cache()
    return out


def _rank_init(geo, tasks, oracle_dir):
    """One emulated MPI rank of the reference: assemble its share of the blocks (as
    ACA_worker does on every rank, src/Hmatrix.py:1014-1066) and keep them."""
    if oracle_dir not in sys.path:
        sys.path.insert(0, oracle_dir)
    import qd_oracle
    qd_oracle._pool_init(geo)
    _W["blocks"] = [qd_oracle._pool_block(t) for t in tasks]


def _rank_mvm(args):
    """This rank's part of the six products (blocks_process_MVM on its local blocks)."""
    import qd_oracle
    x1, x2 = args
    ho = object.__new__(qd_oracle.OracleOperator)
    ho.blocks = _W["blocks"]
    return qd_oracle.operator_mvm(ho)(x1, x2)


def _rank_ready(_):
    return len(_W["blocks"])


def _maps_with(name):
    try:
        return sorted({l.split()[-1] for l in open("/proc/self/maps") if name in l and l.split()[-1].startswith("/")})
    except OSError:
        return []


def run_reference(args, rank, world):
    """The reference's CPU path on the host cores, on the GPU arm's workload and step
    counts.  Nothing of the product's compute path is loaded here: the mesh and the
    initial state come from the host-only input modules (pure numpy restatements of
    read_mshV2 / Init_condition, pinned bitwise to the reference), the operator is
    assembled on the CPU by the oracle (C Green's function + numpy ACA+, relative
    tolerance 1e-5 as in the workload) in worker processes that emulate the
    reference's MPI ranks -- each assembles and keeps its share of the blocks, as
    ACA_worker does -- and every step runs the oracle's simu_forward with the six
    block-loop MVMs split over those ranks and summed (the reference's
    reduce(SUM), src/QDsim.py:906-922)."""
    if rank != 0:
        print(json.dumps({"impl": "reference", "rank": rank, "skipped": "rank 0 runs the CPU arm"}), file=sys.stderr)
        return
    import multiprocessing as mp
    import qd_oracle
    from pyquake3d_b200 import QDsim, read_mshV2
    from pyquake3d_b200.hmatrix import aca_start_indices
    t0 = time.perf_counter()
    msh, para = make_case(rank)
    nodes, tris = read_mshV2(msh)
    sim = QDsim(tris, nodes, para, device="cpu", precision="fp64")
    st = sim.tree_block.struct
    tol = float(sim.Para0.get("ACA tolerance", 0.01))
    rel = sim.Para0.get("ACA relative tolerance", "False") == "True"
    starts = aca_start_indices(st.blocks, int(sim.Para0.get("ACA seed", 0)))
    geo = qd_oracle.Geometry(sim.xg, sim.eleVec, sim.nodelst, sim.elelst, sim.mu, sim.lambda_)
    tasks, si = [], 0
    for b in st.blocks:
        s0 = None
        if b.aca:
            s0 = starts[si]
            si += 1
        tasks.append((np.asarray(b.row.indices), np.asarray(b.col.indices), bool(b.aca), s0, tol, rel))
    cores = os.cpu_count() or 1
    nproc = max(1, min(cores, 64))
    # balance the ranks by assembly cost (largest first, to the least loaded rank)
    cost = [len(t[0]) * len(t[1]) if not t[2] else 60 * (len(t[0]) + len(t[1])) for t in tasks]
    share, load = [[] for _ in range(nproc)], np.zeros(nproc)
    for i in np.argsort(cost)[::-1]:
        r = int(np.argmin(load))
        share[r].append(tasks[i])
        load[r] += cost[i]
    ctx = mp.get_context("spawn")
    odir = os.path.join(REPO, "oracle")
    pools = [ctx.Pool(1, initializer=_rank_init, initargs=(geo, share[r], odir)) for r in range(nproc)]
    nblk = sum(p.apply(_rank_ready, (0,)) for p in pools)
    assert nblk == len(tasks)
    t_asm = time.perf_counter() - t0

    def mvm(x1, x2):
        res = [p.apply_async(_rank_mvm, ((x1, x2),)) for p in pools]
        parts = [r.get() for r in res]
        return tuple(sum(p[k] for p in parts) for k in range(3))   # the reference's reduce(SUM)

    ost = qd_oracle.OracleStepper(qd_oracle.sim_state(sim), mvm, sim.V0, sim.mu, sim.Cs, sim.RelTol, sim.fix_Tn)
    dttry = sim.htry
    # the GPU arm's step counts; larger requests are capped so the arm ends in minutes
    nwarm = min(args.warmup, 20)
    nsteps = max(1, min(args.steps, 200))
    for _ in range(nwarm):
        _, dttry = ost.simu_forward(dttry)
    t1 = time.perf_counter()
    for _ in range(nsteps):
        _, dttry = ost.simu_forward(dttry)
    dt = time.perf_counter() - t1
    for p in pools:
        p.close()
    v = nsteps / dt
    line = {"metric": METRIC, "impl": "reference", "value": v, "unit": "steps/s", "n_gpus": world,
            "steps": nsteps, "warmup": nwarm, "ms_per_step": 1e3 * dt / nsteps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": CASE + " (%d triangles, H-matrix leaf %d, eta 2, ACA %s %g)" % (
                           st.n, st.mini_leaf, "relative" if rel else "absolute", tol),
                       "path": "reference CPU path: operator assembled on the CPU (C Green's function, numpy ACA+) "
                               "by %d processes emulating the MPI ranks, each keeping its blocks; per step the six "
                               "block-loop MVMs on every rank + sum and DP5(4), numpy FP64" % nproc,
                       "assembly_s": round(t_asm, 1),
                       "steps_requested": args.steps, "warmup_requested": args.warmup},
            "cpu_baseline": {"value": v, "unit": "steps/s", "cores": nproc, "kind": "port",
                             "sample": "%d steps of the %d-triangle case after %d warm-up steps" % (nsteps, st.n, nwarm)},
            "e2e": {"value": v, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "repo_libraries_loaded": [m for m in _maps_with(".so") if m.startswith(REPO)]}
    print(json.dumps(line))


# --------------------------------------------------------------------- our arm
def run_partition(args, rank, world, local):
    """ONE fault (the workload) row-partitioned over the ranks, strong scaling: each
    rank assembles and applies the operator of its tree-order rows and steps those
    rows; per step one all-gather of the slip-rate deficit, and per attempt one
    all-reduce (max) of the error maxima, with the step-size controller on the
    device (PartitionedStepper.enqueue_device_step: no host read inside a step;
    G steps captured in a CUDA graph, collectives included).  value = accepted
    steps of the one fault / max over ranks of the timed region."""
    import torch
    import torch.distributed as dist
    from pyquake3d_b200 import QDsim, read_mshV2
    from pyquake3d_b200 import partition as P
    dev = "cuda:%d" % local

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(v):
        if world == 1:
            return v
        t = torch.tensor([v], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    msh, para = make_case(rank)                 # the same fault on every rank (seeded mesh)
    nodes, tris = read_mshV2(msh)
    t0 = time.perf_counter()
    sim = QDsim(tris, nodes, para, device=dev, precision=args.precision)
    st = sim.tree_block.struct
    t_host = time.perf_counter() - t0
    b = P.row_partition(st, world)
    be = P.DeviceRowBackend(sim, st, int(b[rank]), int(b[rank + 1]), precision=args.precision, device=dev)
    torch.cuda.synchronize()
    t_asm = max_over_ranks(time.perf_counter() - t0 - t_host)
    comm = P.TorchComm(use_dist=dist.is_initialized())
    ps = P.PartitionedStepper([be], comm, sim.RelTol, attempts=args.attempts)
    plan = be.op.plan(args.precision)

    # warm-up (device-controlled, one host read at the end), then the graph
    ps.run_device(args.warmup, sim.htry, chunk=args.warmup)
    G = 50
    graph = ps.capture(G)
    ok = max_over_ranks(0.0 if graph is not None else 1.0) == 0.0
    if not ok:
        graph = None                       # every rank launches alike
    torch.cuda.synchronize()
    pc0 = be.pc.cpu().numpy()
    if pc0[P.PC_HALT] != 0:
        raise RuntimeError("partitioned step halted during capture warm-up")
    clk = Clocks(local)
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    # G steps per replay (or G eager steps), then one host read of the control block; a
    # step that needed more than the attempt slots halted the device sequence and is
    # finished here by the host controller, inside the timed region, before the next
    # chunk: every rank reads the same block and takes the same path
    e0.record()
    done, halts = 0, 0
    prev = int(pc0[P.PC_STEPS])
    while done < args.steps:
        if graph is not None:
            graph.replay()
        else:
            for _ in range(G):
                ps.enqueue_device_step()
        pc1 = be.pc.cpu().numpy()
        if pc1[P.PC_STATUS] != 0:
            raise RuntimeError("time step failed in the partitioned run")
        done += int(pc1[P.PC_STEPS]) - prev
        if pc1[P.PC_HALT] != 0:
            halts += 1
            ps.time, ps.steps, ps.rejects = float(pc1[P.PC_TIME]), int(pc1[P.PC_STEPS]), int(pc1[P.PC_REJ])
            h, dtnext = ps._attempts(float(pc1[P.PC_H]), int(pc1[P.PC_NRJCT]), False)
            be.pc_resume(ps, dtnext, h)
            done += 1
        prev = int(be.pc[P.PC_STEPS].item())
    e1.record()
    torch.cuda.synchronize()
    barrier()
    clocks = clk.stop()
    t = max_over_ranks(e0.elapsed_time(e1) / 1e3)
    halted = halts > 0
    del graph                              # holds NCCL calls: released before the group

    # this rank's H-matvec alone (its rows' blocks), CUDA events
    for _ in range(5):
        be.op.matvec(be.xg_buf, args.precision, slots_only=True)
    torch.cuda.synchronize()
    m0, m1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    m0.record()
    for _ in range(50):
        be.op.matvec(be.xg_buf, args.precision, slots_only=True)
    m1.record()
    torch.cuda.synchronize()
    t_mv_rank = m0.elapsed_time(m1) / 1e3 / 50
    t_mv = max_over_ranks(t_mv_rank)
    bytes_all = float(plan["alg_bytes"])
    if world > 1:
        bt = torch.tensor([bytes_all], dtype=torch.float64, device=dev)
        dist.all_reduce(bt)
        bytes_all = float(bt.item())
    hbm, peak_kind = peaks()

    # end to end: the host reads the control block after every step (h, time, counters)
    ne = min(args.steps, 100)
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    hs = ps.run_device(ne, float(be.pc[P.PC_H]), chunk=1)
    e1.record()
    torch.cuda.synchronize()
    t_e2e = max_over_ranks(e0.elapsed_time(e1) / 1e3)
    nl = (2 if plan["n_utasks"] > 0 or args.precision == "mixed" else 1) + 2 * args.attempts + 2
    rows = int(b[rank + 1] - b[rank])
    line = {
        "metric": METRIC, "value": done / t, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * t / max(done, 1), "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None,
        "dtype": {"fp32": "f32 operator, f64 state", "bf16": "bf16+f32 operator, f64 state", "fp64": "f64",
                  "mixed": "f32+f16+i8 operator, f32 accumulation, f64 state"}[args.precision],
        "data": "synthetic",
        "config": {"workload": CASE + " (%d triangles), one fault" % sim.xg.shape[0],
                   "parallelism": "row partition x%d" % world, "precision": args.precision,
                   "collectives": "NCCL" if dist.is_initialized() else "none (one rank, one process)",
                   "rows_per_rank": [int(b[r + 1] - b[r]) for r in range(world)],
                   "attempt_slots": args.attempts, "cuda_graph_steps": G if ok else 0,
                   "l2": "inputs larger than L2 (operator %.2f GB per step over all ranks)" % (bytes_all / 1e9),
                   "host_setup_s": round(t_host, 2), "assembly_s": round(t_asm, 2)},
        "steps_done": done, "halted": halted, "host_finished_steps": halts,
        "roofline": {"bound": "hbm", "achieved": bytes_all / t_mv / 1e9, "peak": hbm * world, "unit": "GB/s",
                     "frac": bytes_all / t_mv / 1e9 / (hbm * world), "traffic": None,
                     "kernel": "H-matvec of every rank's rows (slowest rank's time), %d GPUs" % world,
                     "alg_bytes": bytes_all, "ms": 1e3 * t_mv, "peak_source": peak_kind},
        "step_overhead_ms": 1e3 * (t / max(done, 1) - t_mv),
        "e2e": {"value": ne / t_e2e, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 128,
                "steps": ne, "path": "PartitionedStepper.run_device(chunk=1): the control block to the host "
                                     "after every step (its accepted h)"},
        "cpu_baseline": None,
        "gpu_launches": nl * done,
        "clocks": clocks,
        "rank0_rows": rows, "rank0_matvec_ms": 1e3 * t_mv_rank, "e2e_last_h": hs[-1] if hs else None,
    }
    if rank == 0:
        print(json.dumps(line))
    if dist.is_initialized():
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--cpu-budget", type=float, default=20.0)
    ap.add_argument("--case", default=CASE, help="workload (profiling uses a smaller one)")
    ap.add_argument("--no-vmode", action="store_true", help="skip the V-mode study")
    ap.add_argument("--vmode-steps", type=int, default=60)
    ap.add_argument("--vmode120-steps", type=int, default=30, help="config 3 (curved120k) V-mode study; 0 skips")
    ap.add_argument("--no-ensemble", action="store_true", help="skip the 32-fault ensemble study")
    ap.add_argument("--ensemble-steps", type=int, default=500)
    ap.add_argument("--accuracy-steps", type=int, default=500,
                    help="horizon of the error study against the FP64 path (dt replay)")
    ap.add_argument("--precision", default="mixed", choices=["fp32", "bf16", "fp64", "mixed"],
                    help="operator storage of the headline path (mixed and fp32 meet the 1e-5 slip target)")
    ap.add_argument("--parallelism", default="auto", choices=["auto", "partition", "replicas"],
                    help="several GPUs: partition = one fault row-partitioned over the ranks (strong scaling, "
                         "the default for N > 1); replicas = one fault per rank")
    ap.add_argument("--attempts", type=int, default=3, help="attempt slots per partitioned step")
    ap.add_argument("--no-configs", action="store_true", help="skip the plain2k and thrust20k configurations")
    ap.add_argument("--config0-steps", type=int, default=2000, help="plain2k (dense FP64) steps")
    ap.add_argument("--config1-steps", type=int, default=20000, help="thrust20k (FP32 low rank) steps")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    set_case(args.case)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        # CPU only: rank 0 runs the reference's path on the host cores, the other ranks
        # exit at once (no process group, no CUDA context)
        run_reference(args, rank, world)
        return

    import torch
    import torch.distributed as dist
    if world > 1 or "TORCHELASTIC_RUN_ID" in os.environ:
        # a process group whenever launched by torchrun (one rank included: the
        # partitioned path then runs its collectives through NCCL)
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    torch.cuda.set_device(local)
    if args.parallelism == "partition" or (args.parallelism == "auto" and world > 1):
        run_partition(args, rank, world, local)
        return

    # batched ensemble of 32 independent faults (one launch per step for all); run first,
    # on an empty device: its ACA workspaces (all live until packing) are the run's peak
    ensemble = None
    if not args.no_ensemble and world == 1:
        ensemble = ensemble_study(args.ensemble_steps, 200)
        import gc
        gc.collect()
        torch.cuda.empty_cache()

    # the two smaller configurations at their full step counts: plain2k (dense FP64
    # operator, 2,000 steps) and thrust20k (FP32 low rank, 20,000 steps; mixed beside it)
    configs = None
    if not args.no_configs and world == 1:
        configs = {}
        for name, prec, k, marks, extra in (("plain2k", "fp64", args.config0_steps, (500, 2000), ()),
                                            ("thrust20k", "fp32", args.config1_steps, (500, 2000, 20000), ("mixed",))):
            try:
                configs[name] = config_study(name, prec, k, 10.0, marks, extra=extra)
            except RuntimeError as e:       # recorded in the line; the headline still runs
                configs[name] = {"error": str(e)}
        import gc
        gc.collect()
        torch.cuda.empty_cache()

    from pyquake3d_b200 import QDsim, read_mshV2
    from pyquake3d_b200.qdsim import DeviceStepper
    msh, para = make_case(rank)
    nodes, tris = read_mshV2(msh)
    t0 = time.perf_counter()
    sim = QDsim(tris, nodes, para, device="cuda:%d" % local, precision=args.precision)
    sim.tree_block.want = ("fp64", "bf16", "fp32", "mixed")
    t_host = time.perf_counter() - t0
    op = sim.tree_block.op()
    t_asm = time.perf_counter() - t0 - t_host
    kS, kD = op.ranks()
    head = args.precision
    steppers = {p: DeviceStepper(sim, op, p) for p in ("fp32", "bf16", "fp64", "mixed")}
    plans = {p: op.plan(p) for p in steppers}

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(v):
        if world == 1:
            return v
        t = torch.tensor([v], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    graphs = {}

    def timed_steps(stepper, k, dttry, use_graph=True):
        """k steps; with use_graph, replays of a captured graph of G steps (k multiple of G)."""
        G = 100
        g = None
        if use_graph and k % G == 0 and k >= G:
            key = id(stepper)
            if key not in graphs:
                graphs[key] = stepper.capture(G)
            g = graphs[key]
        if g is None:
            stepper.set_history(k)
        stepper.ctrl[0] = dttry
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        if g is not None:
            for _ in range(k // G):
                g.replay()
        else:
            for i in range(k):
                stepper.launch(i)
        e1.record()
        torch.cuda.synchronize()
        barrier()
        c = stepper.ctrl.cpu().numpy()
        if c[4] != 0:
            raise RuntimeError("step failed with status %d" % int(c[4]))
        return e0.elapsed_time(e1) / 1e3, float(c[0])

    # warm-up of every path, then the timed region of the headline path with clock sampling
    dts = {}
    for p, st in steppers.items():
        _, dts[p] = timed_steps(st, args.warmup, sim.htry, use_graph=False)
    timing = {}
    clk = Clocks(local)
    timing[head], dts[head] = timed_steps(steppers[head], args.steps, dts[head])
    clocks = clk.stop()
    hist = steppers[head].hist.view(-1, 6).cpu().numpy()[:min(args.steps, steppers[head].hist_cap)]
    graph_used = graphs.get(id(steppers[head])) is not None
    for p in steppers:
        if p != head:
            timing[p], dts[p] = timed_steps(steppers[p], args.steps, dts[p])
    timing = {p: max_over_ranks(t) for p, t in timing.items()}
    steps_total = args.steps * world
    rate = {p: steps_total / t for p, t in timing.items()}

    # H-matvec alone (k_dense_v + k_u as the step runs them), CUDA events on the launching stream
    def time_matvec(stepper, reps=50):
        for _ in range(5):
            op.matvec(stepper.x, stepper.precision, slots_only=True)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            op.matvec(stepper.x, stepper.precision, slots_only=True)
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 1e3 / reps
    hbm, peak_kind = peaks()
    mv = {}
    for p, st in steppers.items():
        t = time_matvec(st)
        mv[p] = {"ms": 1e3 * t, "GBs": plans[p]["alg_bytes"] / t / 1e9, "alg_bytes": int(plans[p]["alg_bytes"]),
                 "frac": plans[p]["alg_bytes"] / t / 1e9 / hbm, "stored_bytes": int(plans[p]["stored_bytes"])}

    # Green's-function assembly roofline (FP64 compute bound)
    gf = gf_roofline(op, sim.tree_block.struct)

    # accuracy vs the FP64 path at equal times (dt replay of the FP64 run), at several horizons
    # (a fixed horizon, independent of the timed step count)
    accuracy = accuracy_study(sim, op, args.accuracy_steps, precisions=("bf16", "fp32", "mixed"))
    # the same comparison at common times, each run with its own step sizes
    accuracy["common_times"] = {p: accuracy_common_times(sim, op, p, args.accuracy_steps) for p in ("fp32", "mixed")}

    # V-mode: DP5(4) with one H-matvec per stage and a Newton solve for V; MLP seed
    # trained on the run's own solves (hand-written kernels)
    vmode = None
    if not args.no_vmode:
        vmode = vmode_study(sim, op, args.vmode_steps, prec="mixed")

    # config 3 (curved120k, heterogeneous friction) in V-mode with the gated MLP, on an
    # operator of its own; the 60k steppers stay resident beside it
    vmode120 = None
    if not args.no_vmode and args.vmode120_steps > 0 and world == 1:
        vmode120 = vmode_config3(args.vmode120_steps)

    # end to end through the reference call surface (QDsim.simu_forward) with the
    # reference main loop's per-step host traffic
    mixed = steppers[head]
    sim._dev = mixed
    ne = min(args.steps, 300)
    # one untimed step first: the loop's steady state, where each step's H-matvec was
    # enqueued by the call before; the timed region then ends with one such pre-launched
    # H-matvec, so it holds exactly ne steps of device work
    _, dttry = sim.simu_forward(dts[head])
    sim.snapshot_async(("slipv", "Tt"))           # allocates the mapped host buffers once
    torch.cuda.synchronize()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(ne):
        h, dttry = sim.simu_forward(dttry)
        done, _ = sim.snapshot_async(("slipv", "Tt"))   # slip rate and traction of this step to the host
    done.synchronize()                                   # the last snapshot is inside the timed region
    e1.record()
    torch.cuda.synchronize()
    t_e2e = max_over_ranks(e0.elapsed_time(e1) / 1e3)
    e2e = {"value": ne * world / t_e2e, "unit": "steps/s", "h2d_bytes_per_step": 8,
           "d2h_bytes_per_step": int(12 * 8 + 2 * 8 * sim.xg.shape[0]), "steps": ne,
           "path": "QDsim.simu_forward per step (control block to mapped host memory; the next step's "
                   "H-matvec enqueued before the host waits) + slip-rate and traction vectors to pinned "
                   "host memory (QDsim.snapshot_async: gather on a side stream, copy-engine transfer)"}

    # the reference main loop verbatim (src/main.py:161-184): after every step it reads
    # max |slipv1|, max |slipv2| and keeps the slipv and Tt arrays (device-backed QDsim
    # attributes, prefetched by the step after the first reads)
    nl = min(args.steps, 300)
    _, dttry = sim.simu_forward(dttry)
    _ = (sim.slipv1, sim.slipv2, sim.slipv, sim.Tt)
    torch.cuda.synchronize()
    barrier()
    kept_v, kept_t = [], []
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(nl):
        h, dtnext = sim.simu_forward(dttry)
        _ = (np.max(np.abs(sim.slipv1)), np.max(np.abs(sim.slipv2)))
        kept_v.append(sim.slipv)
        kept_t.append(sim.Tt)
        dttry = dtnext
    e1.record()
    torch.cuda.synchronize()
    t_loop = max_over_ranks(e0.elapsed_time(e1) / 1e3)
    e2e["reference_loop"] = {
        "value": nl * world / t_loop, "unit": "steps/s", "steps": nl,
        "path": "src/main.py's loop unchanged: simu_forward, np.max(np.abs(slipv1|slipv2)), SLIPV.append(slipv), "
                "Tt.append(Tt) every step (four 8n-byte vectors to the host per step)"}
    del kept_v, kept_t

    # CPU baseline: the reference's step on the same operator (rank 0, N=1)
    cpu = None
    pinned = None
    if rank == 0 and world == 1 and not args.no_cpu:
        import qd_oracle
        from pyquake3d_b200 import QDsim as Q2
        ho = export_host_operator(op)
        host = Q2(tris, nodes, para, device="cuda:0", precision="bf16")
        crate, k, secs, ost, hs = cpu_reference_steps(ho, qd_oracle.sim_state(host), host.V0, host.mu, host.Cs,
                                                      args.cpu_budget, dttry=host.htry, reltol=host.RelTol,
                                                      fix_tn=host.fix_Tn)
        cpu = {"value": crate, "unit": "steps/s", "cores": 1, "kind": "port",
               "sample": "%d steps (%.1f s) of the same 60k workload: six block-loop MVMs + DP5(4), "
                         "numpy FP64, one process" % (k, secs)}
        del ho
        # the device FP64 path pinned to the oracle over those steps (same operator)
        pinned = pin_fp64_to_oracle(host, op, ost, hs)

    traffic = None
    tp = os.path.join(REPO, "profiles", "hmatvec_traffic.json")
    if os.path.exists(tp):
        try:
            traffic = json.load(open(tp)).get("bytes_per_matvec_" + head)
        except (ValueError, OSError):
            traffic = None
    nlaunch_step = (2 if plans[head]["n_utasks"] > 0 else 1) + 1
    prec_text = {"fp32": "fp32 operator (near field + low rank), fp64 state and slip",
                 "bf16": "bf16 low rank / fp32 near field, fp64 state and slip",
                 "fp64": "fp64 operator and state",
                 "mixed": "fp32 near field / low-rank terms in fp32, fp16 or int8 by weight, fp64 state and slip"}
    err_head = accuracy.get(head, [{}])[-1] if head in accuracy else {}
    line = {
        "metric": METRIC, "value": rate[head], "unit": "steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * timing[head] / args.steps, "higher_is_better": True,
        # one fault: with more GPUs the default (partition) splits this same fault, so the
        # total work is fixed; --parallelism replicas adds a fault per GPU instead
        "scaling": "weak" if (world > 1 and args.parallelism == "replicas") else "strong", "vs_baseline": None,
        "dtype": {"fp32": "f32 operator, f64 state", "bf16": "bf16+f32 operator, f64 state", "fp64": "f64",
                  "mixed": "f32+f16+i8 operator, f32 accumulation, f64 state"}[head],
        "data": "synthetic",
        "config": {"workload": CASE + " (%d triangles)" % sim.xg.shape[0], "precision": prec_text[head],
                   "leaf": int(sim.tree_block.mini_leaf), "eta": 2.0, "aca": "relative 1e-5",
                   "mean_rank": float(np.mean(np.concatenate([kS, kD]))), "max_rank": int(max(kS.max(), kD.max())),
                   "l2": "inputs larger than L2 (operator %.2f GB per step)" % (plans[head]["alg_bytes"] / 1e9),
                   "parallelism": "replicas x%d" % world if world > 1 else "single GPU", "host_setup_s": round(t_host, 2),
                   "assembly_s": round(t_asm, 2), "assembly_breakdown": {k: round(v, 3) for k, v in op.timings.items()}},
        "roofline": {"bound": "hbm", "achieved": mv[head]["GBs"], "peak": hbm, "unit": "GB/s",
                     "frac": mv[head]["frac"], "traffic": traffic,
                     "kernel": "H-matvec (k_v + k_du), " + prec_text[head].split(",")[0],
                     "alg_bytes": mv[head]["alg_bytes"], "ms": mv[head]["ms"], "peak_source": peak_kind},
        "slip_rel_err_vs_fp64": err_head.get("slip"),
        "err_vs_fp64_at_horizon": dict(err_head, horizon_steps=args.accuracy_steps) if err_head else None,
        "plain_fp64": {"steps_per_s": rate["fp64"], "ms_per_step": 1e3 * timing["fp64"] / args.steps,
                       "hmatvec": mv["fp64"]},
        "mixed_vs_plain": rate[head] / rate["fp64"],
        "all_precisions": {p: {"steps_per_s": rate[p], "ms_per_step": 1e3 * timing[p] / args.steps,
                               "hmatvec": mv[p], "vs_fp64": rate[p] / rate["fp64"]} for p in steppers},
        "mixed_storage": {"tolerance": plans["mixed"]["mixed"]["tol"],
                          "terms_fp32_fp16_int8": [int(sum(c)) for c in plans["mixed"]["mixed"]["class_terms"]],
                          "stored_bytes": int(plans["mixed"]["stored_bytes"])},
        "accuracy_vs_fp64": accuracy,
        "fp64_pinned_to_oracle": pinned,
        "vmode": vmode,
        "vmode_curved120k": vmode120,
        "ensemble": ensemble,
        "configs": configs,
        "gf_assembly": gf,
        "sim": {"time_s": float(hist[-1, 2]), "last_dt": float(hist[-1, 0]), "rejects": int(hist[:, 5].sum())},
        "e2e": e2e,
        "cpu_baseline": cpu,
        "gpu_launches": nlaunch_step * args.steps,
        "cuda_graph": graph_used,
        "clocks": clocks,
    }
    if rank == 0:
        print(json.dumps(line))
    if dist.is_initialized():
        dist.barrier()
        dist.destroy_process_group()

if __name__ == "__main__":
    main()
