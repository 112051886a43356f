"""Work-item shape tuner of the batched H-matvec.

The matvec's packed operator does not depend on how it is cut into work items,
so the tuner re-plans an assembled operator in place (DeviceHMatrix.set_shapes)
and times each candidate with CUDA events on the launching stream:
  dense_chunk  column groups per dense work item (one warp, 32 rows),
  v_chunk      column groups per V work item (the chunk partials of t = V x),
  u_rows       rows per U task (one CTA).
Coordinate descent from the current shapes, two sweeps over the three knobs;
a candidate is kept only when it beats the best time by more than the noise
margin.  The winners are written per GPU model and storage into the plan cache
(pyquake3d_b200/plan_cache.json), one entry per workload size; DeviceHMatrix
reads the entry tuned on the size closest to its own when it builds a plan.

    python -m pyquake3d_b200.autotune --case curved60k --precisions fp32,mixed,fp64 \
        [--out plan_cache.json]

With --time-only it builds the case, times one H-matvec per storage with the plan
cache's shapes (3 warm-up and --reps timed launches) and prints the times: the
driver of the matvec profiles.
"""
import argparse
import json
import os
import sys
import tempfile

CANDIDATES = {"dense_chunk": (4, 8, 16, 32, 64), "v_chunk": (8, 16, 32, 64, 128, 256), "u_rows": (256, 512, 1024)}


def time_matvec(op, dtype, x, reps=30):
    """Mean device time (s) of one H-matvec (slots only, as the step uses it)."""
    import torch
    for _ in range(3):
        op.matvec(x, dtype, slots_only=True)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        op.matvec(x, dtype, slots_only=True)
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / 1e3 / reps


def tune(op, dtype, sweeps=2, margin=0.01, reps=30, log=None):
    """Coordinate descent over CANDIDATES; returns (shapes dict, seconds, trials)."""
    import torch
    x = op.new_x(dtype)
    x.copy_(torch.randn_like(x) * 1e-9)
    cur = dict(zip(("dense_chunk", "v_chunk", "u_rows"), op.shapes(dtype)))
    op.set_shapes(dtype, **cur)
    best = time_matvec(op, dtype, x, reps)
    trials = [dict(cur, ms=1e3 * best)]
    for _ in range(sweeps):
        changed = False
        for knob, values in CANDIDATES.items():
            for v in values:
                if v == cur[knob]:
                    continue
                cand = dict(cur, **{knob: v})
                op.set_shapes(dtype, **cand)
                t = time_matvec(op, dtype, x, reps)
                trials.append(dict(cand, ms=1e3 * t))
                if log:
                    log("%s %s: %.1f us" % (dtype, cand, 1e6 * t))
                if t < best * (1.0 - margin):
                    best, cur, changed = t, cand, True
            op.set_shapes(dtype, **cur)
        if not changed:
            break
    op.set_shapes(dtype, **cur)
    return cur, best, trials


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--case", default="curved60k")
    ap.add_argument("--precisions", default="fp32,mixed,fp64,bf16")
    ap.add_argument("--out", default=None, help="plan cache to update (default: the package's plan_cache.json)")
    ap.add_argument("--reps", type=int, default=30)
    ap.add_argument("--time-only", action="store_true", help="time the matvec with the cached shapes, no tuning")
    args = ap.parse_args()
    import torch
    from . import meshgen
    from .hmatrix import PLAN_CACHE
    from .qdsim import QDsim
    from .mesh import read_mshV2
    precs = args.precisions.split(",")
    d = os.path.join(tempfile.gettempdir(), "pq3d_tune_" + args.case)
    msh, para = meshgen.make_case(args.case, d)
    nodes, tris = read_mshV2(msh)
    sim = QDsim(tris, nodes, para, precision=precs[0])
    sim.tree_block.want = tuple(sorted(set(["fp64"] + precs)))
    op = sim.tree_block.op()
    if args.time_only:
        for p in precs:
            x = op.new_x(p)
            x.copy_(torch.randn_like(x) * 1e-9)
            t = time_matvec(op, p, x, args.reps)
            P = op.plan(p)
            out = dict(case=args.case, n=int(op.n), precision=p, shapes=op.shapes(p), us=round(1e6 * t, 1),
                       alg_bytes=int(P["alg_bytes"]), GBs=round(P["alg_bytes"] / t / 1e9, 1))
            if p == "mixed":
                out["terms_fp32_fp16_int8"] = [int(sum(c)) for c in P["mixed"]["class_terms"]]
            print(json.dumps(out))
        return
    op.use_plan_cache = False            # tune from the built-in defaults
    gpu = torch.cuda.get_device_name(op.dev)
    out = args.out or PLAN_CACHE
    cache = json.load(open(out)) if os.path.exists(out) else {}
    ent = cache.setdefault(gpu, {})
    for p in precs:
        shapes, t, trials = tune(op, p, reps=args.reps, log=lambda m: print(m, file=sys.stderr))
        default = [r for r in trials if (r["dense_chunk"], r["v_chunk"], r["u_rows"]) ==
                   (op.DENSE_CHUNK_GROUPS[{"fp64": 0, "fp32": 1, "bf16": 2, "mixed": 3}[p]],
                    op.V_CHUNK_GROUPS[{"fp64": 0, "fp32": 1, "bf16": 2, "mixed": 3}[p]], op.U_ROWS)]
        new = dict(shapes, us=round(1e6 * t, 1), workload="%s (%d triangles)" % (args.case, op.n), n=int(op.n),
                   default_us=round(1e3 * default[0]["ms"], 1) if default else None, trials=len(trials))
        # one entry per workload size: replace this workload's, keep the others'
        old = ent.get(p)
        olds = [] if old is None else ([old] if isinstance(old, dict) else list(old))
        ent[p] = [e for e in olds if e.get("workload") != new["workload"]] + [new]
        print(json.dumps({p: new}))
    with open(out, "w") as f:
        json.dump(cache, f, indent=1, sort_keys=True)
    print("plan cache:", out)


if __name__ == "__main__":
    main()
