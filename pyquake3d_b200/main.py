"""Command-line driver: the run loop of the reference's src/main.py on one GPU.

    python -m pyquake3d_b200.main -g fault.msh -p parameter.txt

Same inputs and outputs as the reference driver (src/main.py:42-235):
  state.txt           header (:83-99), one line per step (:177), end time (:234-235)
  Init.vtk            initial state (:126-127)
  out_vtk/stepI.vtk   every `outsteps` steps when outputvtk is True (:215-218)
  out_slipvTt/slipv_I.npy, Tt_I.npy
                      slip rate / shear traction of every step since the previous
                      output, when outputSLIPV / outputTt are True (:198-207)
  out_txt/            gridded maps when outputmatrix is True (:219-221)
  Corefunc directory  operator checkpoint when `save Corefunc` is True; a matching
                      checkpoint found there is loaded instead of assembling (:101-107)

Steps between two outputs run back to back on the device (one matvec + one step
kernel each, no host synchronization); the per-step state.txt values come from
the step kernel's history rows, and per-step slip-rate / traction snapshots are
device-to-device copies taken between launches.
"""
import argparse
import os
import sys
import time

import numpy as np

from .mesh import read_mshV2
from .output import StateLog
from .qdsim import QDsim
from . import _lib


BANNER = """# ----------------------------------------------------------------------------
# PyQuake3D quasi-dynamic SEAS hot path on one B200 (pyquake3d_b200)
# * 3D non-planar quasi-dynamic earthquake cycle simulations
# * H-matrix operator assembled and applied on the GPU
# * rate-and-state aging law, adaptive Dormand-Prince 5(4)
# * VTK / state.txt output in the reference formats
# ----------------------------------------------------------------------------"""


def output_points(total, outsteps):
    return [i for i in range(total) if i % outsteps == 0]


def step_ranges(total, outsteps):
    """[(first, last_exclusive)] covering range(total); each range ends right after an
    output step or at the end of the run."""
    ends = [i + 1 for i in output_points(total, outsteps)]
    if not ends or ends[-1] != total:
        ends.append(total)
    out, a = [], 0
    for e in ends:
        if e > a:
            out.append((a, e))
            a = e
    return out


def run(fnamegeo, fnamePara, steps=None, quiet=False, precision=None):
    nodelst, elelst = read_mshV2(fnamegeo)
    sim = QDsim(elelst, nodelst, fnamePara, precision=precision)
    if not quiet:
        print(BANNER)
        print("Input msh geometry file:", fnamegeo, flush=True)
        print("Input parameter file:", fnamePara, flush=True)
        print("Number of Node", nodelst.shape, flush=True)
        print("Number of Element", elelst.shape, flush=True)
    log = StateLog("state.txt", sim, fnamegeo, fnamePara, nodelst, elelst)
    loaded, _ = sim.get_block_core()
    if not quiet:
        print("jud_coredir", loaded)
        print("Hmatrix reading..." if loaded else "Start to calculate Hmatrix...", flush=True)
    sim.ouputVTK("Init.vtk")
    if not loaded:
        sim.tree_block.master(sim.Corefunc_directory, sim.tree_block.blocks_to_process, 0,
                              save_corefunc=sim.save_corefunc)
    P = sim.Para0
    total = int(P["totaloutputsteps"]) if steps is None else int(steps)
    outsteps = int(P["outsteps"])
    want_v = P.get("outputSLIPV") == "True"
    want_t = P.get("outputTt") == "True"
    want_vtk = P.get("outputvtk") == "True"
    want_txt = P.get("outputmatrix") == "True"
    st = sim._ensure_device()
    torch = st.torch
    iperm = torch.as_tensor(np.argsort(st.perm), device=st.op.dev)
    os.makedirs("out_vtk", exist_ok=True)
    t0 = time.perf_counter()
    dttry = sim.htry
    for a, b in step_ranges(total, outsteps):
        k = b - a
        st.set_history(k)
        st.ctrl[0] = float(dttry)
        snap_v = torch.empty((k, st.n), dtype=torch.float64, device=st.op.dev) if want_v else None
        snap_t = torch.empty((k, st.n), dtype=torch.float64, device=st.op.dev) if want_t else None
        for j in range(k):
            st.launch(j)
            if snap_v is not None:
                snap_v[j].copy_(st.t["slipv"])
            if snap_t is not None:
                snap_t[j].copy_(st.t["Tt"])
        c = st.ctrl.cpu().numpy()
        if c[4] != 0:
            log.close(time.perf_counter() - t0)
            raise _lib.Pq3dError(f"time step failed at step {a + int(c[8]) - st.steps}: status {int(c[4])}")
        hist = st.hist.view(-1, 6).cpu().numpy()[:k]
        st.steps += k
        st.time = float(c[2])
        sim.time = st.time
        dttry = float(c[0])
        for j in range(k):
            i = a + j
            h, tt, v1, v2 = hist[j, 0], hist[j, 2], hist[j, 3], hist[j, 4]
            log.step(i, h, v1, v2, tt)
            if not quiet and i % 20 == 0:
                print("iteration:", i, flush=True)
                print("dt:", h, " max_vel1:", v1, " max_vel2:", v2, " Seconds:", tt, "  Days:", tt / 3600 / 24,
                      "year", tt / 3600 / 24 / 365, flush=True)
        i = b - 1
        if i % outsteps == 0:
            if want_v or want_t:
                os.makedirs("out_slipvTt", exist_ok=True)
            if want_v:
                np.save("out_slipvTt/slipv_%d" % i, snap_v[:, iperm].cpu().numpy())
            if want_t:
                np.save("out_slipvTt/Tt_%d" % i, snap_t[:, iperm].cpu().numpy())
            if want_vtk:
                sim.ouputVTK("out_vtk/step" + str(i) + ".vtk")
            if want_txt:
                sim.outputtxt("step" + str(i))
    elapsed = time.perf_counter() - t0
    sim.sync_to_host()
    if not quiet:
        print(f"Program run time: {elapsed:.6f} sec")
    log.close(elapsed)
    return sim


def main(argv=None):
    ap = argparse.ArgumentParser(description="Quasi-dynamic earthquake-cycle simulation on one GPU.")
    ap.add_argument("-g", "--inputgeo", required=True, help="Input msh geometry file to execute")
    ap.add_argument("-p", "--inputpara", required=True, help="Input parameter file to process")
    ap.add_argument("--steps", type=int, default=None, help="override totaloutputsteps")
    ap.add_argument("--precision", default=None, help="operator storage: fp64 | fp32 | bf16")
    args = ap.parse_args(argv)
    run(args.inputgeo, args.inputpara, steps=args.steps, precision=args.precision)
    return 0


if __name__ == "__main__":
    sys.exit(main())
