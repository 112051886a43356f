"""Generate the golden fixtures in tests/golden/ by running the REFERENCE itself.

Run in a container that has the reference tree: the --ref argument, else the
PQ3D_REFERENCE environment variable, else a tree named `reference` beside this
repository's checkout:

    python tests/golden/make_golden.py [--ref <reference tree>]

What it does:
  * builds the reference's TDstressFS_C.cpp from source (oracle/Makefile, target
    `ref`) -- the shipped binary is never used;
  * imports the reference's Python modules (src/readmsh.py, src/QDsim.py,
    src/Hmatrix.py, src/SH_greenfunction.py) with single-rank stand-ins for
    mpi4py and no-op stand-ins for matplotlib and pyvista (plotting and VTK
    reading are off the hot path), from a scratch directory holding
    src/TDstressFS_C.so, the relative path Hmatrix.py loads;
  * records reference outputs:
      gf_cases.npz      stress/strain of TDstressFS_C and TDstressEachSourceAtReceiver_C
                        (full and half space) on fixed and random receivers,
                        including on-plane, on-edge and vertex points, plus
                        the numpy twin SH_greenfunction.TDstressFS
      tiny_case.npz     a 576-element jittered planar fault: frames, initial
                        state, block structure, ACA ranks and factors of
                        a few blocks, the six operator products on fixed
                        vectors, and 30 simu_forward steps (seeded ACA starts)
      hs_cases.npz      half-space stress/strain of TDstressFS_C with jud_halfspace
                        (the C++ path the reference's ACA rows/columns use) and of
                        SH_greenfunction.TDstressHS (the numpy path its dense
                        blocks use) for triangles at depth, touching the free
                        surface, with a vertical side and vertical; receivers at
                        depth, near and on the surface
      tiny_hs_case.npz  the tiny case with `Half space: True` (its top edge lies on
                        the free surface): operator products and 30 steps
      output_case.npz   seeded state fields on the tiny mesh and the SHA-256 of
                        the files QDsim.ouputVTK and QDsim.outputtxt write
                        for them (output formats, byte for byte)
The fixtures are small (< 1 MB) and are what the CPU tests pin against.
"""
import argparse
import os
import shutil
import subprocess
import sys
import tempfile
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def install_stubs():
    class Comm:
        def Get_rank(self):
            return 0

        def Get_size(self):
            return 1

        def bcast(self, x, root=0):
            return x

        def reduce(self, x, op=None, root=0):
            return x

        def Barrier(self):
            pass

    mpi = types.ModuleType("mpi4py.MPI")
    mpi.COMM_WORLD = Comm()
    mpi.SUM = "sum"
    mpi.Wtime = __import__("time").time
    pkg = types.ModuleType("mpi4py")
    pkg.MPI = mpi
    sys.modules["mpi4py"] = pkg
    sys.modules["mpi4py.MPI"] = mpi

    class Anything(types.ModuleType):
        def __getattr__(self, name):
            return lambda *a, **k: None

    mpl = Anything("matplotlib")
    plt = Anything("matplotlib.pyplot")
    plt.rcParams = {}
    cols = Anything("matplotlib.colors")
    mpl.pyplot = plt
    mpl.colors = cols
    sys.modules["matplotlib"] = mpl
    sys.modules["matplotlib.pyplot"] = plt
    sys.modules["matplotlib.colors"] = cols
    sys.modules["pyvista"] = Anything("pyvista")


def gf_cases(lib, SH):
    import ctypes
    D = ctypes.POINTER(ctypes.c_double)
    lib.TDstressFS_C.argtypes = [D, D, D, ctypes.c_size_t, D, D, D] + [ctypes.c_double] * 5 + [ctypes.c_bool, D, D]
    lib.TDstressEachSourceAtReceiver_C.argtypes = [ctypes.c_double] * 3 + [D, D, D, ctypes.c_size_t] + \
        [ctypes.c_double] * 5 + [ctypes.c_bool, D, D]
    p = lambda a: a.ctypes.data_as(D)
    out = {}
    # (1) the fixed inputs of the reference's own main() (src/TDstressFS_C.cpp:2004-2023)
    X = np.array([48771.61733949, -48484.78117283, 48775.26818703])
    Y = np.array([30000., 15000., 3000.])
    Z = np.array([-13944.10291502, -20994.9909562, -12042.91174556])
    P1 = np.array([-49019.8529842, 0., -13632.75018015])
    P2 = np.array([-49294.4187163, 3000., -14516.85867197])
    P3 = np.array([-48427.27119853, 0., -14642.195744633])
    mu = lam = 32038120320.0
    for hs in (False, True):
        s, e = np.zeros(18), np.zeros(18)
        lib.TDstressFS_C(p(X), p(Y), p(Z), 3, p(P1), p(P2), p(P3), 1.0, 0.5, 0.0, mu, lam, hs, p(s), p(e))
        out["main_%s_stress" % ("hs" if hs else "fs")] = s.reshape(3, 6)
        out["main_%s_strain" % ("hs" if hs else "fs")] = e.reshape(3, 6)
    out["main_X"], out["main_Y"], out["main_Z"] = X, Y, Z
    out["main_P"] = np.stack([P1, P2, P3])
    # (2) random triangles and receivers, with special points
    rng = np.random.default_rng(1234)
    tris, recs = [], []
    for t in range(12):
        c = np.array([rng.uniform(-5e3, 5e3), rng.uniform(-5e3, 5e3), rng.uniform(-20e3, -8e3)])
        P = c + rng.normal(size=(3, 3)) * 1500.0
        if t == 11:   # vertical triangle
            P[:, 1] = c[1]
        R = c + rng.normal(size=(160, 3)) * 4000.0
        Rz = R.copy()
        # special receivers: vertices, edge midpoints, centroid, on-plane outside points
        cen = P.mean(axis=0)
        mids = [(P[0] + P[1]) / 2, (P[1] + P[2]) / 2, (P[2] + P[0]) / 2]
        extra = [P[0], P[1], P[2], cen] + mids + [cen + 2.5 * (P[0] - cen), cen + 2.5 * (mids[1] - cen),
                                                   2 * P[1] - P[0], cen + 1e-3 * np.cross(P[1] - P[0], P[2] - P[0])]
        R = np.concatenate([Rz, np.array(extra)])
        tris.append(P)
        recs.append(R)
    tris = np.array(tris)
    recs = np.array(recs)
    out["rand_P"], out["rand_R"] = tris, recs
    for Ss, Ds, tag in ((1.0, 0.0, "ss"), (0.0, 1.0, "ds"), (0.7, -0.4, "mix")):
        S = np.zeros(recs.shape[:2] + (6,))
        E = np.zeros_like(S)
        SH_S = np.zeros_like(S)
        for t in range(len(tris)):
            R = np.ascontiguousarray(recs[t])
            n = len(R)
            s, e = np.zeros(6 * n), np.zeros(6 * n)
            x, y, z = (np.ascontiguousarray(R[:, k]) for k in range(3))
            lib.TDstressFS_C(p(x), p(y), p(z), n, p(tris[t, 0].copy()), p(tris[t, 1].copy()), p(tris[t, 2].copy()),
                             Ss, Ds, 0.0, mu, lam, False, p(s), p(e))
            S[t], E[t] = s.reshape(n, 6), e.reshape(n, 6)
            st, _ = SH.TDstressFS(x.copy(), y.copy(), z.copy(), tris[t, 0].copy(), tris[t, 1].copy(),
                                  tris[t, 2].copy(), Ss, Ds, 0.0, mu, lam)
            SH_S[t] = np.asarray(st).T
        out["rand_%s_stress" % tag], out["rand_%s_strain" % tag], out["rand_%s_numpy" % tag] = S, E, SH_S
    # (3) one receiver, many sources (TDstressEachSourceAtReceiver_C)
    r = recs[0, 5]
    n = len(tris)
    P1f, P2f, P3f = (np.ascontiguousarray(tris[:, k].ravel()) for k in range(3))
    s, e = np.zeros(6 * n), np.zeros(6 * n)
    lib.TDstressEachSourceAtReceiver_C(r[0], r[1], r[2], p(P1f), p(P2f), p(P3f), n, 1.0, 0.0, 0.0, mu, lam, False,
                                       p(s), p(e))
    out["each_R"], out["each_stress"], out["each_strain"] = r, s.reshape(n, 6), e.reshape(n, 6)
    out["mu"], out["lam"] = mu, lam
    return out


def tiny_case(workdir, QDsim_mod, readmsh, Hmatrix):
    sys.path.insert(0, REPO)
    from pyquake3d_b200 import meshgen
    msh, para = meshgen.make_case("tiny", os.path.join(workdir, "tiny"), n_target=600)
    nodes, tris = readmsh.read_mshV2(msh)
    sim = QDsim_mod.QDsim(tris, nodes, para)
    out = {"nodes": nodes, "tris": tris, "eleVec": sim.eleVec, "xg": sim.xg}
    for k in ("Tno", "Tt1o", "Tt2o", "state", "slipv1", "slipv2", "slipv", "a", "b", "dc", "f0", "rake",
              "shear_loading", "normal_loading", "slipvC", "Tt", "fric"):
        out["init_" + k] = np.array(getattr(sim, k), dtype=np.float64)
    tb = sim.tree_block
    tb.blocks_to_process = []
    tb.collect_blocks(tb.root_block)
    blocks = tb.blocks_to_process
    rc = [np.asarray(b.row_cluster) for b in blocks]
    cc = [np.asarray(b.col_cluster) for b in blocks]
    out["blk_m"] = np.array([len(r) for r in rc])
    out["blk_n"] = np.array([len(c) for c in cc])
    out["blk_rows"] = np.concatenate(rc)
    out["blk_cols"] = np.concatenate(cc)
    SEED = 7
    np.random.seed(SEED)
    for b in blocks:
        tb.ACA_worker(b)
    out["aca_seed"] = SEED
    out["blk_aca"] = np.array([bool(b.judaca) for b in blocks])
    ks, kd, fac = [], [], {}
    na = 0
    for i, b in enumerate(blocks):
        if b.judaca:
            ks.append(b.ACA_dictS["U_ACA_A1s"].shape[1])
            kd.append(b.ACA_dictD["U_ACA_A1d"].shape[1])
            if na < 3:
                for key in ("U_ACA_A1s", "V_ACA_A1s", "U_ACA_A2s", "V_ACA_A2s", "U_ACA_Bs", "V_ACA_Bs"):
                    fac["f%d_%s" % (i, key)] = np.asarray(b.ACA_dictS[key], dtype=np.float64)
                for key in ("U_ACA_A1d", "V_ACA_A1d", "U_ACA_A2d", "V_ACA_A2d", "U_ACA_Bd", "V_ACA_Bd"):
                    fac["f%d_%s" % (i, key)] = np.asarray(b.ACA_dictD[key], dtype=np.float64)
                na += 1
    out["aca_kS"], out["aca_kD"] = np.array(ks), np.array(kd)
    out.update(fac)
    # operator products on fixed vectors
    rng = np.random.default_rng(99)
    X = rng.standard_normal((2, len(sim.xg))) * 1e-9
    out["mvm_x"] = X
    for op in ("A1s", "A2s", "Bs", "A1d", "A2d", "Bd"):
        x = X[0] if op.endswith("s") else X[1]
        out["mvm_" + op] = tb.blocks_process_MVM(x, blocks, op)
    # time stepping
    sim.local_blocks = blocks
    hs, dts, ts = [], [], []
    dttry = sim.htry
    snaps = {}
    for i in range(30):
        h, dtnext = sim.simu_forward(dttry)
        hs.append(h)
        dts.append(dtnext)
        ts.append(sim.time)
        dttry = dtnext
        if i in (0, 29):
            for k in ("Tno", "Tt1o", "Tt2o", "state", "slipv1", "slipv2", "slipv", "slip1", "slip2", "slip", "rake"):
                snaps["step%d_%s" % (i + 1, k)] = np.array(getattr(sim, k), dtype=np.float64)
    out["steps_h"], out["steps_dtnext"], out["steps_time"] = np.array(hs), np.array(dts), np.array(ts)
    out.update(snaps)
    with open(para) as f:
        out["parameter_txt"] = np.array(f.read())
    with open(os.path.join(os.path.dirname(para), "tinyparam.dat")) as f:
        out["param_dat"] = np.array(f.read())
    with open(msh) as f:
        out["msh"] = np.array(f.read())
    return out


def hs_cases(lib, SH):
    """Half-space fixtures (see the module docstring)."""
    import ctypes
    D = ctypes.POINTER(ctypes.c_double)
    lib.TDstressFS_C.argtypes = [D, D, D, ctypes.c_size_t, D, D, D] + [ctypes.c_double] * 5 + [ctypes.c_bool, D, D]
    lib.TDstressEachSourceAtReceiver_C.argtypes = [ctypes.c_double] * 3 + [D, D, D, ctypes.c_size_t] + \
        [ctypes.c_double] * 5 + [ctypes.c_bool, D, D]
    p = lambda a: a.ctypes.data_as(D)
    mu = lam = 32038120320.0
    rng = np.random.default_rng(2024)
    tris, kinds = [], []
    for t in range(8):                          # at depth
        c = np.array([rng.uniform(-5e3, 5e3), rng.uniform(-5e3, 5e3), rng.uniform(-15e3, -3e3)])
        tris.append(c + rng.normal(size=(3, 3)) * 1500.0)
        kinds.append("deep")
    for k, nz in enumerate((1, 2, 2)):          # one or two vertices on the free surface z = 0
        c = np.array([rng.uniform(-3e3, 3e3), rng.uniform(-3e3, 3e3), -2e3])
        P = c + rng.normal(size=(3, 3)) * 1500.0
        P[:, 2] = -np.abs(P[:, 2])
        P[:nz, 2] = 0.0
        tris.append(P)
        kinds.append("surface%d_%d" % (nz, k))
    # a side along z (P1 -> P2 vertical) and a vertical triangle without vertical sides
    tris.append(np.array([[1000.0, 500.0, -3000.0], [1000.0, 500.0, -6000.0], [3500.0, 1500.0, -4500.0]]))
    kinds.append("vertical_side")
    tris.append(np.array([[-2000.0, 1000.0, -2500.0], [2500.0, 1000.0, -4000.0], [300.0, 1000.0, -7000.0]]))
    kinds.append("vertical")
    # the vertical side as the second and third side of the triangle
    base = tris[-2]
    tris.append(base[[2, 0, 1]].copy())
    kinds.append("vertical_side2")
    tris.append(base[[1, 2, 0]].copy())
    kinds.append("vertical_side3")
    tris = np.array(tris)
    recs = []
    for P in tris:
        c = P.mean(axis=0)
        R = c + rng.normal(size=(80, 3)) * 4000.0
        R[:, 2] = -np.abs(R[:, 2])
        R[:10, 2] = -rng.uniform(0.5, 20.0, 10)       # near the surface
        R[10:16, 2] = 0.0                                # on the surface
        recs.append(R)
    recs = np.array(recs)
    out = {"hs_P": tris, "hs_R": recs, "hs_kind": np.array(kinds), "mu": mu, "lam": lam}
    for Ss, Ds, Ts, tag in ((1.0, 0.0, 0.0, "ss"), (0.0, 1.0, 0.0, "ds"), (0.7, -0.4, 0.25, "mix")):
        S = np.zeros(recs.shape[:2] + (6,))
        E = np.zeros_like(S)
        N = np.full_like(S, np.nan)
        for t in range(len(tris)):
            R = np.ascontiguousarray(recs[t])
            n = len(R)
            s, e = np.zeros(6 * n), np.zeros(6 * n)
            x, y, z = (np.ascontiguousarray(R[:, k]) for k in range(3))
            lib.TDstressFS_C(p(x), p(y), p(z), n, p(tris[t, 0].copy()), p(tris[t, 1].copy()), p(tris[t, 2].copy()),
                             Ss, Ds, Ts, mu, lam, True, p(s), p(e))
            S[t], E[t] = s.reshape(n, 6), e.reshape(n, 6)
            st, _ = SH.TDstressHS(x.copy(), y.copy(), z.copy(), tris[t, 0].copy(), tris[t, 1].copy(),
                                  tris[t, 2].copy(), Ss, Ds, Ts, mu, lam)
            N[t] = np.asarray(st).T
        out["hs_%s_stress" % tag], out["hs_%s_strain" % tag], out["hs_%s_numpy" % tag] = S, E, N
    # one receiver, all sources
    r = np.array([400.0, -300.0, -2500.0])
    P1f, P2f, P3f = (np.ascontiguousarray(tris[:, k].ravel()) for k in range(3))
    n = len(tris)
    s, e = np.zeros(6 * n), np.zeros(6 * n)
    lib.TDstressEachSourceAtReceiver_C(r[0], r[1], r[2], p(P1f), p(P2f), p(P3f), n, 0.0, 1.0, 0.0, mu, lam, True,
                                       p(s), p(e))
    out["hs_each_R"], out["hs_each_stress"], out["hs_each_strain"] = r, s.reshape(n, 6), e.reshape(n, 6)
    return out


OUTPUT_FIELDS = ("Tno", "Tt", "Tt1o", "Tt2o", "rake", "state", "slipv", "slipv1", "slipv2", "a", "b", "dc", "fric",
                 "slip", "slip1", "slip2", "slipvC")


def output_fields(nodes, tris, xg, seed=11):
    """Seeded state of the tiny mesh spanning the magnitudes a run produces."""
    rng = np.random.default_rng(seed)
    n = len(tris)
    f = dict(nodelst=np.asarray(nodes, dtype=np.float64), elelst=np.asarray(tris), xg=np.asarray(xg, dtype=np.float64))
    f["Tno"] = rng.uniform(20, 80, n)
    f["Tt1o"] = rng.normal(0, 20, n)
    f["Tt2o"] = rng.normal(0, 20, n)
    f["Tt"] = np.sqrt(f["Tt1o"] ** 2 + f["Tt2o"] ** 2)
    f["rake"] = np.arctan2(f["Tt2o"], f["Tt1o"])
    f["state"] = rng.uniform(0.5, 0.9, n)
    f["slipv1"] = 10.0 ** rng.uniform(-14, 0.5, n) * rng.choice([-1, 1], n)
    f["slipv2"] = 10.0 ** rng.uniform(-14, 0.5, n) * rng.choice([-1, 1], n)
    f["slipv"] = np.sqrt(f["slipv1"] ** 2 + f["slipv2"] ** 2)
    f["a"] = rng.uniform(0.005, 0.025, n)
    f["b"] = rng.uniform(0.01, 0.02, n)
    f["dc"] = rng.uniform(0.005, 0.05, n)
    f["fric"] = f["Tt"] / f["Tno"]
    f["slip1"] = rng.normal(0, 3, n)
    f["slip2"] = rng.normal(0, 3, n)
    f["slip"] = np.sqrt(f["slip1"] ** 2 + f["slip2"] ** 2)
    f["slipvC"] = np.full(n, 1e-9) * rng.uniform(0.5, 1.5, n)
    f["maxsize"] = 0.9
    return f


def output_case(work, QDsim_mod):
    import hashlib
    import types as _types
    t = np.load(os.path.join(HERE, "tiny_case.npz"))
    f = output_fields(t["nodes"], t["tris"], t["xg"])
    obj = _types.SimpleNamespace(**f)
    out = {k: v for k, v in f.items() if k in OUTPUT_FIELDS}
    d = os.path.join(work, "outcase")
    os.makedirs(d)
    cwd = os.getcwd()
    os.chdir(d)
    try:
        QDsim_mod.QDsim.ouputVTK(obj, "ref.vtk")
        QDsim_mod.QDsim.outputtxt(obj, "step5")
        files = ["ref.vtk"] + ["out_txt/" + x for x in sorted(os.listdir("out_txt"))]
        for fn in files:
            with open(fn, "rb") as fh:
                out["sha256:" + fn] = np.array(hashlib.sha256(fh.read()).hexdigest())
    finally:
        os.chdir(cwd)
    out["output_seed"] = 11
    out["maxsize"] = np.array(f["maxsize"])
    return out


def tiny_hs_case(work, QDsim_mod, readmsh):
    """The tiny fault (its top edge on the free surface) with `Half space: True`:
    the reference's six operator products on fixed vectors and 30 simu_forward
    steps (same seeded ACA starts as tiny_case)."""
    t = np.load(os.path.join(HERE, "tiny_case.npz"))
    d = os.path.join(work, "tiny_hs")
    os.makedirs(d)
    with open(os.path.join(d, "tiny.msh"), "w") as f:
        f.write(str(t["msh"]))
    with open(os.path.join(d, "tinyparam.dat"), "w") as f:
        f.write(str(t["param_dat"]))
    para_txt = str(t["parameter_txt"]).replace("Half space: False", "Half space: True")
    assert "Half space: True" in para_txt
    with open(os.path.join(d, "parameter.txt"), "w") as f:
        f.write(para_txt)
    nodes, tris = readmsh.read_mshV2(os.path.join(d, "tiny.msh"))
    sim = QDsim_mod.QDsim(tris, nodes, os.path.join(d, "parameter.txt"))
    assert sim.tree_block.halfspace_jud
    tb = sim.tree_block
    tb.blocks_to_process = []
    tb.collect_blocks(tb.root_block)
    blocks = tb.blocks_to_process
    np.random.seed(int(t["aca_seed"]))
    for b in blocks:
        tb.ACA_worker(b)
    out = {"parameter_txt": np.array(para_txt), "aca_seed": t["aca_seed"]}
    ks = [b.ACA_dictS["U_ACA_A1s"].shape[1] for b in blocks if b.judaca]
    kd = [b.ACA_dictD["U_ACA_A1d"].shape[1] for b in blocks if b.judaca]
    out["aca_kS"], out["aca_kD"] = np.array(ks), np.array(kd)
    X = t["mvm_x"]
    out["mvm_x"] = X
    for op in ("A1s", "A2s", "Bs", "A1d", "A2d", "Bd"):
        x = X[0] if op.endswith("s") else X[1]
        out["mvm_" + op] = tb.blocks_process_MVM(x, blocks, op)
    sim.local_blocks = blocks
    hs, ts = [], []
    dttry = sim.htry
    for i in range(30):
        h, dtnext = sim.simu_forward(dttry)
        hs.append(h)
        ts.append(sim.time)
        dttry = dtnext
    out["steps_h"], out["steps_time"] = np.array(hs), np.array(ts)
    for k in ("Tno", "Tt1o", "state", "slip1", "slip"):
        out["step30_" + k] = np.array(getattr(sim, k), dtype=np.float64)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("PQ3D_REFERENCE") or
                    os.path.abspath(os.path.join(REPO, os.pardir, "reference")))
    ap.add_argument("--only", default=None, help="regenerate one fixture: gf | tiny | hs | tiny_hs | output")
    args = ap.parse_args()
    ref_src = os.path.join(args.ref, "src")
    subprocess.run(["make", "-C", os.path.join(REPO, "oracle"), "ref", "REFSRC=" + os.path.join(ref_src, "TDstressFS_C.cpp")],
                   check=True)
    work = tempfile.mkdtemp(prefix="pq3d_golden_")
    os.makedirs(os.path.join(work, "src"))
    shutil.copy(os.path.join(REPO, "oracle", "_ref", "TDstressFS_C.so"), os.path.join(work, "src", "TDstressFS_C.so"))
    install_stubs()
    sys.path.insert(0, ref_src)
    cwd = os.getcwd()
    os.chdir(work)
    try:
        import ctypes
        import SH_greenfunction
        import readmsh
        import Hmatrix
        import QDsim
        lib = ctypes.CDLL(os.path.join(work, "src", "TDstressFS_C.so"))
        if args.only in (None, "gf"):
            g = gf_cases(lib, SH_greenfunction)
            np.savez_compressed(os.path.join(HERE, "gf_cases.npz"), **g)
        if args.only in (None, "tiny"):
            t = tiny_case(work, QDsim, readmsh, Hmatrix)
            np.savez_compressed(os.path.join(HERE, "tiny_case.npz"), **t)
        if args.only in (None, "hs"):
            h = hs_cases(lib, SH_greenfunction)
            np.savez_compressed(os.path.join(HERE, "hs_cases.npz"), **h)
        if args.only in (None, "tiny_hs"):
            th = tiny_hs_case(work, QDsim, readmsh)
            np.savez_compressed(os.path.join(HERE, "tiny_hs_case.npz"), **th)
        if args.only in (None, "output"):
            o = output_case(work, QDsim)
            np.savez_compressed(os.path.join(HERE, "output_case.npz"), **o)
    finally:
        os.chdir(cwd)
        shutil.rmtree(work, ignore_errors=True)
    for f in ("gf_cases.npz", "tiny_case.npz", "hs_cases.npz", "tiny_hs_case.npz", "output_case.npz"):
        print(f, os.path.getsize(os.path.join(HERE, f)), "bytes")


if __name__ == "__main__":
    main()
