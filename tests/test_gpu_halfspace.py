"""GPU: half-space Green's function and the half-space operator.

* the drop-ins with jud_halfspace=True against the reference's compiled library
  (tests/golden/hs_cases.npz: triangles at depth, touching the free surface,
  with a side along z in each position, vertical; receivers at depth, within
  20 m of the surface and on it) and against the reference's own main() inputs;
* hs_mode 1 against the reference's numpy TDstressHS;
* half-space traction pairs on the tiny fault (top edge on the free surface)
  against the oracle's restatement;
* QDsim with `Half space: True`: operator products and the 30-step dt sequence
  of the reference's own run (tests/golden/tiny_hs_case.npz), also with the
  rows split over two emulated ranks; a half-space ensemble against its faults
  run alone.
Tolerances: Green's-function values 1e-9 of each receiver's largest component;
operator products 1e-6 of their maximum (ACA+ magnifies ~1e-11 entry
differences through small pivots; ranks are identical); steps 1e-8."""
import ctypes
import os

import numpy as np
import pytest

import qd_oracle
from conftest import GOLDEN
from pyquake3d_b200 import _lib

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

D = ctypes.POINTER(ctypes.c_double)


def _p(a):
    return a.ctypes.data_as(D)


@pytest.fixture(scope="module")
def lib():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return _lib.load()


@pytest.fixture(scope="module")
def hs():
    return dict(np.load(os.path.join(GOLDEN, "hs_cases.npz")))


def _close(got, ref, tol=1e-9):
    scale = np.abs(ref).max(axis=-1, keepdims=True)
    return (np.abs(got - ref) <= tol * scale).all()


@pytest.mark.parametrize("tag,b", [("ss", (1.0, 0.0, 0.0)), ("ds", (0.0, 1.0, 0.0)), ("mix", (0.7, -0.4, 0.25))])
def test_dropin_halfspace_matches_reference_library(lib, hs, tag, b):
    mu, lam = float(hs["mu"]), float(hs["lam"])
    for t in range(len(hs["hs_P"])):
        R, P = np.ascontiguousarray(hs["hs_R"][t]), hs["hs_P"][t]
        n = len(R)
        x, y, z = (np.ascontiguousarray(R[:, k]) for k in range(3))
        s, e = np.zeros(6 * n), np.zeros(6 * n)
        lib.TDstressFS_C(_p(x), _p(y), _p(z), n, _p(P[0].copy()), _p(P[1].copy()), _p(P[2].copy()), *b, mu, lam,
                         True, _p(s), _p(e))
        assert _close(s.reshape(n, 6), hs["hs_%s_stress" % tag][t]), (t, hs["hs_kind"][t])
        assert _close(e.reshape(n, 6), hs["hs_%s_strain" % tag][t]), (t, hs["hs_kind"][t])


def test_dropin_halfspace_main_inputs_and_each_source(lib, hs, gf_golden):
    g = gf_golden
    P = g["main_P"]
    s, e = np.zeros(18), np.zeros(18)
    X, Y, Z = (np.ascontiguousarray(g[k]) for k in ("main_X", "main_Y", "main_Z"))
    lib.TDstressFS_C(_p(X), _p(Y), _p(Z), 3, _p(P[0].copy()), _p(P[1].copy()), _p(P[2].copy()), 1.0, 0.5, 0.0,
                     float(g["mu"]), float(g["lam"]), True, _p(s), _p(e))
    assert _close(s.reshape(3, 6), g["main_hs_stress"]) and _close(e.reshape(3, 6), g["main_hs_strain"])
    r = hs["hs_each_R"]
    n = len(hs["hs_P"])
    P1f, P2f, P3f = (np.ascontiguousarray(hs["hs_P"][:, k].ravel()) for k in range(3))
    s, e = np.zeros(6 * n), np.zeros(6 * n)
    lib.TDstressEachSourceAtReceiver_C(r[0], r[1], r[2], _p(P1f), _p(P2f), _p(P3f), n, 0.0, 1.0, 0.0,
                                       float(hs["mu"]), float(hs["lam"]), True, _p(s), _p(e))
    assert _close(s.reshape(n, 6), hs["hs_each_stress"])


@pytest.mark.parametrize("tag,b", [("ss", (1.0, 0.0, 0.0)), ("ds", (0.0, 1.0, 0.0))])
def test_exact_mode_matches_reference_numpy(lib, hs, tag, b):
    mu, lam = float(hs["mu"]), float(hs["lam"])
    for t in range(len(hs["hs_P"])):
        R, P = hs["hs_R"][t], hs["hs_P"][t]
        n = len(R)
        dR = torch.tensor(np.ascontiguousarray(R.T), dtype=torch.float64, device="cuda")
        dP = torch.tensor(P.reshape(1, 9), dtype=torch.float64, device="cuda")
        out = torch.zeros(12 * n, dtype=torch.float64, device="cuda")
        _lib.check(lib.pq3d_stress_points(dR[0].data_ptr(), dR[1].data_ptr(), dR[2].data_ptr(), n, dP.data_ptr(), 1,
                                          b[0], b[1], b[2], mu, lam, 1, out.data_ptr(), out[6 * n:].data_ptr(),
                                          _lib.stream_ptr()), "stress_points")
        s = out[:6 * n].cpu().numpy().reshape(n, 6)
        assert _close(s, hs["hs_%s_numpy" % tag][t]), (t, hs["hs_kind"][t])


def test_halfspace_traction_pairs_match_oracle(lib, tiny_sim):
    s = tiny_sim
    n = s.xg.shape[0]
    cols = np.arange(0, n, 12)
    rows = np.arange(n)
    R, C = np.meshgrid(rows, cols, indexing="ij")
    dev = dict(device="cuda")
    xg = torch.tensor(s.xg, dtype=torch.float64, **dev)
    ev = torch.tensor(s.eleVec, dtype=torch.float64, **dev)
    nodes = torch.tensor(s.nodelst, dtype=torch.float64, **dev)
    tri = torch.tensor(np.asarray(s.elelst, dtype=np.int64), **dev)
    rec = torch.empty((n * lib.pq3d_src_record_bytes() + 7) // 8, dtype=torch.float64, **dev)
    hsr = torch.empty((n * lib.pq3d_hs_record_bytes() + 7) // 8, dtype=torch.float64, **dev)
    st = _lib.stream_ptr()
    _lib.check(lib.pq3d_src_records(nodes.data_ptr(), tri.data_ptr(), n, rec.data_ptr(), st), "rec")
    _lib.check(lib.pq3d_hs_records(nodes.data_ptr(), tri.data_ptr(), n, hsr.data_ptr(), st), "hs")
    r_t = torch.tensor(R.ravel(), **dev)
    c_t = torch.tensor(C.ravel(), **dev)
    out = torch.zeros(6 * R.size, dtype=torch.float64, **dev)
    _lib.check(lib.pq3d_traction_pairs(xg.data_ptr(), ev.data_ptr(), rec.data_ptr(), r_t.data_ptr(), c_t.data_ptr(),
                                       R.size, s.mu, s.lambda_, out.data_ptr(), hsr.data_ptr(), 2, st), "pairs")
    got = out.cpu().numpy().reshape(n, len(cols), 6)
    geo = qd_oracle.Geometry(s.xg, s.eleVec, s.nodelst, s.elelst, s.mu, s.lambda_, hs_mode=2)
    ref = geo.gf_block(rows, cols, 3)            # 6 x m x n: A1s A2s Bs A1d A2d Bd
    for k in range(6):
        scale = np.abs(ref[k]).max()
        assert np.abs(got[:, :, k] - ref[k]).max() <= 1e-10 * scale, k


@pytest.fixture(scope="module")
def tiny_hs_files(tmp_path_factory, tiny_golden):
    g = dict(np.load(os.path.join(GOLDEN, "tiny_hs_case.npz")))
    d = tmp_path_factory.mktemp("tiny_hs")
    (d / "tiny.msh").write_text(str(tiny_golden["msh"]))
    (d / "tinyparam.dat").write_text(str(tiny_golden["param_dat"]))
    (d / "parameter.txt").write_text(str(g["parameter_txt"]))
    return str(d / "tiny.msh"), str(d / "parameter.txt"), g


def test_halfspace_simulation_follows_reference(lib, tiny_hs_files):
    from pyquake3d_b200 import QDsim, read_mshV2
    msh, para, g = tiny_hs_files
    nodes, tris = read_mshV2(msh)
    sim = QDsim(tris, nodes, para)
    assert sim.halfspace_jud
    sim.Para0["ACA seed"] = str(int(g["aca_seed"]))
    op = sim.tree_block.op()
    kS, kD = op.ranks()
    assert np.array_equal(kS, g["aca_kS"]) and np.array_equal(kD, g["aca_kD"])
    X = g["mvm_x"]
    y = op.apply(X[0], np.zeros_like(X[0]), "fp64")
    yd = op.apply(np.zeros_like(X[1]), X[1], "fp64")
    for k, name in enumerate(("A1", "A2", "B")):
        for got, sfx in ((y[k], "s"), (yd[k], "d")):
            ref = g["mvm_%s%s" % (name, sfx)]
            assert np.abs(got - ref).max() <= 1e-6 * np.abs(ref).max(), name + sfx
    dttry = sim.htry
    hs = []
    for _ in range(30):
        h, dttry = sim.simu_forward(dttry)
        hs.append(h)
    np.testing.assert_allclose(hs, g["steps_h"], rtol=1e-8)
    sim.sync_to_host()
    for k in ("Tno", "Tt1o", "state", "slip1", "slip"):
        ref = g["step30_" + k]
        assert np.abs(getattr(sim, k) - ref).max() <= 1e-7 * np.abs(ref).max(), k


def test_halfspace_ensemble_follows_single_fault_runs(lib, tmp_path):
    """Faults reaching the free surface, `Half space: True`, stepped together follow the
    same faults run alone (FP64 operators)."""
    from pyquake3d_b200 import QDsim, read_mshV2
    from pyquake3d_b200.ensemble import Ensemble
    from pyquake3d_b200.meshgen import ensemble_faults
    files = ensemble_faults(str(tmp_path), n_faults=2, seed=7, lo=300, hi=700, edge=1.0)
    for _, para in files:
        txt = open(para).read().replace("Half space: False", "Half space: True")
        open(para, "w").write(txt)

    def sims():
        out = []
        for msh, para in files:
            nodes, tris = read_mshV2(msh)
            out.append(QDsim(tris, nodes, para, precision="fp64"))
        return out
    E = Ensemble(sims(), precision="fp64")
    assert E.op.halfspace == 2
    hist = E.run(15, [s.htry for s in E.sims])
    for f, s in enumerate(sims()):
        h1 = s._ensure_device().run(15, s.htry)
        np.testing.assert_allclose(hist[:, f, 0], h1[:, 0], rtol=1e-9)


def test_halfspace_two_ranks_follow_reference(lib, tiny_hs_files):
    from pyquake3d_b200 import QDsim, read_mshV2
    from pyquake3d_b200.partition import DeviceRowBackend, PartitionedStepper, TorchComm, row_partition
    msh, para, g = tiny_hs_files
    nodes, tris = read_mshV2(msh)
    sim = QDsim(tris, nodes, para)
    sim.Para0["ACA seed"] = str(int(g["aca_seed"]))
    st = sim.tree_block.struct
    b = row_partition(st, 2)
    ps = PartitionedStepper([DeviceRowBackend(sim, st, b[r], b[r + 1], precision="fp64") for r in range(2)],
                            TorchComm(use_dist=False), sim.RelTol)
    dttry = sim.htry
    hs = []
    for _ in range(30):
        h, dttry = ps.step(dttry)
        hs.append(h)
    np.testing.assert_allclose(hs, g["steps_h"], rtol=1e-8)
