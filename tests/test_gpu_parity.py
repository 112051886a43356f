"""GPU parity: libpq3d.so kernels against the oracle and the reference's golden outputs.

Tolerances (FP64 paths): Green's function entries 1e-10 of the per-receiver
maximum; operator products 1e-10 (plain FP64) of max|y|; the FP64 stepper
follows the reference's adaptive step sequence to 1e-8 relative.
Mixed precision: FP32 operator 1e-5 and BF16 low-rank 3e-3 of max|y|."""
import ctypes

import numpy as np
import pytest

import qd_oracle
from pyquake3d_b200 import _lib
from pyquake3d_b200.hmatrix import DeviceHMatrix, aca_start_indices

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

D = ctypes.POINTER(ctypes.c_double)
SINGULAR = np.r_[160:163, 164:167]   # vertices and edge midpoints of the golden receivers


def _p(a):
    return a.ctypes.data_as(D)


@pytest.fixture(scope="module")
def lib():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return _lib.load()


def test_dropin_TDstressFS_C_matches_reference(lib, gf_golden):
    g = gf_golden
    regular = np.setdiff1d(np.arange(g["rand_R"].shape[1]), SINGULAR)
    for tag, (Ss, Ds) in (("ss", (1.0, 0.0)), ("ds", (0.0, 1.0)), ("mix", (0.7, -0.4))):
        for t in range(len(g["rand_P"])):
            R, P = g["rand_R"][t], g["rand_P"][t]
            n = len(R)
            s, e = np.zeros(6 * n), np.zeros(6 * n)
            x, y, z = (np.ascontiguousarray(R[:, k]) for k in range(3))
            lib.TDstressFS_C(_p(x), _p(y), _p(z), n, _p(P[0].copy()), _p(P[1].copy()), _p(P[2].copy()), Ss, Ds, 0.0,
                             float(g["mu"]), float(g["lam"]), False, _p(s), _p(e))
            s = s.reshape(n, 6)
            ref = g["rand_%s_stress" % tag][t]
            sc = np.abs(ref[regular]).max(axis=1, keepdims=True)
            assert (np.abs(s[regular] - ref[regular]) <= 1e-10 * sc).all(), (tag, t)
            zero = np.all(ref[regular] == 0.0, axis=1)
            assert (s[regular][zero] == 0.0).all()   # zero-strain configuration away from singular points


def test_dropin_each_source_matches_reference(lib, gf_golden):
    g = gf_golden
    P = g["rand_P"]
    n = len(P)
    P1f, P2f, P3f = (np.ascontiguousarray(P[:, k].ravel()) for k in range(3))
    s, e = np.zeros(6 * n), np.zeros(6 * n)
    r = g["each_R"]
    lib.TDstressEachSourceAtReceiver_C(r[0], r[1], r[2], _p(P1f), _p(P2f), _p(P3f), n, 1.0, 0.0, 0.0, float(g["mu"]),
                                       float(g["lam"]), False, _p(s), _p(e))
    ref = g["each_stress"]
    assert (np.abs(s.reshape(n, 6) - ref) <= 1e-10 * np.abs(ref).max(axis=1, keepdims=True)).all()


def test_main_inputs(lib, gf_golden):
    g = gf_golden
    P = g["main_P"]
    s, e = np.zeros(18), np.zeros(18)
    X, Y, Z = (np.ascontiguousarray(g[k]) for k in ("main_X", "main_Y", "main_Z"))
    lib.TDstressFS_C(_p(X), _p(Y), _p(Z), 3, _p(P[0].copy()), _p(P[1].copy()), _p(P[2].copy()), 1.0, 0.5, 0.0,
                     float(g["mu"]), float(g["lam"]), False, _p(s), _p(e))
    ref = g["main_fs_stress"]
    assert (np.abs(s.reshape(3, 6) - ref) <= 1e-10 * np.abs(ref).max(axis=1, keepdims=True)).all()


@pytest.fixture(scope="module")
def tiny_op(lib, tiny_sim, tiny_golden):
    s = tiny_sim
    op = DeviceHMatrix(s.tree_block.struct, s.xg, s.eleVec, s.nodelst, s.elelst, s.mu, s.lambda_, aca_tol=0.01,
                       aca_rel=False, aca_seed=int(tiny_golden["aca_seed"]))
    return op.assemble(("fp64", "fp32", "bf16"))


def test_traction_pairs_all_pairs(lib, tiny_sim):
    s = tiny_sim
    geo = qd_oracle.Geometry(s.xg, s.eleVec, s.nodelst, s.elelst, s.mu, s.lambda_)
    n = len(s.xg)
    rows = np.arange(n)
    ref = geo.gf_block(rows, rows, 3)            # 6 x n x n
    op_rows = torch.tensor(np.repeat(rows, n), device="cuda")
    op_cols = torch.tensor(np.tile(rows, n), device="cuda")
    dev = DeviceHMatrix.__new__(DeviceHMatrix)
    f64 = dict(dtype=torch.float64, device="cuda")
    xg, ev = torch.tensor(s.xg, **f64), torch.tensor(s.eleVec, **f64)
    nodes = torch.tensor(s.nodelst, **f64)
    tri = torch.tensor(s.elelst.astype(np.int64), device="cuda")
    rec = torch.empty(n * lib.pq3d_src_record_bytes() // 8, **f64)
    st = _lib.stream_ptr()
    _lib.check(lib.pq3d_src_records(nodes.data_ptr(), tri.data_ptr(), n, rec.data_ptr(), st), "records")
    out = torch.empty(n * n * 6, **f64)
    _lib.check(lib.pq3d_traction_pairs(xg.data_ptr(), ev.data_ptr(), rec.data_ptr(), op_rows.data_ptr(),
                                       op_cols.data_ptr(), n * n, s.mu, s.lambda_, out.data_ptr(), None, 0, st),
               "pairs")
    got = out.cpu().numpy().reshape(n, n, 6).transpose(2, 0, 1)
    del dev
    scale = np.abs(ref).max(axis=(0, 2))[None, :, None]
    assert np.abs(got - ref).max(axis=(0, 2)).max() >= 0
    assert (np.abs(got - ref) <= 1e-10 * scale).all()


def test_aca_ranks_and_pivots_match_oracle(tiny_op, tiny_golden):
    kS, kD = tiny_op.ranks()
    # same seeded starts and pivot rules as the reference: ranks agree block by block
    assert np.array_equal(kS, tiny_golden["aca_kS"])
    assert np.array_equal(kD, tiny_golden["aca_kD"])


@pytest.mark.parametrize("dtype,tol", [("fp64", 1e-10), ("fp32", 1e-5), ("bf16", 3e-3)])
def test_hmatvec_matches_reference_mvm(tiny_op, tiny_golden, dtype, tol):
    """Errors are measured against the operator scale (max over the six products):
    on this planar fault the normal-stress operators B are analytically zero and
    numerically rounding noise (~1e-15 of A1), so their own maximum is no scale."""
    g = tiny_golden
    X = g["mvm_x"]
    scale = max(np.abs(g["mvm_" + op]).max() for op in ("A1s", "A2s", "Bs", "A1d", "A2d", "Bd"))
    y1, y2, yB = tiny_op.apply(X[0], np.zeros_like(X[0]), dtype)
    for y, op in ((y1, "A1s"), (y2, "A2s"), (yB, "Bs")):
        ref = g["mvm_" + op]
        assert np.abs(y - ref).max() <= tol * scale, (dtype, op, np.abs(y - ref).max() / scale)
    y1, y2, yB = tiny_op.apply(np.zeros_like(X[1]), X[1], dtype)
    for y, op in ((y1, "A1d"), (y2, "A2d"), (yB, "Bd")):
        ref = g["mvm_" + op]
        assert np.abs(y - ref).max() <= tol * scale, (dtype, op, np.abs(y - ref).max() / scale)


def test_hmatvec_linearity_and_determinism(tiny_op):
    rng = np.random.default_rng(3)
    n = tiny_op.n
    a, b = rng.standard_normal((2, 2, n))
    ya = np.array(tiny_op.apply(a[0], a[1], "fp64"))
    yb = np.array(tiny_op.apply(b[0], b[1], "fp64"))
    yab = np.array(tiny_op.apply(a[0] + 2 * b[0], a[1] + 2 * b[1], "fp64"))
    assert np.abs(yab - (ya + 2 * yb)).max() <= 1e-12 * np.abs(yab).max()   # scale: all components
    again = np.array(tiny_op.apply(a[0], a[1], "fp64"))
    assert np.array_equal(ya, again)   # slot reduction: bitwise reproducible


def test_stepper_follows_reference_30_steps(lib, tiny_files, tiny_golden):
    from pyquake3d_b200 import QDsim, read_mshV2
    g = tiny_golden
    nodes, tris = read_mshV2(tiny_files[0])
    sim = QDsim(tris, nodes, tiny_files[1])
    sim.Para0["ACA seed"] = str(int(g["aca_seed"]))
    dttry = sim.htry
    hs = []
    for i in range(30):
        h, dtnext = sim.simu_forward(dttry)
        hs.append(h)
        dttry = dtnext
        if i == 0:
            sim.sync_to_host()
            for k in ("Tno", "Tt1o", "Tt2o", "state", "slip1"):
                ref = g["step1_" + k]
                assert np.abs(getattr(sim, k) - ref).max() <= 1e-9 * np.abs(ref).max(), k
    np.testing.assert_allclose(hs, g["steps_h"], rtol=1e-8)
    sim.sync_to_host()
    for k in ("Tno", "Tt1o", "state", "slip1", "slip"):
        ref = g["step30_" + k]
        assert np.abs(getattr(sim, k) - ref).max() <= 1e-7 * np.abs(ref).max(), k
