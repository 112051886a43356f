"""GPU: the benchmark workloads at full size, through size-independent properties.

The oracle cannot assemble or step 20k-60k elements in seconds, so at these
sizes the product is checked by properties that hold at any size:

* sampled rows of the H-matvec against exact rows of the operator computed with
  the Green's-function pairs kernel (pinned to the reference's library on the
  golden vectors): the hierarchical approximation stays within a small multiple
  of the ACA tolerance;
* linearity and bitwise determinism of the matvec in every storage precision;
* stepping: a CUDA graph of steps and the same steps launched eagerly are
  bitwise equal, and the FP32 operator's trajectory stays within the 1e-5 slip
  target of the FP64 one on the FP64 step sizes;
* the row-partitioned step (two ranks emulated in one process) follows the
  fused single-GPU step at the 20k thrust workload;
* plain2k (one dense FP64 block) is small enough for the oracle itself: its
  operator rows and 50 adaptive steps against the oracle on the same operator;
* curved60k and thrust20k: the device-assembled FP64 operator copied to the
  host drives the oracle's simu_forward for 12 adaptive steps beside the device
  FP64 stepper (h and state pinned to the oracle) and the FP32-operator stepper
  on the oracle's step sizes (slip, V and theta within the 1e-5 target);
* curved120k in V-mode: the MLP-seeded and the undamped-start runs agree.

Workloads: plain2k (1,936 triangles, vertical strike-slip), thrust20k (20,480
triangles, 30-degree thrust), curved60k (59,696 triangles, rough strike-slip
fault with a branch) and curved120k (the same geometry refined, heterogeneous
a-b and normal stress), generated by pyquake3d_b200.meshgen with fixed seeds."""
import numpy as np
import pytest

from pyquake3d_b200 import _lib

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return _lib.load()


def _case(name, tmp_path_factory, precision):
    from pyquake3d_b200 import QDsim, meshgen, read_mshV2
    msh, para = meshgen.make_case(name, str(tmp_path_factory.mktemp(name)))
    nodes, tris = read_mshV2(msh)
    return QDsim(tris, nodes, para, precision=precision)


@pytest.fixture(scope="module")
def c60(lib, tmp_path_factory):
    sim = _case("curved60k", tmp_path_factory, "fp32")
    sim.tree_block.want = ("fp64", "fp32", "bf16", "mixed")
    return sim, sim.tree_block.op()


def _exact_rows(lib, sim, rows):
    """The six operator planes (A1s, A2s, Bs, A1d, A2d, Bd) of receivers `rows`
    against every source, from the Green's-function pairs kernel: 6 x m x n."""
    n = len(sim.xg)
    f64 = dict(dtype=torch.float64, device="cuda")
    xg, ev = torch.tensor(sim.xg, **f64), torch.tensor(sim.eleVec, **f64)
    nodes = torch.tensor(sim.nodelst, **f64)
    tri = torch.tensor(sim.elelst.astype(np.int64), device="cuda")
    rec = torch.empty(n * lib.pq3d_src_record_bytes() // 8, **f64)
    st = _lib.stream_ptr()
    _lib.check(lib.pq3d_src_records(nodes.data_ptr(), tri.data_ptr(), n, rec.data_ptr(), st), "records")
    m = len(rows)
    pr = torch.tensor(np.repeat(rows, n), device="cuda")
    pc = torch.arange(n, device="cuda").repeat(m)
    out = torch.empty(m * n * 6, **f64)
    _lib.check(lib.pq3d_traction_pairs(xg.data_ptr(), ev.data_ptr(), rec.data_ptr(), pr.data_ptr(), pc.data_ptr(),
                                       m * n, sim.mu, sim.lambda_, out.data_ptr(), None, 0, st), "pairs")
    return out.view(m, n, 6).permute(2, 0, 1)


def test_sampled_rows_match_exact_operator(lib, c60):
    """ACA at relative tolerance eps per block: over 48 sampled receivers, each
    traction-rate component of the H-matvec is within 20 eps (relative L2) of
    the product with the exact operator rows, in FP64 and FP32 storage."""
    sim, op = c60
    eps = float(sim.Para0.get("ACA tolerance"))
    assert sim.Para0.get("ACA relative tolerance") == "True" and eps <= 1e-4
    n = op.n
    rng = np.random.default_rng(11)
    rows = np.sort(rng.choice(n, 48, replace=False))
    x1, x2 = rng.standard_normal((2, n)) * 1e-9
    G = _exact_rows(lib, sim, rows)
    X1, X2 = torch.tensor(x1, device="cuda"), torch.tensor(x2, device="cuda")
    exact = [(G[c] @ X1 + G[c + 3] @ X2).cpu().numpy() for c in range(3)]
    for dtype, tol in (("fp64", 20 * eps), ("fp32", 20 * eps), ("mixed", 20 * eps)):
        y = op.apply(x1, x2, dtype)
        for c in range(3):
            err = np.linalg.norm(y[c][rows] - exact[c]) / np.linalg.norm(exact[c])
            assert err <= tol, (dtype, c, err)


def test_matvec_linearity_and_determinism(c60):
    sim, op = c60
    n = op.n
    rng = np.random.default_rng(12)
    a, b = rng.standard_normal((2, 2, n)) * 1e-9
    for dtype, tol in (("fp64", 1e-12), ("fp32", 1e-5), ("bf16", 1e-5), ("mixed", 1e-5)):
        ya = np.array(op.apply(a[0], a[1], dtype))
        yb = np.array(op.apply(b[0], b[1], dtype))
        yab = np.array(op.apply(a[0] + 2 * b[0], a[1] + 2 * b[1], dtype))
        assert np.abs(yab - (ya + 2 * yb)).max() <= tol * np.abs(yab).max(), dtype
        assert np.array_equal(ya, np.array(op.apply(a[0], a[1], dtype))), dtype   # bitwise reproducible


def _state(st):
    return {k: st.t[k].cpu().numpy().copy() for k in ("slip", "slipv", "psi", "Tno", "Tt")}


def test_graph_equals_eager_steps(c60):
    from pyquake3d_b200.qdsim import DeviceStepper
    sim, op = c60
    a, b = DeviceStepper(sim, op, "fp32"), DeviceStepper(sim, op, "fp32")
    ha = a.run(100, sim.htry)
    g = b.capture(100)
    assert g is not None
    b.ctrl[0] = sim.htry
    g.replay()
    torch.cuda.synchronize()
    hb = b.hist.view(-1, 6).cpu().numpy()[:100]
    assert np.array_equal(ha, hb)
    sa, sb = _state(a), _state(b)
    for k in sa:
        assert np.array_equal(sa[k], sb[k]), k


@pytest.mark.parametrize("prec", ["fp32", "mixed"])
def test_operator_within_slip_target_of_fp64(c60, prec):
    """On the FP64 run's step sizes (dt replay), 100 steps: slip relative L2
    error of the FP32- and mixed-storage runs below the 1e-5 target."""
    from pyquake3d_b200.qdsim import DeviceStepper
    sim, op = c60
    ref = DeviceStepper(sim, op, "fp64")
    h = ref.run(100, sim.htry)[:, 0]
    mix = DeviceStepper(sim, op, prec)
    mix.set_replay(torch.tensor(h, device="cuda"))
    mix.run(100, sim.htry)
    s64, s32 = ref.t["slip"].cpu().numpy(), mix.t["slip"].cpu().numpy()
    err = np.linalg.norm(s32 - s64) / np.linalg.norm(s64)
    assert err < 1e-5, err
    assert abs(mix.time - ref.time) <= 1e-12 * ref.time


def test_two_ranks_follow_fused_step_thrust20k(lib, tmp_path_factory):
    """Row partition over two ranks (emulated in one process) against the fused
    single-GPU step on the 20k thrust fault, FP64 operator, 20 steps: the same
    step sizes and states to 1e-9 (the ranks' row sums add the same products in
    another order)."""
    from pyquake3d_b200.partition import DeviceRowBackend, PartitionedStepper, TorchComm, row_partition
    from pyquake3d_b200.qdsim import DeviceStepper
    sim = _case("thrust20k", tmp_path_factory, "fp64")
    op = sim.tree_block.op()
    st = sim.tree_block.struct
    ref = DeviceStepper(sim, op, "fp64")
    h_ref = ref.run(20, sim.htry)[:, 0]
    b = row_partition(st, 2)
    backends = [DeviceRowBackend(sim, st, b[r], b[r + 1], precision="fp64") for r in range(2)]
    ps = PartitionedStepper(backends, TorchComm(use_dist=False), sim.RelTol)
    dt = sim.htry
    hs = []
    for _ in range(20):
        h, dt = ps.step(dt)
        hs.append(h)
    np.testing.assert_allclose(hs, h_ref, rtol=1e-9)
    for k in ("slip", "psi", "Tt"):
        got = np.concatenate([be.get(k) for be in backends])
        want = ref.t[k].cpu().numpy()
        assert np.abs(got - want).max() <= 1e-9 * np.abs(want).max(), k


def test_two_ranks_device_controller_graph_thrust20k(lib, tmp_path_factory):
    """The row partition with the controller on the device, 20 steps as two
    replays of a captured 10-step graph (collectives and control kernels
    included), mixed storage, two ranks emulated in one process: the fused
    single-GPU mixed step's sizes and states (the ranks' operators hold the same
    term classes; their FP32 sums run in another order)."""
    from pyquake3d_b200 import partition as P
    from pyquake3d_b200.qdsim import DeviceStepper
    sim = _case("thrust20k", tmp_path_factory, "mixed")
    op = sim.tree_block.op()
    st = sim.tree_block.struct
    ref = DeviceStepper(sim, op, "mixed")
    h_ref = ref.run(21, sim.htry)[:, 0]
    b = P.row_partition(st, 2)
    backends = [P.DeviceRowBackend(sim, st, b[r], b[r + 1], precision="mixed") for r in range(2)]
    ps = P.PartitionedStepper(backends, P.TorchComm(use_dist=False), sim.RelTol, attempts=3)
    h1 = ps.run_device(1, sim.htry, chunk=1)
    g = ps.capture(10)
    assert g is not None
    torch.cuda.synchronize()
    hs = list(h1)
    for _ in range(2):
        s0 = int(backends[0].pc[P.PC_STEPS].item())
        g.replay()
        torch.cuda.synchronize()
        pc = backends[0].pc.cpu().numpy()
        assert pc[P.PC_HALT] == 0 and pc[P.PC_STATUS] == 0
        assert int(pc[P.PC_STEPS]) - s0 == 10
        hs.append(float(pc[P.PC_LASTH]))
    np.testing.assert_allclose(hs, h_ref[[0, 10, 20]], rtol=1e-6)
    for be in backends:
        np.testing.assert_array_equal(be.pc.cpu().numpy()[:13], backends[0].pc.cpu().numpy()[:13])
    np.testing.assert_allclose(float(backends[0].pc[P.PC_TIME]), h_ref.sum(), rtol=1e-6)
    for k in ("slip", "psi", "Tt"):
        got = np.concatenate([be.get(k) for be in backends])
        want = ref.t[k].cpu().numpy()
        assert np.abs(got - want).max() <= 1e-6 * np.abs(want).max(), k


def test_plain2k_device_follows_oracle_on_same_operator(lib, tmp_path_factory):
    """plain2k at full size (1,936 triangles, one dense FP64 block): sampled rows
    of the device-assembled operator equal the C oracle's Green's function to
    1e-10 of each plane's scale, and 50 adaptive device steps follow the
    oracle's simu_forward on the same operator (copied to the host): h to 1e-9,
    state to 1e-8."""
    import qd_oracle
    from pyquake3d_b200.hmatrix import export_blocks
    from pyquake3d_b200.qdsim import DeviceStepper
    sim = _case("plain2k", tmp_path_factory, "fp64")
    op = sim.tree_block.op()
    blocks = export_blocks(op)
    assert len(blocks) == 1 and blocks[0][0] == "dense"
    _, rows, cols, M = blocks[0]
    geo = qd_oracle.Geometry(sim.xg, sim.eleVec, sim.nodelst, sim.elelst, sim.mu, sim.lambda_)
    pick = np.random.default_rng(13).choice(len(rows), 16, replace=False)
    ref = geo.gf_block(rows[pick], cols, 3)
    # planar vertical fault: the normal-stress planes B are rounding noise, so the
    # scale of every plane is the operator's maximum
    assert np.abs(M[:, pick, :] - ref).max() <= 1e-10 * np.abs(ref).max()
    ho = object.__new__(qd_oracle.OracleOperator)
    ho.blocks = blocks
    ost = qd_oracle.OracleStepper(qd_oracle.sim_state(sim), qd_oracle.operator_mvm(ho), sim.V0, sim.mu, sim.Cs,
                                  sim.RelTol, sim.fix_Tn)
    dst = DeviceStepper(sim, op, "fp64")
    dt_o = dt_d = sim.htry
    for i in range(50):
        h_o, dt_o = ost.simu_forward(dt_o)
        h_d, dt_d = dst.step(dt_d)
        assert abs(h_d - h_o) <= 1e-9 * abs(h_o), i
    for name, dev in (("slip1", "slip1"), ("state", "psi"), ("Tno", "Tno"), ("Tt1o", "Tt1o")):
        r = getattr(ost, name)
        assert np.abs(dst.get(dev) - r).max() <= 1e-8 * np.abs(r).max(), name


def test_vmode_curved120k_mlp_seed_matches_newton(lib, tmp_path_factory):
    """curved120k at full size (V-mode with the Newton-seeding MLP): the MLP is
    trained on the run's own logged solves; Newton judges every start, so the
    MLP-seeded run and the undamped-start run take the same steps (time to 1e-9)
    and reach the same slip (1e-9), with at most 1% of solves falling back."""
    from pyquake3d_b200.vmode import MLPTrainer, VStepper
    sim = _case("curved120k", tmp_path_factory, "fp32")
    op = sim.tree_block.op()
    logger = VStepper(sim, op, "fp32", seed_mode=1, log_cap=1 << 20)
    logger.run(10, chunk=2)
    tr = MLPTrainer(seed=0)
    hist = tr.fit(logger.samples(), epochs=10, batch=8192, lr=3e-3)
    assert hist[-1] < 0.2 * hist[0]
    del logger
    runs = {}
    for mode in (1, 2):
        st = VStepper(sim, op, "fp32", seed_mode=mode, mlp_params=tr.P if mode == 2 else None)
        c = st.run(10, chunk=2)
        runs[mode] = (c.copy(), st.get("slip1"), st.newton_stats())
        del st
    assert int(runs[1][0][8]) == int(runs[2][0][8]) == 10
    np.testing.assert_allclose(runs[2][0][2], runs[1][0][2], rtol=1e-9)
    assert np.linalg.norm(runs[2][1] - runs[1][1]) <= 1e-9 * np.linalg.norm(runs[1][1])
    s = runs[2][2]
    assert s["fallbacks"] <= 0.01 * s["solves"], s


def _theta(psi, dc, f0, b, V0):
    """State variable theta = (Dc / V0) exp((psi - f0) / b) of the log-state psi."""
    return dc / V0 * np.exp((psi - f0) / b)


def _pin_to_oracle(sim, op, nsteps=12):
    """Device FP64 and FP32 steppers against the oracle's simu_forward on the device's
    own FP64 operator copied to the host (the operator the reference path would
    apply, pinned blockwise by the parity tests).  Returns the worst errors."""
    import qd_oracle
    from pyquake3d_b200.hmatrix import export_blocks
    from pyquake3d_b200.qdsim import DeviceStepper
    ho = object.__new__(qd_oracle.OracleOperator)
    ho.blocks = export_blocks(op)
    ost = qd_oracle.OracleStepper(qd_oracle.sim_state(sim), qd_oracle.operator_mvm(ho), sim.V0, sim.mu, sim.Cs,
                                  sim.RelTol, sim.fix_Tn)
    d64 = DeviceStepper(sim, op, "fp64")
    dt_o = dt_d = sim.htry
    hs = []
    for i in range(nsteps):
        h_o, dt_o = ost.simu_forward(dt_o)
        h_d, dt_d = d64.step(dt_d)
        assert abs(h_d - h_o) <= 1e-9 * abs(h_o), (i, h_d, h_o)
        hs.append(h_o)
    del ho
    out = {}
    for name, dev in (("slip1", "slip1"), ("slip2", "slip2"), ("state", "psi"), ("Tno", "Tno"), ("Tt1o", "Tt1o"),
                      ("slipv", "slipv")):
        r = getattr(ost, name)
        out["fp64_" + name] = float(np.abs(d64.get(dev) - r).max() / np.abs(r).max())
    # FP32 and mixed operators on the oracle's step sizes
    rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))
    slip_o = np.sqrt(ost.slip1 ** 2 + ost.slip2 ** 2)
    th_o = _theta(ost.state, ost.dc, ost.f0, ost.b, sim.V0)
    for prec in [p for p in ("fp32", "mixed") if p in op.plans]:
        d32 = DeviceStepper(sim, op, prec)
        d32.set_replay(torch.tensor(hs, dtype=torch.float64, device="cuda"))
        d32.run(nsteps, sim.htry)
        out[prec + "_slip"] = rel(np.sqrt(d32.get("slip1") ** 2 + d32.get("slip2") ** 2), slip_o)
        out[prec + "_V"] = rel(d32.get("slipv"), ost.slipv)
        out[prec + "_theta"] = rel(_theta(d32.get("psi"), ost.dc, ost.f0, ost.b, sim.V0), th_o)
    return out


def test_curved60k_pinned_to_oracle(c60):
    """curved60k: 12 adaptive steps of the oracle's simu_forward on the device's FP64
    operator (copied to the host) beside the device FP64 stepper (h to 1e-9, state
    to 1e-8) and the FP32- and mixed-storage steppers on the oracle's step sizes
    (slip, V and theta relative L2 within the 1e-5 target)."""
    sim, op = c60
    e = _pin_to_oracle(sim, op)
    for k, v in e.items():
        lim = 1e-8 if k.startswith("fp64") else 1e-5
        assert v <= lim, (k, v, e)


def test_thrust20k_pinned_to_oracle(lib, tmp_path_factory):
    """thrust20k (20,480 triangles, ACA relative 1e-4): the same pin as curved60k."""
    sim = _case("thrust20k", tmp_path_factory, "fp32")
    sim.tree_block.want = ("fp64", "fp32", "mixed")
    op = sim.tree_block.op()
    e = _pin_to_oracle(sim, op)
    for k, v in e.items():
        lim = 1e-8 if k.startswith("fp64") else 1e-5
        assert v <= lim, (k, v, e)
