"""V-mode on the GPU (no reference counterpart; checked against the project's FP64
oracle oracle/vmode_oracle.py) and the Newton-seeding MLP: gradients of the
hand-written training kernels vs the FP64 oracle, training on the stepper's own
solves, and the Newton iterations it saves.  Tolerances: V-mode state 1e-8
(same controller, same step sequence), MLP gradients 1e-4 of each tensor's scale."""
import numpy as np
import pytest

import qd_oracle
import vmode_oracle as vo
from pyquake3d_b200.hmatrix import aca_start_indices

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return True


def _case(tmp, name, n):
    from pyquake3d_b200 import QDsim, meshgen, read_mshV2
    msh, para = meshgen.make_case(name, str(tmp), n_target=n)
    nodes, tris = read_mshV2(msh)
    return QDsim(tris, nodes, para, precision="fp64")


def test_vmode_follows_oracle(gpu, tmp_path_factory):
    from pyquake3d_b200.vmode import VStepper
    sim = _case(tmp_path_factory.mktemp("vm"), "tiny", 300)
    op = sim.tree_block.op()
    st = sim.tree_block.struct
    geo = qd_oracle.Geometry(sim.xg, sim.eleVec, sim.nodelst, sim.elelst, sim.mu, sim.lambda_)
    oop = qd_oracle.OracleOperator(geo, [(b.row.indices, b.col.indices, b.aca) for b in st.blocks],
                                   aca_start_indices(st.blocks, 0), eps=0.01)
    ref = vo.VModeOracle(qd_oracle.sim_state(sim), qd_oracle.operator_mvm(oop), sim.V0, sim.mu, sim.Cs)
    dev = VStepper(sim, op, "fp64", seed_mode=1)
    dev.start(1e-3)
    h = 1e-3
    for _ in range(12):
        _, h = ref.step(h)
    c = dev.run(12, max_attempts=200, chunk=1)
    assert int(c[8]) == 12
    np.testing.assert_allclose(c[2], ref.time, rtol=1e-8)
    for name, r in (("slip1", ref.s1), ("psi", ref.psi)):
        d = dev.get(name)
        assert np.linalg.norm(d - r) <= 1e-8 * np.linalg.norm(r), name


def test_mlp_gradient_matches_fp64_oracle(gpu):
    from pyquake3d_b200.vmode import MLPTrainer, mlp_init_params, mlp_unflatten
    tr = MLPTrainer(seed=3)
    rng = np.random.default_rng(4)
    X = rng.standard_normal((512, 6)).astype(np.float32)
    Xd = torch.tensor(X, device="cuda")
    g, loss = tr.grad(Xd, Xd[:, 5:])
    P = mlp_unflatten(tr.P.double().cpu().numpy())
    L, gr = vo.mlp_loss_grad(P, X[:, :5].astype(np.float64), X[:, 5].astype(np.float64))
    g = g.double().cpu().numpy()
    flat = np.concatenate([gr["W1"].ravel(), gr["b1"], gr["W2"].ravel(), gr["b2"], gr["W3"].ravel(), gr["b3"]])
    for sl in (slice(0, 320), slice(320, 384), slice(384, 4480), slice(4480, 4544), slice(4544, 4608), slice(4608, 4609)):
        assert np.abs(g[sl] - flat[sl]).max() <= 1e-4 * np.abs(flat[sl]).max() + 1e-7
    assert abs(loss - L) <= 1e-5 * L


def test_mlp_seed_trained_on_own_solves_cuts_newton_iterations(gpu, tmp_path_factory):
    from pyquake3d_b200.vmode import MLPTrainer, VStepper
    sim = _case(tmp_path_factory.mktemp("nuc"), "tinynuc", 400)
    op = sim.tree_block.op()
    # 1. log converged solves from plain Newton (undamped start)
    logger = VStepper(sim, op, "fp64", seed_mode=1, log_cap=300000)
    logger.run(30, chunk=2)
    data = logger.samples()
    assert data.shape[0] > 20000
    # 2. train on the GPU with the hand-written kernels
    tr = MLPTrainer(seed=0)
    hist = tr.fit(data, epochs=40, batch=4096, lr=3e-3)
    assert hist[-1] < 0.2 * hist[0]
    # 3. same steps with the undamped start, the previous-rate start, the MLP start and
    # the gated MLP start (network only where the undamped start's first Newton
    # correction is large)
    runs = {}
    for mode in (1, 0, 2, 3):
        st = VStepper(sim, op, "fp64", seed_mode=mode, mlp_params=tr.P if mode >= 2 else None)
        c = st.run(20, chunk=2)
        runs[mode] = (st.newton_stats(), c, st.get("slip1"))
    # Newton judges every start: the solutions agree
    base = runs[1][2]
    for mode in (0, 2, 3):
        assert np.linalg.norm(runs[mode][2] - base) <= 1e-9 * np.linalg.norm(base)
        np.testing.assert_allclose(runs[mode][1][2], runs[1][1][2], rtol=1e-9)
    # the trained network saves iterations against the undamped start (mean and worst case);
    # gated, it takes fewer iterations on average than either classical start (measured:
    # 1.61 against 1.79 undamped and 1.91 previous-rate; worst case 9 against 15 and 4)
    stats = {m: r[0] for m, r in runs.items()}
    assert stats[2]["mean"] < stats[1]["mean"], stats
    assert stats[2]["max"] < stats[1]["max"], stats
    assert stats[3]["mean"] < min(stats[0]["mean"], stats[1]["mean"]), stats
    assert stats[3]["max"] < stats[1]["max"], stats
    for m in (2, 3):
        assert stats[m]["fallbacks"] <= 0.01 * stats[m]["solves"], stats
