"""GPU: the row-partitioned step with ranks emulated in one process.

Each rank is a DeviceRowBackend (its own operator over its rows, the row-range
step kernels); the ranks of one process are reduced by TorchComm on the host
side of plain launches, so no kernel waits for another.  Two ranks follow the
reference's 30-step dt sequence of the tiny case (FP64 operator, 1e-8 as the
single-GPU stepper), and three ranks (low-rank blocks shared across cuts) follow
the fused single-GPU step on the FP32 operator."""
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


def _sim(files, seed):
    from pyquake3d_b200 import QDsim, read_mshV2
    nodes, tris = read_mshV2(files[0])
    sim = QDsim(tris, nodes, files[1])
    sim.Para0["ACA seed"] = str(seed)
    return sim


def _run(sim, R, precision, steps, slack=0.02):
    from pyquake3d_b200.partition import DeviceRowBackend, PartitionedStepper, TorchComm, row_partition
    st = sim.tree_block.struct
    b = row_partition(st, R, slack=slack)
    backends = [DeviceRowBackend(sim, st, b[r], b[r + 1], precision=precision) for r in range(R)]
    ps = PartitionedStepper(backends, TorchComm(use_dist=False), sim.RelTol)
    dttry = sim.htry
    hs = []
    for _ in range(steps):
        h, dttry = ps.step(dttry)
        hs.append(h)
    return np.array(hs), backends, b


def test_two_ranks_follow_reference(lib, tiny_files, tiny_golden):
    g = tiny_golden
    sim = _sim(tiny_files, int(g["aca_seed"]))
    hs, backends, b = _run(sim, 2, "fp64", 30)
    np.testing.assert_allclose(hs, g["steps_h"], rtol=1e-8)
    slip = np.concatenate([be.get("slip") for be in backends])
    ref = g["step30_slip"][sim.tree_block.struct.perm]
    assert np.abs(slip - ref).max() <= 1e-7 * np.abs(ref).max()


def test_three_ranks_with_shared_blocks_follow_fused_step(lib, tiny_files, tiny_golden):
    seed = int(tiny_golden["aca_seed"])
    sim = _sim(tiny_files, seed)
    hs, backends, b = _run(sim, 3, "fp32", 30, slack=0.0)
    assert sum(1 for be in backends for blk in be.rs.blocks if hasattr(blk, "rows")) > 0
    ref_sim = _sim(tiny_files, seed)
    ref_sim.precision = "fp32"
    st = ref_sim._ensure_device()
    h1 = st.run(30, ref_sim.htry)[:, 0]
    np.testing.assert_allclose(hs, h1, rtol=1e-9)
    slip = np.concatenate([be.get("slip1") for be in backends])
    ref = st.t["slip1"].cpu().numpy()
    assert np.abs(slip - ref).max() <= 1e-9 * np.abs(ref).max()
