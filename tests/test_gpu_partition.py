"""GPU: the row-partitioned step with ranks emulated in one process.

Each rank is a DeviceRowBackend (its own operator over its rows, the row-range
step kernels); the ranks of one process are reduced by TorchComm on the host
side of plain launches, so no kernel waits for another.  Two ranks follow the
reference's 30-step dt sequence of the tiny case (FP64 operator, 1e-8 as the
single-GPU stepper), and three ranks (low-rank blocks shared across cuts) follow
the fused single-GPU step on the FP32 operator.  With the controller on the
device (pq3d_rk_rows_control) the two ranks take the same decisions without a
host read per attempt, and a step that outruns the attempt slots is finished by
the host controller exactly as the host-controlled run takes it."""
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


def _backends(sim, R, precision, slack=0.02):
    from pyquake3d_b200.partition import DeviceRowBackend, row_partition
    st = sim.tree_block.struct
    b = row_partition(st, R, slack=slack)
    return [DeviceRowBackend(sim, st, b[r], b[r + 1], precision=precision) for r in range(R)]


@pytest.mark.parametrize("chunk", [1, 10])
def test_device_controller_follows_reference(lib, tiny_files, tiny_golden, chunk):
    """The controller on the device (a fixed launch sequence per step, the host
    reading the control block once per chunk) takes the reference's decisions."""
    from pyquake3d_b200.partition import PartitionedStepper, TorchComm
    g = tiny_golden
    sim = _sim(tiny_files, int(g["aca_seed"]))
    backends = _backends(sim, 2, "fp64")
    ps = PartitionedStepper(backends, TorchComm(use_dist=False), sim.RelTol, attempts=3)
    out = ps.run_device(30, sim.htry, chunk=chunk)
    if chunk == 1:
        np.testing.assert_allclose(out, g["steps_h"], rtol=1e-8)
    else:
        np.testing.assert_allclose(out[0], g["steps_h"][-1], rtol=1e-8)
    assert ps.steps == 30
    np.testing.assert_allclose(ps.time, np.sum(g["steps_h"]), rtol=1e-8)
    slip = np.concatenate([be.get("slip") for be in backends])
    ref = g["step30_slip"][sim.tree_block.struct.perm]
    assert np.abs(slip - ref).max() <= 1e-7 * np.abs(ref).max()
    assert all(be.pc[4].item() == 0.0 and be.pc[10].item() == 0.0 for be in backends)


@pytest.mark.parametrize("attempts,k", [(1, 36), (3, 40)])
def test_device_controller_halts_and_host_finishes(lib, tiny_files, tiny_golden, attempts, k):
    """A first trial size of 2^k times the initial one (about 2 and 35 years; the
    oracle rejects it 5 and 9 times, NaN attempts among the latter): the first step
    outruns the attempt slots, the device halts it, the host finishes it with the
    same controller and the device run resumes; steps, rejections, sizes and state
    equal the host-controlled run from the same trial size."""
    from pyquake3d_b200.partition import PartitionedStepper, TorchComm
    seed = int(tiny_golden["aca_seed"])
    sim_a = _sim(tiny_files, seed)
    sim_b = _sim(tiny_files, seed)
    dttry = sim_a.htry * 2.0 ** k
    ba = _backends(sim_a, 2, "fp64")
    pa = PartitionedStepper(ba, TorchComm(use_dist=False), sim_a.RelTol, attempts=attempts)
    ha = pa.run_device(12, dttry, chunk=1)
    bb = _backends(sim_b, 2, "fp64")
    pb = PartitionedStepper(bb, TorchComm(use_dist=False), sim_b.RelTol)
    hb = []
    dt = dttry
    for _ in range(12):
        h, dt = pb.step(dt)
        hb.append(h)
    assert pb.rejects > attempts                 # the first step did outrun the slots
    np.testing.assert_allclose(ha, hb, rtol=1e-12)
    assert (pa.steps, pa.rejects) == (pb.steps, pb.rejects)
    for x, y in zip(ba, bb):
        np.testing.assert_allclose(x.get("slip1"), y.get("slip1"), rtol=1e-12, atol=1e-300)
        np.testing.assert_allclose(x.get("psi"), y.get("psi"), rtol=1e-12)


def test_bench_partition_arm(lib):
    """bench.py's row-partition arm (what `bench.py --gpus N` runs) on one GPU and one
    rank, thrust20k: the timed region completes its steps (graph replays of 50 steps,
    any step that outran the attempt slots finished by the host controller inside the
    region) and the JSON line carries the strong-scaling fields."""
    import json
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK", "TORCHELASTIC_RUN_ID")}
    r = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--parallelism", "partition", "--case",
                        "thrust20k", "--steps", "50", "--warmup", "3", "--no-cpu"], cwd=root, env=env,
                       capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["scaling"] == "strong" and line["n_gpus"] == 1
    assert line["steps_done"] >= 50 and line["value"] > 0
    assert line["halted"] == (line["host_finished_steps"] > 0)
    assert line["config"]["cuda_graph_steps"] == 50
    assert line["gpu_launches"] > 0 and line["e2e"]["value"] > 0
