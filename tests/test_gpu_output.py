"""GPU: operator checkpoint round trip and the command-line driver on the tiny case.

* a checkpointed operator, loaded into a fresh DeviceHMatrix, gives bitwise the
  same products as the assembled one, for every stored precision (the mixed
  storage's term classes, class arrays and scales included);
* the driver (pyquake3d_b200.main.run) follows the reference's 30-step dt sequence
  (state.txt, %f of h), writes Init.vtk, out_vtk/stepI.vtk and the per-step slip
  rate / traction dumps of the reference layout, and a second run that loads the
  checkpoint written by the first reproduces its state.txt lines exactly."""
import os
import shutil

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


def test_checkpoint_roundtrip_bitwise(lib, tiny_sim, tiny_golden, tmp_path):
    from pyquake3d_b200 import checkpoint
    from pyquake3d_b200.hmatrix import DeviceHMatrix
    s = tiny_sim
    kw = dict(aca_tol=0.01, aca_rel=False, aca_seed=int(tiny_golden["aca_seed"]))
    op = DeviceHMatrix(s.tree_block.struct, s.xg, s.eleVec, s.nodelst, s.elelst, s.mu, s.lambda_, **kw)
    op.assemble(("fp64", "fp32", "bf16", "mixed"))
    p = str(tmp_path / checkpoint.FILE_NAME)
    checkpoint.save_operator(op, p, s.xg, s.eleVec)
    op2 = DeviceHMatrix(s.tree_block.struct, s.xg, s.eleVec, s.nodelst, s.elelst, s.mu, s.lambda_, **kw)
    checkpoint.load_operator(op2, p, s.xg, s.eleVec)
    rng = np.random.default_rng(3)
    x1, x2 = rng.standard_normal((2, s.xg.shape[0])) * 1e-9
    for d in ("fp64", "fp32", "bf16", "mixed"):
        a = op.apply(x1, x2, d)
        b = op2.apply(x1, x2, d)
        for u, v in zip(a, b):
            assert np.array_equal(u, v), d
    # another mesh: refused
    ev = s.eleVec.copy()
    ev[0, 0] += 1e-9
    op3 = DeviceHMatrix(s.tree_block.struct, s.xg, ev, s.nodelst, s.elelst, s.mu, s.lambda_, **kw)
    with pytest.raises(_lib.Pq3dError):
        checkpoint.load_operator(op3, p, s.xg, ev)


def _case_dir(tmp, tiny_files, tiny_golden):
    msh, para = tiny_files
    src = os.path.dirname(msh)
    d = tmp / "case"
    d.mkdir()
    shutil.copy(msh, d / "tiny.msh")
    shutil.copy(os.path.join(src, "tinyparam.dat"), d / "tinyparam.dat")
    keys = {"Corefunc directory": str(tmp / "core"), "save Corefunc": "True", "outsteps": "10",
            "outputvtk": "True", "outputSLIPV": "True", "outputTt": "True",
            "ACA seed": str(int(tiny_golden["aca_seed"]))}
    lines = []
    for ln in str(tiny_golden["parameter_txt"]).splitlines():
        k = ln.split(":")[0].strip() if ":" in ln else None
        lines.append(f"{k}: {keys.pop(k)}" if k in keys else ln)
    lines += [f"{k}: {v}" for k, v in keys.items()]
    (d / "parameter.txt").write_text("\n".join(lines) + "\n")
    return str(d / "tiny.msh"), str(d / "parameter.txt")


def _step_lines(path):
    lines = open(path).read().splitlines()
    i = lines.index("iteration time_step(s) maximum_slip_rate(m/s) time(s) time(h)")
    return [ln for ln in lines[i + 1:] if not ln.startswith(("Program end", "Time taken"))]


def test_driver_outputs_and_checkpoint_reload(lib, tiny_files, tiny_golden, tmp_path, monkeypatch):
    from pyquake3d_b200.main import run
    g = tiny_golden
    msh, para = _case_dir(tmp_path, tiny_files, g)
    run1 = tmp_path / "run1"
    run1.mkdir()
    monkeypatch.chdir(run1)
    sim = run(msh, para, steps=30, quiet=True)
    steps = _step_lines("state.txt")
    assert len(steps) == 30
    cols = np.array([[float(v) for v in ln.split()] for ln in steps])
    assert np.array_equal(cols[:, 0], np.arange(30))
    np.testing.assert_allclose(cols[:, 1], g["steps_h"], atol=1.5e-6, rtol=1e-8)
    np.testing.assert_allclose(cols[:, 4], g["steps_time"], atol=1.5e-6, rtol=1e-8)
    np.testing.assert_allclose(cols[29, 3], np.abs(g["step30_slipv2"]).max(), rtol=1e-7)
    assert os.path.exists("Init.vtk")
    assert sorted(os.listdir("out_vtk")) == ["step0.vtk", "step10.vtk", "step20.vtk"]
    v0 = np.load("out_slipvTt/slipv_0.npy")
    v20 = np.load("out_slipvTt/slipv_20.npy")
    t10 = np.load("out_slipvTt/Tt_10.npy")
    n = sim.xg.shape[0]
    assert v0.shape == (1, n) and v20.shape == (10, n) and t10.shape == (10, n)
    ref = g["step1_slipv"]
    assert np.abs(v0[0] - ref).max() <= 1e-9 * np.abs(ref).max()
    assert os.path.exists(tmp_path / "core" / "operator.pq3d")
    vtk = open("out_vtk/step20.vtk").read()
    assert "CELL_DATA %d SCALARS Normal_[MPa] float" % n in vtk
    # second run: the operator comes from the checkpoint, the run is identical
    run2 = tmp_path / "run2"
    run2.mkdir()
    monkeypatch.chdir(run2)
    from pyquake3d_b200 import QDsim, read_mshV2
    nodes, tris = read_mshV2(msh)
    probe = QDsim(tris, nodes, para)
    loaded, blocks = probe.get_block_core()
    assert loaded and len(blocks) == len(probe.tree_block.struct.blocks)
    run(msh, para, steps=30, quiet=True)
    assert _step_lines("state.txt") == steps


def test_async_snapshots_match_state(lib, tiny_files):
    """QDsim.snapshot_async: host copies gathered on a side stream into mapped host
    memory (alternating buffers) equal the synchronous read-back of the same step,
    step after step, while the next step's H-matvec is already enqueued."""
    from pyquake3d_b200 import QDsim, read_mshV2
    nodes, tris = read_mshV2(tiny_files[0])
    sim = QDsim(tris, nodes, tiny_files[1])
    dttry = sim.htry
    pending = []
    for i in range(6):
        h, dttry = sim.simu_forward(dttry)
        st = sim._ensure_device()
        ref = {k: st.get(k) for k in ("slipv", "Tt")}
        done, host = sim.snapshot_async(("slipv", "Tt"))
        pending.append((done, host, ref))
        if len(pending) == 2:               # a buffer stays valid until the snapshot after next
            d0, h0, r0 = pending.pop(0)
            d0.synchronize()
            for k in ("slipv", "Tt"):
                assert np.array_equal(h0[k], r0[k]), (i, k)
