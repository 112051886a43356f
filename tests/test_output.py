"""Output path (VTK, gridded maps, state.txt, driver step ranges) and the operator
checkpoint file format, on the CPU.  The VTK and map files are compared byte for
byte (SHA-256) with what the reference's QDsim.ouputVTK / QDsim.outputtxt wrote
for the same state (tests/golden/output_case.npz, made by make_golden.py)."""
import hashlib
import json
import os
import types

import numpy as np
import pytest

from conftest import GOLDEN


@pytest.fixture(scope="module")
def out_case(tiny_golden):
    d = dict(np.load(os.path.join(GOLDEN, "output_case.npz")))
    ns = types.SimpleNamespace(nodelst=tiny_golden["nodes"], elelst=tiny_golden["tris"], xg=tiny_golden["xg"],
                               maxsize=float(d["maxsize"]))
    for k, v in d.items():
        if not k.startswith("sha256:") and k not in ("maxsize", "output_seed"):
            setattr(ns, k, v)
    return ns, {k[7:]: str(v) for k, v in d.items() if k.startswith("sha256:")}


def _sha(path):
    with open(path, "rb") as f:
        return hashlib.sha256(f.read()).hexdigest()


def test_vtk_bytes_match_reference(out_case, tmp_path):
    from pyquake3d_b200.output import write_vtk
    ns, sums = out_case
    p = tmp_path / "s.vtk"
    write_vtk(ns, str(p))
    assert _sha(p) == sums["ref.vtk"]
    text = p.read_text()
    assert text.startswith("# vtk DataFile Version 3.0\ntest\nASCII\nDATASET  UNSTRUCTURED_GRID\n")
    assert text.count("SCALARS ") == 18


def test_gridded_maps_match_reference(out_case, tmp_path, monkeypatch):
    from pyquake3d_b200.output import write_txt
    ns, sums = out_case
    monkeypatch.chdir(tmp_path)
    write_txt(ns, "step5")
    files = ["out_txt/" + f for f in sorted(os.listdir("out_txt"))]
    assert files == sorted(k for k in sums if k.startswith("out_txt/"))
    for f in files:
        assert _sha(f) == sums[f], f


def test_state_log_lines(tmp_path):
    from pyquake3d_b200.output import StateLog
    sim = types.SimpleNamespace(Cs=3464.0, lambda_=3.2e10, mu=3.2e10, YoungsM=8e10, possonratio=0.25, maxsize=1.0,
                                ave_elesize=0.5, hRA=1234.5, A0=99.0)
    p = tmp_path / "state.txt"
    log = StateLog(str(p), sim, "a.msh", "p.txt", np.zeros((5, 3)), np.zeros((7, 3)))
    log.step(3, 0.125, 1e-9, 2.5e-12, 86400.0)
    log.close(1.5)
    lines = p.read_text().splitlines()
    assert lines[3] == "Number of Node:5" and lines[4] == "Number of Element:7"
    assert lines[14] == "iteration time_step(s) maximum_slip_rate(m/s) time(s) time(h)"
    assert lines[15] == "%d %f %f %.16e %f %f" % (3, 0.125, 1e-9, 2.5e-12, 86400.0, 1.0)
    assert lines[15].startswith("3 0.125000 0.000000 2.49999")
    assert lines[-1] == "Time taken: 1.50 seconds"


@pytest.mark.parametrize("total,outsteps", [(1, 100), (10, 3), (250, 100), (201, 100), (7, 1), (5, 10)])
def test_step_ranges_cover_run_and_end_at_outputs(total, outsteps):
    from pyquake3d_b200.main import step_ranges
    r = step_ranges(total, outsteps)
    assert r[0][0] == 0 and r[-1][1] == total
    assert all(a < b for a, b in r) and all(r[i][1] == r[i + 1][0] for i in range(len(r) - 1))
    outs = {i for i in range(total) if i % outsteps == 0}
    ends = {b - 1 for _, b in r}
    assert outs <= ends and ends - outs <= {total - 1}


class _FakeOp:
    """Enough of DeviceHMatrix (host tensors) to exercise the checkpoint file format."""

    DENSE_CHUNK_GROUPS = {0: 64, 1: 16, 2: 16}
    V_CHUNK_GROUPS = {0: 128, 1: 32, 2: 32}
    U_ROWS = 512

    def __init__(self):
        import torch
        from pyquake3d_b200 import _lib
        self.n = 40
        self.mu = self.lam = 3.2e10
        self.aca_tol, self.aca_rel, self.aca_seed, self.kcap = 1e-4, True, 0, 96
        self.s = types.SimpleNamespace(mini_leaf=32, eta=2.0, min_size=16)
        self.dense_recs = np.zeros(3, dtype=_lib.DENSE_BLOCK)
        self.dense_recs["m"] = [4, 5, 6]
        self.aca_ranks = np.array([3, 0, 7, 2], dtype=np.int32)
        self.aca_flags = np.array([0, 2, 0, 0], dtype=np.int32)
        g = torch.Generator().manual_seed(0)
        self.dense64 = torch.randn(1000, generator=g, dtype=torch.float64)
        self.dense32 = self.dense64.float()
        self.plans = {"bf16": dict(U=torch.randn(77, generator=g).bfloat16(), V=torch.randn(99, generator=g).bfloat16()),
                      "fp32": dict(U=torch.randn(5000, generator=g), V=torch.randn(123, generator=g))}
        self.assembled = True


def test_checkpoint_file_roundtrip(tmp_path):
    from pyquake3d_b200 import checkpoint
    op = _FakeOp()
    xg = np.random.default_rng(0).normal(size=(40, 3))
    ev = np.random.default_rng(1).normal(size=(40, 9))
    p = str(tmp_path / checkpoint.FILE_NAME)
    h = checkpoint.save_operator(op, p, xg, ev)
    assert os.path.getsize(p) % checkpoint.ALIGN == 0
    hr = checkpoint.read_header(p)
    assert hr["fingerprint"] == h["fingerprint"] == checkpoint.op_fingerprint(op, xg, ev)
    assert hr["precisions"] == ["bf16", "fp32"]
    for t in hr["sections"]:
        assert (hr["_data0"] + t["offset"]) % checkpoint.ALIGN == 0
    np.testing.assert_array_equal(checkpoint._read(p, hr, "aca_ranks"), op.aca_ranks)
    np.testing.assert_array_equal(checkpoint._read(p, hr, "dense64"), op.dense64.numpy())
    np.testing.assert_array_equal(checkpoint._read(p, hr, "U_fp32"), op.plans["fp32"]["U"].numpy())
    ub = checkpoint._read(p, hr, "U_bf16")
    import torch
    assert torch.equal(torch.from_numpy(ub.view(np.int16)).view(torch.bfloat16), op.plans["bf16"]["U"])
    recs = checkpoint._read(p, hr, "dense_recs").view(op.dense_recs.dtype)
    np.testing.assert_array_equal(recs["m"], [4, 5, 6])


def test_checkpoint_fingerprint_sensitivity():
    from pyquake3d_b200 import checkpoint
    op = _FakeOp()
    xg = np.zeros((40, 3))
    ev = np.zeros((40, 9))
    f0 = checkpoint.op_fingerprint(op, xg, ev)
    xg2 = xg.copy()
    xg2[5, 1] = 1e-12
    assert checkpoint.op_fingerprint(op, xg2, ev) != f0
    op.aca_tol = 1e-5
    assert checkpoint.op_fingerprint(op, xg, ev) != f0


def test_checkpoint_rejects_foreign_files(tmp_path):
    from pyquake3d_b200 import checkpoint, _lib
    p = tmp_path / "x.pq3d"
    p.write_bytes(b"not a checkpoint at all")
    with pytest.raises(_lib.Pq3dError):
        checkpoint.read_header(str(p))
    hb = json.dumps(dict(version=99)).encode()
    import struct
    p.write_bytes(checkpoint.MAGIC + struct.pack("<Q", len(hb)) + hb)
    with pytest.raises(_lib.Pq3dError):
        checkpoint.read_header(str(p))


def test_checkpoint_fingerprint_covers_half_space():
    from pyquake3d_b200 import checkpoint
    op = _FakeOp()
    xg, ev = np.zeros((40, 3)), np.zeros((40, 9))
    fps = set()
    for hs in (0, 1, 2):
        op.halfspace = hs
        fps.add(checkpoint.op_fingerprint(op, xg, ev))
    assert len(fps) == 3
